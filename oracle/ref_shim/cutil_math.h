// cutil_math.h -- host stand-in for the CUDA SDK vector helpers the
// reference includes (TEST INFRASTRUCTURE).  Written from the mathematics:
// component-wise operators, the dot product in x, y, z order, length as the
// square root of the dot product, and normalize as v * (1 / sqrt(dot(v, v)))
// (the SDK's host form of rsqrtf is 1 / sqrtf).  Every operation is one IEEE
// float rounding (the recipe builds with -ffp-contract=off).
#pragma once
#include <cmath>
#include "vector_types.h"

typedef unsigned int uint;

inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
inline float fminf_(float a, float b) { return a < b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline uint min(uint a, uint b) { return a < b ? a : b; }
inline uint max(uint a, uint b) { return a > b ? a : b; }
inline float min(float a, float b) { return a < b ? a : b; }
// mixed signed / unsigned arguments compare as unsigned (the CUDA overloads)
inline uint min(int a, uint b) { return min((uint)a, b); }
inline uint min(uint a, int b) { return min(a, (uint)b); }
inline uint max(int a, uint b) { return max((uint)a, b); }
inline uint max(uint a, int b) { return max(a, (uint)b); }
inline float max(float a, float b) { return a > b ? a : b; }
inline float clamp(float f, float a, float b) { return fmaxf(a, fminf(f, b)); }

inline float3 make_float3(float x, float y, float z) { float3 r; r.x = x; r.y = y; r.z = z; return r; }
inline float3 make_float3(float s) { return make_float3(s, s, s); }
inline float3 make_float3(float4 a) { return make_float3(a.x, a.y, a.z); }
inline float4 make_float4(float x, float y, float z, float w) { float4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }
inline float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
inline float4 make_float4(float3 a) { return make_float4(a.x, a.y, a.z, 0.0f); }
inline float4 make_float4(float s) { return make_float4(s, s, s, s); }
inline int3 make_int3(int x, int y, int z) { int3 r; r.x = x; r.y = y; r.z = z; return r; }
inline uint2 make_uint2(uint x, uint y) { uint2 r; r.x = x; r.y = y; return r; }
inline uint3 make_uint3(uint x, uint y, uint z) { uint3 r; r.x = x; r.y = y; r.z = z; return r; }
inline uint4 make_uint4(uint x, uint y, uint z, uint w) { uint4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }

inline int3 operator+(int3 a, int3 b) { return make_int3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
inline float3 operator/(float s, float3 a) { return make_float3(s / a.x, s / a.y, s / a.z); }
inline void operator+=(float3& a, float3 b) { a = a + b; }
inline void operator-=(float3& a, float3 b) { a = a - b; }
inline void operator*=(float3& a, float s) { a = a * s; }
inline void operator/=(float3& a, float s) { a = a / s; }
inline float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline float4 operator-(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
inline float4 operator*(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline float4 operator/(float4 a, float s) { return make_float4(a.x / s, a.y / s, a.z / s, a.w / s); }
inline void operator+=(float4& a, float4 b) { a = a + b; }

inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float length(float3 v) { return sqrtf(dot(v, v)); }
inline float length(float4 v) { return sqrtf(dot(v, v)); }
inline float3 normalize(float3 v) { float invLen = rsqrtf(dot(v, v)); return v * invLen; }
inline float3 floor(float3 v) { return make_float3(floorf(v.x), floorf(v.y), floorf(v.z)); }
inline float3 cross(float3 a, float3 b) { return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
