// vector_types.h -- host stand-in for the CUDA vector types the reference's
// device code uses, so that its __host__ __device__ functions compile with
// g++ (TEST INFRASTRUCTURE: the oracle's check against the reference itself).
#pragma once

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct int4 { int x, y, z, w; };
struct uint2 { unsigned int x, y; };
struct uint3 { unsigned int x, y, z; };
struct uint4 { unsigned int x, y, z, w; };
struct dim3 { unsigned int x = 1, y = 1, z = 1; };
