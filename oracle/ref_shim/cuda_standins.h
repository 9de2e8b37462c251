// cuda_standins.h -- force-included before the reference's device sources
// when the oracle's check compiles them on the host (TEST INFRASTRUCTURE).
// CUDA keywords become plain C++, a texture is a pointer to a host array and
// tex1Dfetch reads it, so the reference's own __device__ functions run on the
// CPU unchanged.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#define __host__
#define __device__
#define __global__
#define __constant__
#define __shared__ static
#define __forceinline__ inline

enum cudaTextureReadMode { cudaReadModeElementType = 0 };
template <class T, int Dim = 1, int Mode = 0>
struct texture {
  const T* data = nullptr;
};
template <class T, int Dim, int Mode>
inline T tex1Dfetch(const texture<T, Dim, Mode>& t, int i) { return t.data[i]; }

inline int __mul24(int a, int b) { return a * b; }
inline unsigned int __umul24(unsigned int a, unsigned int b) { return a * b; }

#include "cutil_math.h"

// Built-in indices: the host runs a kernel body for one thread at a time,
// with blockDim = 1 and blockIdx.x = the thread's global index (set by the
// caller before each call).
inline uint3 threadIdx = {0, 0, 0}, blockIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1};
inline void __syncthreads() {}

// The runtime calls the kernel files' host hooks make: a texture is bound by
// pointing it at the array; a symbol copy is a plain copy.
typedef int cudaError_t;
constexpr cudaError_t cudaSuccess = 0;
template <class T, int D, int M>
inline cudaError_t cudaBindTexture(size_t* offset, texture<T, D, M>& t, const void* ptr, size_t bytes = 0) {
  (void)offset; (void)bytes;
  t.data = static_cast<const T*>(ptr);
  return cudaSuccess;
}
template <class T, int D, int M>
inline cudaError_t cudaUnbindTexture(texture<T, D, M>& t) { t.data = nullptr; return cudaSuccess; }
template <class T>
inline cudaError_t cudaMemcpyToSymbol(T& symbol, const void* src, size_t bytes) {
  std::memcpy(&symbol, src, bytes);
  return cudaSuccess;
}
