/*
 * ref_shim.h -- test infrastructure only (not part of the product).
 *
 * A tiny host-side stand-in for the CUDA runtime so that the reference's own
 * compress/decompress sources (cucm_compress_v2.cu, cucm_decompress_v2.cu)
 * compile with g++ and run on the CPU.  make_ref.py rewrites every kernel
 * launch `k<<<g, b>>>(args);` into `shim_launch(g, b, [&] { k(args); });`,
 * which runs the kernel body once per (block, thread) in index order.
 *
 * Serial execution gives the same results as the GPU for these kernels: no
 * kernel reads what another thread of the same launch writes, the only
 * atomics are commutative integer adds, and no warp-level primitives are
 * used.  Launches on the legacy default stream are ordered, exactly like the
 * sequential loop here.
 *
 * The executables built from this shim are the checker that pins the C
 * restatement in oracle/cucm_oracle.c, and the CPU baseline that bench.py's
 * reference arm times.
 */
#pragma once

#include <cctype>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline

struct shim_dim3 {
  unsigned x, y, z;
};
extern shim_dim3 blockIdx, threadIdx, blockDim, gridDim;

template <typename F>
static inline void shim_launch(unsigned long long grid, unsigned long long block, F body) {
  gridDim.x = (unsigned)grid;
  blockDim.x = (unsigned)block;
  gridDim.y = gridDim.z = blockDim.y = blockDim.z = 1;
  blockIdx.y = blockIdx.z = threadIdx.y = threadIdx.z = 0;
  for (unsigned long long b = 0; b < grid; b++) {
    blockIdx.x = (unsigned)b;
    for (unsigned long long t = 0; t < block; t++) {
      threadIdx.x = (unsigned)t;
      body();
    }
  }
}

typedef int cudaError_t;
enum { cudaSuccess = 0 };
enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3
};

static inline const char *cudaGetErrorString(cudaError_t) { return "no error"; }
static inline cudaError_t cudaGetLastError() { return cudaSuccess; }
static inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
static inline cudaError_t cudaDeviceReset() { return cudaSuccess; }

/* Zero-filled, like the fresh device memory the reference sees on its first
 * allocations: its decoder reads never-written entries of d_realsmhashes
 * (cucm_decompress_v2.cu:876) when a chunk's only unit is partial, and a
 * garbage hash would index far outside the StateMap. */
template <typename T>
static inline cudaError_t cudaMalloc(T **p, size_t n) {
  *p = (T *)calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : 2;
}
static inline cudaError_t cudaFree(void *p) {
  free(p);
  return cudaSuccess;
}
static inline cudaError_t cudaMemset(void *p, int v, size_t n) {
  memset(p, v, n);
  return cudaSuccess;
}
static inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) {
  memmove(d, s, n);
  return cudaSuccess;
}
#define cudaMemcpyToSymbol(sym, src, n) (memcpy((void *)&(sym), (src), (n)), cudaSuccess)

/* int atomicAdd with two's-complement wrap, as the hardware does. */
static inline int atomicAdd(int *p, long long v) {
  int old = *p;
  *p = (int)((unsigned)old + (unsigned)(int)v);
  return old;
}
static inline int __clz(int x) { return x == 0 ? 32 : __builtin_clz((unsigned)x); }

/* The only library call on the path: cub's inclusive prefix sum. */
namespace cub {
struct DeviceScan {
  template <typename T>
  static cudaError_t InclusiveSum(void *tmp, size_t &bytes, const T *in, T *out, long long n) {
    if (tmp == nullptr) {
      bytes = 16;
      return cudaSuccess;
    }
    T acc = 0;
    for (long long i = 0; i < n; i++) {
      acc += in[i];
      out[i] = acc;
    }
    return cudaSuccess;
  }
};
}  // namespace cub
