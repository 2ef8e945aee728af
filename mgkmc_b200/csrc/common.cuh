// Shared definitions for the mgkmc B200 kernels: status codes, error capture,
// complex helpers and deterministic block reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/mgkmc.h"

namespace mgk {

// Thread-local text of the last error, returned by mgk_last_error().
void set_error(const char* fmt, ...);

#define MGK_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess) {                                                        \
      ::mgk::set_error("%s:%d %s -> %s", __FILE__, __LINE__, #call,                 \
                       cudaGetErrorString(_e));                                     \
      return (_e == cudaErrorMemoryAllocation) ? MGK_OOM : MGK_CUDA_ERROR;          \
    }                                                                               \
  } while (0)

#define MGK_REQUIRE(cond, ...)                                                      \
  do {                                                                              \
    if (!(cond)) {                                                                  \
      ::mgk::set_error(__VA_ARGS__);                                                \
      return MGK_BAD_ARG;                                                           \
    }                                                                               \
  } while (0)

// ---------------------------------------------------------------- complex ---
template <typename T> struct cpx;
template <> struct cpx<double> { using t = double2; };
template <> struct cpx<float> { using t = float2; };
template <typename T> using C_t = typename cpx<T>::t;

template <typename C> __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C r; r.x = a; r.y = b; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
// multiply by SIGN*i  (SIGN = -1: forward DFT kernel, +1: inverse)
template <int SIGN, typename C> __device__ __forceinline__ C cmul_i(C a) {
  return SIGN < 0 ? mk<C>(a.y, -a.x) : mk<C>(-a.y, a.x);
}

// ------------------------------------------------------ block reductions ---
// Deterministic: fixed tree over warps, result valid in thread 0.
template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <typename T> __device__ T block_sum(T v, T* red /* >= 32 entries */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  T r = 0;
  if (wid == 0) {
    r = lane < nw ? red[lane] : T(0);
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes` (never lowers it: plans of different sizes share kernels).
cudaError_t raise_smem(const void* fn, size_t bytes);

}  // namespace mgk
