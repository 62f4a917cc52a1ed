// Shared helpers of libigmb200: status handling, error text, reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/igm_b200.h"

namespace igm {

// Records a formatted message for igm_last_error() on this host thread.
void set_error(const char* fmt, ...);

#define IGM_CHECK_ARG(cond, code, ...)      \
  do {                                      \
    if (!(cond)) {                          \
      ::igm::set_error(__VA_ARGS__);        \
      return (code);                        \
    }                                       \
  } while (0)

// Counts kernel launches (igm_launch_count) and returns IGM_ERR_CUDA with the
// error text when the last launch failed.  Called after every launch.
void note_launch();
inline int launch_status(const char* what) {
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return IGM_ERR_CUDA;
  }
  return IGM_OK;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Deterministic block sum of a double (fixed tree; result valid in the thread
// with linear id 0).  `tid` is the linear thread index in the block.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh, int tid) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = tid & 31, warp = tid >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (tid == 0) {
    for (int w = 0; w < NT / 32; ++w) r += sh[w];
  }
  return r;
}

// Atomic max of a non-negative float through its bit pattern (non-negative
// IEEE floats order like their unsigned integer images).
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
  atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}

template <typename T> struct Math;
template <> struct Math<float> {
  static __device__ __forceinline__ float rcbrt(float x) { return rcbrtf(x); }
  static __device__ __forceinline__ float cbrt(float x) { return cbrtf(x); }
  static __device__ __forceinline__ float pow(float x, float y) { return powf(x, y); }
  static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
};
template <> struct Math<double> {
  static __device__ __forceinline__ double rcbrt(double x) { return ::rcbrt(x); }
  static __device__ __forceinline__ double cbrt(double x) { return ::cbrt(x); }
  static __device__ __forceinline__ double pow(double x, double y) { return ::pow(x, y); }
  static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
};

}  // namespace igm
