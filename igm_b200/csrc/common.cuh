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

// Programmatic dependent launch along the emulator's kernel chain: a kernel
// launched by launch_pdl may start (launch, shared-memory and barrier setup)
// once every CTA of the previous kernel in the stream has called
// grid_dep_launch(); it calls grid_dep_wait() -- which returns when that grid
// has completed and its writes are visible -- before it touches global memory
// or allocates tensor memory.  Every kernel launched by launch_pdl must call
// grid_dep_wait() first; for a kernel launched plainly both are no-ops.
// Only the persistent tensor-core convolutions trigger early (one CTA per SM,
// so a following convolution's CTAs take each SM as it frees); the small
// kernels only wait, because dependents launched at their start would sit on
// the SMs they still need (measured: the 16-layer forward 0.54 ms with the
// convolutions triggering, 0.60 ms with every kernel triggering, 0.57 ms
// without programmatic launches).
#ifndef IGM_PDL
#define IGM_PDL 1
#endif

__device__ __forceinline__ void grid_dep_wait() {
#if IGM_PDL
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
#endif
}
__device__ __forceinline__ void grid_dep_launch() {
#if IGM_PDL
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
#endif
}

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = IGM_PDL ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...);
}

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
