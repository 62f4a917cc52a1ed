// Fixed-order reductions of per-CTA partial sums, shared by the finishing kernels
// (csrc/cnn.cu) and the fused backward convolution (csrc/conv.cu), so both sum
// the same partials in the same order (deterministic, and the same bits).
#pragma once

#include <cuda_runtime.h>

namespace igm {

constexpr int kFinCols = 32;  // output channels of a finished weight-gradient row
constexpr int kFinWarps = 8;  // warps of the fixed-order partial-sum kernels
constexpr int kRedBatch = 8;  // partials whose loads a lane issues before adding them

// fixed xor-shuffle tree over the 32 lanes: the same order on every run, the
// total in every lane
__device__ __forceinline__ float warp_sum_fixed(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the partials p = warp, warp + kFinWarps, ... of the entries (kh + jj,
// jj) of one (kw, ci) accumulator row of a weight-gradient partial
// [n_parts][kw][128][JN * 32] (lane = output channel); NSP adjacent input
// channels summed (the first layer's split input).  kRedBatch partials are
// loaded before they are added (absent ones add +0).
template <int JN, int NSP>
__device__ __forceinline__ float finish_sum(const float* part, int n_parts, int warp, int lane, int kw, int kh,
                                            int ci, int cw) {
  constexpr int wn = JN * kFinCols;
  float acc = 0.f;
  for (int p0 = warp; p0 < n_parts; p0 += kFinWarps * kRedBatch) {
    float v[kRedBatch][JN][NSP];
#pragma unroll
    for (int u = 0; u < kRedBatch; ++u) {
      const int p = p0 + u * kFinWarps;
      const float* base = part + ((size_t)(p < n_parts ? p : 0) * 3 + kw) * 128 * wn;
#pragma unroll
      for (int jj = 0; jj < JN; ++jj)
#pragma unroll
        for (int sp = 0; sp < NSP; ++sp)
          v[u][jj][sp] = p < n_parts ? base[(size_t)((kh + jj) * cw + ci + sp) * wn + jj * kFinCols + lane] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kRedBatch; ++u)
#pragma unroll
      for (int jj = 0; jj < JN; ++jj)
#pragma unroll
        for (int sp = 0; sp < NSP; ++sp) acc += v[u][jj][sp];
  }
  return acc;
}

// One warp's sum of out-element i of partials [n_parts][stride]: lane l adds the
// partials l, l + 32, ... in order (kRedBatch loads issued first), then the
// fixed tree; the total in every lane.
__device__ __forceinline__ float partial_sum(const float* part, int n_parts, int stride, int i, int lane) {
  float s = 0.f;
  for (int p0 = lane; p0 < n_parts; p0 += 32 * kRedBatch) {
    float v[kRedBatch];
#pragma unroll
    for (int u = 0; u < kRedBatch; ++u) {
      const int p = p0 + 32 * u;
      v[u] = p < n_parts ? part[(size_t)p * stride + i] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kRedBatch; ++u) s += v[u];
  }
  return warp_sum_fixed(s);
}

}  // namespace igm
