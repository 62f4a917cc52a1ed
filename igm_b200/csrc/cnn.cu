// CUDA-core kernels around the tensor-core convolutions of the CNN emulator:
// input windows, the 1x1 output head (forward and backward), weight packing
// for the UMMA B operands, deterministic partial-sum reductions, the mapping
// of the weight-gradient accumulators to the Keras kernel layout, and the
// Keras-legacy Adam update with per-variable clip-by-norm.
//
// Reference: igm/processes/iceflow/emulate/neural_network.py:9-66 (network),
// igm/processes/iceflow/utils.py:133-158 (fieldin_to_X / Y_to_UV layouts),
// emulate.py:116-152 (inference + mask), emulate.py:22-35 and :267 (Adam,
// epsilon, clipnorm), emulate.py:283-308 (patches).
//
// Parameter vector (fp32, Keras order): for each 3x3 layer l: kernel
// [3][3][cin_l][32] then bias [32]; then the head kernel [1][1][32][nout] and
// bias [nout].  cin_0 = the number of input fields (5), cin_l = 32 after.
#include <cuda_bf16.h>

#include "common.cuh"
#include "reduce.cuh"

namespace igm {

constexpr int kF = 32;  // filters
static_assert(kF == kFinCols, "the finishing reductions sum 32-channel rows");

__device__ __forceinline__ float bf_lo(uint32_t w) {
  return __low2float(*reinterpret_cast<const __nv_bfloat162*>(&w));
}
__device__ __forceinline__ float bf_hi(uint32_t w) {
  return __high2float(*reinterpret_cast<const __nv_bfloat162*>(&w));
}
__device__ __forceinline__ uint32_t bf_pack(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

// offsets (in floats) of the parameters of layer l (0-based; l == L is the head)
__host__ __device__ inline size_t w_offset(int l, int cin0, int nout) {
  (void)nout;
  if (l == 0) return 0;
  const size_t l0 = (size_t)9 * cin0 * kF + kF;
  const size_t li = (size_t)9 * kF * kF + kF;
  return l0 + (size_t)(l - 1) * li;
}
__host__ __device__ inline size_t b_offset(int l, int cin0, int nout, int L) {
  if (l < L) return w_offset(l, cin0, nout) + (size_t)9 * (l == 0 ? cin0 : kF) * kF;
  return w_offset(L, cin0, nout) + (size_t)kF * nout;
}
__host__ __device__ inline size_t param_count(int L, int cin0, int nout) {
  return w_offset(L, cin0, nout) + (size_t)kF * nout + nout;
}

// ---------------------------------------------------------------------------
// weight packing: fp32 Keras layout -> bf16 UMMA B operands, ordered so that
// for one (kw, 8-channel k-chunk) the three kernel rows follow each other:
//  forward  layer l: [kw][k-chunk (ci)][kh][co][8]   (layer 0: 2 k-chunks over the split
//           input channels 3c + {0, 1, 2} of field c: W_h, W_h, W_l; zero for c >= cin0)
//  dgrad    layer l>=1: [kw'][k-chunk (co)][kh'][ci][8], flipped: kh' = 2 - kh, kw' = 2 - kw
// ---------------------------------------------------------------------------
__global__ void pack_kernel(const float* params, int L, int cin0, int nout, __nv_bfloat16* wf, __nv_bfloat16* wb) {
  grid_dep_wait();
  const size_t n0 = (size_t)9 * 2 * kF * 8;   // layer 0, forward
  const size_t ni = (size_t)9 * 4 * kF * 8;   // other layers, per pack
  const size_t total_f = n0 + (size_t)(L - 1) * ni;
  const size_t total = total_f + (size_t)(L - 1) * ni;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    if (i < total_f) {
      int l, rem;
      int c8;
      if (i < n0) { l = 0; rem = (int)i; c8 = 2; }
      else { l = 1 + (int)((i - n0) / ni); rem = (int)((i - n0) % ni); c8 = 4; }
      const int e = rem % 8, co = (rem / 8) % kF, kh = (rem / (8 * kF)) % 3, kc = (rem / (24 * kF)) % c8,
                kw = rem / (24 * kF * c8);
      const int ci = kc * 8 + e;
      float v = 0.f;
      if (l == 0) {
        // layer 0 reads the split input (x_h, x_l, x_h per field): weights W_h, W_h, W_l with
        // W_h = bf16(W), W_l = bf16(W - W_h), so that x W ~ x_h W_h + x_l W_h + x_h W_l
        const int c = ci / 3, part = ci - 3 * c;
        if (c < cin0) {
          const float w = params[w_offset(0, cin0, nout) + (((size_t)kh * 3 + kw) * cin0 + c) * kF + co];
          const float wh = __bfloat162float(__float2bfloat16_rn(w));
          v = part == 2 ? w - wh : wh;
        }
      } else {
        v = params[w_offset(l, cin0, nout) + (((size_t)kh * 3 + kw) * kF + ci) * kF + co];
      }
      wf[i] = __float2bfloat16_rn(v);
    } else {
      const size_t j = i - total_f;
      const int l = 1 + (int)(j / ni);
      const int rem = (int)(j % ni);
      const int e = rem % 8, ci = (rem / 8) % kF, khp = (rem / (8 * kF)) % 3, kc = (rem / (24 * kF)) % 4,
                kwp = rem / (24 * kF * 4);
      const int co = kc * 8 + e;
      const int kh = 2 - khp, kw = 2 - kwp;
      const float v = params[w_offset(l, cin0, nout) + (((size_t)kh * 3 + kw) * kF + ci) * kF + co];
      wb[j] = __float2bfloat16_rn(v);
    }
  }
}

// ---------------------------------------------------------------------------
// input windows: fields [Ny][Nx] -> X bf16 [B][h][2][w][8] (channels thk, usurf,
// arrhenius, slidingco, dX, scaled; zero above) and optional fp32 copies of
// the windowed fields [B][h][w] for the energy
// ---------------------------------------------------------------------------
struct InputArgs {
  int B, h, w, Ny, Nx;
  const float* f[4];
  float dx;
  float scale[5];
  int y0[IGM_MAX_WINDOWS], x0[IGM_MAX_WINDOWS];
  __nv_bfloat16* X;
  float* out[4];
};

__global__ void input_kernel(const InputArgs a) {
  grid_dep_wait();
  const size_t plane = (size_t)a.h * a.w;
  const size_t total = plane * a.B;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / plane);
    const int rem = (int)(i - (size_t)b * plane);
    const int y = rem / a.w, x = rem - (rem / a.w) * a.w;
    const size_t src = (size_t)(a.y0[b] + y) * a.Nx + (a.x0[b] + x);
    float v[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      v[c] = a.f[c][src];
      if (a.out[c]) a.out[c][i] = v[c];
    }
    if (a.X) {
      // each scaled field x as three BF16 channels (x_h, x_l, x_h) with x_h = bf16(x),
      // x_l = bf16(x - x_h); channel 15 is zero
      float ch[16];
      const float xs[5] = {v[0] * a.scale[0], v[1] * a.scale[1], v[2] * a.scale[2], v[3] * a.scale[3],
                           a.dx * a.scale[4]};
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const float hi = __bfloat162float(__float2bfloat16_rn(xs[c]));
        ch[3 * c] = hi;
        ch[3 * c + 1] = xs[c] - hi;
        ch[3 * c + 2] = hi;
      }
      ch[15] = 0.f;
      uint4 c0, c1;
      c0.x = bf_pack(ch[0], ch[1]);
      c0.y = bf_pack(ch[2], ch[3]);
      c0.z = bf_pack(ch[4], ch[5]);
      c0.w = bf_pack(ch[6], ch[7]);
      c1.x = bf_pack(ch[8], ch[9]);
      c1.y = bf_pack(ch[10], ch[11]);
      c1.z = bf_pack(ch[12], ch[13]);
      c1.w = bf_pack(ch[14], ch[15]);
      uint4* X = reinterpret_cast<uint4*>(a.X);
      const size_t row = ((size_t)b * a.h + y) * 2;
      X[(row + 0) * a.w + x] = c0;
      X[(row + 1) * a.w + x] = c1;
    }
  }
}

// ---------------------------------------------------------------------------
// head forward: Y = A16 Wh + bh, written as planar U [B][Nz][H][W], V [B][Nz][H][W]
// (Y_to_UV: channels [0,Nz) are U, [Nz, 2Nz) are V), masked where thk <= 0
// ---------------------------------------------------------------------------
// Two output channels per packed FP32x2 fma (the weights read as float4 rows,
// the activation broadcast); each output accumulates over ci in order, as one
// scalar fma chain would.  NJ >= 2 nz, multiple of 4 (padded weight rows).
template <int NJ>
__global__ void __launch_bounds__(256) head_fwd_kernel(int B, int H, int W, int nz, const __nv_bfloat16* act,
                                                       const float* wh, const float* bh, float out_scale, float* U,
                                                       float* V, const float* thk_mask) {
  grid_dep_wait();
  static_assert(NJ % 4 == 0, "NJ");
  __shared__ __align__(16) float sw[kF * NJ + NJ];  // [32][NJ] then bias [NJ]
  const int nout = 2 * nz;
  for (int i = threadIdx.x; i < kF * NJ; i += blockDim.x) {
    const int ci = i / NJ, j = i - (i / NJ) * NJ;
    sw[i] = j < nout ? wh[ci * nout + j] : 0.f;
  }
  for (int i = threadIdx.x; i < NJ; i += blockDim.x) sw[kF * NJ + i] = i < nout ? bh[i] : 0.f;
  __syncthreads();
  const size_t plane = (size_t)H * W;
  const size_t total = plane * B;
  const uint4* A = reinterpret_cast<const uint4*>(act);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    // keeps the weight reads inside the loop: hoisted, they would stay live in registers
    asm volatile("" ::: "memory");
    const size_t b = i / plane;
    const size_t rem = i - b * plane;
    const size_t y = rem / W, x = rem - y * W;
    // every load of the pixel (activation and ice mask) is issued before the arithmetic
    uint4 u[4];
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) u[ch] = A[((b * H + y) * 4 + ch) * W + x];
    const float mk = thk_mask != nullptr ? thk_mask[i] : 1.f;
    float2 acc[NJ / 2];
#pragma unroll
    for (int q = 0; q < NJ / 2; ++q) acc[q] = make_float2(0.f, 0.f);
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      const uint32_t wv[4] = {u[ch].x, u[ch].y, u[ch].z, u[ch].w};
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int ci = ch * 8 + e;
        const float av = (e & 1) ? bf_hi(wv[e >> 1]) : bf_lo(wv[e >> 1]);
        const float2 aa = make_float2(av, av);
        const float4* wr = reinterpret_cast<const float4*>(sw + ci * NJ);
#pragma unroll
        for (int q = 0; q < NJ / 4; ++q) {
          const float4 w4 = wr[q];
          acc[2 * q] = __ffma2_rn(aa, make_float2(w4.x, w4.y), acc[2 * q]);
          acc[2 * q + 1] = __ffma2_rn(aa, make_float2(w4.z, w4.w), acc[2 * q + 1]);
        }
      }
    }
    const bool keep = mk > 0.f;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      if (j >= nout) break;
      const float sacc = (j & 1) ? acc[j >> 1].y : acc[j >> 1].x;
      float sv = (sacc + sw[kF * NJ + j]) * out_scale;
      if (!keep) sv = 0.f;
      float* dst = j < nz ? U : V;
      const int k = j < nz ? j : j - nz;
      dst[(b * nz + k) * plane + rem] = sv;
    }
  }
}

// ---------------------------------------------------------------------------
// head backward: from dU, dV (planar) and A16:
//   dPre16 = (dY Wh^T) * LeakyReLU'(A16)  (bf16, row-chunked),
//   partials per block of dWh [32][nout], dbh [nout] and db16 [32].
// ---------------------------------------------------------------------------
// Work split: a warp takes 32 consecutive pixels; each lane loads its pixel,
// computes that pixel's dPre16 and stages the operands in the warp's shared
// memory; then lane l owns input channel ci = l and accumulates the outer
// products over the 32 pixels (dWh[l][:], db16[l]) from broadcast reads --
// no block barrier inside the pixel loop.  Warps are summed in a fixed order
// at the end (deterministic).  NJ >= nout is the per-lane accumulator count.
constexpr int kHeadWarps = 8;
template <int NJ>
struct HeadBwdSmem {
  static constexpr int GS = NJ + 4;                     // output-gradient row stride (16-byte aligned rows)
  static constexpr int WARP = 32 * 33 * 2 + 32 * GS;    // per warp: activations, masked dPre, gradients
  static constexpr int RED = kF * NJ + NJ + kF;         // per-warp results for the final sum
  static constexpr int FLOATS = NJ * kF + kHeadWarps * (WARP > RED ? WARP : RED);
};
template <int NJ>
__global__ void __launch_bounds__(kHeadWarps * 32, 2)
    head_bwd_kernel(int B, int H, int W, int nz, const __nv_bfloat16* act, const float* wh, const float* dU,
                    const float* dV, float out_scale, float alpha, __nv_bfloat16* dpre, float* partial) {
  grid_dep_wait();
  using SM_ = HeadBwdSmem<NJ>;
  constexpr int GS = SM_::GS;
  extern __shared__ __align__(16) float sm[];
  const int nout = 2 * nz;
  float* swT = sm;  // [NJ][32]: swT[j][ci] = Wh[ci][j]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* wbase = sm + NJ * kF + warp * (SM_::WARP > SM_::RED ? SM_::WARP : SM_::RED);
  float* sA = wbase;            // [32 pixels][33]
  float* sP = sA + 32 * 33;     // [32 pixels][33]
  float* sG = sP + 32 * 33;     // [32 pixels][GS]
  for (int i = threadIdx.x; i < NJ * kF; i += blockDim.x) {
    const int j = i / kF, ci = i - (i / kF) * kF;
    swT[i] = j < nout ? wh[ci * nout + j] : 0.f;
  }
  __syncthreads();
  float accw[NJ];
#pragma unroll
  for (int j = 0; j < NJ; ++j) accw[j] = 0.f;
  float accb[NJ / 32];
#pragma unroll
  for (int q = 0; q < NJ / 32; ++q) accb[q] = 0.f;
  float accd = 0.f;
  const size_t plane = (size_t)H * W;
  const size_t total = plane * B;
  const size_t nchunks = (total + 31) / 32;
  const size_t nw = (size_t)gridDim.x * kHeadWarps;
  const uint4* A = reinterpret_cast<const uint4*>(act);
  uint4* DP = reinterpret_cast<uint4*>(dpre);
  for (size_t chunk = (size_t)blockIdx.x * kHeadWarps + warp; chunk < nchunks; chunk += nw) {
    const size_t i = chunk * 32 + lane;
    const bool ok = i < total;
    int b = 0, y = 0, x = 0;
    size_t rem = 0;
    if (ok) {
      b = (int)(i / plane);
      rem = i - (size_t)b * plane;
      y = (int)(rem / W);
      x = (int)(rem - (size_t)y * W);
    }
    // this lane's pixel: activations into its sA row, output gradients into g and its sG row
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      uint4 u = make_uint4(0, 0, 0, 0);
      if (ok) u = A[(((size_t)b * H + y) * 4 + ch) * W + x];
      const uint32_t wv[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        sA[lane * 33 + ch * 8 + 2 * e] = bf_lo(wv[e]);
        sA[lane * 33 + ch * 8 + 2 * e + 1] = bf_hi(wv[e]);
      }
    }
    float g[NJ];
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      float v = 0.f;
      if (ok && j < nout) {
        const float* src = j < nz ? dU : dV;
        const int k = j < nz ? j : j - nz;
        v = src[((size_t)b * nz + k) * plane + rem] * out_scale;
      }
      g[j] = v;
      sG[lane * GS + j] = v;
    }
    // dPre16 = (dY Wh^T) * LeakyReLU'(A16)
    float da[kF];
#pragma unroll
    for (int ci = 0; ci < kF; ++ci) da[ci] = 0.f;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      if (j >= nout) break;
      const float4* wr = reinterpret_cast<const float4*>(swT + j * kF);
#pragma unroll
      for (int q = 0; q < kF / 4; ++q) {
        const float4 w4 = wr[q];
        da[4 * q + 0] = fmaf(g[j], w4.x, da[4 * q + 0]);
        da[4 * q + 1] = fmaf(g[j], w4.y, da[4 * q + 1]);
        da[4 * q + 2] = fmaf(g[j], w4.z, da[4 * q + 2]);
        da[4 * q + 3] = fmaf(g[j], w4.w, da[4 * q + 3]);
      }
    }
#pragma unroll
    for (int ci = 0; ci < kF; ++ci) {
      da[ci] *= sA[lane * 33 + ci] > 0.f ? 1.f : alpha;
      sP[lane * 33 + ci] = da[ci];
    }
    if (ok) {
#pragma unroll
      for (int ch = 0; ch < 4; ++ch) {
        uint4 o;
        o.x = bf_pack(da[ch * 8 + 0], da[ch * 8 + 1]);
        o.y = bf_pack(da[ch * 8 + 2], da[ch * 8 + 3]);
        o.z = bf_pack(da[ch * 8 + 4], da[ch * 8 + 5]);
        o.w = bf_pack(da[ch * 8 + 6], da[ch * 8 + 7]);
        DP[(((size_t)b * H + y) * 4 + ch) * W + x] = o;
      }
    }
    __syncwarp();
    // lane = input channel: outer products over the warp's 32 pixels
    for (int p = 0; p < 32; ++p) {
      const float av = sA[p * 33 + lane];
      accd += sP[p * 33 + lane];
      const float4* gr = reinterpret_cast<const float4*>(sG + p * GS);
#pragma unroll
      for (int q = 0; q < NJ / 4; ++q) {
        if (4 * q >= nout) break;
        const float4 g4 = gr[q];
        accw[4 * q + 0] = fmaf(av, g4.x, accw[4 * q + 0]);
        accw[4 * q + 1] = fmaf(av, g4.y, accw[4 * q + 1]);
        accw[4 * q + 2] = fmaf(av, g4.z, accw[4 * q + 2]);
        accw[4 * q + 3] = fmaf(av, g4.w, accw[4 * q + 3]);
      }
#pragma unroll
      for (int q = 0; q < NJ / 32; ++q) accb[q] += sG[p * GS + lane + 32 * q];
    }
    __syncwarp();  // this warp's staging area is rewritten by its next chunk
  }
  // per-warp results, then the fixed-order sum over the block's warps
  __syncthreads();
  float* red = wbase;  // [32 * NJ] dWh, [NJ] dbh, [32] db16
#pragma unroll
  for (int j = 0; j < NJ; ++j) red[lane * NJ + j] = accw[j];
#pragma unroll
  for (int q = 0; q < NJ / 32; ++q) red[kF * NJ + lane + 32 * q] = accb[q];
  red[kF * NJ + NJ + lane] = accd;
  __syncthreads();
  const int stride = SM_::WARP > SM_::RED ? SM_::WARP : SM_::RED;
  const int npairs = kF * nout;
  float* out = partial + (size_t)blockIdx.x * (npairs + nout + kF);
  const float* r0 = sm + NJ * kF;
  for (int o = threadIdx.x; o < npairs + nout + kF; o += blockDim.x) {
    int src;
    if (o < npairs) {
      const int ci = o / nout, j = o - (o / nout) * nout;
      src = ci * NJ + j;
    } else if (o < npairs + nout) {
      src = kF * NJ + (o - npairs);
    } else {
      src = kF * NJ + NJ + (o - npairs - nout);
    }
    float s = 0.f;
    for (int w2 = 0; w2 < kHeadWarps; ++w2) s += r0[w2 * stride + src];
    out[o] = s;
  }
}

// ---------------------------------------------------------------------------
// head backward for up to 32 outputs, pixel part: dPre16 = (dY Wh^T) *
// LeakyReLU'(A16) and dY itself as a row-chunked bf16 [B][H][4][W][8] tensor
// (outputs beyond 2 Nz zero), from which the tensor-core weight-gradient kernel
// forms dWh = A16^T dY (its centre tap, igm_cnn_head_wgrad_finish).  A warp
// takes 32 consecutive pixels per chunk (lane = pixel).  Each lane keeps its
// own running sums of dY (dbh) and dPre16 (db16) in registers; at the end fixed
// xor trees add the lanes and the warps are added in a fixed order, giving the
// per-CTA partials [dbh (2 Nz)][db16 (32)] (deterministic).  NJ = 2 Nz rounded
// up to a multiple of 4.
// ---------------------------------------------------------------------------
constexpr int kHpWarps = 8;

template <int NJ>
struct HeadPx {
  uint4 a[4];   // A16 of the pixel, 32 bf16 channels
  float g[NJ];  // dY of the pixel (output_scale applied), 0 beyond 2 Nz
  bool ok;
  size_t o;     // uint4 index of channel chunk 0 of the pixel
};

// The loads are unconditional (lanes past the end and outputs past 2 Nz read a
// valid element and select 0), so the compiler issues all of them back to back.
template <int NJ>
__device__ __forceinline__ void head_px_load(HeadPx<NJ>& q, size_t chunk, size_t total, size_t plane, int H, int W,
                                             int nz, int nout, const uint4* A, const float* dU, const float* dV,
                                             float out_scale, int lane) {
  const size_t i = chunk * 32 + lane;
  q.ok = i < total;
  const size_t ic = q.ok ? i : 0;
  const size_t b = ic / plane;
  const size_t rem = ic - b * plane;
  const size_t y = rem / W;
  const size_t x = rem - y * W;
  q.o = ((b * H + y) * 4) * W + x;
#pragma unroll
  for (int ch = 0; ch < 4; ++ch) {
    const uint4 v = A[q.o + (size_t)ch * W];
    q.a[ch] = q.ok ? v : make_uint4(0, 0, 0, 0);
  }
  const float* pu = dU + b * nz * plane + rem;
  const float* pv = dV + b * nz * plane + rem;
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int k = j < nz ? j : min(j - nz, nz - 1);
    const float v = (j < nz ? pu : pv)[(size_t)k * plane];
    q.g[j] = (q.ok && j < nout) ? v * out_scale : 0.f;
  }
}

template <int NJ, bool PARAMS>
__global__ void __launch_bounds__(kHpWarps * 32, 2)
    head_bwd_px_kernel(int B, int H, int W, int nz, const __nv_bfloat16* act, const float* wh, const float* dU,
                       const float* dV, float out_scale, float alpha, __nv_bfloat16* dpre, __nv_bfloat16* dyb,
                       float* partial) {
  grid_dep_wait();
  static_assert(NJ % 4 == 0 && NJ <= kF, "NJ");
  __shared__ __align__(16) float swT[NJ * kF];  // [j][ci] = Wh[ci][j], 0 for j >= 2 nz
  __shared__ float red[kHpWarps][NJ + kF];
  const int nout = 2 * nz;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < NJ * kF; i += blockDim.x) {
    const int j = i / kF, ci = i - (i / kF) * kF;
    swT[i] = j < nout ? wh[ci * nout + j] : 0.f;
  }
  __syncthreads();
  // this lane's sums of dY (j) and dPre16 (ci) for the parameter gradients, channel pairs
  float2 accb[PARAMS ? NJ / 2 : 1], accd[PARAMS ? kF / 2 : 1];
#pragma unroll
  for (int q = 0; q < (PARAMS ? NJ / 2 : 1); ++q) accb[q] = make_float2(0.f, 0.f);
#pragma unroll
  for (int q = 0; q < (PARAMS ? kF / 2 : 1); ++q) accd[q] = make_float2(0.f, 0.f);
  const size_t plane = (size_t)H * W;
  const size_t total = plane * B;
  const size_t nchunks = (total + 31) / 32;
  const size_t nwarps = (size_t)gridDim.x * kHpWarps;
  const uint4* A = reinterpret_cast<const uint4*>(act);
  uint4* DP = reinterpret_cast<uint4*>(dpre);
  uint4* DY = reinterpret_cast<uint4*>(dyb);
  for (size_t chunk = (size_t)blockIdx.x * kHpWarps + warp; chunk < nchunks; chunk += nwarps) {
    // keeps the weight reads below inside the loop: hoisted, 32 NJ of them would stay live in registers
    asm volatile("" ::: "memory");
    HeadPx<NJ> cur;
    head_px_load<NJ>(cur, chunk, total, plane, H, W, nz, nout, A, dU, dV, out_scale, lane);
    if (PARAMS) {
#pragma unroll
      for (int q = 0; q < NJ / 2; ++q)
        accb[q] = __fadd2_rn(accb[q], make_float2(cur.g[2 * q], cur.g[2 * q + 1]));
    }
    // dPre = dY Wh^T, two channels per packed fma, in two halves of the input channels (16 each)
    // so that only half of the sums are live at once
#pragma unroll
    for (int hf = 0; hf < 2; ++hf) {
      float2 da[kF / 4];
#pragma unroll
      for (int q = 0; q < kF / 4; ++q) da[q] = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const float2 gg = make_float2(cur.g[j], cur.g[j]);
        const float4* wr = reinterpret_cast<const float4*>(swT + j * kF + hf * (kF / 2));
#pragma unroll
        for (int q = 0; q < kF / 8; ++q) {
          const float4 w4 = wr[q];
          da[2 * q] = __ffma2_rn(gg, make_float2(w4.x, w4.y), da[2 * q]);
          da[2 * q + 1] = __ffma2_rn(gg, make_float2(w4.z, w4.w), da[2 * q + 1]);
        }
      }
#pragma unroll
      for (int cc = 0; cc < 2; ++cc) {
        const int ch = 2 * hf + cc;  // 8-channel chunk
        const uint32_t wv[4] = {cur.a[ch].x, cur.a[ch].y, cur.a[ch].z, cur.a[ch].w};
        uint32_t pk[4], yk[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int c = ch * 8 + 2 * e;
          const float2 m = make_float2(bf_lo(wv[e]) > 0.f ? 1.f : alpha, bf_hi(wv[e]) > 0.f ? 1.f : alpha);
          const float2 d = __fmul2_rn(da[(c - hf * (kF / 2)) >> 1], m);
          if (PARAMS) accd[c >> 1] = __fadd2_rn(accd[c >> 1], d);
          pk[e] = bf_pack(d.x, d.y);
          yk[e] = c < NJ ? bf_pack(cur.g[c], cur.g[c + 1]) : 0u;
        }
        if (cur.ok) {
          DP[cur.o + (size_t)ch * W] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          if (PARAMS) DY[cur.o + (size_t)ch * W] = make_uint4(yk[0], yk[1], yk[2], yk[3]);
        }
      }
    }
  }
  if (!PARAMS) return;  // uniform: no partials in the data-only variant
#pragma unroll
  for (int q = 0; q < NJ / 2; ++q) {
    const float x0 = warp_sum_fixed(accb[q].x), x1 = warp_sum_fixed(accb[q].y);
    if (lane == 0) {
      red[warp][2 * q] = x0;
      red[warp][2 * q + 1] = x1;
    }
  }
#pragma unroll
  for (int q = 0; q < kF / 2; ++q) {
    const float x0 = warp_sum_fixed(accd[q].x), x1 = warp_sum_fixed(accd[q].y);
    if (lane == 0) {
      red[warp][NJ + 2 * q] = x0;
      red[warp][NJ + 2 * q + 1] = x1;
    }
  }
  __syncthreads();
  float* out = partial + (size_t)blockIdx.x * (nout + kF);
  const int t = threadIdx.x;
  if (t < nout + kF) {
    const int src = t < nout ? t : NJ + (t - nout);
    float v = 0.f;
#pragma unroll
    for (int w2 = 0; w2 < kHpWarps; ++w2) v += red[w2][src];
    out[t] = v;
  }
}

// head kernel gradient from igm_conv3x3_wgrad partials over (A16, dY): the centre
// tap (kh = kw = 1), i.e. accumulator entries (r, jj) with r - jj = 1, kw = 1.
__global__ void __launch_bounds__(kFinWarps * 32) head_wgrad_finish_kernel(const float* part, int n_parts, int nout,
                                                                           float* out) {
  grid_dep_wait();
  __shared__ float red[kFinWarps][kF];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int cw = 32, jn = 2;
  for (int ci = blockIdx.x; ci < kF; ci += gridDim.x) {
    red[warp][lane] = finish_sum<jn, 1>(part, n_parts, warp, lane, 1, 1, ci, cw);
    __syncthreads();
    if (warp == 0) {
      float tsum = 0.f;
#pragma unroll
      for (int w2 = 0; w2 < kFinWarps; ++w2) tsum += red[w2][lane];
      if (lane < nout) out[(size_t)ci * nout + lane] = tsum;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// First layer in FP32 on CUDA cores: the raw fields (surface elevation of
// ~3000 m varying by a few metres per cell) cannot be rounded to BF16 without
// losing the surface slope that drives the flow, so the 5 -> 32 layer reads
// the FP32 fields and writes BF16 activations.  Input channels in fieldin
// order: thk, usurf, arrhenius, slidingco (windowed copies [B][H][W]) and the
// constant dX channel; zero outside the window ("same" padding of X).
// ---------------------------------------------------------------------------
struct L1Args {
  int B, H, W, cin;
  const float* f[4];
  float dxs;        // dx * scale of the dX channel
  float scale[4];   // fixed input scales
  const float* w;   // [3][3][cin][32]
  const float* b;   // [32]
  float alpha;
  __nv_bfloat16* out;  // [B][H][4][W][8]
};

__device__ __forceinline__ void l1_inputs(const L1Args& a, int b, int y, int x, float (&in)[9][5]) {
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
    const bool ok = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
    const size_t o = ((size_t)b * a.H + (ok ? yy : 0)) * a.W + (ok ? xx : 0);
#pragma unroll
    for (int c = 0; c < 4; ++c) in[t][c] = ok ? a.f[c][o] * a.scale[c] : 0.f;
    in[t][4] = ok ? a.dxs : 0.f;
  }
}

__global__ void __launch_bounds__(256) layer1_fwd_kernel(const L1Args a) {
  grid_dep_wait();
  __shared__ __align__(16) float sw[9 * 5 * kF + kF];
  for (int i = threadIdx.x; i < 9 * a.cin * kF; i += blockDim.x) sw[i] = a.w[i];
  if (threadIdx.x < kF) sw[9 * 5 * kF + threadIdx.x] = a.b[threadIdx.x];
  __syncthreads();
  const size_t plane = (size_t)a.H * a.W;
  const size_t total = plane * a.B;
  uint4* O = reinterpret_cast<uint4*>(a.out);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / plane);
    const size_t rem = i - (size_t)b * plane;
    const int y = (int)(rem / a.W), x = (int)(rem - (size_t)y * a.W);
    float in[9][5];
    l1_inputs(a, b, y, x, in);
    // two output channels per packed FP32x2 fma; each channel accumulates in (tap, c) order
    float2 acc[kF / 2];
#pragma unroll
    for (int q = 0; q < kF / 2; ++q) acc[q] = make_float2(sw[9 * 5 * kF + 2 * q], sw[9 * 5 * kF + 2 * q + 1]);
#pragma unroll
    for (int t = 0; t < 9; ++t)
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        if (c >= a.cin) break;
        const float2 vv = make_float2(in[t][c], in[t][c]);
        const float4* wr = reinterpret_cast<const float4*>(&sw[(t * a.cin + c) * kF]);
#pragma unroll
        for (int q = 0; q < kF / 4; ++q) {
          const float4 w4 = wr[q];
          acc[2 * q] = __ffma2_rn(vv, make_float2(w4.x, w4.y), acc[2 * q]);
          acc[2 * q + 1] = __ffma2_rn(vv, make_float2(w4.z, w4.w), acc[2 * q + 1]);
        }
      }
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      float z[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int co = ch * 8 + e;
        const float v = (co & 1) ? acc[co >> 1].y : acc[co >> 1].x;
        z[e] = v > 0.f ? v : a.alpha * v;
      }
      uint4 o;
      o.x = bf_pack(z[0], z[1]);
      o.y = bf_pack(z[2], z[3]);
      o.z = bf_pack(z[4], z[5]);
      o.w = bf_pack(z[6], z[7]);
      O[(((size_t)b * a.H + y) * 4 + ch) * a.W + x] = o;
    }
  }
}

// dW1[t][c][co] = sum_p X[p + off(t)][c] * G[p][co], per-block partials [9*cin*32].
// A warp takes 32 consecutive pixels: each lane stages its pixel's 3x3x5
// input window and its 32 output gradients in the warp's shared memory, then
// lane l owns output channel co = l and accumulates the 45 (tap, channel)
// products over the 32 pixels from broadcast reads.  Warps are summed in a
// fixed order at the end (deterministic).
constexpr int kL1Warps = 8;
constexpr int kL1XS = 48;  // window row stride (16-byte aligned rows)
constexpr int kL1Warp = 32 * kL1XS + 32 * 33;
constexpr int kL1Red = 45 * kF;
constexpr int kL1Stride = kL1Warp > kL1Red ? kL1Warp : kL1Red;
__global__ void __launch_bounds__(kL1Warps * 32, 2) layer1_wgrad_kernel(const L1Args a, const __nv_bfloat16* g,
                                                                       float* partial) {
  grid_dep_wait();
  extern __shared__ __align__(16) float sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* sX = sm + warp * kL1Stride;  // [32 pixels][48]
  float* sG = sX + 32 * kL1XS;        // [32 pixels][33]
  float acc[45];
#pragma unroll
  for (int k = 0; k < 45; ++k) acc[k] = 0.f;
  const size_t plane = (size_t)a.H * a.W;
  const size_t total = plane * a.B;
  const size_t nchunks = (total + 31) / 32;
  const size_t nw = (size_t)gridDim.x * kL1Warps;
  const uint4* G = reinterpret_cast<const uint4*>(g);
  for (size_t chunk = (size_t)blockIdx.x * kL1Warps + warp; chunk < nchunks; chunk += nw) {
    const size_t i = chunk * 32 + lane;
    if (i < total) {
      const int b = (int)(i / plane);
      const size_t rem = i - (size_t)b * plane;
      const int y = (int)(rem / a.W), x = (int)(rem - (size_t)y * a.W);
      float in[9][5];
      l1_inputs(a, b, y, x, in);
#pragma unroll
      for (int tp = 0; tp < 9; ++tp)
#pragma unroll
        for (int c = 0; c < 5; ++c) sX[lane * kL1XS + tp * 5 + c] = in[tp][c];
#pragma unroll
      for (int ch = 0; ch < 4; ++ch) {
        const uint4 u = G[(((size_t)b * a.H + y) * 4 + ch) * a.W + x];
        const uint32_t wv[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          sG[lane * 33 + ch * 8 + 2 * e] = bf_lo(wv[e]);
          sG[lane * 33 + ch * 8 + 2 * e + 1] = bf_hi(wv[e]);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < 45; ++k) sX[lane * kL1XS + k] = 0.f;
#pragma unroll
      for (int k = 0; k < kF; ++k) sG[lane * 33 + k] = 0.f;
    }
    __syncwarp();
    for (int p = 0; p < 32; ++p) {
      const float gp = sG[p * 33 + lane];
      const float4* xr = reinterpret_cast<const float4*>(sX + p * kL1XS);
#pragma unroll
      for (int q = 0; q < 11; ++q) {
        const float4 x4 = xr[q];
        acc[4 * q + 0] = fmaf(x4.x, gp, acc[4 * q + 0]);
        acc[4 * q + 1] = fmaf(x4.y, gp, acc[4 * q + 1]);
        acc[4 * q + 2] = fmaf(x4.z, gp, acc[4 * q + 2]);
        acc[4 * q + 3] = fmaf(x4.w, gp, acc[4 * q + 3]);
      }
      acc[44] = fmaf(sX[p * kL1XS + 44], gp, acc[44]);
    }
    __syncwarp();  // this warp's staging area is rewritten by its next chunk
  }
  __syncthreads();
  float* red = sm + warp * kL1Stride;  // [45][32]
#pragma unroll
  for (int k = 0; k < 45; ++k) red[k * kF + lane] = acc[k];
  __syncthreads();
  const int nw_out = 9 * a.cin * kF;
  for (int o = threadIdx.x; o < nw_out; o += blockDim.x) {
    const int co = o % kF, c = (o / kF) % a.cin, tp = o / (kF * a.cin);
    const int src = (tp * 5 + c) * kF + co;
    float s = 0.f;
    for (int w2 = 0; w2 < kL1Warps; ++w2) s += sm[w2 * kL1Stride + src];
    partial[(size_t)blockIdx.x * nw_out + o] = s;
  }
}

// ---------------------------------------------------------------------------
// reductions of per-block partials (fixed order -> deterministic)
// ---------------------------------------------------------------------------
// One warp per output element: lane l sums the partials l, l + 32, ... in
// order, then a fixed xor-shuffle tree (warp_sum_fixed) adds the 32 lane sums
// -- the same order on every run.

// A lane issues the loads of kRedBatch partials before it adds any of them; the
// additions keep the order p = lane, lane + 32, ... (absent partials add +0).
__global__ void reduce_partials_kernel(const float* part, int n_parts, int len, int stride, float* out,
                                       int accumulate) {
  grid_dep_wait();
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < len; i += nw) {
    const float s = partial_sum(part, n_parts, stride, i, lane);
    if (lane == 0) out[i] = accumulate ? out[i] + s : s;
  }
}

// wgrad raw partials [n_parts][kw][128][jn * 32] -> Keras kernel gradient [kh][kw][cin][32].
// Accumulator row m = r * cw + ci (input row r of the M window, cw = 8 * C/8 of the
// layer's input tensor), column jj * 32 + co (output row jj of the N window); the
// product belongs to kernel row kh = r - jj, so dW[kh] sums the jn pairs r = kh + jj.
// jn = 2 for C = 32, 4 for C = 16.
// A CTA owns the 32 output channels of one (tap, ci): lane = co reads the partials
// coalesced, warp w sums partials w, w + 8, ... in order, and the 8 warp sums are
// added in a fixed order -- deterministic.
__global__ void __launch_bounds__(kFinWarps * 32) wgrad_finish_kernel(const float* part, int n_parts, int cin,
                                                                      int cw, float* out) {
  grid_dep_wait();
  __shared__ float red[kFinWarps][kF];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int groups = 9 * cin;
  for (int gi = blockIdx.x; gi < groups; gi += gridDim.x) {
    const int ci = gi % cin, tap = gi / cin;
    const int kh = tap / 3, kw = tap % 3;
    red[warp][lane] = cw == 32 ? finish_sum<2, 1>(part, n_parts, warp, lane, kw, kh, ci, cw)
                               : finish_sum<4, 1>(part, n_parts, warp, lane, kw, kh, ci, cw);
    __syncthreads();
    if (warp == 0) {
      float tsum = 0.f;
#pragma unroll
      for (int w2 = 0; w2 < kFinWarps; ++w2) tsum += red[w2][lane];
      out[(size_t)gi * kF + lane] = tsum;
    }
    __syncthreads();
  }
}

// Layer 0 (split input): the weight gradient of field c is the sum of the raw
// gradients of its x_h and x_l channels (3c, 3c + 1); the duplicate x_h channel
// (3c + 2, weights W_l) only carries the weights' low part and is not a variable.
__global__ void __launch_bounds__(kFinWarps * 32) wgrad_finish_split_kernel(const float* part, int n_parts, int cin,
                                                                            float* out) {
  grid_dep_wait();
  __shared__ float red[kFinWarps][kF];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int cw = 16, jn = 4;  // the 16-channel input tensor's partial layout
  const int groups = 9 * cin;
  for (int gi = blockIdx.x; gi < groups; gi += gridDim.x) {
    const int c = gi % cin, tap = gi / cin;
    const int kh = tap / 3, kw = tap % 3;
    red[warp][lane] = finish_sum<jn, 2>(part, n_parts, warp, lane, kw, kh, 3 * c, cw);
    __syncthreads();
    if (warp == 0) {
      float tsum = 0.f;
#pragma unroll
      for (int w2 = 0; w2 < kFinWarps; ++w2) tsum += red[w2][lane];
      out[(size_t)gi * kF + lane] = tsum;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Adam (Keras legacy): per-variable clip_by_norm, then
//   m += (g - m)(1 - b1); v += (g^2 - v)(1 - b2); x -= lr_t m / (sqrt(v) + eps)
// ---------------------------------------------------------------------------
// The squared norms in two deterministic stages: one CTA per chunk of
// kNormChunk elements of a variable (partial sums after the norms in the
// scratch), then one warp per variable adds its chunks in a fixed order.
constexpr size_t kNormChunk = 4096;

struct AdamVars {
  int n;
  size_t off[IGM_MAX_VARS + 1];
  int cbase[IGM_MAX_VARS + 1];  // first chunk of each variable; cbase[n] = number of chunks
};

static int norm_chunks(size_t len) { return (int)((len + kNormChunk - 1) / kNormChunk); }

__global__ void __launch_bounds__(256) grad_norm_parts_kernel(const float* g, const AdamVars vars, double* parts) {
  grid_dep_wait();
  __shared__ double sh[8];
  const int b = blockIdx.x;
  int v = 0;
  while (v + 1 < vars.n && b >= vars.cbase[v + 1]) ++v;
  const size_t lo = vars.off[v] + (size_t)(b - vars.cbase[v]) * kNormChunk;
  const size_t hi = min(vars.off[v + 1], lo + kNormChunk);
  double s = 0.0;
  for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += (double)g[i] * g[i];
  s = block_sum<256>(s, sh, threadIdx.x);
  if (threadIdx.x == 0) parts[b] = s;
}

__global__ void grad_norm_finish_kernel(const double* parts, const AdamVars vars, double* norms) {
  grid_dep_wait();
  const int v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (v >= vars.n) return;  // uniform per warp
  double s = 0.0;
  for (int c = vars.cbase[v] + lane; c < vars.cbase[v + 1]; c += 32) s += parts[c];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) norms[v] = sqrt(s);
}

__global__ void adam_kernel(float* x, const float* g, float* m, float* v, const AdamVars vars, const double* norms,
                            float lr_t, float b1, float b2, float eps, float clipnorm) {
  grid_dep_wait();
  const size_t total = vars.off[vars.n];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    int k = 0;
    while (k + 1 < vars.n && i >= vars.off[k + 1]) ++k;
    float gi = g[i];
    if (clipnorm > 0.f) {
      const float nrm = (float)norms[k];
      gi = gi * clipnorm / (nrm > clipnorm ? nrm : clipnorm);
    }
    float mi = m[i], vi = v[i];
    mi += (gi - mi) * (1.f - b1);
    vi += (gi * gi - vi) * (1.f - b2);
    m[i] = mi;
    v[i] = vi;
    x[i] -= (mi * lr_t) / (sqrtf(vi) + eps);
  }
}

static int grid_for(size_t n, int per = 256) {
  size_t b = (n + per - 1) / per;
  if (b > 148 * 8) b = 148 * 8;
  return (int)(b < 1 ? 1 : b);
}

// ---------------------------------------------------------------------------
// Input gradient of the first layer: from dPre0 (the gradient of the first
// layer's pre-activation, bf16 row-chunked [B][H][4][W][8], as the second
// layer's dgrad leaves it) to the gradient of each raw input field,
//   dField_c[y][x] = scale_c sum_{kh,kw,co} dPre0[y-kh+1][x-kw+1][co] W0[kh][kw][c][co]
// with the FP32 weights (the transposed "same" convolution; the BF16 split of
// the inputs is a representation of the same x, so its gradient is x's).
// A CTA stages the 10 x 34 halo tile of dPre0 in shared memory and produces
// an 8 x 32 tile of pixels, one per thread; the weights in shared memory too.
// ---------------------------------------------------------------------------
struct InputGradScales { float s[8]; };

constexpr int kIgTY = 8, kIgTX = 32;  // output tile of one CTA (256 threads, one pixel each)

template <int NG>
__global__ void __launch_bounds__(256) input_grad_kernel(int B, int H, int W, int cin, const __nv_bfloat16* dpre,
                                                         const float* w0, InputGradScales sc, float* out) {
  grid_dep_wait();
  __shared__ __align__(16) float sw[9 * NG * kF];                // [tap][c][co] of the fields computed
  __shared__ uint4 tile[kIgTY + 2][4][kIgTX + 2];                // dPre0 rows y0-1 .. y0+8, 8-channel chunks
  for (int i = threadIdx.x; i < 9 * NG * kF; i += blockDim.x) {
    const int tap = i / (NG * kF), r = i - tap * NG * kF;
    sw[i] = w0[(size_t)tap * cin * kF + r];
  }
  const int b = blockIdx.z, y0 = blockIdx.y * kIgTY, x0 = blockIdx.x * kIgTX;
  const uint4* D = reinterpret_cast<const uint4*>(dpre);
  for (int i = threadIdx.x; i < (kIgTY + 2) * 4 * (kIgTX + 2); i += blockDim.x) {
    const int hy = i / (4 * (kIgTX + 2)), rem = i - hy * 4 * (kIgTX + 2);
    const int ch = rem / (kIgTX + 2), hx = rem - ch * (kIgTX + 2);
    const int yy = y0 - 1 + hy, xx = x0 - 1 + hx;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);  // bf16 zeros: the "same" padding
    if (yy >= 0 && yy < H && xx >= 0 && xx < W) val = D[(((size_t)b * H + yy) * 4 + ch) * W + xx];
    tile[hy][ch][hx] = val;
  }
  __syncthreads();
  const int r = threadIdx.x / kIgTX, c = threadIdx.x - r * kIgTX;
  const int y = y0 + r, x = x0 + c;
  float acc[NG];
#pragma unroll
  for (int k = 0; k < NG; ++k) acc[k] = 0.f;
#pragma unroll
  for (int kh = 0; kh < 3; ++kh) {
#pragma unroll
    for (int kw = 0; kw < 3; ++kw) {
      // dPre0[y - kh + 1][x - kw + 1] sits at tile[r + 2 - kh][.][c + 2 - kw]
      const float* wt = sw + (kh * 3 + kw) * NG * kF;
#pragma unroll
      for (int ch = 0; ch < 4; ++ch) {
        const uint4 u = tile[r + 2 - kh][ch][c + 2 - kw];
        const uint32_t wv[4] = {u.x, u.y, u.z, u.w};
        float d[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) d[e] = (e & 1) ? bf_hi(wv[e >> 1]) : bf_lo(wv[e >> 1]);
#pragma unroll
        for (int k = 0; k < NG; ++k) {
          const float4 wa = *reinterpret_cast<const float4*>(wt + k * kF + ch * 8);
          const float4 wb = *reinterpret_cast<const float4*>(wt + k * kF + ch * 8 + 4);
          const float wk[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
          for (int e = 0; e < 8; ++e) acc[k] = fmaf(d[e], wk[e], acc[k]);
        }
      }
    }
  }
  if (y < H && x < W) {
    const size_t plane = (size_t)H * W, rem = (size_t)y * W + x;
#pragma unroll
    for (int k = 0; k < NG; ++k) out[((size_t)b * NG + k) * plane + rem] = acc[k] * sc.s[k];
  }
}

}  // namespace igm

using namespace igm;

extern "C" size_t igm_cnn_param_count(int nb_layers, int cin, int nout) {
  if (nb_layers < 1 || cin < 1 || cin > 8 || nout < 1 || nout > 2 * IGM_MAX_NZ) return 0;
  return param_count(nb_layers, cin, nout);
}

extern "C" size_t igm_cnn_param_offset(int nb_layers, int cin, int nout, int layer, int bias) {
  if (layer < 0 || layer > nb_layers) return (size_t)-1;
  return bias ? b_offset(layer, cin, nout, nb_layers) : w_offset(layer, cin, nout);
}

extern "C" int igm_cnn_pack_weights(int nb_layers, int cin, int nout, const float* params, void* wpack_fwd,
                                    void* wpack_bwd, void* stream) {
  IGM_CHECK_ARG(nb_layers >= 1 && cin >= 1 && cin <= 8 && nout >= 1, IGM_ERR_BAD_SHAPE,
                "igm_cnn_pack_weights: bad network shape");
  IGM_CHECK_ARG(params && wpack_fwd && (wpack_bwd || nb_layers == 1), IGM_ERR_BAD_ARGUMENT,
                "igm_cnn_pack_weights: NULL argument");
  const size_t total = (size_t)9 * 2 * kF * 8 + (size_t)(nb_layers - 1) * 9 * 4 * kF * 8 * 2;
  launch_pdl(pack_kernel, dim3(grid_for(total)), dim3(256), 0, as_stream(stream), params, nb_layers, cin, nout,
                                                              (__nv_bfloat16*)wpack_fwd, (__nv_bfloat16*)wpack_bwd);
  return launch_status("pack_kernel");
}

extern "C" int igm_cnn_input(int batch, int h, int w, int ny, int nx, const float* thk, const float* usurf,
                             const float* arrhenius, const float* slidingco, double dx, const float* scales,
                             const int* win_y0, const int* win_x0, void* X, float* thk_out, float* usurf_out,
                             float* arrhenius_out, float* slidingco_out, void* stream) {
  IGM_CHECK_ARG(batch >= 1 && batch <= IGM_MAX_WINDOWS && h >= 1 && w >= 1, IGM_ERR_BAD_SHAPE,
                "igm_cnn_input: bad shape (batch must be <= %d)", IGM_MAX_WINDOWS);
  IGM_CHECK_ARG(thk && usurf && arrhenius && slidingco && scales && win_y0 && win_x0, IGM_ERR_BAD_ARGUMENT,
                "igm_cnn_input: NULL argument");
  InputArgs a{};
  a.B = batch; a.h = h; a.w = w; a.Ny = ny; a.Nx = nx;
  a.f[0] = thk; a.f[1] = usurf; a.f[2] = arrhenius; a.f[3] = slidingco;
  a.dx = (float)dx;
  for (int c = 0; c < 5; ++c) a.scale[c] = scales[c];
  for (int b = 0; b < batch; ++b) {
    IGM_CHECK_ARG(win_y0[b] >= 0 && win_x0[b] >= 0 && win_y0[b] + h <= ny && win_x0[b] + w <= nx,
                  IGM_ERR_BAD_SHAPE, "igm_cnn_input: window %d outside the domain", b);
    a.y0[b] = win_y0[b];
    a.x0[b] = win_x0[b];
  }
  a.X = (__nv_bfloat16*)X;
  a.out[0] = thk_out; a.out[1] = usurf_out; a.out[2] = arrhenius_out; a.out[3] = slidingco_out;
  launch_pdl(input_kernel, dim3(grid_for((size_t)batch * h * w)), dim3(256), 0, as_stream(stream), a);
  return launch_status("input_kernel");
}

static int l1_args(L1Args* a, int batch, int h, int w, int cin, const float* thk, const float* usurf,
                   const float* arrhenius, const float* slidingco, double dx, const float* scales, const float* w1,
                   const float* b1, float alpha) {
  IGM_CHECK_ARG(batch >= 1 && h >= 1 && w >= 1 && cin >= 1 && cin <= 5, IGM_ERR_BAD_SHAPE,
                "igm_cnn_layer1: bad shape (cin must be 1..5)");
  IGM_CHECK_ARG(thk && usurf && arrhenius && slidingco && scales && w1, IGM_ERR_BAD_ARGUMENT,
                "igm_cnn_layer1: NULL argument");
  a->B = batch; a->H = h; a->W = w; a->cin = cin;
  a->f[0] = thk; a->f[1] = usurf; a->f[2] = arrhenius; a->f[3] = slidingco;
  for (int c = 0; c < 4; ++c) a->scale[c] = scales[c];
  a->dxs = (float)dx * scales[4];
  a->w = w1;
  a->b = b1;
  a->alpha = alpha;
  return IGM_OK;
}

extern "C" int igm_cnn_layer1_forward(int batch, int h, int w, int cin, const float* thk, const float* usurf,
                                      const float* arrhenius, const float* slidingco, double dx, const float* scales,
                                      const float* w1, const float* b1, float alpha, void* act, void* stream) {
  L1Args a{};
  int rc = l1_args(&a, batch, h, w, cin, thk, usurf, arrhenius, slidingco, dx, scales, w1, b1, alpha);
  if (rc) return rc;
  IGM_CHECK_ARG(b1 && act, IGM_ERR_BAD_ARGUMENT, "igm_cnn_layer1_forward: NULL argument");
  a.out = (__nv_bfloat16*)act;
  launch_pdl(layer1_fwd_kernel, dim3(grid_for((size_t)batch * h * w)), dim3(256), 0, as_stream(stream), a);
  return launch_status("layer1_fwd_kernel");
}

extern "C" int igm_cnn_layer1_wgrad(int batch, int h, int w, int cin, const float* thk, const float* usurf,
                                    const float* arrhenius, const float* slidingco, double dx, const float* scales,
                                    const void* g, float* partials, int n_parts, void* stream) {
  L1Args a{};
  const float dummy = 0.f;
  int rc = l1_args(&a, batch, h, w, cin, thk, usurf, arrhenius, slidingco, dx, scales, &dummy, nullptr, 0.f);
  if (rc) return rc;
  IGM_CHECK_ARG(g && partials && n_parts >= 1, IGM_ERR_BAD_ARGUMENT, "igm_cnn_layer1_wgrad: bad argument");
  constexpr size_t smem = (size_t)kL1Warps * kL1Stride * sizeof(float);
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(layer1_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
      set_error("layer1_wgrad smem attribute: %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
    configured = true;
  }
  launch_pdl(layer1_wgrad_kernel, dim3(n_parts), dim3(kL1Warps * 32), smem, as_stream(stream), a, (const __nv_bfloat16*)g, partials);
  return launch_status("layer1_wgrad_kernel");
}

extern "C" int igm_cnn_head_forward(int batch, int h, int w, int nz, const void* act, const float* head_w,
                                    const float* head_b, float out_scale, float* U, float* V, const float* thk_mask,
                                    void* stream) {
  IGM_CHECK_ARG(batch >= 1 && h >= 1 && w >= 1 && nz >= 1 && nz <= IGM_MAX_NZ, IGM_ERR_BAD_SHAPE,
                "igm_cnn_head_forward: bad shape");
  IGM_CHECK_ARG(act && head_w && head_b && U && V, IGM_ERR_BAD_ARGUMENT, "igm_cnn_head_forward: NULL argument");
  const int nout = 2 * nz;
  const int grid = grid_for((size_t)batch * h * w);
  cudaStream_t st = as_stream(stream);
  const __nv_bfloat16* A = (const __nv_bfloat16*)act;
  if (nout <= 32) {
    switch ((nout + 3) / 4) {
#define IGM_HEAD_FWD(Q)                                                                                      \
  case Q:                                                                                                    \
    launch_pdl(head_fwd_kernel<4 * Q>, dim3(grid), dim3(256), 0, st, batch, h, w, nz, A, head_w, head_b, out_scale, U, V, thk_mask); \
    break;
      IGM_HEAD_FWD(1) IGM_HEAD_FWD(2) IGM_HEAD_FWD(3) IGM_HEAD_FWD(4) IGM_HEAD_FWD(5) IGM_HEAD_FWD(6)
      IGM_HEAD_FWD(7) IGM_HEAD_FWD(8)
#undef IGM_HEAD_FWD
      default:
        return IGM_ERR_BAD_SHAPE;
    }
  } else if (nout <= 64)
    launch_pdl(head_fwd_kernel<64>, dim3(grid), dim3(256), 0, st, batch, h, w, nz, A, head_w, head_b, out_scale, U, V, thk_mask);
  else
    launch_pdl(head_fwd_kernel<128>, dim3(grid), dim3(256), 0, st, batch, h, w, nz, A, head_w, head_b, out_scale, U, V, thk_mask);
  return launch_status("head_fwd_kernel");
}

extern "C" size_t igm_cnn_head_partial_len(int nz) { return (size_t)kF * 2 * nz + 2 * nz + kF; }

template <int NJ>
static int head_bwd_launch(int batch, int h, int w, int nz, const void* act, const float* head_w, const float* dU,
                           const float* dV, float out_scale, float alpha, void* dpre, float* partials, int n_parts,
                           cudaStream_t st) {
  constexpr size_t smem = (size_t)HeadBwdSmem<NJ>::FLOATS * sizeof(float);
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(head_bwd_kernel<NJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
      set_error("head_bwd smem attribute: %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
    configured = true;
  }
  launch_pdl(head_bwd_kernel<NJ>, dim3(n_parts), dim3(kHeadWarps * 32), smem, st, batch, h, w, nz, (const __nv_bfloat16*)act, head_w, dU,
                                                                dV, out_scale, alpha, (__nv_bfloat16*)dpre, partials);
  return launch_status("head_bwd_kernel");
}

extern "C" int igm_cnn_head_backward(int batch, int h, int w, int nz, const void* act, const float* head_w,
                                     const float* dU, const float* dV, float out_scale, float alpha, void* dpre,
                                     float* partials, int n_parts, void* stream) {
  IGM_CHECK_ARG(batch >= 1 && h >= 1 && w >= 1 && nz >= 1 && nz <= IGM_MAX_NZ && n_parts >= 1, IGM_ERR_BAD_SHAPE,
                "igm_cnn_head_backward: bad shape");
  IGM_CHECK_ARG(act && head_w && dU && dV && dpre && partials, IGM_ERR_BAD_ARGUMENT,
                "igm_cnn_head_backward: NULL argument");
  const int nout = 2 * nz;
  cudaStream_t st = as_stream(stream);
  if (nout <= 32) return head_bwd_launch<32>(batch, h, w, nz, act, head_w, dU, dV, out_scale, alpha, dpre, partials,
                                             n_parts, st);
  if (nout <= 64) return head_bwd_launch<64>(batch, h, w, nz, act, head_w, dU, dV, out_scale, alpha, dpre, partials,
                                             n_parts, st);
  return head_bwd_launch<128>(batch, h, w, nz, act, head_w, dU, dV, out_scale, alpha, dpre, partials, n_parts, st);
}


extern "C" int igm_cnn_head_backward_tc(int batch, int h, int w, int nz, const void* act, const float* head_w,
                                        const float* dU, const float* dV, float out_scale, float alpha, void* dpre,
                                        void* dy_bf16, float* partials, int n_parts, void* stream) {
  IGM_CHECK_ARG(batch >= 1 && h >= 1 && w >= 1 && nz >= 1 && 2 * nz <= kF && n_parts >= 1, IGM_ERR_BAD_SHAPE,
                "igm_cnn_head_backward_tc: bad shape (needs 2 nz <= 32)");
  IGM_CHECK_ARG(act && head_w && dU && dV && dpre && ((dy_bf16 == nullptr) == (partials == nullptr)),
                IGM_ERR_BAD_ARGUMENT, "igm_cnn_head_backward_tc: NULL argument");
  cudaStream_t st = as_stream(stream);
  const __nv_bfloat16* a16 = (const __nv_bfloat16*)act;
  __nv_bfloat16 *dp = (__nv_bfloat16*)dpre, *dy = (__nv_bfloat16*)dy_bf16;
  const bool params = partials != nullptr;  // NULL dy_bf16 and partials: the data gradient only
  switch ((2 * nz + 3) / 4) {
#define IGM_HEAD_PX(Q)                                                                                              \
  case Q:                                                                                                           \
    if (params)                                                                                                     \
      launch_pdl(head_bwd_px_kernel<4 * Q, true>, dim3(n_parts), dim3(kHpWarps * 32), 0, st, batch, h, w, nz, a16, head_w, dU, dV,     \
                                                                         out_scale, alpha, dp, dy, partials);       \
    else                                                                                                            \
      launch_pdl(head_bwd_px_kernel<4 * Q, false>, dim3(n_parts), dim3(kHpWarps * 32), 0, st, batch, h, w, nz, a16, head_w, dU, dV,    \
                                                                          out_scale, alpha, dp, dy, partials);      \
    break;
    IGM_HEAD_PX(1) IGM_HEAD_PX(2) IGM_HEAD_PX(3) IGM_HEAD_PX(4) IGM_HEAD_PX(5) IGM_HEAD_PX(6) IGM_HEAD_PX(7)
    IGM_HEAD_PX(8)
#undef IGM_HEAD_PX
    default:
      return IGM_ERR_BAD_SHAPE;
  }
  return launch_status("head_bwd_px_kernel");
}

extern "C" int igm_cnn_head_wgrad_finish(const float* partials, int n_parts, int nout, float* out, void* stream) {
  IGM_CHECK_ARG(partials && out && n_parts >= 1 && nout >= 1 && nout <= kF, IGM_ERR_BAD_ARGUMENT,
                "igm_cnn_head_wgrad_finish: bad argument");
  launch_pdl(head_wgrad_finish_kernel, dim3(kF), dim3(kFinWarps * 32), 0, as_stream(stream), partials, n_parts, nout, out);
  return launch_status("head_wgrad_finish_kernel");
}

extern "C" int igm_reduce_partials(const float* partials, int n_parts, int len, int stride, float* out,
                                   int accumulate, void* stream) {
  IGM_CHECK_ARG(partials && out && n_parts >= 1 && len >= 0 && stride >= len, IGM_ERR_BAD_ARGUMENT,
                "igm_reduce_partials: bad argument");
  if (len == 0) return IGM_OK;
  launch_pdl(reduce_partials_kernel, dim3(grid_for((size_t)len * 32)), dim3(256), 0, as_stream(stream), partials, n_parts, len, stride,
                                                                                   out, accumulate);
  return launch_status("reduce_partials_kernel");
}

extern "C" int igm_cnn_wgrad_finish(const float* partials, int n_parts, int cin, int cin_tensor, float* out,
                                    void* stream) {
  IGM_CHECK_ARG(partials && out && n_parts >= 1, IGM_ERR_BAD_ARGUMENT, "igm_cnn_wgrad_finish: bad argument");
  IGM_CHECK_ARG((cin_tensor == 16 || cin_tensor == 32) && cin >= 1 && cin <= cin_tensor, IGM_ERR_BAD_SHAPE,
                "igm_cnn_wgrad_finish: bad channel counts");
  launch_pdl(wgrad_finish_kernel, dim3(9 * cin), dim3(kFinWarps * 32), 0, as_stream(stream), partials, n_parts, cin, cin_tensor, out);
  return launch_status("wgrad_finish_kernel");
}

extern "C" int igm_cnn_wgrad_finish_split(const float* partials, int n_parts, int cin, float* out, void* stream) {
  IGM_CHECK_ARG(partials && out && n_parts >= 1, IGM_ERR_BAD_ARGUMENT, "igm_cnn_wgrad_finish_split: bad argument");
  IGM_CHECK_ARG(cin >= 1 && cin <= 5, IGM_ERR_BAD_SHAPE, "igm_cnn_wgrad_finish_split: 1..5 input fields");
  // the kernel reads the 16-channel weight-gradient partials with row groups of 4 (3 x 128 x 4 x 32 floats)
  IGM_CHECK_ARG(igm_conv3x3_wgrad_partial_len(16) == (size_t)3 * 128 * 4 * kF, IGM_ERR_UNSUPPORTED,
                "igm_cnn_wgrad_finish_split: the weight-gradient partial layout is not the one this kernel reads");
  launch_pdl(wgrad_finish_split_kernel, dim3(9 * cin), dim3(kFinWarps * 32), 0, as_stream(stream), partials, n_parts, cin, out);
  return launch_status("wgrad_finish_split_kernel");
}

extern "C" size_t igm_adam_norms_len(int n_vars, const size_t* var_offsets) {
  if (n_vars < 1 || n_vars > IGM_MAX_VARS || !var_offsets) return 0;
  size_t len = (size_t)n_vars;
  for (int i = 0; i < n_vars; ++i)
    len += var_offsets[i + 1] > var_offsets[i] ? (size_t)norm_chunks(var_offsets[i + 1] - var_offsets[i]) : 0;
  return len;
}

extern "C" int igm_adam_clipnorm(int n_vars, const size_t* var_offsets, float* params, const float* grads,
                                 float* m, float* v, double* norms, double lr, double beta_1, double beta_2,
                                 double epsilon, double clipnorm, int64_t iteration, void* stream) {
  IGM_CHECK_ARG(n_vars >= 1 && n_vars <= IGM_MAX_VARS, IGM_ERR_BAD_ARGUMENT, "igm_adam_clipnorm: 1..%d variables",
                IGM_MAX_VARS);
  IGM_CHECK_ARG(var_offsets && params && grads && m && v && norms, IGM_ERR_BAD_ARGUMENT,
                "igm_adam_clipnorm: NULL argument");
  AdamVars vars{};
  vars.n = n_vars;
  for (int i = 0; i <= n_vars; ++i) vars.off[i] = var_offsets[i];
  vars.cbase[0] = 0;
  for (int i = 0; i < n_vars; ++i) {
    IGM_CHECK_ARG(var_offsets[i + 1] > var_offsets[i], IGM_ERR_BAD_ARGUMENT, "igm_adam_clipnorm: empty variable %d",
                  i);
    vars.cbase[i + 1] = vars.cbase[i] + norm_chunks(var_offsets[i + 1] - var_offsets[i]);
  }
  const double t = (double)iteration;
  const float b1p = powf((float)beta_1, (float)t), b2p = powf((float)beta_2, (float)t);
  const float lr_t = (float)lr * sqrtf(1.f - b2p) / (1.f - b1p);
  cudaStream_t st = as_stream(stream);
  double* parts = norms + n_vars;
  launch_pdl(grad_norm_parts_kernel, dim3(vars.cbase[n_vars]), dim3(256), 0, st, grads, vars, parts);
  int rc = launch_status("grad_norm_parts_kernel");
  if (rc) return rc;
  launch_pdl(grad_norm_finish_kernel, dim3((n_vars + 3) / 4), dim3(128), 0, st, parts, vars, norms);
  if ((rc = launch_status("grad_norm_finish_kernel"))) return rc;
  launch_pdl(adam_kernel, dim3(grid_for(vars.off[n_vars])), dim3(256), 0, st, params, grads, m, v, vars, norms, lr_t, (float)beta_1,
                                                         (float)beta_2, (float)epsilon, (float)clipnorm);
  return launch_status("adam_kernel");
}

extern "C" int igm_cnn_input_gradient(int batch, int h, int w, int cin, int n_grad, const void* dpre0,
                                      const float* w0, const double* scales, float* out, void* stream) {
  IGM_CHECK_ARG(batch >= 1 && h >= 1 && w >= 1 && cin >= 1 && cin <= 8 && n_grad >= 1 && n_grad <= cin,
                IGM_ERR_BAD_SHAPE, "igm_cnn_input_gradient: bad shape");
  IGM_CHECK_ARG(dpre0 && w0 && scales && out, IGM_ERR_BAD_ARGUMENT, "igm_cnn_input_gradient: NULL argument");
  InputGradScales sc{};
  for (int c = 0; c < n_grad; ++c) sc.s[c] = (float)scales[c];
  IGM_CHECK_ARG(batch <= 65535, IGM_ERR_BAD_SHAPE, "igm_cnn_input_gradient: batch above 65535");
  const dim3 grid((w + kIgTX - 1) / kIgTX, (h + kIgTY - 1) / kIgTY, batch);
  cudaStream_t st = as_stream(stream);
  const __nv_bfloat16* d = (const __nv_bfloat16*)dpre0;
  switch (n_grad) {
#define IGM_IG(C)                                                                      \
  case C:                                                                              \
    launch_pdl(input_grad_kernel<C>, dim3(grid), dim3(256), 0, st, batch, h, w, cin, d, w0, sc, out);      \
    break;
    IGM_IG(1) IGM_IG(2) IGM_IG(3) IGM_IG(4) IGM_IG(5) IGM_IG(6) IGM_IG(7) IGM_IG(8)
#undef IGM_IG
  }
  return launch_status("input_grad_kernel");
}
