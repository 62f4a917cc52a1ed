// 3x3 "same" convolutions of the CNN emulator on the 5th-generation tensor
// cores (tcgen05.mma kind::f16, BF16 operands, FP32 accumulation in TMEM).
//
// Reference: igm/processes/iceflow/emulate/neural_network.py:9-66 (Keras
// Conv2D(3x3, padding="same") + LeakyReLU(0.01)); the backward passes are the
// data and weight gradients Keras' GradientTape computes for it
// (emulate.py:252).
//
// Activation layout ("row-chunked"): bf16 [B][H][C/8][W][8].  A haloed input
// tile (R+2 rows, 130 pixels) lands in shared memory as [row][chunk][pixel][8]
// -- one ~2 KB bulk copy per (row, chunk), because each is contiguous in
// global memory -- which IS the canonical no-swizzle K-major UMMA layout for
// "pixels x channels" (8-pixel core matrices of 16-byte rows).  Rows/pixels
// outside the domain are zero-filled (the zero "same" padding).  Each of the
// nine taps is then just a shifted descriptor start address:
// (row + dy) * row_stride + (dx) * 16 bytes.
//
// Forward / dgrad kernel (persistent, one CTA per SM, 10 warps):
//   warp 0  producer: bulk copies of the input tile (and TMEM allocator),
//   warp 1  MMA issuer: per tile of R = 8 rows (R + 2 input rows x 3 kernel
//           columns x C/16 MMAs of M=128 pixels, the kernel rows folded into N),
//           K=16, into R TMEM accumulators,
//   warps 2-9 epilogue, two per TMEM lane quarter (each half of the rows):
//           TMEM -> registers (one pixel per thread), bias + LeakyReLU (forward)
//           or the LeakyReLU derivative mask of the previous activation (dgrad,
//           plus the bias-gradient partial sums), bf16 store.
//   Two input stages and two accumulator sets overlap load, MMA and epilogue
//   (rows, stages and sets are build-time constants; 8 / 2 / 2 measured best).
// Weight-gradient kernel: D[(input row, ci)][co] += X^T G over the pixels of
// four output rows per work item, with both operands MN-major: M = 128 spans
// 128/(C/8*8) consecutive input rows x C input channels (row stride = C/8
// chunk strides, so the M groups are uniformly strided), one accumulator per
// horizontal tap; the four output rows share one input tile of 3 + 4 rows.
#include <cuda_bf16.h>

#include "common.cuh"
#include "reduce.cuh"
#include "tc.cuh"

namespace igm {

constexpr int kTW = 128;        // pixels per tile row (the UMMA M)
constexpr int kBoxW = kTW + 2;  // with the 1-pixel halo on each side
constexpr int kCout = 32;       // output channels
constexpr int kWRowsN = 3 * kCout;  // B-operand rows per (dx, k-chunk) of a weight pack: (dy, channel)
constexpr int kConvThreads = 192;      // weight-gradient kernel: producer, MMA issuer, 4 epilogue warps
// forward / dgrad kernel: producer, MMA issuer and kConvEpiWarps epilogue warps -- two per TMEM lane
// quarter, each finishing half of a tile's rows, so that every scheduler has two epilogue warps to
// interleave
constexpr int kConvEpiWarps = 8;
constexpr int kConvFwdThreads = 64 + 32 * kConvEpiWarps;

enum ConvEpi { kEpiFwdLeaky = 0, kEpiDgrad = 1 };

struct ConvArgs {
  int B, H, W;
  int tiles_w, tiles_h, n_tiles;
  const __nv_bfloat16* x;      // input activation [B][H][C8_IN][W][8]
  const __nv_bfloat16* wpack;  // [9][C8_IN][32][8]
  const float* bias;           // [32] (forward)
  const __nv_bfloat16* amask;  // dgrad: previous activation [B][H][4][W][8]
  __nv_bfloat16* out;          // [B][H][4][W][8]
  float* db_partial;           // dgrad: [gridDim.x][32] or NULL
  float alpha;
  int* err;
};

// Input stages of the forward / dgrad pipeline and output rows per tile (build-time
// tuning constants; R must keep 2 R 32 TMEM columns a power of two: 2, 4 or 8).
#ifndef IGM_CONV_STAGES
#define IGM_CONV_STAGES 2
#endif
#ifndef IGM_CONV_ROWS
#define IGM_CONV_ROWS 8
#endif
// TMEM accumulator sets of the forward / dgrad pipeline (2 or 4; NACC R 32 columns a power of two)
#ifndef IGM_CONV_ACC_SETS
#define IGM_CONV_ACC_SETS 2
#endif

template <int C8_IN, int R>
struct ConvGeom {
  static constexpr int NST = IGM_CONV_STAGES;                 // input stages
  static constexpr uint32_t P = kBoxW * 16;                   // chunk plane stride (bytes)
  static constexpr uint32_t RS = C8_IN * P;                   // row stride
  static constexpr uint32_t STAGE = (R + 2) * RS;             // one input stage
  static constexpr uint32_t WBYTES = 9 * C8_IN * kCout * 16;  // packed weights
  static constexpr uint32_t OFF_W = NST * STAGE;
  static constexpr uint32_t OFF_BAR = OFF_W + WBYTES;
  static constexpr int NACC = IGM_CONV_ACC_SETS;              // accumulator sets
  static constexpr uint32_t TMEM_COLS = NACC * R * kCout;
  static_assert(TMEM_COLS <= 512 && (TMEM_COLS & (TMEM_COLS - 1)) == 0, "TMEM columns: a power of two <= 512");
  static_assert(2 * NST + 2 * NACC <= 16, "barrier slots");
  static constexpr uint32_t SMEM = OFF_BAR + 16 * 8 + 16 + 32 * 4 + 1024;
};

__device__ __forceinline__ void set_err(int* err, int code) {
  if (err) atomicExch(err, code);
}

// Loads, with one full warp, the tile of a row-chunked activation (bf16
// [B][H][c8][W][8]) covering rows gy0 .. gy0+rows-1 and pixels gx0 .. gx0+npx-1
// into shared memory as [row][chunk][pixel][8] (plane stride npx * 16 bytes).
// Every (row, chunk) plane is one contiguous run in global memory: one lane
// issues one bulk copy for its in-domain part; pixels and rows outside the
// domain are zero-filled with shared-memory stores ("same" zero padding),
// made visible to the tensor cores by a proxy fence before the arrival.
// Lane 0 arrives on `bar` with the number of bytes the copies will deliver.
__device__ __forceinline__ void load_tile(const __nv_bfloat16* act, int H, int W, int c8, int b, int gy0, int rows,
                                          int gx0, int npx, unsigned char* dst, uint64_t* bar, int lane) {
  const int nplanes = rows * c8;
  const uint32_t P = (uint32_t)npx * 16;
  const int xa = gx0 < 0 ? 0 : gx0;                // first in-domain pixel
  const int xb = gx0 + npx > W ? W : gx0 + npx;     // one past the last
  const uint32_t run = xb > xa ? (uint32_t)(xb - xa) * 16 : 0;
  uint32_t mine = 0;
  for (int p = lane; p < nplanes; p += 32) {
    const int gy = gy0 + p / c8;
    uint4* plane = reinterpret_cast<uint4*>(dst + (size_t)p * P);
    const uint4 z = make_uint4(0, 0, 0, 0);
    if (gy < 0 || gy >= H || run == 0) {
      for (int q = 0; q < npx; ++q) plane[q] = z;
    } else {
      for (int q = 0; q < xa - gx0; ++q) plane[q] = z;
      for (int q = xb - gx0; q < npx; ++q) plane[q] = z;
      mine += run;
    }
  }
  uint32_t total = mine;
  for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
  tc::fence_proxy_async_smem();
  __syncwarp();
  if (lane == 0) tc::mbar_expect_tx(bar, total);
  __syncwarp();
  for (int p = lane; p < nplanes; p += 32) {
    const int gy = gy0 + p / c8, c = p % c8;
    if (gy >= 0 && gy < H && run > 0) {
      const __nv_bfloat16* src = act + ((((size_t)b * H + gy) * c8 + c) * W + xa) * 8;
      tc::bulk_load(dst + (size_t)p * P + (size_t)(xa - gx0) * 16, src, run, bar);
    }
  }
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

template <int C8_IN, int R, int EPI>
__global__ void __launch_bounds__(kConvFwdThreads, 1) conv3x3_kernel(const ConvArgs a) {
  using G = ConvGeom<C8_IN, R>;
  constexpr int NST = G::NST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::OFF_BAR);
  uint64_t* full = bars;               // [NST] loads -> MMA
  uint64_t* empty = bars + NST;        // [NST] MMA -> loads
  constexpr int NACC = G::NACC;
  uint64_t* tfull = bars + 2 * NST;    // [NACC] MMA -> epilogue
  uint64_t* tempty = bars + 2 * NST + NACC;  // [NACC] epilogue -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + G::OFF_BAR + 128);
  float* sbias = reinterpret_cast<float*>(smem + G::OFF_BAR + 144);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // the next kernel may launch now: its CTAs wait for this grid to complete (grid_dep_wait)
  grid_dep_launch();
  grid_dep_wait();  // inputs, weights and outputs are touched only after the previous grid completed
  // packed weights -> shared memory, bias, barriers
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.wpack);
    uint4* dst = reinterpret_cast<uint4*>(smem + G::OFF_W);
    for (int i = threadIdx.x; i < (int)(G::WBYTES / 16); i += kConvFwdThreads) dst[i] = src[i];
    if (threadIdx.x < kCout) sbias[threadIdx.x] = (EPI == kEpiFwdLeaky && a.bias) ? a.bias[threadIdx.x] : 0.f;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < NACC; ++s) {
      tc::mbar_init(&tfull[s], 1);
      tc::mbar_init(&tempty[s], 32 * kConvEpiWarps);
    }
    tc::fence_mbar_init();
  }
  tc::fence_proxy_async_smem();
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, G::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t sbase = tc::smem_u32(smem);

  if (warp == 0) {
    // ---------------- producer: bulk copies of the haloed input tile ----------------
    for (int it = 0, t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
      const int s = it % NST, use = it / NST;
      if (!tc::mbar_wait(&empty[s], (use & 1) ^ 1)) {
        if (lane == 0) set_err(a.err, 1);
        break;
      }
      const int txi = t % a.tiles_w, rest = t / a.tiles_w;
      const int tyi = rest % a.tiles_h, b = rest / a.tiles_h;
      load_tile(a.x, a.H, a.W, C8_IN, b, tyi * R - 1, R + 2, txi * kTW - 1, kBoxW, smem + s * G::STAGE, &full[s],
                lane);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      // descriptors as (low word + compile-time offset, fixed high word): a few integer
      // instructions per MMA keep this one thread ahead of the tensor cores
      constexpr uint32_t a_hi = tc::desc_hi(128), b_hi = tc::desc_hi(128);
      const uint32_t w_lo = tc::desc_lo(sbase + G::OFF_W, kWRowsN * 16);
      for (int it = 0, t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
        const int s = it % NST, use = it / NST, acc = it % NACC, ause = it / NACC;
        if (!tc::mbar_wait(&tempty[acc], (ause & 1) ^ 1) || !tc::mbar_wait(&full[s], use & 1)) {
          set_err(a.err, 2);
          break;
        }
        tc::tc_fence_after();
        const uint32_t in_lo = tc::desc_lo(sbase + s * G::STAGE, G::P);
        const uint32_t dset = tmem + (uint32_t)(acc * R * kCout);
        // Input row i (global row y0 - 1 + i) feeds output rows o = i - dy through kernel row dy.
        // One MMA covers all of its valid dy at once (N = 32 ndy): output row o accumulates at
        // TMEM column 32 (R - 1 - o), so consecutive dy land in consecutive 32-column blocks.
        // Each activation tile is thus read once per (dx, k-step), not once per tap.
#pragma unroll
        for (int i = 0; i < R + 2; ++i) {
          constexpr int dmax = 2;
          const int dlo = i - (R - 1) > 0 ? i - (R - 1) : 0;
          const int dhi = i < dmax ? i : dmax;
          const int ndy = dhi - dlo + 1;
          const uint32_t dcol = dset + (uint32_t)(kCout * (R - 1 - i + dlo));
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
            for (int ks = 0; ks < C8_IN / 2; ++ks) {
              const uint32_t aoff = (i * G::RS + dx * 16 + ks * 2 * G::P) >> 4;
              const uint32_t boff = (((dx * C8_IN + ks * 2) * kWRowsN + dlo * kCout) * 16) >> 4;
              const uint64_t ad = tc::desc_join(in_lo + aoff, a_hi);
              if (dx == 0 && ks == 0 && dlo == 0) {
                // output row i starts here: initialise its accumulator alone, then add to the rows above
                tc::mma_bf16(dcol, ad, tc::desc_join(w_lo + boff, b_hi), tc::make_idesc_bf16(128, kCout, false, false),
                             0u);
                if (ndy > 1)
                  tc::mma_bf16(dcol + kCout, ad, tc::desc_join(w_lo + boff + ((kCout * 16) >> 4), b_hi),
                               tc::make_idesc_bf16(128, kCout * (ndy - 1), false, false), 1u);
              } else {
                tc::mma_bf16(dcol, ad, tc::desc_join(w_lo + boff, b_hi),
                             tc::make_idesc_bf16(128, kCout * ndy, false, false), 1u);
              }
            }
          }
        }
        tc::mma_commit(&empty[s]);
        tc::mma_commit(&tfull[acc]);
      }
    }
  } else {
    // ---------------- epilogue (warps 2 .. 2 + kConvEpiWarps - 1) ----------------
    static_assert(kConvEpiWarps == 8 && R % 2 == 0, "two epilogue warps per lane quarter, each half the rows");
    constexpr int RH = R / 2;         // rows of a tile this warp finishes
    const int q = warp & 3;           // TMEM lane quarter this warp may access
    const int r0 = ((warp - 2) >> 2) * RH;  // its first row
    const int p = q * 32 + lane;      // pixel within the tile = TMEM lane
    float dbacc[kCout];
#pragma unroll
    for (int c = 0; c < kCout; ++c) dbacc[c] = 0.f;
    for (int it = 0, t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
      const int use = it / NACC, acc = it % NACC;
      const int txi = t % a.tiles_w, rest = t / a.tiles_w;
      const int tyi = rest % a.tiles_h, b = rest / a.tiles_h;
      const int x = txi * kTW + p;
      // dgrad: the activation mask of this warp's rows is requested before waiting for the
      // accumulators, so its latency overlaps the MMAs of this tile
      uint4 mk[EPI == kEpiDgrad ? RH : 1][4];
      if (EPI == kEpiDgrad) {
        const uint4* am = reinterpret_cast<const uint4*>(a.amask);
#pragma unroll
        for (int r = 0; r < RH; ++r) {
          const int y = tyi * R + r0 + r;
          const bool ok = y < a.H && x < a.W;
          const size_t pix = ok ? (((size_t)b * a.H + y) * 4) * a.W + x : 0;
#pragma unroll
          for (int ch = 0; ch < 4; ++ch) mk[r][ch] = ok ? am[pix + (size_t)ch * a.W] : make_uint4(0, 0, 0, 0);
        }
      }
      if (!tc::mbar_wait(&tfull[acc], use & 1)) {
        set_err(a.err, 3);
        break;
      }
      tc::tc_fence_after();
#pragma unroll
      for (int rr = 0; rr < RH; ++rr) {
        const int r = r0 + rr;  // row of the tile
        uint32_t v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((acc * R + (R - 1 - r)) * kCout), v);
        tc::tmem_wait_ld();
        const int y = tyi * R + r;
        if (y < a.H && x < a.W) {
          const size_t pix = (((size_t)b * a.H + y) * 4) * a.W + x;  // chunk 0 of this pixel, in 8-element units
          float f[kCout];
#pragma unroll
          for (int c = 0; c < kCout; ++c) f[c] = __uint_as_float(v[c]);
          if (EPI == kEpiFwdLeaky) {
#pragma unroll
            for (int c = 0; c < kCout; ++c) {
              const float z = f[c] + sbias[c];
              f[c] = z > 0.f ? z : a.alpha * z;
            }
          } else {
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) {
              const uint4 mv = mk[EPI == kEpiDgrad ? rr : 0][ch];
              const uint32_t mw[4] = {mv.x, mv.y, mv.z, mv.w};
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&mw[e]);
                const float lo = __low2float(h), hi = __high2float(h);
                const int c = ch * 8 + e * 2;
                f[c] *= lo > 0.f ? 1.f : a.alpha;
                f[c + 1] *= hi > 0.f ? 1.f : a.alpha;
              }
            }
#pragma unroll
            for (int c = 0; c < kCout; ++c) dbacc[c] += f[c];
          }
          uint4* o = reinterpret_cast<uint4*>(a.out);
#pragma unroll
          for (int ch = 0; ch < 4; ++ch) {
            uint4 w;
            w.x = pack_bf16x2(f[ch * 8 + 0], f[ch * 8 + 1]);
            w.y = pack_bf16x2(f[ch * 8 + 2], f[ch * 8 + 3]);
            w.z = pack_bf16x2(f[ch * 8 + 4], f[ch * 8 + 5]);
            w.w = pack_bf16x2(f[ch * 8 + 6], f[ch * 8 + 7]);
            o[pix + (size_t)ch * a.W] = w;
          }
        }
      }
      tc::tc_fence_before();
      tc::mbar_arrive(&tempty[acc]);
    }
    if (EPI == kEpiDgrad && a.db_partial) {
      // deterministic CTA reduction of the bias-gradient partial sums
#pragma unroll
      for (int c = 0; c < kCout; ++c) {
        float v = dbacc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        dbacc[c] = v;
      }
      float* red = reinterpret_cast<float*>(smem + G::OFF_W);  // weights no longer needed after the last MMA
      // wait until every MMA of this CTA completed before reusing the weight area
      if (lane == 0) {
#pragma unroll
        for (int c = 0; c < kCout; ++c) red[(warp - 2) * kCout + c] = dbacc[c];
      }
    }
  }
  __syncthreads();
  if (EPI == kEpiDgrad && a.db_partial && threadIdx.x < kCout) {
    const float* red = reinterpret_cast<const float*>(smem + G::OFF_W);
    float sum = red[threadIdx.x];
#pragma unroll
    for (int w = 1; w < kConvEpiWarps; ++w) sum += red[w * kCout + threadIdx.x];  // fixed order
    a.db_partial[(size_t)blockIdx.x * kCout + threadIdx.x] = sum;
  }
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, G::TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// forward of a stack of 32 -> 32 channel layers in one persistent launch
// ---------------------------------------------------------------------------
// conv3x3_kernel<4, R, fwd> per layer, for layers k = 0 .. nlayers-1 of a stack
// (layer k reads the output of layer k - 1), with the tile pipeline running on
// across the layer boundaries: each CTA takes the same tiles in every layer, and
// before it loads tile t of layer k its producer waits until the (up to nine)
// tiles of layer k - 1 around t are stored -- a per-tile flag set to this
// launch's epoch.  Those are the only tiles whose outputs tile t reads, and the
// only tiles of layer k - 1 that read the rows tile t overwrites when layers
// alternate between two buffers, so the wait also orders that reuse.  A CTA's
// own earlier tiles never wait on its later ones, so with every CTA resident (a
// cooperative launch) all waits end; each is bounded all the same.  Each
// layer's weights are copied into one of two shared-memory buffers on the
// barrier of that layer's first tile.
constexpr int kStackMax = 16;

struct StackArgs {
  int B, H, W;
  int tiles_w, tiles_h, n_tiles;  // per layer
  int nlayers;
  const __nv_bfloat16* in;        // input of layer 0 [B][H][4][W][8]
  __nv_bfloat16* out[kStackMax];  // output of layer k
  const __nv_bfloat16* wpack[kStackMax];
  const float* bias[kStackMax];
  int* flags;                     // [nlayers][n_tiles]
  int epoch;
  float alpha;
  int* err;
};

template <int R>
__global__ void __launch_bounds__(kConvFwdThreads, 1) conv3x3_stack_kernel(const StackArgs a) {
  using G = ConvGeom<4, R>;
  constexpr int NST = G::NST, NACC = G::NACC;
  constexpr uint32_t OFF_BAR = G::OFF_W + 2 * G::WBYTES;  // two weight buffers
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + OFF_BAR);
  uint64_t* full = bars;
  uint64_t* empty = bars + NST;
  uint64_t* tfull = bars + 2 * NST;
  uint64_t* tempty = bars + 2 * NST + NACC;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + OFF_BAR + 128);
  volatile int* abort_epi = reinterpret_cast<volatile int*>(smem + OFF_BAR + 132);  // an epilogue wait gave up
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int per = a.n_tiles;
  // Layer k's tiles t = first(k) + j * gridDim.x: the CTAs that take the layer's last, partial round
  // of tiles move on by (per mod gridDim.x) each layer, so over the stack every CTA takes about the
  // same number of tiles (a fixed assignment would let the same CTAs take one tile more in every
  // layer, and the others wait for them)
  const int ncta = (int)gridDim.x, rem = per % ncta;
  auto first = [&](int k) { return ((int)blockIdx.x + ncta - (int)(((long long)k * rem) % ncta)) % ncta; };

  if (threadIdx.x == 0) {
    *abort_epi = 0;
    for (int s = 0; s < NST; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < NACC; ++s) {
      tc::mbar_init(&tfull[s], 1);
      tc::mbar_init(&tempty[s], 32 * kConvEpiWarps);
    }
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, G::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t sbase = tc::smem_u32(smem);

  if (warp == 0) {
    // ---------------- producer ----------------
    int it = 0;
    bool ok = true;
    for (int k = 0; k < a.nlayers && ok; ++k) {
      const __nv_bfloat16* src = k == 0 ? a.in : a.out[k - 1];
      for (int t = first(k); t < per; t += gridDim.x, ++it) {
        const int s = it % NST, use = it / NST;
        if (!tc::mbar_wait(&empty[s], (use & 1) ^ 1)) {
          if (lane == 0) set_err(a.err, 31);
          ok = false;
          break;
        }
        const int txi = t % a.tiles_w, rest = t / a.tiles_w;
        const int tyi = rest % a.tiles_h, b = rest / a.tiles_h;
        if (k > 0) {
          // the tiles of layer k - 1 whose outputs this tile reads
          bool got = true;
          if (lane < 9) {
            const int ny = tyi + lane / 3 - 1, nx = txi + lane % 3 - 1;
            if (ny >= 0 && ny < a.tiles_h && nx >= 0 && nx < a.tiles_w) {
              const int* f = a.flags + (size_t)(k - 1) * per + ((size_t)b * a.tiles_h + ny) * a.tiles_w + nx;
              uint32_t n = 0;
              while (tc::ld_acquire_gpu(f) != a.epoch) {
                if (++n > (1u << 22)) {
                  got = false;
                  break;
                }
                __nanosleep(64);
              }
            }
          }
          if (!__all_sync(0xffffffffu, got)) {
            if (lane == 0) set_err(a.err, 32);
            ok = false;
            break;
          }
          tc::fence_proxy_async_global();  // the acquired data is read next by the bulk-copy (async) proxy
        }
        unsigned char* st = smem + s * G::STAGE;
        if (t == first(k) && lane == 0) {
          // this layer's weights, on the barrier of its first tile (their buffer's last reader, layer
          // k - 2, completed: the commit that released this stage covers every earlier MMA)
          tc::mbar_expect_tx_only(&full[s], G::WBYTES);
          tc::bulk_load(smem + G::OFF_W + (k & 1) * G::WBYTES, a.wpack[k], G::WBYTES, &full[s]);
        }
        __syncwarp();
        load_tile(src, a.H, a.W, 4, b, tyi * R - 1, R + 2, txi * kTW - 1, kBoxW, st, &full[s], lane);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t a_hi = tc::desc_hi(128), b_hi = tc::desc_hi(128);
      int it = 0;
      bool ok = true;
      for (int k = 0; k < a.nlayers && ok; ++k) {
        const uint32_t w_lo = tc::desc_lo(sbase + G::OFF_W + (k & 1) * G::WBYTES, kWRowsN * 16);
        for (int t = first(k); t < per; t += gridDim.x, ++it) {
          const int s = it % NST, use = it / NST, acc = it % NACC, ause = it / NACC;
          if (!tc::mbar_wait(&tempty[acc], (ause & 1) ^ 1) || !tc::mbar_wait(&full[s], use & 1)) {
            set_err(a.err, 33);
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const uint32_t in_lo = tc::desc_lo(sbase + s * G::STAGE, G::P);
          const uint32_t dset = tmem + (uint32_t)(acc * R * kCout);
#pragma unroll
          for (int i = 0; i < R + 2; ++i) {
            const int dlo = i - (R - 1) > 0 ? i - (R - 1) : 0;
            const int dhi = i < 2 ? i : 2;
            const int ndy = dhi - dlo + 1;
            const uint32_t dcol = dset + (uint32_t)(kCout * (R - 1 - i + dlo));
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
              for (int ks = 0; ks < 2; ++ks) {
                const uint32_t aoff = (i * G::RS + dx * 16 + ks * 2 * G::P) >> 4;
                const uint32_t boff = (((dx * 4 + ks * 2) * kWRowsN + dlo * kCout) * 16) >> 4;
                const uint64_t ad = tc::desc_join(in_lo + aoff, a_hi);
                if (dx == 0 && ks == 0 && dlo == 0) {
                  tc::mma_bf16(dcol, ad, tc::desc_join(w_lo + boff, b_hi),
                               tc::make_idesc_bf16(128, kCout, false, false), 0u);
                  if (ndy > 1)
                    tc::mma_bf16(dcol + kCout, ad, tc::desc_join(w_lo + boff + ((kCout * 16) >> 4), b_hi),
                                 tc::make_idesc_bf16(128, kCout * (ndy - 1), false, false), 1u);
                } else {
                  tc::mma_bf16(dcol, ad, tc::desc_join(w_lo + boff, b_hi),
                               tc::make_idesc_bf16(128, kCout * ndy, false, false), 1u);
                }
              }
            }
          }
          tc::mma_commit(&empty[s]);
          tc::mma_commit(&tfull[acc]);
        }
      }
    }
  } else {
    // ---------------- epilogue (warps 2 .. 9) ----------------
    constexpr int RH = R / 2;
    const int q = warp & 3;
    const int r0 = ((warp - 2) >> 2) * RH;
    const int p = q * 32 + lane;
    int it = 0;
    bool ok = true;
    for (int k = 0; k < a.nlayers && ok; ++k) {
      float bias[kCout];
#pragma unroll
      for (int c = 0; c < kCout; ++c) bias[c] = __ldg(a.bias[k] + c);
      uint4* o = reinterpret_cast<uint4*>(a.out[k]);
      for (int t = first(k); t < per; t += gridDim.x, ++it) {
        const int use = it / NACC, acc = it % NACC;
        const int txi = t % a.tiles_w, rest = t / a.tiles_w;
        const int tyi = rest % a.tiles_h, b = rest / a.tiles_h;
        const int x = txi * kTW + p;
        if (!tc::mbar_wait(&tfull[acc], use & 1)) {
          set_err(a.err, 34);
          ok = false;
        }
        tc::tc_fence_after();
#pragma unroll
        for (int rr = 0; rr < RH && ok; ++rr) {
          const int r = r0 + rr;
          uint32_t v[32];
          tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((acc * R + (R - 1 - r)) * kCout), v);
          tc::tmem_wait_ld();
          const int y = tyi * R + r;
          if (y < a.H && x < a.W) {
            const size_t pix = (((size_t)b * a.H + y) * 4) * a.W + x;
            float f[kCout];
#pragma unroll
            for (int c = 0; c < kCout; ++c) {
              const float z = __uint_as_float(v[c]) + bias[c];
              f[c] = z > 0.f ? z : a.alpha * z;
            }
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) {
              uint4 w;
              w.x = pack_bf16x2(f[ch * 8 + 0], f[ch * 8 + 1]);
              w.y = pack_bf16x2(f[ch * 8 + 2], f[ch * 8 + 3]);
              w.z = pack_bf16x2(f[ch * 8 + 4], f[ch * 8 + 5]);
              w.w = pack_bf16x2(f[ch * 8 + 6], f[ch * 8 + 7]);
              o[pix + (size_t)ch * a.W] = w;
            }
          }
        }
        tc::tc_fence_before();
        tc::mbar_arrive(&tempty[acc]);
        // the tile's output is complete once all eight epilogue warps stored their rows: publish it;
        // the eight warps leave together when any of them gave up a wait (the shared abort flag,
        // written before the barrier, read after it), so none is left alone at the next barrier
        tc::fence_proxy_async_global();
        if (!ok) *abort_epi = 1;
        asm volatile("bar.sync 1, %0;\n" ::"n"(32 * kConvEpiWarps) : "memory");
        if (*abort_epi) {
          ok = false;
          break;
        }
        if (warp == 2 && lane == 0) {
          __threadfence();
          tc::st_release_gpu(a.flags + (size_t)k * per + t, a.epoch);
        }
      }
    }
  }
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, G::TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// weight gradient
// ---------------------------------------------------------------------------
struct WgradArgs {
  int B, H, W;
  int segs_w, yblocks, n_items;
  const __nv_bfloat16* x;  // layer input [B][H][C8_IN][W][8]
  const __nv_bfloat16* g;  // gradient w.r.t. the pre-activation [B][H][4][W][8]
  float* partial;  // [gridDim.x][3][128][32]
  int* err;
  int centre_only;  // only the kw = 1 accumulators (a 1x1 convolution's weight gradient)
};

// Output rows per work item of the weight-gradient kernel, and its input stages.
// The 16-channel input tensor keeps 4 rows: the finish kernel of the first layer
// (csrc/cnn.cu) reads its partials with the row-group width that gives (JN = 4).
// For 32 channels JN = 2 for 2 or 4 rows, so the partial layout does not depend on
// the build-time choice IGM_WGRAD_ROWS_32 (2 or 4) / IGM_WGRAD_STAGES_32.
#ifndef IGM_WGRAD_ROWS_32
#define IGM_WGRAD_ROWS_32 4
#endif
#ifndef IGM_WGRAD_STAGES_32
#define IGM_WGRAD_STAGES_32 2
#endif

template <int C8_IN>
struct WgradGeom {
  static constexpr int WR = C8_IN == 4 ? IGM_WGRAD_ROWS_32 : 4;  // output rows per work item
  static constexpr int NROW = 128 / (C8_IN * 8);         // input rows covered by M = 128
  // output rows covered by N: every one of them finds its three kernel rows in the M window
  static constexpr int JN = (NROW - 2) < WR ? (NROW - 2) : WR;
  static_assert(C8_IN != 4 || JN == 2, "the 32-channel partial layout has row groups of 2");
  static_assert(C8_IN != 2 || JN == 4, "the 16-channel partial layout has row groups of 4");
  static constexpr int NGRP = WR / JN;                   // MMA row groups per item
  static constexpr int WN = JN * kCout;                  // accumulator width per kw
  static constexpr int XROWS = WR - JN + NROW;           // input rows of one item
  static constexpr uint32_t P = kBoxW * 16;              // X chunk plane stride
  static constexpr uint32_t RS = C8_IN * P;              // X row stride
  static constexpr uint32_t XBYTES = XROWS * RS;         // X stage
  static constexpr uint32_t GP = kTW * 16;               // G chunk plane stride
  static constexpr uint32_t GBYTES = WR * 4 * GP;        // G stage (32 channels, WR rows)
  static constexpr uint32_t STAGE = XBYTES + GBYTES;
  static constexpr int NST = C8_IN == 4 ? IGM_WGRAD_STAGES_32 : 2;
  static constexpr uint32_t OFF_BAR = NST * STAGE;
  static constexpr uint32_t TMEM_COLS = 3 * WN <= 256 ? 256 : 512;
  static_assert(2 * NST + 1 <= 8, "barrier slots");
  static constexpr uint32_t SMEM = OFF_BAR + 8 * 8 + 16 + 1024;
  static_assert(WR % JN == 0, "whole row groups per item");
  static_assert(OFF_BAR + 8 * 8 + 16 + 1024 <= 232448, "shared memory");
};

template <int C8_IN>
__global__ void __launch_bounds__(kConvThreads, 1) conv3x3_wgrad_kernel(const WgradArgs a) {
  using G = WgradGeom<C8_IN>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::OFF_BAR);
  uint64_t* full = bars;               // [NST]
  uint64_t* empty = bars + G::NST;     // [NST]
  uint64_t* done = bars + 2 * G::NST;  // [1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + G::OFF_BAR + 64);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  grid_dep_launch();
  grid_dep_wait();
  if (threadIdx.x == 0) {
    for (int s = 0; s < G::NST; ++s) {
      tc::mbar_init(&full[s], 2);  // the X and the G tile loads each arrive once
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, G::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t sbase = tc::smem_u32(smem);
  const int my_items = blockIdx.x < a.n_items ? (a.n_items - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (warp == 0) {
    for (int it = 0, t = blockIdx.x; t < a.n_items; t += gridDim.x, ++it) {
      const int s = it % G::NST, use = it / G::NST;
      if (!tc::mbar_wait(&empty[s], (use & 1) ^ 1)) {
        if (lane == 0) set_err(a.err, 11);
        break;
      }
      const int sx = t % a.segs_w, rest = t / a.segs_w;
      const int y0 = (rest % a.yblocks) * G::WR, b = rest / a.yblocks;
      load_tile(a.x, a.H, a.W, C8_IN, b, y0 - 1, G::XROWS, sx * kTW - 1, kBoxW, smem + s * G::STAGE, &full[s], lane);
      load_tile(a.g, a.H, a.W, 4, b, y0, G::WR, sx * kTW, kTW, smem + s * G::STAGE + G::XBYTES, &full[s], lane);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = tc::make_idesc_bf16(128, G::WN, true, true);
      constexpr uint32_t x_hi = tc::desc_hi(G::P), g_hi = tc::desc_hi(G::GP);
      for (int it = 0, t = blockIdx.x; t < a.n_items; t += gridDim.x, ++it) {
        const int s = it % G::NST, use = it / G::NST;
        if (!tc::mbar_wait(&full[s], use & 1)) {
          set_err(a.err, 12);
          break;
        }
        tc::tc_fence_after();
        // A: M = (input row, ci) groups of 8 channels every P bytes; K = pixels, 8-pixel groups 128 B apart.
        // B: N = (output row, co) groups of 8 every GP bytes; K = pixels.
        const uint32_t x_lo = tc::desc_lo(sbase + s * G::STAGE, 128);
        const uint32_t g_lo = tc::desc_lo(sbase + s * G::STAGE + G::XBYTES, 128);
        // Row group q: output rows y0 + q JN + jj (N = (jj, co)) against input rows
        // y0 - 1 + q JN + m (M = (m, ci)); the product lands at kernel row kh = m - jj.
#pragma unroll 1
        for (int q = 0; q < G::NGRP; ++q) {
          const uint32_t xq = x_lo + ((q * G::JN * G::RS) >> 4), gq = g_lo + ((q * G::JN * 4 * G::GP) >> 4);
          const uint32_t acc0 = (it > 0 || q > 0) ? 1u : 0u;
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
            if (a.centre_only && dx != 1) continue;
#pragma unroll
            for (int ks = 0; ks < kTW / 16; ++ks) {
              const uint64_t ad = tc::desc_join(xq + ((dx * 16 + ks * 256) >> 4), x_hi);
              const uint64_t bd = tc::desc_join(gq + ((ks * 256) >> 4), g_hi);
              tc::mma_bf16(tmem + dx * G::WN, ad, bd, idesc, ks > 0 ? 1u : acc0);
            }
          }
        }
        tc::mma_commit(&empty[s]);
      }
      tc::mma_commit(done);
    }
  } else {
    const int q = warp & 3;
    const int m = q * 32 + lane;  // accumulator row: (input row slot, ci)
    bool ok = true;
    if (my_items > 0) {
      ok = tc::mbar_wait(done, 0);
      if (!ok) set_err(a.err, 13);
      tc::tc_fence_after();
    }
#pragma unroll 1
    for (int dx = 0; dx < 3; ++dx) {
#pragma unroll 1
      for (int cb = 0; cb < G::WN; cb += 32) {
        uint32_t v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(dx * G::WN + cb), v);
        tc::tmem_wait_ld();
        float4* dst =
            reinterpret_cast<float4*>(a.partial + (((size_t)blockIdx.x * 3 + dx) * 128 + m) * G::WN + cb);
#pragma unroll
        for (int c = 0; c < 32; c += 4) {
          float4 f;
          const bool z = my_items == 0 || !ok;
          f.x = z ? 0.f : __uint_as_float(v[c + 0]);
          f.y = z ? 0.f : __uint_as_float(v[c + 1]);
          f.z = z ? 0.f : __uint_as_float(v[c + 2]);
          f.w = z ? 0.f : __uint_as_float(v[c + 3]);
          dst[c / 4] = f;
        }
      }
    }
    tc::tc_fence_before();
  }
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, G::TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// fused backward of a 32 -> 32 channel layer: data gradient + weight gradient
// ---------------------------------------------------------------------------
// Both gradients of layer l read the gradient G_l of its pre-activation, and the
// data gradient's LeakyReLU mask is the layer's input X = act_{l-1}, which the
// weight gradient reads as well.  One kernel streams each 4-row tile of G_l and
// of X once (haloed boxes, 6 rows x 130 pixels), and per tile
//   * accumulates the data gradient in TMEM exactly as conv3x3_kernel<4, 4, dgrad>
//     does (A = the G box, B = the flipped weights), the epilogue masking it with
//     the X box read from shared memory (no global mask read) and storing
//     G_{l-1}, with the per-CTA bias-gradient sums;
//   * adds X^T G over the tile's pixels into the CTA's weight-gradient
//     accumulators exactly as conv3x3_wgrad_kernel<4> does for its 4-row work
//     item (A = the X box, MN-major; B = rows 1..4 of the G box from pixel 1).
// The work items are the weight-gradient kernel's (the same 4-row blocks in the
// same order per CTA), so the partials are those of conv3x3_wgrad_kernel<4>
// bit for bit, and each output row's data gradient sums its taps in the order of
// conv3x3_kernel's.  Shared memory: 2 stages x (G box + X box) + the weights;
// TMEM: 2 x 4 x 32 data-gradient columns, then 3 x 64 weight-gradient columns.
// A stage is released when its MMAs completed (one commit) and each of the 8
// epilogue warps has read its mask rows (one arrival each).
struct BwdGeom {
  static constexpr int R = 4;                           // output rows per tile
  static constexpr int C8 = 4;                          // 32 channels
  static constexpr int NST = 2;
  static constexpr int NACC = 2;                        // data-gradient accumulator sets
  static constexpr uint32_t P = kBoxW * 16;             // chunk plane stride
  static constexpr uint32_t RS = C8 * P;                // row stride
  static constexpr uint32_t BOX = (R + 2) * RS;         // one haloed box
  static constexpr uint32_t STAGE = 2 * BOX;            // G box, then X box
  static constexpr uint32_t WBYTES = 9 * C8 * kCout * 16;
  static constexpr uint32_t OFF_W = NST * STAGE;
  static constexpr uint32_t OFF_BAR = OFF_W + WBYTES;
  static constexpr uint32_t OFF_RED = OFF_BAR + 256;    // the finishing reductions' [8][32] exchange
  static constexpr uint32_t SMEM = OFF_RED + kFinWarps * kFinCols * 4 + 1024;
  // weight gradient (conv3x3_wgrad_kernel<4>'s item geometry)
  static constexpr int NROW = 128 / (C8 * 8);           // input rows per M = 128
  static constexpr int JN = NROW - 2;                   // output rows per MMA (N = JN x 32)
  static constexpr int NGRP = R / JN;
  static constexpr int WN = JN * kCout;
  static constexpr uint32_t DCOLS = NACC * R * kCout;   // data-gradient TMEM columns
  static constexpr uint32_t TMEM_COLS = 512;
  static_assert(JN == WgradGeom<4>::JN && WN == WgradGeom<4>::WN && R == WgradGeom<4>::WR,
                "the weight-gradient partials keep conv3x3_wgrad_kernel<4>'s layout");
  static_assert(DCOLS + 3 * WN <= TMEM_COLS, "TMEM columns");
  static_assert(SMEM <= 232448, "shared memory");
};

struct BwdArgs {
  int B, H, W;
  int tiles_w, tiles_h, n_tiles;
  const __nv_bfloat16* g;      // G_l [B][H][4][W][8]
  const __nv_bfloat16* x;      // X = act_{l-1} [B][H][4][W][8]
  const __nv_bfloat16* wpack;  // the layer's dgrad pack [9][4][32][8]
  __nv_bfloat16* out;          // G_{l-1} [B][H][4][W][8]
  float* db_partial;           // [gridDim.x][32]
  float* w_partial;            // [gridDim.x][3][128][WN]
  float alpha;
  int* err;
  // the previous launch's (the layer above's) partials and where their sums go; NULL: none
  const float* prev_w_partial;  // [gridDim.x][3][128][WN] -> prev_w_out [3][3][32][32]
  const float* prev_db_partial; // [gridDim.x][32] -> prev_db_out [32]
  float* prev_w_out;
  float* prev_db_out;
};

__global__ void __launch_bounds__(kConvFwdThreads, 1) conv3x3_bwd_kernel(const BwdArgs a) {
  using G = BwdGeom;
  constexpr int R = G::R, NST = G::NST, NACC = G::NACC;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::OFF_BAR);
  uint64_t* full = bars;                     // [NST] both boxes landed
  uint64_t* empty = bars + NST;              // [NST] MMAs done + masks read
  uint64_t* tfull = bars + 2 * NST;          // [NACC]
  uint64_t* tempty = bars + 2 * NST + NACC;  // [NACC]
  uint64_t* done = bars + 2 * NST + 2 * NACC;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + G::OFF_BAR + 128);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  grid_dep_launch();
  grid_dep_wait();
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.wpack);
    uint4* dst = reinterpret_cast<uint4*>(smem + G::OFF_W);
    for (int i = threadIdx.x; i < (int)(G::WBYTES / 16); i += kConvFwdThreads) dst[i] = src[i];
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      tc::mbar_init(&full[s], 2);                   // the two boxes' loads
      tc::mbar_init(&empty[s], 1 + kConvEpiWarps);  // MMA commit + one arrival per epilogue warp
    }
    for (int s = 0; s < NACC; ++s) {
      tc::mbar_init(&tfull[s], 1);
      tc::mbar_init(&tempty[s], 32 * kConvEpiWarps);
    }
    tc::mbar_init(done, 1);
    tc::fence_mbar_init();
  }
  tc::fence_proxy_async_smem();
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, G::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t sbase = tc::smem_u32(smem);
  const int my_tiles = (int)blockIdx.x < a.n_tiles ? (a.n_tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

  if (warp == 0) {
    // ---------------- producer ----------------
    for (int it = 0, t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
      const int s = it % NST, use = it / NST;
      if (!tc::mbar_wait(&empty[s], (use & 1) ^ 1)) {
        if (lane == 0) set_err(a.err, 21);
        break;
      }
      const int txi = t % a.tiles_w, rest = t / a.tiles_w;
      const int tyi = rest % a.tiles_h, b = rest / a.tiles_h;
      unsigned char* st = smem + s * G::STAGE;
      load_tile(a.g, a.H, a.W, G::C8, b, tyi * R - 1, R + 2, txi * kTW - 1, kBoxW, st, &full[s], lane);
      load_tile(a.x, a.H, a.W, G::C8, b, tyi * R - 1, R + 2, txi * kTW - 1, kBoxW, st + G::BOX, &full[s], lane);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t d_hi = tc::desc_hi(128), p_hi = tc::desc_hi(G::P);
      constexpr uint32_t wg_idesc = tc::make_idesc_bf16(128, G::WN, true, true);
      const uint32_t w_lo = tc::desc_lo(sbase + G::OFF_W, kWRowsN * 16);
      const uint32_t wtm = tmem + G::DCOLS;  // weight-gradient accumulators [3][WN]
      bool ok = true;
      for (int it = 0, t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
        const int s = it % NST, use = it / NST, acc = it % NACC, ause = it / NACC;
        if (!tc::mbar_wait(&tempty[acc], (ause & 1) ^ 1) || !tc::mbar_wait(&full[s], use & 1)) {
          set_err(a.err, 22);
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const uint32_t gbox = sbase + s * G::STAGE, xbox = gbox + G::BOX;
        // data gradient: conv3x3_kernel's sliding-window accumulation over the G box
        const uint32_t in_lo = tc::desc_lo(gbox, G::P);
        const uint32_t dset = tmem + (uint32_t)(acc * R * kCout);
#pragma unroll
        for (int i = 0; i < R + 2; ++i) {
          const int dlo = i - (R - 1) > 0 ? i - (R - 1) : 0;
          const int dhi = i < 2 ? i : 2;
          const int ndy = dhi - dlo + 1;
          const uint32_t dcol = dset + (uint32_t)(kCout * (R - 1 - i + dlo));
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
            for (int ks = 0; ks < G::C8 / 2; ++ks) {
              const uint32_t aoff = (i * G::RS + dx * 16 + ks * 2 * G::P) >> 4;
              const uint32_t boff = (((dx * G::C8 + ks * 2) * kWRowsN + dlo * kCout) * 16) >> 4;
              const uint64_t ad = tc::desc_join(in_lo + aoff, d_hi);
              if (dx == 0 && ks == 0 && dlo == 0) {
                tc::mma_bf16(dcol, ad, tc::desc_join(w_lo + boff, d_hi), tc::make_idesc_bf16(128, kCout, false, false),
                             0u);
                if (ndy > 1)
                  tc::mma_bf16(dcol + kCout, ad, tc::desc_join(w_lo + boff + ((kCout * 16) >> 4), d_hi),
                               tc::make_idesc_bf16(128, kCout * (ndy - 1), false, false), 1u);
              } else {
                tc::mma_bf16(dcol, ad, tc::desc_join(w_lo + boff, d_hi),
                             tc::make_idesc_bf16(128, kCout * ndy, false, false), 1u);
              }
            }
          }
        }
        // weight gradient: conv3x3_wgrad_kernel<4>'s item over the X box and rows 1..R of the G box
        const uint32_t x_lo = tc::desc_lo(xbox, 128), g_lo = tc::desc_lo(gbox + G::RS + 16, 128);
#pragma unroll 1
        for (int q = 0; q < G::NGRP; ++q) {
          const uint32_t xq = x_lo + ((q * G::JN * G::RS) >> 4), gq = g_lo + ((q * G::JN * G::RS) >> 4);
          const uint32_t acc0 = (it > 0 || q > 0) ? 1u : 0u;
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
            for (int ks = 0; ks < kTW / 16; ++ks) {
              const uint64_t ad = tc::desc_join(xq + ((dx * 16 + ks * 256) >> 4), p_hi);
              const uint64_t bd = tc::desc_join(gq + ((ks * 256) >> 4), p_hi);
              tc::mma_bf16(wtm + dx * G::WN, ad, bd, wg_idesc, ks > 0 ? 1u : acc0);
            }
          }
        }
        tc::mma_commit(&empty[s]);
        tc::mma_commit(&tfull[acc]);
      }
      if (ok) tc::mma_commit(done);
    }
  } else {
    // ---------------- epilogue (warps 2 .. 9) ----------------
    constexpr int RH = R / 2;
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int r0 = half * RH;
    const int p = q * 32 + lane;
    if (a.prev_w_partial) {
      // The layer above's weight and bias gradients from its partials, while this kernel's first
      // tiles load: the eight epilogue warps are the eight warps of wgrad_finish_kernel (one
      // (tap, ci) row per step, the same partials in the same order) and of reduce_partials_kernel.
      static_assert(kConvEpiWarps == kFinWarps, "the epilogue warps are the finishing reduction's warps");
      float(*red)[kFinCols] = reinterpret_cast<float(*)[kFinCols]>(smem + G::OFF_RED);
      const int ew = warp - 2;
      for (int gi = blockIdx.x; gi < 9 * kCout; gi += gridDim.x) {
        const int ci = gi % kCout, tap = gi / kCout;
        red[ew][lane] = finish_sum<2, 1>(a.prev_w_partial, (int)gridDim.x, ew, lane, tap % 3, tap / 3, ci, 32);
        asm volatile("bar.sync 1, %0;\n" ::"n"(32 * kConvEpiWarps) : "memory");
        if (ew == 0) {
          float tsum = 0.f;
#pragma unroll
          for (int w2 = 0; w2 < kFinWarps; ++w2) tsum += red[w2][lane];
          a.prev_w_out[(size_t)gi * kFinCols + lane] = tsum;
        }
        asm volatile("bar.sync 1, %0;\n" ::"n"(32 * kConvEpiWarps) : "memory");
      }
      if (ew == 0)
        for (int i = blockIdx.x; i < kCout; i += gridDim.x) {
          const float sdb = partial_sum(a.prev_db_partial, (int)gridDim.x, kCout, i, lane);
          if (lane == 0) a.prev_db_out[i] = sdb;
        }
    }
    float dbacc[kCout];
#pragma unroll
    for (int c = 0; c < kCout; ++c) dbacc[c] = 0.f;
    bool ok = true;
    for (int it = 0, t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
      const int s = it % NST, use = it / NST, acc = it % NACC, ause = it / NACC;
      const int txi = t % a.tiles_w, rest = t / a.tiles_w;
      const int tyi = rest % a.tiles_h, b = rest / a.tiles_h;
      const int x = txi * kTW + p;
      if (!tc::mbar_wait(&full[s], use & 1)) {
        set_err(a.err, 23);
        ok = false;
        break;
      }
      // this warp's mask rows from the X box (row r of the tile = box row r + 1, pixel p = box pixel p + 1)
      uint4 mk[RH][4];
      const unsigned char* xb = smem + s * G::STAGE + G::BOX;
#pragma unroll
      for (int rr = 0; rr < RH; ++rr)
#pragma unroll
        for (int ch = 0; ch < 4; ++ch)
          mk[rr][ch] = *reinterpret_cast<const uint4*>(xb + (r0 + rr + 1) * G::RS + ch * G::P + (p + 1) * 16);
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&empty[s]);
      if (!tc::mbar_wait(&tfull[acc], ause & 1)) {
        set_err(a.err, 24);
        ok = false;
        break;
      }
      tc::tc_fence_after();
#pragma unroll
      for (int rr = 0; rr < RH; ++rr) {
        const int r = r0 + rr;
        uint32_t v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((acc * R + (R - 1 - r)) * kCout), v);
        tc::tmem_wait_ld();
        const int y = tyi * R + r;
        if (y < a.H && x < a.W) {
          const size_t pix = (((size_t)b * a.H + y) * 4) * a.W + x;
          float f[kCout];
#pragma unroll
          for (int c = 0; c < kCout; ++c) f[c] = __uint_as_float(v[c]);
#pragma unroll
          for (int ch = 0; ch < 4; ++ch) {
            const uint32_t mw[4] = {mk[rr][ch].x, mk[rr][ch].y, mk[rr][ch].z, mk[rr][ch].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&mw[e]);
              const float lo = __low2float(h), hi = __high2float(h);
              const int c = ch * 8 + e * 2;
              f[c] *= lo > 0.f ? 1.f : a.alpha;
              f[c + 1] *= hi > 0.f ? 1.f : a.alpha;
            }
          }
#pragma unroll
          for (int c = 0; c < kCout; ++c) dbacc[c] += f[c];
          uint4* o = reinterpret_cast<uint4*>(a.out);
#pragma unroll
          for (int ch = 0; ch < 4; ++ch) {
            uint4 w;
            w.x = pack_bf16x2(f[ch * 8 + 0], f[ch * 8 + 1]);
            w.y = pack_bf16x2(f[ch * 8 + 2], f[ch * 8 + 3]);
            w.z = pack_bf16x2(f[ch * 8 + 4], f[ch * 8 + 5]);
            w.w = pack_bf16x2(f[ch * 8 + 6], f[ch * 8 + 7]);
            o[pix + (size_t)ch * a.W] = w;
          }
        }
      }
      tc::tc_fence_before();
      tc::mbar_arrive(&tempty[acc]);
    }
    // weight-gradient accumulators -> this CTA's partials: warp (q, half) takes lane quarter q and
    // the half-th 32 of each kernel column's WN = 64 accumulator columns
    if (ok && my_tiles > 0) {
      ok = tc::mbar_wait(done, 0);
      if (!ok) set_err(a.err, 25);
      tc::tc_fence_after();
    }
    const int m = q * 32 + lane;
#pragma unroll 1
    for (int dx = 0; dx < 3; ++dx) {
      const int cb = half * 32;
      uint32_t v[32];
      tc::tmem_ld32(tmem + G::DCOLS + ((uint32_t)(q * 32) << 16) + (uint32_t)(dx * G::WN + cb), v);
      tc::tmem_wait_ld();
      float4* dst = reinterpret_cast<float4*>(a.w_partial + (((size_t)blockIdx.x * 3 + dx) * 128 + m) * G::WN + cb);
#pragma unroll
      for (int c = 0; c < 32; c += 4) {
        const bool z = my_tiles == 0 || !ok;
        float4 f4;
        f4.x = z ? 0.f : __uint_as_float(v[c + 0]);
        f4.y = z ? 0.f : __uint_as_float(v[c + 1]);
        f4.z = z ? 0.f : __uint_as_float(v[c + 2]);
        f4.w = z ? 0.f : __uint_as_float(v[c + 3]);
        dst[c / 4] = f4;
      }
    }
    // bias-gradient partial sums: warp reduction, then a fixed-order CTA sum below
#pragma unroll
    for (int c = 0; c < kCout; ++c) {
      float v = dbacc[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      dbacc[c] = v;
    }
    // every MMA of this CTA has completed (the last tfull / done wait), so the weight area is free
    float* red = reinterpret_cast<float*>(smem + G::OFF_W);
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < kCout; ++c) red[(warp - 2) * kCout + c] = dbacc[c];
    }
    tc::tc_fence_before();
  }
  __syncthreads();
  if (threadIdx.x < kCout) {
    const float* red = reinterpret_cast<const float*>(smem + G::OFF_W);
    float sum = red[threadIdx.x];
#pragma unroll
    for (int w = 1; w < kConvEpiWarps; ++w) sum += red[w * kCout + threadIdx.x];  // fixed order
    a.db_partial[(size_t)blockIdx.x * kCout + threadIdx.x] = sum;
  }
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, G::TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <typename K>
static int set_smem(K kernel, uint32_t bytes, bool* done) {
  if (!*done) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) {
      set_error("conv smem attribute: %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
    *done = true;
  }
  return IGM_OK;
}

constexpr int kRows = IGM_CONV_ROWS;
static_assert(kRows == 2 || kRows == 4 || kRows == 8, "IGM_CONV_ROWS: 2, 4 or 8");

template <int C8_IN, int EPI>
static int conv_launch(int B, int H, int W, const void* x, const void* wpack, const float* bias, const void* amask,
                       void* y, float* db_partial, int db_slots, float alpha, int* err, cudaStream_t st) {
  using G = ConvGeom<C8_IN, kRows>;
  static bool configured = false;
  int rc = set_smem(conv3x3_kernel<C8_IN, kRows, EPI>, G::SMEM, &configured);
  if (rc) return rc;
  IGM_CHECK_ARG(((uintptr_t)x & 15) == 0 && ((uintptr_t)y & 15) == 0, IGM_ERR_BAD_ARGUMENT,
                "igm_conv3x3: activations must be 16-byte aligned");
  ConvArgs a{};
  a.B = B; a.H = H; a.W = W;
  a.x = (const __nv_bfloat16*)x;
  a.tiles_w = (W + kTW - 1) / kTW;
  a.tiles_h = (H + kRows - 1) / kRows;
  a.n_tiles = B * a.tiles_w * a.tiles_h;
  a.wpack = (const __nv_bfloat16*)wpack;
  a.bias = bias;
  a.amask = (const __nv_bfloat16*)amask;
  a.out = (__nv_bfloat16*)y;
  a.alpha = alpha;
  a.err = err;
  int grid = a.n_tiles < sm_count() ? a.n_tiles : sm_count();
  if (db_partial) {
    if (db_slots < grid) grid = db_slots;
    a.db_partial = db_partial;
  }
  if (grid < 1) grid = 1;
  if (db_partial && grid < db_slots) {
    // each CTA writes its own slot of bias-gradient partials; the slots beyond the grid are zeroed
    // here, so the caller's reduction over all db_slots needs no cleared buffer
    cudaError_t e = cudaMemsetAsync(db_partial + (size_t)grid * kCout, 0,
                                    (size_t)(db_slots - grid) * kCout * sizeof(float), st);
    if (e != cudaSuccess) {
      set_error("igm_conv3x3: clearing the partials: %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
  }
  launch_pdl(conv3x3_kernel<C8_IN, kRows, EPI>, dim3(grid), dim3(kConvFwdThreads), G::SMEM, st, a);
  return launch_status("conv3x3_kernel");
}

template <int C8_IN>
static int wgrad_launch(int B, int H, int W, const void* x, const void* g, float* partial, int n_parts, int* err,
                        cudaStream_t st, int centre_only = 0) {
  using G = WgradGeom<C8_IN>;
  static bool configured = false;
  int rc = set_smem(conv3x3_wgrad_kernel<C8_IN>, G::SMEM, &configured);
  if (rc) return rc;
  IGM_CHECK_ARG(((uintptr_t)x & 15) == 0 && ((uintptr_t)g & 15) == 0, IGM_ERR_BAD_ARGUMENT,
                "igm_conv3x3_wgrad: activations must be 16-byte aligned");
  WgradArgs a{};
  a.B = B; a.H = H; a.W = W;
  a.segs_w = (W + kTW - 1) / kTW;
  a.yblocks = (H + G::WR - 1) / G::WR;
  a.n_items = B * a.yblocks * a.segs_w;
  a.x = (const __nv_bfloat16*)x;
  a.g = (const __nv_bfloat16*)g;
  a.partial = partial;
  a.err = err;
  a.centre_only = centre_only;
  launch_pdl(conv3x3_wgrad_kernel<C8_IN>, dim3(n_parts), dim3(kConvThreads), G::SMEM, st, a);
  return launch_status("conv3x3_wgrad_kernel");
}

}  // namespace igm

using namespace igm;

extern "C" int igm_conv3x3(int mode, int batch, int height, int width, int cin, const void* x, const void* wpack,
                           const float* bias, const void* act_mask, void* y, float* db_partials, int db_slots,
                           float alpha, int* err, void* stream) {
  IGM_CHECK_ARG(batch >= 1 && height >= 1 && width >= 1 && batch <= 65535, IGM_ERR_BAD_SHAPE,
                "igm_conv3x3: bad shape %dx%dx%d", batch, height, width);
  IGM_CHECK_ARG(cin == 16 || cin == 32, IGM_ERR_UNSUPPORTED, "igm_conv3x3: cin must be 16 or 32 (got %d)", cin);
  IGM_CHECK_ARG(x && wpack && y, IGM_ERR_BAD_ARGUMENT, "igm_conv3x3: NULL argument");
  IGM_CHECK_ARG(mode == IGM_CONV_FWD_LEAKY || mode == IGM_CONV_DGRAD, IGM_ERR_BAD_ARGUMENT,
                "igm_conv3x3: unknown mode %d", mode);
  IGM_CHECK_ARG(mode != IGM_CONV_DGRAD || act_mask, IGM_ERR_BAD_ARGUMENT, "igm_conv3x3: dgrad needs act_mask");
  IGM_CHECK_ARG(mode != IGM_CONV_FWD_LEAKY || bias, IGM_ERR_BAD_ARGUMENT, "igm_conv3x3: forward needs bias");
  cudaStream_t st = as_stream(stream);
  if (mode == IGM_CONV_FWD_LEAKY) {
    if (cin == 16)
      return conv_launch<2, kEpiFwdLeaky>(batch, height, width, x, wpack, bias, nullptr, y, nullptr, 0, alpha, err, st);
    return conv_launch<4, kEpiFwdLeaky>(batch, height, width, x, wpack, bias, nullptr, y, nullptr, 0, alpha, err, st);
  }
  IGM_CHECK_ARG(cin == 32, IGM_ERR_UNSUPPORTED, "igm_conv3x3: dgrad needs cin == 32");
  return conv_launch<4, kEpiDgrad>(batch, height, width, x, wpack, nullptr, act_mask, y, db_partials, db_slots, alpha,
                                   err, st);
}

extern "C" int igm_conv3x3_wgrad(int batch, int height, int width, int cin, const void* x, const void* g,
                                 float* partials, int n_parts, int* err, void* stream) {
  IGM_CHECK_ARG(batch >= 1 && height >= 1 && width >= 1, IGM_ERR_BAD_SHAPE, "igm_conv3x3_wgrad: bad shape");
  IGM_CHECK_ARG(cin == 16 || cin == 32, IGM_ERR_UNSUPPORTED, "igm_conv3x3_wgrad: cin must be 16 or 32");
  IGM_CHECK_ARG(x && g && partials && n_parts >= 1, IGM_ERR_BAD_ARGUMENT, "igm_conv3x3_wgrad: bad argument");
  cudaStream_t st = as_stream(stream);
  if (cin == 16) return wgrad_launch<2>(batch, height, width, x, g, partials, n_parts, err, st);
  return wgrad_launch<4>(batch, height, width, x, g, partials, n_parts, err, st);
}

extern "C" int igm_conv3x3_backward(int batch, int height, int width, const void* g, const void* wpack_bwd,
                                    const void* x, void* g_prev, float* db_partials, float* w_partials, int n_parts,
                                    float alpha, int* err, const float* prev_w_partials,
                                    const float* prev_db_partials, float* prev_w_out, float* prev_db_out,
                                    void* stream) {
  using G = BwdGeom;
  IGM_CHECK_ARG(batch >= 1 && height >= 1 && width >= 1 && batch <= 65535, IGM_ERR_BAD_SHAPE,
                "igm_conv3x3_backward: bad shape %dx%dx%d", batch, height, width);
  IGM_CHECK_ARG(g && wpack_bwd && x && g_prev && db_partials && w_partials && n_parts >= 1, IGM_ERR_BAD_ARGUMENT,
                "igm_conv3x3_backward: NULL argument");
  IGM_CHECK_ARG(((uintptr_t)g & 15) == 0 && ((uintptr_t)x & 15) == 0 && ((uintptr_t)g_prev & 15) == 0,
                IGM_ERR_BAD_ARGUMENT, "igm_conv3x3_backward: activations must be 16-byte aligned");
  const bool prev = prev_w_partials != nullptr;
  IGM_CHECK_ARG(prev == (prev_db_partials != nullptr) && prev == (prev_w_out != nullptr) &&
                    prev == (prev_db_out != nullptr),
                IGM_ERR_BAD_ARGUMENT, "igm_conv3x3_backward: the four prev_* pointers are all set or all NULL");
  IGM_CHECK_ARG(!prev || (prev_w_partials != w_partials && prev_db_partials != db_partials), IGM_ERR_BAD_ARGUMENT,
                "igm_conv3x3_backward: the previous partials must not be this call's partial buffers");
  static bool configured = false;
  int rc = set_smem(conv3x3_bwd_kernel, G::SMEM, &configured);
  if (rc) return rc;
  BwdArgs a{};
  a.B = batch; a.H = height; a.W = width;
  a.tiles_w = (width + kTW - 1) / kTW;
  a.tiles_h = (height + G::R - 1) / G::R;
  a.n_tiles = batch * a.tiles_w * a.tiles_h;
  a.g = (const __nv_bfloat16*)g;
  a.x = (const __nv_bfloat16*)x;
  a.wpack = (const __nv_bfloat16*)wpack_bwd;
  a.out = (__nv_bfloat16*)g_prev;
  a.db_partial = db_partials;
  a.w_partial = w_partials;
  a.alpha = alpha;
  a.err = err;
  a.prev_w_partial = prev_w_partials;
  a.prev_db_partial = prev_db_partials;
  a.prev_w_out = prev_w_out;
  a.prev_db_out = prev_db_out;
  launch_pdl(conv3x3_bwd_kernel, dim3(n_parts), dim3(kConvFwdThreads), G::SMEM, as_stream(stream), a);
  return launch_status("conv3x3_bwd_kernel");
}

extern "C" int igm_conv3x3_stack(int batch, int height, int width, int nlayers, const void* x, void* const* outs,
                                 const void* const* wpacks, const float* const* biases, int* flags, int epoch,
                                 float alpha, int* err, void* stream) {
  constexpr int R = kRows;
  using G = ConvGeom<4, R>;
  constexpr uint32_t SMEM = G::OFF_W + 2 * G::WBYTES + 128 + 16 + 1024;
  static_assert(SMEM <= 232448, "shared memory");
  IGM_CHECK_ARG(batch >= 1 && height >= 1 && width >= 1 && batch <= 65535, IGM_ERR_BAD_SHAPE,
                "igm_conv3x3_stack: bad shape %dx%dx%d", batch, height, width);
  IGM_CHECK_ARG(nlayers >= 1 && nlayers <= kStackMax, IGM_ERR_BAD_SHAPE, "igm_conv3x3_stack: 1 .. %d layers",
                kStackMax);
  IGM_CHECK_ARG(x && outs && wpacks && biases && flags && epoch != 0, IGM_ERR_BAD_ARGUMENT,
                "igm_conv3x3_stack: NULL argument or zero epoch");
  StackArgs a{};
  a.B = batch; a.H = height; a.W = width;
  a.tiles_w = (width + kTW - 1) / kTW;
  a.tiles_h = (height + R - 1) / R;
  a.n_tiles = batch * a.tiles_w * a.tiles_h;
  a.nlayers = nlayers;
  a.in = (const __nv_bfloat16*)x;
  IGM_CHECK_ARG(((uintptr_t)x & 15) == 0, IGM_ERR_BAD_ARGUMENT, "igm_conv3x3_stack: activations must be 16-byte aligned");
  for (int k = 0; k < nlayers; ++k) {
    IGM_CHECK_ARG(outs[k] && wpacks[k] && biases[k] && ((uintptr_t)outs[k] & 15) == 0 && ((uintptr_t)wpacks[k] & 15) == 0,
                  IGM_ERR_BAD_ARGUMENT, "igm_conv3x3_stack: layer %d: NULL or unaligned pointer", k);
    a.out[k] = (__nv_bfloat16*)outs[k];
    a.wpack[k] = (const __nv_bfloat16*)wpacks[k];
    a.bias[k] = biases[k];
  }
  a.flags = flags;
  a.epoch = epoch;
  a.alpha = alpha;
  a.err = err;
  static bool configured = false;
  int rc = set_smem(conv3x3_stack_kernel<R>, SMEM, &configured);
  if (rc) return rc;
  const int grid = a.n_tiles < sm_count() ? a.n_tiles : sm_count();
  // cooperative: every CTA resident at once, which the inter-CTA tile flags rely on
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kConvFwdThreads);
  cfg.dynamicSmemBytes = SMEM;
  cfg.stream = as_stream(stream);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, conv3x3_stack_kernel<R>, a);
  return launch_status("conv3x3_stack_kernel");
}

extern "C" size_t igm_conv3x3_stack_flags_len(int batch, int height, int width, int nlayers) {
  return (size_t)nlayers * batch * ((width + kTW - 1) / kTW) * ((height + kRows - 1) / kRows);
}

extern "C" int igm_conv1x1_wgrad(int batch, int height, int width, const void* x, const void* g, float* partials,
                                 int n_parts, int* err, void* stream) {
  IGM_CHECK_ARG(batch >= 1 && height >= 1 && width >= 1, IGM_ERR_BAD_SHAPE, "igm_conv1x1_wgrad: bad shape");
  IGM_CHECK_ARG(x && g && partials && n_parts >= 1, IGM_ERR_BAD_ARGUMENT, "igm_conv1x1_wgrad: bad argument");
  return wgrad_launch<4>(batch, height, width, x, g, partials, n_parts, err, as_stream(stream), 1);
}

extern "C" size_t igm_conv3x3_wgrad_partial_len(int cin) {
  if (cin == 32) return (size_t)3 * 128 * WgradGeom<4>::WN;
  if (cin == 16) return (size_t)3 * 128 * WgradGeom<2>::WN;
  return 0;
}

extern "C" int igm_conv_sm_count(void) { return sm_count(); }
