// Blatter-Pattyn energy, its hand-written adjoint, and the fused
// energy + adjoint + Adam solver iteration, as ONE stencil kernel.
//
// Reference: igm/processes/iceflow/energy/cost_shear.py:55-209,
// cost_sliding_weertman.py:23-43, cost_gravity.py:24-69 (staggered grid,
// Lagrange basis), energy/utils.py:11-25, utils/gradient/compute_gradient.py:3-16,
// solve/solve.py:45-114 (the Adam loop with EarlyStopping).
//
// Geometry.  A staggered cell (j,i) has corner nodes a=(j,i), b=(j,i+1),
// c=(j+1,i), d=(j+1,i+1).  Per level k the energy needs, per cell,
//   Us = (d+c+b+a)/4,  Dx = ((b-a)/dx + (d-c)/dx)/2,  Dy = ((c-a)/dx + (d-b)/dx)/2
// for U and V (stag4h and the staggered horizontal derivatives), and per
// layer l (between levels l and l+1) the stag2v averages and the vertical
// derivative (Us[l+1]-Us[l]) / (dzeta[l] max(thk_s, thr)).
//
// Kernel shape.  A tile is 32 cells in x (one per lane) and TYC cell rows;
// each thread evaluates TWO vertically adjacent cells, whose values travel as
// a pair: for float the pair arithmetic runs on sm_100's packed FP32x2 pipe
// (one instruction for both cells), which halves the instruction count of the
// per-cell math that bounds this kernel; a warp reads whole tile rows, free of
// shared-memory bank conflicts.  A tile's cells [j0-1, j0-1+TYC) x
// [i0-1, i0+31) cover every cell touching its (TYC-1) x 31 output nodes, so
// the adjoint (a scatter from cells to their 4 corners) becomes a gather
// inside the CTA with no atomics: the horizontal half by warp shuffles, the
// vertical half through one shared-memory row per warp.
// CTAs are persistent (as many as fit on the device) and walk their tiles
// level by level as one sequence: each level's node tile of U and V (and, in
// solver mode, the Adam moments) arrives by TMA (or cp.async when the row pitch
// is not a multiple of 16 bytes) into a ring of stages kept several levels
// ahead of the one being computed -- across tile boundaries -- and a tile's
// 2-D fields arrive while the previous tile is computed.  Each level's node
// outputs (gradient, or the Adam update) are finished two levels later, when
// all of the layers touching them are done.
//
// Energy reduction: per-cell FP32 densities, FP64 per-thread sums over its
// tiles, FP64 block sums, per-CTA partials in the workspace, and the last CTA
// to finish sums them in a fixed order (deterministic for a given device) and,
// in solver mode, runs EarlyStopping on the device.
#include <stdarg.h>

#include <string.h>

#include <initializer_list>
#include <type_traits>
#include <mutex>

#include "common.cuh"
#include "tc.cuh"

namespace igm {

constexpr int kCW = 32;  // cells per CTA row (one per lane)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Element copy global -> shared through the async-copy unit; src_bytes = 0
// zero-fills the destination without reading (used outside the domain).
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool valid) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(smem_u32(dst)), "l"(src), "n"(sizeof(T)),
               "r"(valid ? (int)sizeof(T) : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Node tiles are loaded as boxes of (TYC + 1) rows x BW columns starting at
// the 16-byte aligned column xs <= i0 - 1; the tile's column 0 (node i0 - 1)
// sits at box column ox = i0 - 1 - xs.  Out-of-domain nodes read as zero.
template <typename T> struct Box {
  static constexpr int AL = 16 / (int)sizeof(T);                   // elements per 16 bytes
  static constexpr int BW = ((kCW + 1 + AL - 1 + AL - 1) / AL) * AL;  // >= 33 + (AL - 1), multiple of AL
};

// ---- cell pairs --------------------------------------------------------------
// Two values of adjacent cells.  float: packed FP32x2 instructions (add, mul,
// fma; a - b as fma(b, -1, a), exact); double: two scalar operations.
template <typename T> struct Two { T x, y; };
template <typename T> __device__ __forceinline__ Two<T> two(T s) { return {s, s}; }
template <typename T> __device__ __forceinline__ Two<T> operator+(Two<T> a, Two<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T> __device__ __forceinline__ Two<T> operator-(Two<T> a, Two<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T> __device__ __forceinline__ Two<T> operator*(Two<T> a, Two<T> b) { return {a.x * b.x, a.y * b.y}; }
template <typename T> __device__ __forceinline__ Two<T> fma2(Two<T> a, Two<T> b, Two<T> c) {
  return {fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)};
}
__device__ __forceinline__ float2 f2(Two<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ Two<float> t2(float2 a) { return {a.x, a.y}; }
template <> __device__ __forceinline__ Two<float> operator+(Two<float> a, Two<float> b) {
  return t2(__fadd2_rn(f2(a), f2(b)));
}
template <> __device__ __forceinline__ Two<float> operator-(Two<float> a, Two<float> b) {
  return t2(__ffma2_rn(f2(b), make_float2(-1.f, -1.f), f2(a)));
}
template <> __device__ __forceinline__ Two<float> operator*(Two<float> a, Two<float> b) {
  return t2(__fmul2_rn(f2(a), f2(b)));
}
template <> __device__ __forceinline__ Two<float> fma2(Two<float> a, Two<float> b, Two<float> c) {
  return t2(__ffma2_rn(f2(a), f2(b), f2(c)));
}
template <typename T> __device__ __forceinline__ Two<T> sel(bool px, bool py, Two<T> a, Two<T> b) {
  return {px ? a.x : b.x, py ? a.y : b.y};
}

// x^(-1/3) for x > 0 (x >= 1e-20 here): 2^(-log2(x)/3) from the hardware
// base-2 logarithm and exponential approximations, refined by one
// Newton-Raphson step for f(y) = y^-3 - x, y <- y (4 - x y^3) / 3.
__device__ __forceinline__ float rcbrt_fast(float x) {
  float l, y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(-0.33333334f * l));
  const float y3 = y * y * y;
  return y * fmaf(-0.33333334f * x, y3, 1.33333337f);
}
template <typename T> __device__ __forceinline__ T rcbrt_k(T x) { return Math<T>::rcbrt(x); }
template <> __device__ __forceinline__ float rcbrt_k<float>(float x) { return rcbrt_fast(x); }
// The same for a pair, the Newton step in pair arithmetic.
template <typename T> __device__ __forceinline__ Two<T> rcbrt2(Two<T> x) { return {rcbrt_k(x.x), rcbrt_k(x.y)}; }
template <> __device__ __forceinline__ Two<float> rcbrt2<float>(Two<float> x) {
  float lx, ly, yx, yy;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(lx) : "f"(x.x));
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(ly) : "f"(x.y));
  const Two<float> e = Two<float>{lx, ly} * two(-0.33333334f);
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(yx) : "f"(e.x));
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(yy) : "f"(e.y));
  const Two<float> y{yx, yy};
  const Two<float> y3 = y * y * y;
  return y * fma2(x * two(-0.33333334f), y3, two(1.33333337f));
}

// Adam's step m * alpha / (sqrt(v) + eps), correctly rounded square root and
// division as TensorFlow's ApplyAdam evaluates it (the solver's trajectory
// amplifies every rounding difference).
template <typename T> __device__ __forceinline__ T adam_step(T m_alpha, T v, T eps) {
  return m_alpha / (Math<T>::sqrt(v) + eps);
}

enum StencilMode { kEnergyOnly = 0, kGradient = 1, kAdamStep = 2 };

// Levels in flight ahead of the one being computed.  The ring also holds the
// level being computed and the two levels whose outputs are still pending
// (their Adam moments and old velocities are read when they are finished).
// The solver mode stages six tiles per level, so it looks two levels less
// ahead to keep two CTAs per SM.
// Energy-only mode: levels in flight and CTAs per SM (build-time constants; 3 ahead with 4 CTAs per
// SM measured best: 115 -> 104 us at 1500^2, the gradient modes keep 4 ahead / 2 CTAs per SM, whose
// registers a third CTA would spill)
#ifndef IGM_STENCIL_AHEAD_E
#define IGM_STENCIL_AHEAD_E 3
#endif
template <int MODE> struct Ring {
  static constexpr int ahead = MODE == kAdamStep ? 2 : (MODE == kEnergyOnly ? IGM_STENCIL_AHEAD_E : 4);
  static constexpr int stages = ahead + 3;
};

template <typename T>
struct StencilArgs {
  int batch, nz, ny, nx;
  T dx, inv_dx;
  T dzeta[IGM_MAX_NZ];
  T inv_dzeta[IGM_MAX_NZ];
  // physics
  T q, inv_p, regu2, sr_lo, sr_hi, thr, Kg, inv_n, s_w, inv_sw, regw2;
  // working units of the kernel: sr2 = k2 sr2w (k2 = 1/(32 dx^2)), clip bounds of sr2w,
  // and the gravity weight of each level, dzeta[k-1] + dzeta[k]
  T k2, lo2, hi2;
  T wgrav[IGM_MAX_NZ];
  int glen3, weert3, fnge;
  // inputs
  const T* thk;
  const T* usurf;
  const T* A;
  const T* C;
  T* U0;
  T* V0;
  // gradient mode
  T* dU;
  T* dV;
  T grad_scale;
  // solver mode
  T* U1;
  T* V1;
  T* mU;
  T* mV;
  T* vU;
  T* vV;
  T lr, b1, b2, eps;
  double es_delta;
  int es_patience, es_enabled, max_iter;
  igm_solver_ctl* ctl;
  double* costs;
  // reduction
  double* partials;
  unsigned int* counter;
  double* terms;
  double inv_count;
  int* err;  // set when a level load never arrived (bounded wait expired)
};

// Tensor maps of the node tiles: U/V of both solver buffers, the Adam moments
// and the 2-D fields.
struct StencilMaps {
  CUtensorMap U0, V0, U1, V1, mU, mV, vU, vV;
  CUtensorMap thk, usurf, A, C;
};

template <typename T, int TYP, int MODE>
struct StencilSmem {
  static constexpr int NR = 2 * TYP + 1, BW = Box<T>::BW;
  // elements per box, rounded up so that every box starts on a 128-byte boundary
  static constexpr int BOXE = ((NR * BW * (int)sizeof(T) + 127) / 128) * 128 / (int)sizeof(T);
  static constexpr bool GRAD = MODE != kEnergyOnly;
  static constexpr bool ADAM = MODE == kAdamStep;
  static constexpr int kStages = Ring<MODE>::stages;
  T N[kStages][2][BOXE];                        // U, V node tiles [NR][BW], ring of levels
  T M[ADAM ? kStages : 1][ADAM ? 4 : 1][BOXE];  // mU, mV, vU, vV node tiles, ring of levels
  T F[2][4][BOXE];                              // thk, usurf, A (then B = 2 A^(-1/n)), c: this tile, next tile
  T Down[GRAD ? 2 : 1][2][TYP][kCW];            // [level parity][U, V]: a thread row's share of the node row below
  double red[3][TYP];
  uint64_t full[kStages];                       // TMA arrival of a level
  uint64_t ffull[2];                            // TMA arrival of a tile's 2-D fields
  unsigned int ticket;
};

// Thread rows per CTA (each thread row = one warp = two cell rows).
#ifndef IGM_STENCIL_ROWS_F32
#define IGM_STENCIL_ROWS_F32 8
#endif
template <typename T> struct ThreadRows { static constexpr int value = IGM_STENCIL_ROWS_F32; };
template <> struct ThreadRows<double> { static constexpr int value = 4; };
#ifndef IGM_STENCIL_MINB_E
#define IGM_STENCIL_MINB_E 4
#endif
#ifndef IGM_STENCIL_MINB_G
#define IGM_STENCIL_MINB_G 2
#endif
template <typename T, int MODE> struct MinBlocks {
  static constexpr int value = (MODE == kEnergyOnly ? IGM_STENCIL_MINB_E : IGM_STENCIL_MINB_G) * 8 / IGM_STENCIL_ROWS_F32;
};
template <int MODE> struct MinBlocks<double, MODE> { static constexpr int value = 2; };

struct TileGeo {
  int j0, i0, xs, ox, b;  // first output node row / column, aligned box column, tile column 0 in the box, batch
};

// Persistent CTAs: CTA c processes tiles c, c + gridDim.x, ... (row-major over
// x, then y, then batch), streaming the sequence (tile, level) through one
// ring, so the loads of a tile's first levels and its 2-D fields are issued
// while the previous tile is still being computed.
template <typename T, int TYP, int MODE, bool TMA, bool STD>
__global__ void __launch_bounds__(kCW* TYP, MinBlocks<T, MODE>::value)
    stencil_kernel(const StencilArgs<T> a, const __grid_constant__ StencilMaps maps) {
  using P = Two<T>;
  using SmemT = StencilSmem<T, TYP, MODE>;
  // STD: the default physics (Glen n = 3, Weertman m = 3, gravitational energy not forced
  // negative), fixed at compile time so that its branches and generic powers drop out
  const bool glen3 = STD || a.glen3, weert3 = STD || a.weert3, fnge = !STD && a.fnge;
  constexpr int TYC = 2 * TYP;  // cell rows per tile
  constexpr int NT = kCW * TYP;
  constexpr int NR = TYC + 1, NC = kCW + 1;
  constexpr int NTILE = NR * NC;
  constexpr int BW = Box<T>::BW;
  constexpr int AL = Box<T>::AL;
  constexpr bool GRAD = MODE != kEnergyOnly;
  constexpr bool ADAM = MODE == kAdamStep;
  constexpr uint32_t kBoxBytes = NR * BW * sizeof(T);
  constexpr int kAhead = Ring<MODE>::ahead, kStages = Ring<MODE>::stages;
  static_assert(kCW == 32, "one warp per thread row");

  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA box destinations: align the base explicitly (the launch reserves 128 extra bytes).
  unsigned char* smem_al = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  SmemT& SM = *reinterpret_cast<SmemT*>(smem_al);

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kCW + tx;
  const int ny = a.ny, nx = a.nx, nz = a.nz;
  const size_t plane = (size_t)ny * nx;
  const int tiles_x = (nx + kCW - 2) / (kCW - 1);
  const int tiles_y = (ny + TYC - 2) / (TYC - 1);
  const int tiles_xy = tiles_x * tiles_y;
  const int ntiles = tiles_xy * a.batch;
  const int my_tiles = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

  const T* Ucur = a.U0;
  const T* Vcur = a.V0;
  T* Unxt = a.U1;
  T* Vnxt = a.V1;
  const CUtensorMap* mapU = &maps.U0;
  const CUtensorMap* mapV = &maps.V0;
  int iter = 0;
  T alpha = 0;
  if (MODE == kAdamStep) {
    iter = __ldcg(&a.ctl->iter);
    const int stopped = __ldcg(&a.ctl->stopped);
    if (stopped || iter >= a.max_iter) return;
    if (iter & 1) {
      mapU = &maps.U1; mapV = &maps.V1; Unxt = a.U0; Vnxt = a.V0;
      Ucur = a.U1; Vcur = a.V1;
    }
    const long long t = __ldcg(&a.ctl->adam_t0) + iter + 1;
    const T one = T(1);
    alpha = a.lr * Math<T>::sqrt(one - Math<T>::pow(a.b2, T(t))) / (one - Math<T>::pow(a.b1, T(t)));
  }

  auto geo = [&](int i) {
    const int t = (int)blockIdx.x + i * (int)gridDim.x;
    const int b = t / tiles_xy, r = t - b * tiles_xy;
    const int yt = r / tiles_x, xt = r - yt * tiles_x;
    TileGeo g;
    g.j0 = yt * (TYC - 1);
    g.i0 = xt * (kCW - 1);
    g.b = b;
    g.xs = g.i0 >= 1 ? ((g.i0 - 1) / AL) * AL : -AL;
    g.ox = g.i0 - 1 - g.xs;
    return g;
  };

  if (tid == 0) {
    for (int st = 0; st < kStages; ++st) tc::mbar_init(&SM.full[st], 1);
    tc::mbar_init(&SM.ffull[0], 1);
    tc::mbar_init(&SM.ffull[1], 1);
    tc::fence_mbar_init();
  }
  __syncthreads();

  // fixed node slots of this thread in a tile (element-wise loads and the B pass)
  constexpr int NSLOT = (NTILE + NT - 1) / NT;
  int slot_r[NSLOT], slot_c[NSLOT];
#pragma unroll
  for (int q = 0; q < NSLOT; ++q) {
    const int idx = tid + q * NT;
    slot_r[q] = idx < NTILE ? idx / NC : -1;
    slot_c[q] = idx < NTILE ? idx - (idx / NC) * NC : 0;
  }
  // this thread: cells (R0, tx) and (R0 + 1, tx) of the tile; output nodes (R0 + e, tx)
  const int R0 = 2 * ty;

  auto issue_fields = [&](const TileGeo& g, int fb) {  // TMA path only
    if (tid == 0) {
      uint64_t* bar = &SM.ffull[fb];
      tc::mbar_expect_tx(bar, 4u * kBoxBytes);
      tc::tma_load_3d(SM.F[fb][0], &maps.thk, g.xs, g.j0 - 1, g.b, bar);
      tc::tma_load_3d(SM.F[fb][1], &maps.usurf, g.xs, g.j0 - 1, g.b, bar);
      tc::tma_load_3d(SM.F[fb][2], &maps.A, g.xs, g.j0 - 1, g.b, bar);
      tc::tma_load_3d(SM.F[fb][3], &maps.C, g.xs, g.j0 - 1, g.b, bar);
    }
  };
  auto issue_level = [&](const TileGeo& g, int k, int st) {
    if (TMA) {
      if (tid == 0) {
        uint64_t* bar = &SM.full[st];
        const int z = g.b * nz + k;
        tc::mbar_expect_tx(bar, (ADAM ? 6u : 2u) * kBoxBytes);
        tc::tma_load_3d(SM.N[st][0], mapU, g.xs, g.j0 - 1, z, bar);
        tc::tma_load_3d(SM.N[st][1], mapV, g.xs, g.j0 - 1, z, bar);
        if (ADAM) {
          tc::tma_load_3d(SM.M[st][0], &maps.mU, g.xs, g.j0 - 1, z, bar);
          tc::tma_load_3d(SM.M[st][1], &maps.mV, g.xs, g.j0 - 1, z, bar);
          tc::tma_load_3d(SM.M[st][2], &maps.vU, g.xs, g.j0 - 1, z, bar);
          tc::tma_load_3d(SM.M[st][3], &maps.vV, g.xs, g.j0 - 1, z, bar);
        }
      }
    } else {
      const size_t lo = ((size_t)g.b * nz + k) * plane;
#pragma unroll
      for (int q = 0; q < NSLOT; ++q) {
        if (slot_r[q] < 0) continue;
        const int gj = g.j0 - 1 + slot_r[q], gi = g.i0 - 1 + slot_c[q];
        const bool ok = gj >= 0 && gj < ny && gi >= 0 && gi < nx;
        const size_t o = lo + (ok ? (size_t)gj * nx + gi : 0);
        const int sm = slot_r[q] * BW + slot_c[q] + g.ox;
        cp_async_elem(SM.N[st][0] + sm, Ucur + o, ok);
        cp_async_elem(SM.N[st][1] + sm, Vcur + o, ok);
        if (ADAM) {
          cp_async_elem(SM.M[st][0] + sm, a.mU + o, ok);
          cp_async_elem(SM.M[st][1] + sm, a.mV + o, ok);
          cp_async_elem(SM.M[st][2] + sm, a.vU + o, ok);
          cp_async_elem(SM.M[st][3] + sm, a.vV + o, ok);
        }
      }
    }
  };
  // issue cursor over the sequence (tile, level)
  int iss_i = 0, iss_k = 0, iss_st = 0;
  TileGeo ig = geo(0);  // geometry of the tile at the cursor
  auto issue_next = [&]() {
    if (TMA && tid != 0) return;  // TMA: only the issuing thread tracks the cursor
    if (iss_i < my_tiles) issue_level(ig, iss_k, iss_st);
    if (!TMA) cp_async_commit();  // one group per sequence position, possibly empty
    iss_st = iss_st + 1 == kStages ? 0 : iss_st + 1;
    if (++iss_k == nz) {
      iss_k = 0;
      if (++iss_i < my_tiles) ig = geo(iss_i);
    }
  };
  if (TMA && my_tiles > 0) issue_fields(ig, 0);
#pragma unroll 1
  for (int q = 0; q < kAhead; ++q) issue_next();

  const T half = T(0.5), quarter = T(0.25);
  const P H = two(half), Q4 = two(quarter), zero = two(T(0));
  const P HI = two(half * a.inv_dx);
  double acc[3] = {0.0, 0.0, 0.0};
  bool load_ok = true;
  int cons_st = 0;         // ring slot of the level being computed
  uint32_t cons_ph = 0;    // its mbarrier phase parity

#pragma unroll 1
  for (int i = 0; i < my_tiles; ++i) {
    const TileGeo g = geo(i);
    const int fb = TMA ? (i & 1) : 0;
    if (TMA) {
      if (tid == 0 && i + 1 < my_tiles) issue_fields(geo(i + 1), fb ^ 1);
      // one thread waits for the transfer; the barrier publishes it to the CTA
      if (tid == 0 && !tc::mbar_wait(&SM.ffull[fb], (uint32_t)((i >> 1) & 1))) load_ok = false;
      __syncthreads();
    }
    // 2-D fields (element-wise path: plain loads) and B = 2 A^(-1/n) in place at in-domain nodes
#pragma unroll
    for (int q = 0; q < NSLOT; ++q) {
      if (slot_r[q] < 0) continue;
      const int gj = g.j0 - 1 + slot_r[q], gi = g.i0 - 1 + slot_c[q];
      const bool ok = gj >= 0 && gj < ny && gi >= 0 && gi < nx;
      const int sm = slot_r[q] * BW + slot_c[q] + g.ox;
      T Av;
      if (TMA) {
        Av = SM.F[fb][2][sm];
      } else {
        const size_t o = (size_t)g.b * plane + (ok ? (size_t)gj * nx + gi : 0);
        SM.F[0][0][sm] = ok ? a.thk[o] : T(0);
        SM.F[0][1][sm] = ok ? a.usurf[o] : T(0);
        SM.F[0][3][sm] = ok ? a.C[o] : T(0);
        Av = ok ? a.A[o] : T(1);
      }
      SM.F[fb][2][sm] = ok ? T(2) * (glen3 ? rcbrt_k<T>(Av) : Math<T>::pow(Av, -a.inv_n)) : T(0);
    }
    // these generic writes precede a later TMA write to the same buffer
    if (TMA) tc::fence_proxy_async_smem();
    __syncthreads();

    // ---- per-cell constants of this tile --------------------------------------------
    // Working units.  Per level the kernel keeps, per cell, the corner sums
    //   S = a+b+c+d (= 4 Us),  DX = (b-a)+(d-c) (= Dx / hx),  DY = (c-a)+(d-b) (= Dy / hx)
    // with hx = 1/(2dx), and per layer the strain components divided by
    // kappa = 1/(4dx), so that the staggered averages need no multiplications
    // and sr2 = kappa^2/2 * sr2w; every scale folds into per-tile constants.
    const int own_sm = R0 * BW + tx + g.ox;
    P thks, Bs, cs, sbx, sby, ssx, ssy;
    bool cok[2], own[2], out_ok[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const T* f0 = SM.F[fb][0] + own_sm + e * BW;
      const T* f1 = SM.F[fb][1] + own_sm + e * BW;
      const T* f2p = SM.F[fb][2] + own_sm + e * BW;
      const T* f3 = SM.F[fb][3] + own_sm + e * BW;
      const T t00 = f0[0], t01 = f0[1], t10 = f0[BW], t11 = f0[BW + 1];
      const T u00 = f1[0], u01 = f1[1], u10 = f1[BW], u11 = f1[BW + 1];
      const T th = (((t11 + t10) + t01) + t00) * quarter;
      const T bs = (((f2p[BW + 1] + f2p[BW]) + f2p[1]) + f2p[0]) * quarter;
      const T cv = (((f3[BW + 1] + f3[BW]) + f3[1]) + f3[0]) * quarter;
      const T b00 = u00 - t00, b01 = u01 - t01, b10 = u10 - t10, b11 = u11 - t11;
      // compute_gradient (staggered): 2 ds / (dx + dx), averaged over the other axis
      const T id = a.inv_dx;
      const T bx = half * ((b11 - b10) * id + (b01 - b00) * id);
      const T by = half * ((b11 - b01) * id + (b10 - b00) * id);
      const T sx = half * ((u11 - u10) * id + (u01 - u00) * id);
      const T sy = half * ((u11 - u01) * id + (u10 - u00) * id);
      if (e == 0) {
        thks.x = th; Bs.x = bs; cs.x = cv; sbx.x = bx; sby.x = by; ssx.x = sx; ssy.x = sy;
      } else {
        thks.y = th; Bs.y = bs; cs.y = cv; sbx.y = bx; sby.y = by; ssx.y = sx; ssy.y = sy;
      }
      const int cj = g.j0 - 1 + R0 + e, ci = g.i0 - 1 + tx;  // cell (j, i) = node (j, i) of its top-left corner
      cok[e] = cj >= 0 && cj < ny - 1 && ci >= 0 && ci < nx - 1;
      own[e] = cok[e] && R0 + e >= 1 && tx >= 1;
      out_ok[e] = R0 + e >= 1 && tx >= 1 && cj < ny && ci < nx;
    }
    // vertical-derivative factor dx / max(thk_s, thr), damped where there is no sliding (times 1/dzeta per layer)
    const P rzc = {(cs.x > T(0) ? a.dx : T(0.01) * a.dx) / (thks.x > a.thr ? thks.x : a.thr),
                   (cs.y > T(0) ? a.dx : T(0.01) * a.dx) / (thks.y > a.thr ? thks.y : a.thr)};
    const P nsbx = sbx * two(T(-1)), nsby = sby * two(T(-1));
    // energy: shear = esc * sum dz bq sr2w; gravity = egc * (ssx sum w S + ssy sum w SV)
    const P esc = thks * Bs * two(a.inv_p * a.k2);
    const P egc = thks * two(a.Kg * T(0.125));
    // adjoint constants (grad_scale folded in; zero for cells outside the domain, whose
    // contributions then vanish without masking)
    const P okm = sel(cok[0], cok[1], two(a.grad_scale), zero);
    const P gshc = esc * okm;                // dE/d(bq sr2w) per unit dzeta
    const P gxc = egc * ssx * okm, gyc = egc * ssy * okm;  // dE/dS, dE/dSV per unit gravity weight
    const P csg = cs * okm * Q4;             // sliding: dE/dS = csg N^(s/2-1) (Us + tb sbx)
    // output node (R0, tx) of level 0 of this tile, as an element offset
    const long long obase = ((long long)g.b * nz) * (long long)plane +
                            (long long)(g.j0 - 1 + R0) * nx + (g.i0 - 1 + tx);

    P e_sh = zero, eGu = zero, eGv = zero, e_slid = zero, e_gf = zero;
    // previous level's corner sums, pending adjoint of the previous level
    P pSu = zero, pSv = zero, pXu = zero, pYu = zero, pXv = zero, pYv = zero;
    P gSu = zero, gXu = zero, gYu = zero, gSv = zero, gXv = zero, gYv = zero;
    P partU = zero, partV = zero;  // own-node sums of the level awaiting its finish
    int st_m1 = 0, st_m2 = 0;      // ring slots of the previous two levels

    auto level_q = [&](const T* t, P& S, P& DX, P& DY) {
      const T* p = t + own_sm;
      const T a0 = p[0], b0 = p[1], a1 = p[BW], b1 = p[BW + 1], a2 = p[2 * BW], b2 = p[2 * BW + 1];
      const T s0 = a0 + b0, s1 = a1 + b1, s2 = a2 + b2;
      const T d0 = b0 - a0, d1 = b1 - a1, d2 = b2 - a2;
      S = {s0 + s1, s1 + s2};
      DX = {d0 + d1, d1 + d2};
      DY = {s1 - s0, s2 - s1};
    };
    // corner contributions of a completed level's adjoint (dE/dS, dE/dDX, dE/dDY);
    // the right-hand corners reach the next lane by shuffles, the node row below
    // this thread row goes through shared memory
    auto flush = [&](int lvl, P gS, P gX, P gY, int f, P& part) {
      const P SmY = gS - gY, SpY = gS + gY;
      const P c00 = SmY - gX, c01 = SmY + gX, c10 = SpY - gX, c11 = SpY + gX;
      const T r1 = c01.y + c11.x;
      const T l0 = __shfl_up_sync(0xffffffffu, c01.x, 1);
      const T l1 = __shfl_up_sync(0xffffffffu, r1, 1);
      const T l2 = __shfl_up_sync(0xffffffffu, c11.y, 1);
      part = c00 + P{l0, c10.x + l1};
      SM.Down[GRAD ? (lvl & 1) : 0][f][ty][tx] = c10.y + l2;
    };
    // node outputs of a flushed level (after a barrier): gradient, or the Adam update
    auto finish = [&](int lvl, int st) {
      const int pb = GRAD ? (lvl & 1) : 0;
      const T upU = ty >= 1 ? SM.Down[pb][0][ty - 1][tx] : T(0);
      const T upV = ty >= 1 ? SM.Down[pb][1][ty - 1][tx] : T(0);
      const long long o0 = obase + (long long)lvl * (long long)plane;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (!out_ok[e]) continue;
        const T gu = e ? partU.y : partU.x + upU;
        const T gv = e ? partV.y : partV.x + upV;
        const long long o = o0 + (e ? nx : 0);
        if (MODE == kGradient) {
          a.dU[o] = gu;
          a.dV[o] = gv;
        } else if (MODE == kAdamStep) {
          const int sm = own_sm + e * BW;
          const T b1c = T(1) - a.b1, b2c = T(1) - a.b2;
          T m = SM.M[st][0][sm], v = SM.M[st][2][sm];
          m += (gu - m) * b1c;
          v += (gu * gu - v) * b2c;
          a.mU[o] = m;
          a.vU[o] = v;
          Unxt[o] = SM.N[st][0][sm] - adam_step<T>(m * alpha, v, a.eps);
          m = SM.M[st][1][sm];
          v = SM.M[st][3][sm];
          m += (gv - m) * b1c;
          v += (gv * gv - v) * b2c;
          a.mV[o] = m;
          a.vV[o] = v;
          Vnxt[o] = SM.N[st][1][sm] - adam_step<T>(m * alpha, v, a.eps);
        }
      }
    };

    // one level of the stream; the first level (sliding, no layer below it) is peeled
    // off at compile time so that the steady-state loop carries no branches on k
    auto level = [&](const int k, auto first_tag) {
      constexpr bool FIRST = decltype(first_tag)::value;
      const int nb = cons_st;
      if (TMA) {
        // level k landed: one thread waits (the others spend no issue slots polling)
        if (tid == 0 && !tc::mbar_wait(&SM.full[nb], cons_ph)) load_ok = false;
      } else {
        cp_async_wait<kAhead - 1>();  // this thread's copies of level k have landed
      }
      __syncthreads();  // level k visible to all; every thread is done with the previous iteration
      issue_next();
      if (GRAD && !FIRST && k >= 2) finish(k - 2, st_m2);

      P cSu, cXu, cYu, cSv, cXv, cYv;
      level_q(SM.N[nb][0], cSu, cXu, cYu);
      level_q(SM.N[nb][1], cSv, cXv, cYv);
      // gravity of level k (weight dzeta[k-1] + dzeta[k]) enters its pending adjoint directly
      const T wk = a.wgrav[k];
      if (!fnge) {
        eGu = fma2(cSu, two(wk), eGu);
        eGv = fma2(cSv, two(wk), eGv);
      }
      P hSu = zero, hXu = zero, hYu = zero, hSv = zero, hXv = zero, hYv = zero;  // pending adjoint of level k
      if (GRAD && !fnge) {
        hSu = gxc * two(wk);
        hSv = gyc * two(wk);
      }

      if (FIRST) {
        // Weertman sliding on the basal level (cost_sliding_weertman.py:23-43)
        const P cUs = cSu * Q4, cVs = cSv * Q4;
        const P tb = fma2(cVs, sby, cUs * sbx);
        const P Nn = fma2(tb, tb, fma2(cUs, cUs, cVs * cVs) + two(a.regw2));
        P Np, dN;  // N^(s/2) and N^(s/2 - 1)
        if (weert3) {
          dN = rcbrt2(Nn);  // N^(-1/3)
          Np = Nn * dN;     // N^(2/3)
        } else {
          Np = {Math<T>::pow(Nn.x, a.s_w * half), Math<T>::pow(Nn.y, a.s_w * half)};
          dN = {Math<T>::pow(Nn.x, a.s_w * half - T(1)), Math<T>::pow(Nn.y, a.s_w * half - T(1))};
        }
        e_slid = cs * Np * two(a.inv_sw);
        if (GRAD) {
          const P gN = csg * dN;
          hSu = fma2(gN, fma2(tb, sbx, cUs), hSu);
          hSv = fma2(gN, fma2(tb, sby, cVs), hSv);
        }
        if (nz == 1) {
          pSu = cSu; pSv = cSv; pXu = cXu; pYu = cYu; pXv = cXv; pYv = cYv;
        }
      }

      if (!FIRST || nz == 1) {
        const int l = FIRST ? 0 : k - 1;  // a layer on the first level exists only when nz == 1
        const T dz = a.dzeta[l];
        const P rz = rzc * two(a.inv_dzeta[l]);
        const P uz = (cSu - pSu) * rz, vz = (cSv - pSv) * rz;
        const P X = fma2(uz, nsbx, pXu + cXu), Y = fma2(uz, nsby, pYu + cYu);
        const P Z = fma2(vz, nsbx, pXv + cXv), W = fma2(vz, nsby, pYv + cYv);
        const P ZY = Z + Y;  // 2 Exy (scaled)
        const P XW = X + W;  // -Ezz (scaled)
        const P hZY = ZY * H;
        P t = X * X;
        t = fma2(W, W, t);
        t = fma2(XW, XW, t);
        t = fma2(ZY, hZY, t);
        const P sr2w = fma2(fma2(vz, vz, uz * uz), H, t);  // sr2 = k2 sr2w
        const P sc = {sr2w.x < a.lo2 ? a.lo2 : (sr2w.x > a.hi2 ? a.hi2 : sr2w.x),
                      sr2w.y < a.lo2 ? a.lo2 : (sr2w.y > a.hi2 ? a.hi2 : sr2w.y)};
        const P base = fma2(sc, two(a.k2), two(a.regu2));
        const P bq = glen3 ? rcbrt2(base) : P{Math<T>::pow(base.x, a.q), Math<T>::pow(base.y, a.q)};
        e_sh = fma2(bq * sr2w, two(dz), e_sh);
        P gXh = zero;  // gravity adjoint of this layer under force_negative_gravitational_energy
        if (fnge) {
          // per layer: twice the staggered u . grad(s) (scaled by 4), kept only where negative
          P uds = fma2(cSv + pSv, ssy, (cSu + pSu) * ssx);
          const bool gax = uds.x < T(0), gay = uds.y < T(0);
          uds = sel(uds.x > T(0), uds.y > T(0), zero, uds);
          e_gf = fma2(uds, two(dz), e_gf);
          gXh = sel(gax, gay, two(dz), zero);
        }
        if (GRAD) {
          const bool in_x = sr2w.x >= a.lo2 && sr2w.x <= a.hi2;
          const bool in_y = sr2w.y >= a.lo2 && sr2w.y <= a.hi2;
          // d(bq sr2)/d sr2 = bq + q bq / base sr2; bq / base = bq^4 for n = 3
          P bq_base;
          if (glen3) {
            const P bq2 = bq * bq;
            bq_base = bq2 * bq2;
          } else {
            bq_base = {bq.x / base.x, bq.y / base.y};
          }
          const P qk = {in_x ? a.q * a.k2 : T(0), in_y ? a.q * a.k2 : T(0)};
          const P G = fma2(qk * bq_base, sr2w, bq) * (gshc * two(dz));  // dE/d sr2w
          const P G2 = G + G;
          const P gX = G2 * fma2(X, two(T(2)), W);
          const P gW = G2 * fma2(W, two(T(2)), X);
          const P gY = G * ZY;
          const P Gu = fma2(gX, nsbx, fma2(gY, nsby, G * uz)) * rz;
          const P Gv = fma2(gY, nsbx, fma2(gW, nsby, G * vz)) * rz;
          P fgu = zero, fgv = zero;  // gravity under force_negative_gravitational_energy
          if (fnge) {
            fgu = gxc * gXh;
            fgv = gyc * gXh;
          }
          if (nz == 1) {  // the only layer couples level 0 with itself
            hXu = gX + gX; hYu = gY + gY; hXv = hYu; hYv = gW + gW;
            hSu = hSu + (fgu - Gu) + (fgu + Gu);
            hSv = hSv + (fgv - Gv) + (fgv + Gv);
          } else {
            // layer l couples level l (pending g*) and level l+1 (pending h*)
            gXu = gXu + gX; gYu = gYu + gY; gXv = gXv + gY; gYv = gYv + gW;
            gSu = gSu + (fgu - Gu);
            gSv = gSv + (fgv - Gv);
            hXu = gX; hYu = gY; hXv = gY; hYv = gW;
            hSu = hSu + (fgu + Gu);
            hSv = hSv + (fgv + Gv);
          }
        }
      }

      if (GRAD) {
        if (!FIRST && nz > 1) {
          flush(k - 1, gSu, gXu, gYu, 0, partU);
          flush(k - 1, gSv, gXv, gYv, 1, partV);
        }
        gSu = hSu; gXu = hXu; gYu = hYu; gSv = hSv; gXv = hXv; gYv = hYv;
      }
      pSu = cSu; pSv = cSv; pXu = cXu; pYu = cYu; pXv = cXv; pYv = cYv;
      st_m2 = st_m1;
      st_m1 = nb;
      if (++cons_st == kStages) {
        cons_st = 0;
        cons_ph ^= 1u;
      }
    };
    level(0, std::true_type{});
#pragma unroll 2
    for (int k = 1; k < nz; ++k) level(k, std::false_type{});
    if (GRAD) {
      __syncthreads();
      if (nz >= 2) finish(nz - 2, st_m2);
      flush(nz - 1, gSu, gXu, gYu, 0, partU);
      flush(nz - 1, gSv, gXv, gYv, 1, partV);
      __syncthreads();
      finish(nz - 1, st_m1);
    }
    // this tile's energy densities (owned cells only)
    const P egrav = fnge ? egc * e_gf : egc * fma2(ssy, eGv, ssx * eGu);
    const P es = sel(own[0], own[1], esc * e_sh, zero);
    const P eg = sel(own[0], own[1], egrav, zero);
    const P el = sel(own[0], own[1], e_slid, zero);
    acc[0] += (double)es.x + (double)es.y;
    acc[1] += (double)el.x + (double)el.y;
    acc[2] += (double)eg.x + (double)eg.y;
  }

  if (!load_ok && a.err) atomicExch(a.err, 1);
  // ---- energy reduction ---------------------------------------------------------
  const int nblocks = gridDim.x;
  const int bid = blockIdx.x;
  // three FP64 sums over the CTA in a fixed order; every thread gets the totals
  auto block_sum3 = [&](double (&r)[3]) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      r[0] += __shfl_xor_sync(0xffffffffu, r[0], o);
      r[1] += __shfl_xor_sync(0xffffffffu, r[1], o);
      r[2] += __shfl_xor_sync(0xffffffffu, r[2], o);
    }
    __syncthreads();
    if (tx == 0) {
      SM.red[0][ty] = r[0];
      SM.red[1][ty] = r[1];
      SM.red[2][ty] = r[2];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int w = 0; w < TYP; ++w) s += SM.red[i][w];
      r[i] = s;
    }
  };
  block_sum3(acc);
  if (tid == 0) {
    a.partials[3 * (size_t)bid + 0] = acc[0];
    a.partials[3 * (size_t)bid + 1] = acc[1];
    a.partials[3 * (size_t)bid + 2] = acc[2];
    __threadfence();
    SM.ticket = atomicAdd(a.counter, 1u);
  }
  __syncthreads();
  if (SM.ticket != (unsigned)(nblocks - 1)) return;
  __threadfence();
  double r[3] = {0.0, 0.0, 0.0};
  for (int i = tid; i < nblocks; i += NT) {
    r[0] += __ldcg(&a.partials[3 * (size_t)i + 0]);
    r[1] += __ldcg(&a.partials[3 * (size_t)i + 1]);
    r[2] += __ldcg(&a.partials[3 * (size_t)i + 2]);
  }
  block_sum3(r);
  const double t0 = r[0], t1 = r[1], t2 = r[2];
  if (tid == 0) {
    *a.counter = 0u;
    const bool lost = a.err && __ldcg(a.err) != 0;
    if (lost) *a.err = 0;  // reported through this launch's terms / status; the next launch starts clean
    if (a.terms) {
      a.terms[0] = lost ? nan("") : t0;
      a.terms[1] = lost ? nan("") : t1;
      a.terms[2] = lost ? nan("") : t2;
    }
    if (MODE == kAdamStep) {
      igm_solver_ctl* ctl = a.ctl;
      const double cost = (t0 + t1 + t2) * a.inv_count;
      a.costs[iter] = cost;
      ctl->last_cost = cost;
      ctl->terms[0] = t0 * a.inv_count;
      ctl->terms[1] = t1 * a.inv_count;
      ctl->terms[2] = t2 * a.inv_count;
      if (lost) {
        ctl->status = IGM_ERR_CUDA;
        ctl->stopped = 1;
      } else if (!isfinite(cost)) {
        ctl->status = IGM_ERR_NAN_DETECTED;
        ctl->stopped = 1;
      } else if (a.es_enabled) {
        if (iter == 0) {
          ctl->best = cost;
          ctl->wait = 0;
        } else {
          const double best = ctl->best;
          const double rel = (best - cost) / fabs(best);
          if (rel > a.es_delta) {
            ctl->best = cost;
            ctl->wait = 0;
          } else {
            const int w = ctl->wait + 1;
            ctl->wait = w;
            if (w >= a.es_patience) ctl->stopped = 1;
          }
        }
      }
      __threadfence();
      ctl->iter = iter + 1;
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static inline int grid_blocks_rows(const igm_grid* g, int tyc, dim3* grid) {
  *grid = dim3((g->nx + kCW - 2) / (kCW - 1), (g->ny + tyc - 2) / (tyc - 1), g->batch);
  return (int)(grid->x * grid->y * grid->z);
}
// The workspace is sized for the smaller tile (more CTAs) so one size fits both dtypes.
static inline int grid_blocks(const igm_grid* g, dim3* grid) { return grid_blocks_rows(g, 8, grid); }

static int check_grid(const igm_grid* g) {
  IGM_CHECK_ARG(g != nullptr, IGM_ERR_BAD_ARGUMENT, "grid is NULL");
  IGM_CHECK_ARG(g->batch >= 1 && g->nz >= 1 && g->nz <= IGM_MAX_NZ && g->ny >= 2 && g->nx >= 2,
                IGM_ERR_BAD_SHAPE, "bad grid shape batch=%d nz=%d ny=%d nx=%d (need batch>=1, 1<=nz<=%d, ny,nx>=2)",
                g->batch, g->nz, g->ny, g->nx, IGM_MAX_NZ);
  IGM_CHECK_ARG(g->dx > 0, IGM_ERR_BAD_ARGUMENT, "dx must be positive (got %g)", g->dx);
  dim3 gr;
  grid_blocks(g, &gr);
  IGM_CHECK_ARG(gr.y <= 65535u && gr.z <= 65535u, IGM_ERR_BAD_SHAPE, "grid too large");
  return IGM_OK;
}

template <typename T>
static void fill_common(StencilArgs<T>& s, const igm_grid* g, const igm_physics* ph, const igm_fields* f) {
  s.batch = g->batch;
  s.nz = g->nz;
  s.ny = g->ny;
  s.nx = g->nx;
  s.dx = (T)g->dx;
  s.inv_dx = (T)(1.0 / g->dx);
  for (int l = 0; l < IGM_MAX_NZ; ++l) {
    s.dzeta[l] = (T)g->dzeta[l];
    s.inv_dzeta[l] = g->dzeta[l] != 0.0 ? (T)(1.0 / g->dzeta[l]) : T(0);
  }
  const double n = ph->exp_glen, m = ph->exp_weertman;
  const double p = 1.0 + 1.0 / n;
  s.q = (T)((p - 2.0) / 2.0);
  s.inv_p = (T)(1.0 / p);
  s.regu2 = (T)(ph->regu_glen * ph->regu_glen);
  s.sr_lo = (T)(ph->min_sr * ph->min_sr);  // float: a denormal, as TF's float32 clip bound
  s.sr_hi = (T)(ph->max_sr * ph->max_sr);  // float: +inf, as TF's float32 clip bound
  s.thr = (T)ph->thr_ice_thk;
  s.Kg = (T)(ph->ice_density * ph->gravity_cst * 1e-6);
  s.inv_n = (T)(1.0 / n);
  s.s_w = (T)(1.0 + 1.0 / m);
  s.inv_sw = (T)(1.0 / (1.0 + 1.0 / m));
  s.regw2 = (T)(ph->regu_weertman * ph->regu_weertman);
  const double k2 = 1.0 / (32.0 * g->dx * g->dx);
  s.k2 = (T)k2;
  s.lo2 = (T)((double)s.sr_lo / k2);
  s.hi2 = (T)((double)s.sr_hi / k2);
  for (int k = 0; k < IGM_MAX_NZ; ++k) {
    double w = 0.0;
    if (k < g->nz) {
      if (g->nz == 1) {
        w = 2.0 * g->dzeta[0];
      } else {
        if (k >= 1) w += g->dzeta[k - 1];
        if (k <= g->nz - 2) w += g->dzeta[k];
      }
    }
    s.wgrav[k] = (T)w;
  }
  s.glen3 = n == 3.0;
  s.weert3 = m == 3.0;
  s.fnge = ph->force_negative_gravitational_energy != 0;
  s.thk = (const T*)f->thk;
  s.usurf = (const T*)f->usurf;
  s.A = (const T*)f->arrhenius;
  s.C = (const T*)f->slidingco;
  s.inv_count = 1.0 / ((double)g->batch * (double)(g->ny - 1) * (double)(g->nx - 1));
}

size_t workspace_bytes_for(const igm_grid* g) {
  dim3 gr;
  const size_t nb = (size_t)grid_blocks(g, &gr);
  return 256 + ((3 * nb * sizeof(double) + 255) / 256) * 256 + 4096;
}

static int bind_workspace(void* ws, size_t bytes, const igm_grid* g, unsigned int** counter, double** partials) {
  IGM_CHECK_ARG(ws != nullptr, IGM_ERR_WORKSPACE, "workspace is NULL");
  const size_t need = workspace_bytes_for(g);
  IGM_CHECK_ARG(bytes >= need, IGM_ERR_WORKSPACE, "workspace too small: %zu < %zu bytes", bytes, need);
  IGM_CHECK_ARG(((uintptr_t)ws & 255) == 0, IGM_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  *counter = (unsigned int*)ws;
  *partials = (double*)((char*)ws + 256);
  return IGM_OK;
}

// 3-D tensor map over [planes][ny][nx] of T with the node-tile box: planes =
// batch * nz for the levels of U, V and the moments, batch for the 2-D fields.
template <typename T>
static int level_map(CUtensorMap* m, const void* base, const igm_grid* g, int planes) {
  tc::EncodeTiledFn enc = tc::encode_tiled_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the CUDA driver");
    return IGM_ERR_CUDA;
  }
  constexpr int TYC = 2 * ThreadRows<T>::value;
  cuuint64_t dims[3] = {(cuuint64_t)g->nx, (cuuint64_t)g->ny, (cuuint64_t)planes};
  cuuint64_t strides[2] = {(cuuint64_t)g->nx * sizeof(T), (cuuint64_t)g->ny * g->nx * sizeof(T)};
  cuuint32_t box[3] = {(cuuint32_t)Box<T>::BW, (cuuint32_t)(TYC + 1), 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                   const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (level tiles) failed (CUresult %d)", (int)r);
    return IGM_ERR_CUDA;
  }
  return IGM_OK;
}

// SM count of the current device, looked up once per device.
static int sm_count_current(int* out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  constexpr int kMaxDevices = 128;
  static int cache[kMaxDevices] = {};
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error("cudaGetDevice: %s", cudaGetErrorString(e));
    return IGM_ERR_CUDA;
  }
  if (cache[dev] == 0) {
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || n <= 0) {
      set_error("cudaDeviceGetAttribute(MultiProcessorCount): %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
    cache[dev] = n;
  }
  *out = cache[dev];
  return IGM_OK;
}

template <typename T>
static int field_maps(StencilMaps* maps, const igm_fields* f, const igm_grid* g) {
  int rc;
  if ((rc = level_map<T>(&maps->thk, f->thk, g, g->batch)) || (rc = level_map<T>(&maps->usurf, f->usurf, g, g->batch)) ||
      (rc = level_map<T>(&maps->A, f->arrhenius, g, g->batch)) || (rc = level_map<T>(&maps->C, f->slidingco, g, g->batch)))
    return rc;
  return IGM_OK;
}

// TMA needs 16-byte aligned bases and a row pitch that is a multiple of 16 bytes.
template <typename T>
static bool tma_usable(const igm_grid* g, std::initializer_list<const void*> ptrs) {
  if (((size_t)g->nx * sizeof(T)) % 16 != 0) return false;
  for (const void* p : ptrs)
    if (p == nullptr || ((uintptr_t)p & 15) != 0) return false;
  return true;
}

// Persistent launch: as many CTAs as fit on the device at once (at most one per tile).
template <typename T, int MODE, bool TMA, bool STD>
static int launch_stencil_t(const StencilArgs<T>& s, const StencilMaps& maps, const igm_grid* g, cudaStream_t st) {
  constexpr int TYP = ThreadRows<T>::value;
  constexpr int TYC = 2 * TYP;
  constexpr size_t smem = sizeof(StencilSmem<T, TYP, MODE>) + 128;
  auto kern = stencil_kernel<T, TYP, MODE, TMA, STD>;
  static int per_sm = 0;
  if (per_sm == 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    int n = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, kCW * TYP, smem);
    if (e != cudaSuccess) {
      set_error("stencil_kernel configuration: %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
    per_sm = n > 0 ? n : 1;
  }
  int sms = 0;
  int rc = sm_count_current(&sms);
  if (rc) return rc;
  const long long ntiles = (long long)((g->nx + kCW - 2) / (kCW - 1)) * ((g->ny + TYC - 2) / (TYC - 1)) * g->batch;
  const long long cap = (long long)per_sm * sms;
  const int grid = (int)(ntiles < cap ? ntiles : cap);
  kern<<<grid, dim3(kCW, TYP), smem, st>>>(s, maps);
  return launch_status("stencil_kernel");
}

template <typename T, int MODE>
static int launch_stencil(const StencilArgs<T>& s, const StencilMaps& maps, bool tma, const igm_grid* g,
                          cudaStream_t st) {
  const bool std_phys = s.glen3 && s.weert3 && !s.fnge;
  if (std_phys)
    return tma ? launch_stencil_t<T, MODE, true, true>(s, maps, g, st) : launch_stencil_t<T, MODE, false, true>(s, maps, g, st);
  return tma ? launch_stencil_t<T, MODE, true, false>(s, maps, g, st) : launch_stencil_t<T, MODE, false, false>(s, maps, g, st);
}

template <typename T>
static int energy_t(const igm_grid* g, const igm_physics* ph, const igm_fields* f, const void* U, const void* V,
                    void* dU, void* dV, double grad_scale, double* terms, void* ws, size_t wsb, cudaStream_t st) {
  StencilArgs<T> s{};
  fill_common(s, g, ph, f);
  s.U0 = (T*)U;
  s.V0 = (T*)V;
  s.dU = (T*)dU;
  s.dV = (T*)dV;
  s.grad_scale = (T)grad_scale;
  s.terms = terms;
  int rc = bind_workspace(ws, wsb, g, &s.counter, &s.partials);
  if (rc) return rc;
  s.err = (int*)((char*)ws + 4);
  StencilMaps maps;
  memset(&maps, 0, sizeof(maps));
  const bool tma = tma_usable<T>(g, {U, V, f->thk, f->usurf, f->arrhenius, f->slidingco});
  if (tma) {
    const int nl = g->batch * g->nz;
    if ((rc = level_map<T>(&maps.U0, U, g, nl)) || (rc = level_map<T>(&maps.V0, V, g, nl)) ||
        (rc = field_maps<T>(&maps, f, g)))
      return rc;
  }
  if (dU) return launch_stencil<T, kGradient>(s, maps, tma, g, st);
  return launch_stencil<T, kEnergyOnly>(s, maps, tma, g, st);
}

template <typename T>
static int solver_t(const igm_grid* g, const igm_physics* ph, const igm_fields* f, void* U0, void* V0, void* U1,
                    void* V1, void* mU, void* mV, void* vU, void* vV, const igm_adam* ad, const igm_early_stop* es,
                    int n_it, int max_iter, igm_solver_ctl* ctl, double* costs, void* ws, size_t wsb,
                    cudaStream_t st) {
  StencilArgs<T> s{};
  fill_common(s, g, ph, f);
  s.U0 = (T*)U0;
  s.V0 = (T*)V0;
  s.U1 = (T*)U1;
  s.V1 = (T*)V1;
  s.mU = (T*)mU;
  s.mV = (T*)mV;
  s.vU = (T*)vU;
  s.vV = (T*)vV;
  s.lr = (T)ad->lr;
  s.b1 = (T)ad->beta_1;
  s.b2 = (T)ad->beta_2;
  s.eps = (T)ad->epsilon;
  s.es_delta = es ? es->relative_min_delta : 0.0;
  s.es_patience = es ? es->patience : 1;
  s.es_enabled = es ? es->enabled : 0;
  s.max_iter = max_iter;
  s.ctl = ctl;
  s.costs = costs;
  s.terms = nullptr;
  s.grad_scale = (T)s.inv_count;
  int rc = bind_workspace(ws, wsb, g, &s.counter, &s.partials);
  if (rc) return rc;
  s.err = (int*)((char*)ws + 4);
  StencilMaps maps;
  memset(&maps, 0, sizeof(maps));
  const bool tma =
      tma_usable<T>(g, {U0, V0, U1, V1, mU, mV, vU, vV, f->thk, f->usurf, f->arrhenius, f->slidingco});
  if (tma) {
    const int nl = g->batch * g->nz;
    if ((rc = level_map<T>(&maps.U0, U0, g, nl)) || (rc = level_map<T>(&maps.V0, V0, g, nl)) ||
        (rc = level_map<T>(&maps.U1, U1, g, nl)) || (rc = level_map<T>(&maps.V1, V1, g, nl)) ||
        (rc = level_map<T>(&maps.mU, mU, g, nl)) || (rc = level_map<T>(&maps.mV, mV, g, nl)) ||
        (rc = level_map<T>(&maps.vU, vU, g, nl)) || (rc = level_map<T>(&maps.vV, vV, g, nl)) ||
        (rc = field_maps<T>(&maps, f, g)))
      return rc;
  }
  for (int i = 0; i < n_it; ++i) {
    rc = launch_stencil<T, kAdamStep>(s, maps, tma, g, st);
    if (rc) return rc;
  }
  return IGM_OK;
}

__global__ void solver_begin_kernel(igm_solver_ctl* ctl, long long t0) {
  ctl->iter = 0;
  ctl->stopped = 0;
  ctl->status = IGM_OK;
  ctl->wait = 0;
  ctl->adam_t0 = t0;
  ctl->best = 0.0;
  ctl->last_cost = 0.0;
  ctl->terms[0] = ctl->terms[1] = ctl->terms[2] = 0.0;
}

// ---------------------------------------------------------------------------
// Reduction scratch of igm_energy_noalloc: a fixed array inside the library.
// The first 256 bytes hold the CTA counter, the rest the per-CTA FP64
// partial sums.  Every device that loads the library keeps this array until
// the process exits.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = (size_t)2 << 20;  // 2 MiB
static __device__ __align__(256) unsigned char g_energy_scratch[kNoAllocScratchBytes];

// Device address of g_energy_scratch for the current device.  In host code the
// array's name only stands in for the symbol; the address is looked up once per
// device (with that device current) and cached.
static int noalloc_scratch(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("igm_energy_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    return IGM_ERR_CUDA;
  }
  constexpr int kMaxDevices = 128;
  static std::mutex mu;
  static void* addr[kMaxDevices] = {};
  IGM_CHECK_ARG(dev >= 0 && dev < kMaxDevices, IGM_ERR_CUDA, "igm_energy_noalloc: device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_energy_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("igm_energy_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
    addr[dev] = p;
  }
  *out = addr[dev];
  return IGM_OK;
}

}  // namespace igm

using namespace igm;

extern "C" int igm_energy_noalloc(int dtype, const igm_grid* grid, const igm_physics* phys, const igm_fields* fields,
                                  const void* U, const void* V, void* dU, void* dV, double grad_scale, double* terms,
                                  void* stream) {
  int rc = check_grid(grid);
  if (rc) return rc;
  IGM_CHECK_ARG(phys && fields && U && V && terms, IGM_ERR_BAD_ARGUMENT, "igm_energy_noalloc: NULL argument");
  IGM_CHECK_ARG((dU == nullptr) == (dV == nullptr), IGM_ERR_BAD_ARGUMENT,
                "igm_energy_noalloc: dU and dV must both be set or both NULL");
  IGM_CHECK_ARG(fields->thk && fields->usurf && fields->arrhenius && fields->slidingco, IGM_ERR_BAD_ARGUMENT,
                "igm_energy_noalloc: NULL field");
  IGM_CHECK_ARG(dtype == IGM_F32 || dtype == IGM_F64, IGM_ERR_BAD_ARGUMENT, "igm_energy_noalloc: unknown dtype %d",
                dtype);
  const size_t need = workspace_bytes_for(grid);
  IGM_CHECK_ARG(need <= kNoAllocScratchBytes, IGM_ERR_WORKSPACE,
                "igm_energy_noalloc: this grid (batch %d x %d x %d) needs %zu bytes of reduction scratch, more than "
                "the library's fixed %zu-byte array; call igm_energy with a workspace instead",
                grid->batch, grid->ny, grid->nx, need, kNoAllocScratchBytes);
  void* ws = nullptr;
  rc = noalloc_scratch(&ws);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  // The CTA counter must start at zero.  Kernels leave it at zero, but a call
  // that failed part-way could not; clearing it costs one 256-byte memset.
  cudaError_t e = cudaMemsetAsync(ws, 0, 256, st);
  if (e != cudaSuccess) {
    set_error("igm_energy_noalloc: clearing the counter: %s", cudaGetErrorString(e));
    return IGM_ERR_CUDA;
  }
  if (dtype == IGM_F32)
    return energy_t<float>(grid, phys, fields, U, V, dU, dV, grad_scale, terms, ws, kNoAllocScratchBytes, st);
  return energy_t<double>(grid, phys, fields, U, V, dU, dV, grad_scale, terms, ws, kNoAllocScratchBytes, st);
}

extern "C" size_t igm_workspace_size(const igm_grid* grid) {
  if (check_grid(grid) != IGM_OK) return 0;
  return workspace_bytes_for(grid);
}

extern "C" int igm_energy(int dtype, const igm_grid* grid, const igm_physics* phys, const igm_fields* fields,
                          const void* U, const void* V, void* dU, void* dV, double grad_scale, double* terms,
                          void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_grid(grid);
  if (rc) return rc;
  IGM_CHECK_ARG(phys && fields && U && V && terms, IGM_ERR_BAD_ARGUMENT, "igm_energy: NULL argument");
  IGM_CHECK_ARG((dU == nullptr) == (dV == nullptr), IGM_ERR_BAD_ARGUMENT, "igm_energy: dU and dV must both be set or both NULL");
  IGM_CHECK_ARG(fields->thk && fields->usurf && fields->arrhenius && fields->slidingco, IGM_ERR_BAD_ARGUMENT,
                "igm_energy: NULL field");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    return energy_t<float>(grid, phys, fields, U, V, dU, dV, grad_scale, terms, workspace, workspace_bytes, st);
  if (dtype == IGM_F64)
    return energy_t<double>(grid, phys, fields, U, V, dU, dV, grad_scale, terms, workspace, workspace_bytes, st);
  set_error("igm_energy: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_solver_begin(igm_solver_ctl* ctl, int64_t adam_iterations, void* stream) {
  IGM_CHECK_ARG(ctl != nullptr, IGM_ERR_BAD_ARGUMENT, "igm_solver_begin: ctl is NULL");
  solver_begin_kernel<<<1, 1, 0, as_stream(stream)>>>(ctl, (long long)adam_iterations);
  return launch_status("solver_begin_kernel");
}

extern "C" int igm_solver_iterate(int dtype, const igm_grid* grid, const igm_physics* phys, const igm_fields* fields,
                                  void* U0, void* V0, void* U1, void* V1, void* mU, void* mV, void* vU, void* vV,
                                  const igm_adam* adam, const igm_early_stop* early_stop, int n_iterations,
                                  int max_iter, igm_solver_ctl* ctl, double* costs, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  int rc = check_grid(grid);
  if (rc) return rc;
  IGM_CHECK_ARG(phys && fields && U0 && V0 && U1 && V1 && mU && mV && vU && vV && adam && ctl && costs,
                IGM_ERR_BAD_ARGUMENT, "igm_solver_iterate: NULL argument");
  IGM_CHECK_ARG(n_iterations >= 0 && max_iter >= 1, IGM_ERR_BAD_ARGUMENT, "igm_solver_iterate: bad iteration counts");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    return solver_t<float>(grid, phys, fields, U0, V0, U1, V1, mU, mV, vU, vV, adam, early_stop, n_iterations,
                           max_iter, ctl, costs, workspace, workspace_bytes, st);
  if (dtype == IGM_F64)
    return solver_t<double>(grid, phys, fields, U0, V0, U1, V1, mU, mV, vU, vV, adam, early_stop, n_iterations,
                            max_iter, ctl, costs, workspace, workspace_bytes, st);
  set_error("igm_solver_iterate: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}
