// 2-D field kernels of the path: velocity reduction (+ mask + CFL max),
// slope-limited upwind thickness transport, surfaces, ELA mass balance and
// the CFL time step.  All are HBM-bound elementwise/stencil passes.
#include "common.cuh"

namespace igm {

// ---------------------------------------------------------------------------
// velbase / velsurf / velbar (iceflow/utils.py:21-51), optional mask
// where(thk > 0, U, 0) (solve.py:116-117), and max(|ubar|, |vbar|) (time.py:36-39)
// ---------------------------------------------------------------------------
template <typename T>
struct VelArgs {
  int batch, nz, ny, nx, mask;
  T* U;
  T* V;
  const T* thk;
  T w[IGM_MAX_NZ];
  T* ubar;
  T* vbar;
  T* ub0;
  T* vb0;
  T* us0;
  T* vs0;
  float* velomax;
};

template <typename T>
__global__ void __launch_bounds__(256) velocity_reduce_kernel(const VelArgs<T> a) {
  const size_t plane = (size_t)a.ny * a.nx;
  const size_t total = plane * a.batch;
  float vmax = 0.f;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t b = idx / plane, p = idx - b * plane;
    const size_t base = b * a.nz * plane + p;
    const bool keep = !a.mask || a.thk[idx] > T(0);
    T su = 0, sv = 0, u0 = 0, v0 = 0, u1 = 0, v1 = 0;
    if (!keep) {
      // masked column: zeros, nothing to read
      for (int k = 0; k < a.nz; ++k) {
        a.U[base + k * plane] = T(0);
        a.V[base + k * plane] = T(0);
      }
    } else {
      // the column's loads issued eight levels at a time (no store in this branch, so they need
      // not wait for one another); the sums in level order, as the reference's reduce_sum
      for (int k0 = 0; k0 < a.nz; k0 += 8) {
        T u[8], v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int k = k0 + q;
          u[q] = k < a.nz ? a.U[base + k * plane] : T(0);
          v[q] = k < a.nz ? a.V[base + k * plane] : T(0);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int k = k0 + q;
          if (k < a.nz) {
            su += u[q] * a.w[k];
            sv += v[q] * a.w[k];
          }
        }
        if (k0 == 0) {
          u0 = u[0];
          v0 = v[0];
        }
        const int kl = a.nz - 1 - k0;
        if (kl >= 0 && kl < 8) {
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (q == kl) {
              u1 = u[q];
              v1 = v[q];
            }
        }
      }
    }
    if (a.ubar) a.ubar[idx] = su;
    if (a.vbar) a.vbar[idx] = sv;
    if (a.ub0) a.ub0[idx] = u0;
    if (a.vb0) a.vb0[idx] = v0;
    if (a.us0) a.us0[idx] = u1;
    if (a.vs0) a.vs0[idx] = v1;
    const float m = fmaxf(fabsf((float)su), fabsf((float)sv));
    vmax = fmaxf(vmax, m);
  }
  if (a.velomax) {
    for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_down_sync(0xffffffffu, vmax, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(a.velomax, vmax);
  }
}

// ---------------------------------------------------------------------------
// transport (compute_divflux_slope_limiter.py:11-65 + thk.py:36-54)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T minmod(T a, T b) {
  const bool pos = a * b > T(0);
  const T fa = fabs(a), fb = fabs(b);
  return (fa < fb && pos) ? a : ((fa > fb && pos) ? b : T(0));
}
template <typename T>
__device__ __forceinline__ T maxmod(T a, T b) {
  const bool pos = a * b > T(0);
  const T fa = fabs(a), fb = fabs(b);
  return (fa < fb && pos) ? b : ((fa > fb && pos) ? a : T(0));
}

template <typename T>
struct TransportArgs {
  int ny, nx, slope;
  T dx, rdx, half_dx, dt_host, ratio, sealevel;  // rdx = 1/dx correctly rounded in T
  const float* dt_dev;
  const T* u;
  const T* v;
  const T* h;
  T* h_out;
  const T* topg;
  const T* smb;
  T* usurf;
  T* lsurf;
  T* divflux;
};

// num / dx, correctly rounded (the IEEE quotient), for dx > 0 and |num| well
// inside the normal range, from the correctly rounded reciprocal rdx = RN(1/dx)
// by Markstein's division step (P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1),
// 1990): q = RN(num rdx) is within one ulp of num/dx, the remainder
// r = num - dx q is exact in one fma, and RN(q + r rdx) is the correctly
// rounded quotient.  A zero numerator is returned as is (keeps its sign).
template <typename T>
__device__ __forceinline__ T div_dx(T num, T dx, T rdx) {
  const T q = num * rdx;
  const T r = fma(-q, dx, num);
  const T d = fma(r, rdx, q);
  return num == T(0) ? num : d;
}

template <typename T>
__device__ __forceinline__ T limited_slope(T hm, T h0, T hp, T dx, T rdx, int slope) {
  // slope of the cell holding h0 from its neighbours hm (left) and hp (right)
  const T sigp = div_dx(hp - h0, dx, rdx), sigm = div_dx(h0 - hm, dx, rdx);
  if (slope == IGM_GODUNOV) return T(0);
  if (slope == IGM_MINMOD) return minmod(sigm, sigp);
  return maxmod(minmod(sigp, T(2) * sigm), minmod(sigm, T(2) * sigp));
}

// A warp owns a strip of 30 columns (lanes 1..30; lanes 0 and 31 carry the
// columns on either side) and walks down a segment of rows.
// x neighbours come from the adjacent lanes by shuffles; in y the thread keeps
// a window of its column (thickness of rows j-1 .. j+2, the slope of cell j and
// the flux through the face below node j), so every slope and face flux of the
// interior is evaluated once.  The loads of a row are issued two rows ahead.
// Each quantity is evaluated with the operations and order of the reference
// (IEEE division by dx through div_dx, no contraction), so the result is
// bit-identical to evaluating each face of the reference on its own.
constexpr int kTmCols = 30;  // interior columns per warp
#ifndef IGM_TM_MIN_ROWS
#define IGM_TM_MIN_ROWS 8
#endif
constexpr int kTmMinRows = IGM_TM_MIN_ROWS;  // shortest row segment of a warp (even)
constexpr int kTmWarps = 4;  // warps per CTA

template <typename T, int SLOPE>
__device__ __forceinline__ T cell_slope(T hm, T h0, T hp, T dx, T rdx) {
  if (SLOPE == IGM_GODUNOV) return T(0);
  const T sigp = div_dx(hp - h0, dx, rdx), sigm = div_dx(h0 - hm, dx, rdx);
  if (SLOPE == IGM_MINMOD) return minmod(sigm, sigp);
  // superbee: maxmod(minmod(sigp, 2 sigm), minmod(sigm, 2 sigp)).  The two minmods' sign tests
  // sigp (2 sigm) > 0 and sigm (2 sigp) > 0 round the same exact product 2 sigp sigm (doubling is
  // exact), so they are one test.
  const T m2 = T(2) * sigm, p2 = T(2) * sigp;
  const bool pos = sigp * m2 > T(0);
  const T fa = fabs(sigp), fb = fabs(m2), fc = fabs(sigm), fd = fabs(p2);
  const T s1 = (fa < fb && pos) ? sigp : ((fa > fb && pos) ? m2 : T(0));
  const T s2 = (fc < fd && pos) ? sigm : ((fc > fd && pos) ? p2 : T(0));
  return maxmod(s1, s2);
}

// upwind flux through a face with velocity uf between cells (hl, sl) and (hr, sr): only the state
// tf.where(u > 0, w, e) keeps is evaluated, with the reference's operations and order
// (w = hl + (half_dx (1 - cu)) sl, e = hr - (half_dx (1 + cu)) sr)
template <typename T>
__device__ __forceinline__ T face_flux(T uf, T hl, T hr, T sl, T sr, T dt, T dx, T rdx, T half_dx) {
  const T cu = div_dx(uf * dt, dx, rdx);
  const bool up = uf > T(0);
  const T h = up ? hl : hr;
  const T c = up ? T(1) - cu : T(1) + cu;
  const T t = half_dx * c * (up ? sl : sr);
  return uf * (up ? h + t : h - t);
}

template <typename T>
struct MarchRow {
  T h2;  // thickness two rows below (j + 2)
  T v1;  // vbar one row below (j + 1)
  T u, tg, sm;
  T he;  // edge lanes: thickness of the column beyond the strip, row j
};

// ROWS: the segment's rows y0-2 .. y1+4 may leave the domain (the first and last
// segments of a strip), so every row index is checked; interior segments skip
// those checks.
template <typename T, int SLOPE, bool ROWS>
__device__ __forceinline__ void transport_march(const TransportArgs<T>& a, int lane, int strip, int y0, int y1) {
  const int nx = a.nx, ny = a.ny;
  const int i = strip * kTmCols - 1 + lane;  // this lane's column
  const bool col = i >= 0 && i < nx;
  const size_t ic = col ? (size_t)i : 0;
  const int ie = lane == 0 ? i - 1 : i + 1;  // the extra column of the edge lanes
  const bool ecol = (lane == 0 || lane == 31) && ie >= 0 && ie < nx;
  const size_t iec = ecol ? (size_t)ie : 0;
  const bool out_lane = lane >= 1 && lane <= kTmCols && col;
  const T dt = a.dt_dev ? (T)(*a.dt_dev) : a.dt_host;
  const T dx = a.dx, rdx = a.rdx, hdx = a.half_dx;
  const T* H = a.h;
  auto at = [&](const T* p, int j, bool ok, size_t c) -> T {
    if (ROWS) return (ok && j >= 0 && j < ny) ? p[(size_t)j * nx + c] : T(0);
    return ok ? p[(size_t)j * nx + c] : T(0);
  };
  // interior segments: every row of the segment is in the domain, so a row's six loads share one
  // element offset (the row's start), computed once
  const T* hc = H + ic;
  const T* vc = a.v + ic;
  const T* uc = a.u + ic;
  const T* tc_ = a.topg + ic;
  const T* sc_ = a.smb ? a.smb + ic : nullptr;
  const T* hec = H + iec;
  const size_t nx1 = (size_t)nx, nx2 = 2 * (size_t)nx;
  auto load_row = [&](int j) {
    MarchRow<T> r;
    if (ROWS) {
      const bool live = j < y1;
      r.h2 = at(H, j + 2, live && col, ic);
      r.v1 = at(a.v, j + 1, live && col, ic);
      r.u = at(a.u, j, live && col, ic);
      r.tg = at(a.topg, j, live && col, ic);
      r.sm = a.smb ? at(a.smb, j, live && col, ic) : T(0);
      r.he = at(H, j, live && ecol, iec);
    } else {
      const size_t o = (size_t)j * nx1;
      r.h2 = col ? hc[o + nx2] : T(0);
      r.v1 = col ? vc[o + nx1] : T(0);
      r.u = col ? uc[o] : T(0);
      r.tg = col ? tc_[o] : T(0);
      r.sm = (sc_ && col) ? sc_[o] : T(0);
      r.he = ecol ? hec[o] : T(0);
    }
    return r;
  };
  // prologue: the y slopes of cells y0-1 and y0 and the flux through face y0
  T hm1 = at(H, y0 - 1, col, ic), h0 = at(H, y0, col, ic), hp1 = at(H, y0 + 1, col, ic);
  T v0 = at(a.v, y0, col, ic);
  T sy0, qs;
  {
    const T hm2 = at(H, y0 - 2, col, ic);
    const T vm1 = at(a.v, y0 - 1, col, ic);
    const T sym1 = cell_slope<T, SLOPE>(hm2, hm1, h0, dx, rdx);
    sy0 = cell_slope<T, SLOPE>(hm1, h0, hp1, dx, rdx);
    const T vf = y0 == 0 ? v0 : T(0.5) * (vm1 + v0);
    qs = face_flux(vf, hm1, h0, sym1, sy0, dt, dx, rdx, hdx);
  }
  auto step = [&](int j, const MarchRow<T>& r) {
    // y: slope of cell j+1, flux through face j+1 (between rows j and j+1)
    const T sy1 = cell_slope<T, SLOPE>(h0, hp1, r.h2, dx, rdx);
    const T vf = (ROWS && j + 1 == ny) ? v0 : T(0.5) * (v0 + r.v1);
    const T qn = face_flux(vf, h0, hp1, sy0, sy1, dt, dx, rdx, hdx);
    // x: slope of this lane's cell, flux through its left face (face i)
    T hl = __shfl_up_sync(0xffffffffu, h0, 1), hr = __shfl_down_sync(0xffffffffu, h0, 1);
    if (lane == 0) hl = r.he;
    if (lane == 31) hr = r.he;
    const T sx = cell_slope<T, SLOPE>(hl, h0, hr, dx, rdx);
    const T sxl = __shfl_up_sync(0xffffffffu, sx, 1);
    const T ul = __shfl_up_sync(0xffffffffu, r.u, 1);
    const T uf = i == 0 ? r.u : (i == nx ? ul : T(0.5) * (ul + r.u));
    const T qw = face_flux(uf, hl, h0, sxl, sx, dt, dx, rdx, hdx);
    const T qe = __shfl_down_sync(0xffffffffu, qw, 1);
    if (out_lane) {
      const T div = div_dx(qe - qw, dx, rdx) + div_dx(qn - qs, dx, rdx);
      T hn = h0 + dt * (r.sm - div);
      hn = hn > T(0) ? hn : T(0);
      const T fl = -a.ratio * hn + a.sealevel;
      const T ls = r.tg > fl ? r.tg : fl;
      const size_t o = (size_t)j * nx + ic;
      a.h_out[o] = hn;
      a.usurf[o] = ls + hn;
      if (a.lsurf) a.lsurf[o] = ls;
      if (a.divflux) a.divflux[o] = div;
    }
    hm1 = h0;
    h0 = hp1;
    hp1 = r.h2;
    v0 = r.v1;
    sy0 = sy1;
    qs = qn;
  };
  MarchRow<T> r0 = load_row(y0), r1 = load_row(y0 + 1);
  for (int j = y0; j < y1; j += 2) {
    const MarchRow<T> r2 = load_row(j + 2);
    step(j, r0);
    const MarchRow<T> r3 = load_row(j + 3);
    if (j + 1 < y1) step(j + 1, r1);
    r0 = r2;
    r1 = r3;
  }
  (void)hm1;
}

template <typename T, int SLOPE>
__global__ void __launch_bounds__(kTmWarps * 32) transport_march_kernel(const TransportArgs<T> a, int n_strips,
                                                                       int rows_per_seg) {
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * kTmWarps + (threadIdx.x >> 5);
  const int strip = gw % n_strips, seg = gw / n_strips;
  const int y0 = seg * rows_per_seg;
  if (y0 >= a.ny) return;  // uniform per warp
  const int y1 = min(y0 + rows_per_seg, a.ny);
  if (y0 >= 2 && y1 + 5 <= a.ny)  // every row loaded (y0-2 .. y1+4) is in the domain
    transport_march<T, SLOPE, false>(a, lane, strip, y0, y1);
  else
    transport_march<T, SLOPE, true>(a, lane, strip, y0, y1);
}

template <typename T>
__global__ void surfaces_kernel(int n, const T* thk, const T* topg, T* lsurf, T* usurf, T ratio, T sealevel) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
    const T h = thk[idx], tg = topg[idx];
    const T fl = -ratio * h + sealevel;
    const T ls = tg > fl ? tg : fl;
    if (lsurf) lsurf[idx] = ls;
    usurf[idx] = ls + h;
  }
}

template <typename T>
__global__ void smb_kernel(int n, const T* usurf, const T* icemask, T* smb, T gabl, T gacc, T ela, T maxacc) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
    T s = usurf[idx] - ela;
    s *= s < T(0) ? gabl : gacc;
    s = s < T(-100) ? T(-100) : (s > maxacc ? maxacc : s);
    if (icemask && !(s < T(0) || icemask[idx] > T(0.5))) s = T(-10);
    smb[idx] = s;
  }
}

template <typename T>
__global__ void absmax2_kernel(int n, const T* a, const T* b, float* out) {
  float m = 0.f;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x)
    m = fmaxf(m, fmaxf(fabsf((float)a[idx]), fabsf((float)b[idx])));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

// force_max_velbar (igm/processes/iceflow/utils.py:182-194, Lagrange basis):
// per node and level, with mag = |(U, V)| (tf.norm of the stacked pair:
// sqrt(U U + V V), no fused multiply-add), U = cap (U / mag) and V = cap
// (V / mag) where mag >= cap, else unchanged; IEEE division, as the reference
// graph.
template <typename T>
__global__ void force_max_velbar_kernel(size_t n, T* U, T* V, T cap) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const T u = U[i], v = V[i];
    // this unit is compiled with -fmad=false and IEEE division / square root
    const T mag = Math<T>::sqrt(u * u + v * v);
    if (mag >= cap) {
      U[i] = cap * (u / mag);
      V[i] = cap * (v / mag);
    }
  }
}

__global__ void cfl_dt_kernel(const float* velomax, float* dt, float cfl_dx, float step_max) {
  const float vm = *velomax;
  float d = step_max;
  if (vm > 0.f) {
    const float c = cfl_dx / vm;
    d = c < step_max ? c : step_max;
  }
  *dt = d;
}

static int grid1d(size_t n) {
  size_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

template <typename T>
static int velocity_t(int batch, int nz, int ny, int nx, void* U, void* V, const void* thk, int mask,
                      const double* w, void* ubar, void* vbar, void* ub0, void* vb0, void* us0, void* vs0,
                      float* velomax, cudaStream_t st) {
  VelArgs<T> a{};
  a.batch = batch; a.nz = nz; a.ny = ny; a.nx = nx; a.mask = mask;
  a.U = (T*)U; a.V = (T*)V; a.thk = (const T*)thk;
  for (int k = 0; k < nz; ++k) a.w[k] = (T)w[k];
  a.ubar = (T*)ubar; a.vbar = (T*)vbar; a.ub0 = (T*)ub0; a.vb0 = (T*)vb0; a.us0 = (T*)us0; a.vs0 = (T*)vs0;
  a.velomax = velomax;
  if (velomax) {
    cudaError_t e = cudaMemsetAsync(velomax, 0, sizeof(float), st);
    if (e != cudaSuccess) {
      set_error("igm_velocity_reduce: %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
  }
  velocity_reduce_kernel<T><<<grid1d((size_t)batch * ny * nx), 256, 0, st>>>(a);
  return launch_status("velocity_reduce_kernel");
}

template <typename T>
static int transport_t(int ny, int nx, double dx, const void* u, const void* v, const void* h, void* h_out,
                       const void* topg, const void* smb, void* usurf, void* lsurf, void* divflux, double dt,
                       const float* dt_dev, int slope, double ratio, double sealevel, cudaStream_t st) {
  TransportArgs<T> a{};
  a.ny = ny; a.nx = nx; a.slope = slope;
  a.dx = (T)dx; a.half_dx = (T)(0.5 * dx); a.dt_host = (T)dt; a.ratio = (T)ratio; a.sealevel = (T)sealevel;
  a.rdx = T(1) / a.dx;  // host IEEE division in T: the correctly rounded reciprocal
  a.dt_dev = dt_dev;
  a.u = (const T*)u; a.v = (const T*)v; a.h = (const T*)h; a.h_out = (T*)h_out; a.topg = (const T*)topg;
  a.smb = (const T*)smb; a.usurf = (T*)usurf; a.lsurf = (T*)lsurf; a.divflux = (T*)divflux;
  // segments of rows sized for about 32 resident warps per SM, at least kTmMinRows rows
  const int n_strips = (nx + kTmCols - 1) / kTmCols;
  const long long target = 148LL * 32;
  int rows = (int)((n_strips * (long long)ny + target - 1) / target);
  rows = rows < kTmMinRows ? kTmMinRows : rows;
  rows += rows & 1;
  const long long warps = (long long)n_strips * ((ny + rows - 1) / rows);
  const int grid = (int)((warps + kTmWarps - 1) / kTmWarps);
  if (slope == IGM_GODUNOV)
    transport_march_kernel<T, IGM_GODUNOV><<<grid, kTmWarps * 32, 0, st>>>(a, n_strips, rows);
  else if (slope == IGM_MINMOD)
    transport_march_kernel<T, IGM_MINMOD><<<grid, kTmWarps * 32, 0, st>>>(a, n_strips, rows);
  else
    transport_march_kernel<T, IGM_SUPERBEE><<<grid, kTmWarps * 32, 0, st>>>(a, n_strips, rows);
  return launch_status("transport_march_kernel");
}

// ---------------------------------------------------------------------------
// vertical velocity, vert_flow version 2, kinematic method
// (vert_flow/vert_flow_v2.py:17-37, 62-87, 126-147; vert_disc.py:17-23)
// ---------------------------------------------------------------------------
template <typename T>
struct VertFlowArgs {
  int nz, ny, nx;
  T dx, rdx;               // rdx = RN(1/dx) in T
  T lev[IGM_MAX_NZ];       // levels (zeta map of compute_levels)
  T w[IGM_MAX_NZ];         // vert_weight
  const T* U;
  const T* V;
  const T* topg;
  const T* thk;
  T* W;
};

template <typename T>
__device__ __forceinline__ T ieee_div(T a, T b);
template <>
__device__ __forceinline__ float ieee_div<float>(float a, float b) { return __fdiv_rn(a, b); }
template <>
__device__ __forceinline__ double ieee_div<double>(double a, double b) { return __ddiv_rn(a, b); }

// A warp owns a strip of 30 columns (lanes 1..30; lanes 0 and 31 carry the
// columns on either side) and kVfRows rows plus the row above and below; each
// thread keeps, for its column's kVfRows + 2 nodes, the running sums of the
// layer walk in registers: the layer height z_k - topg (the scan of
// thk (level[l+1] - level[l])) and the weighted sums of U and V.  Per layer it
// forms the layer surface topg + z_k and the fluxes (mean U) z_k, (mean V) z_k
// of those nodes; y neighbours are the thread's own registers, x neighbours
// come from the adjacent lanes by shuffles -- no shared memory, no barrier.
// Operation order and rounding follow the reference (no contraction: this unit
// is built with -fmad=false; every quotient is the correctly rounded one, by
// Markstein's step from the divisor's correctly rounded reciprocal -- dx, and
// per layer the sum of the weights), so W is bit-identical.
constexpr int kVfRows = 8;   // output rows per warp
constexpr int kVfCols = 30;  // output columns per warp
constexpr int kVfWarps = 4;  // warps per CTA
template <typename T>
__global__ void __launch_bounds__(kVfWarps * 32) vert_flow_kernel(const VertFlowArgs<T> a, int n_strips) {
  constexpr int R = kVfRows + 2;
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * kVfWarps + (threadIdx.x >> 5);
  const int strip = gw % n_strips, seg = gw / n_strips;
  const int nx = a.nx, ny = a.ny;
  const int j0 = seg * kVfRows;
  if (j0 >= ny) return;  // uniform per warp
  const int i = strip * kVfCols - 1 + lane;
  const bool col = i >= 0 && i < nx;
  const size_t ic = col ? (size_t)i : 0;
  const size_t plane = (size_t)ny * nx;
  const bool out_lane = lane >= 1 && lane <= kVfCols && col;
  const T dx = a.dx, rdx = a.rdx;
  T tg[R], th[R], zh[R], su[R], sv[R];
  bool in[R];
  size_t off[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 - 1 + r;
    in[r] = col && j >= 0 && j < ny;
    off[r] = in[r] ? (size_t)j * nx + ic : 0;
    tg[r] = in[r] ? a.topg[off[r]] : T(0);
    th[r] = in[r] ? a.thk[off[r]] : T(0);
    zh[r] = T(0);
    su[r] = T(0);
    sv[r] = T(0);
  }
  T sw = T(0);
  for (int k = 0; k < a.nz; ++k) {
    T u[R], v[R], z[R], qx[R], qy[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      u[r] = in[r] ? a.U[(size_t)k * plane + off[r]] : T(0);
      v[r] = in[r] ? a.V[(size_t)k * plane + off[r]] : T(0);
    }
    sw = k == 0 ? a.w[0] : sw + a.w[k];
    const T rsw = ieee_div(T(1), sw);  // the layer's one divisor: Markstein's step from its reciprocal
    const T ddz = k > 0 ? a.lev[k] - a.lev[k - 1] : T(0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (k > 0) {
        const T dzl = th[r] * ddz;
        zh[r] = k == 1 ? dzl : zh[r] + dzl;
      }
      const T wu = a.w[k] * u[r], wv = a.w[k] * v[r];
      su[r] = k == 0 ? wu : su[r] + wu;
      sv[r] = k == 0 ? wv : sv[r] + wv;
      z[r] = tg[r] + zh[r];
      qx[r] = div_dx(su[r], sw, rsw) * zh[r];
      qy[r] = div_dx(sv[r], sw, rsw) * zh[r];
    }
#pragma unroll
    for (int r = 1; r <= kVfRows; ++r) {
      const int j = j0 - 1 + r;
      const T zl = __shfl_up_sync(0xffffffffu, z[r], 1), zr = __shfl_down_sync(0xffffffffu, z[r], 1);
      const T ql = __shfl_up_sync(0xffffffffu, qx[r], 1), qr = __shfl_down_sync(0xffffffffu, qx[r], 1);
      if (!out_lane || j >= ny) continue;
      // faces of the layer surface (compute_gradient_layers_tf)
      const T zw = i == 0 ? T(1.5) * z[r] - T(0.5) * zr : T(0.5) * zl + T(0.5) * z[r];
      const T ze = i == nx - 1 ? T(1.5) * z[r] - T(0.5) * zl : T(0.5) * z[r] + T(0.5) * zr;
      const T zs = j == 0 ? T(1.5) * z[r] - T(0.5) * z[r + 1] : T(0.5) * z[r - 1] + T(0.5) * z[r];
      const T zn = j == ny - 1 ? T(1.5) * z[r] - T(0.5) * z[r - 1] : T(0.5) * z[r] + T(0.5) * z[r + 1];
      // faces of the fluxes (compute_divflux_layers)
      const T fw = i == 0 ? qx[r] : T(0.5) * (ql + qx[r]);
      const T fe = i == nx - 1 ? qx[r] : T(0.5) * (qx[r] + qr);
      const T fs = j == 0 ? qy[r] : T(0.5) * (qy[r - 1] + qy[r]);
      const T fn = j == ny - 1 ? qy[r] : T(0.5) * (qy[r] + qy[r + 1]);
      const T sx = div_dx(ze - zw, dx, rdx), sy = div_dx(zn - zs, dx, rdx);
      const T div = div_dx(fe - fw, dx, rdx) + div_dx(fn - fs, dx, rdx);
      a.W[(size_t)k * plane + off[r]] = (-div + u[r] * sx) + v[r] * sy;
    }
  }
}

// vert_flow version 2, incompressibility method (vert_flow_v2.py:40-57 with
// gradx/grady_non_flat_layers_tf :168-199), uniform spacing dX = dx.  Same
// warp layout as vert_flow_kernel; a thread walks its column's nodes up the
// layers carrying the layer height above the bed (the scan of
// thk (level[k] - level[k-1])), the running sum of dz (du/dx + dv/dy) and the
// lower layer-face values of U and V, with U, V of the next layer loaded one
// layer ahead.  x neighbours (U and the layer surface Z) by shuffles, y
// neighbours (V and Z) from the thread's own rows.  Operation order and
// rounding follow the reference: division by dx by Markstein's step, by
// vert_weight thk (per node) in IEEE division; no contraction.
template <typename T>
__global__ void __launch_bounds__(kVfWarps * 32) vert_flow_incomp_kernel(const VertFlowArgs<T> a, int n_strips) {
  constexpr int R = kVfRows + 2;
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * kVfWarps + (threadIdx.x >> 5);
  const int strip = gw % n_strips, seg = gw / n_strips;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int j0 = seg * kVfRows;
  if (j0 >= ny) return;  // uniform per warp
  const int i = strip * kVfCols - 1 + lane;
  const bool col = i >= 0 && i < nx;
  const size_t ic = col ? (size_t)i : 0;
  const size_t plane = (size_t)ny * nx;
  const bool out_lane = lane >= 1 && lane <= kVfCols && col;
  const T dx = a.dx, rdx = a.rdx, h = T(0.5), o5 = T(1.5);
  // x and y derivative of a field from this node (c), its x neighbours (l, r) and its
  // y neighbours (s, n), with the reference's one-sided border faces
  auto ddx = [&](T l, T c, T r) {
    const T fw = i == 0 ? o5 * c - h * r : h * l + h * c;
    const T fe = i == nx - 1 ? o5 * c - h * l : h * c + h * r;
    return div_dx(fe - fw, dx, rdx);
  };
  auto ddy = [&](int j, T s_, T c, T n_) {
    const T fs = j == 0 ? o5 * c - h * n_ : h * s_ + h * c;
    const T fn = j == ny - 1 ? o5 * c - h * s_ : h * c + h * n_;
    return div_dx(fn - fs, dx, rdx);
  };
  T tg[R], th[R], zc[R], uc[R], vc[R], ufl[R], vfl[R], cum[R], base[R];
  bool in[R];
  size_t off[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 - 1 + r;
    in[r] = col && j >= 0 && j < ny;
    off[r] = in[r] ? (size_t)j * nx + ic : 0;
    tg[r] = in[r] ? a.topg[off[r]] : T(0);
    th[r] = in[r] ? a.thk[off[r]] : T(0);
    uc[r] = in[r] ? a.U[off[r]] : T(0);
    vc[r] = in[r] ? a.V[off[r]] : T(0);
    ufl[r] = uc[r];  // the bed face is U_0 itself
    vfl[r] = vc[r];
    zc[r] = T(0);
    cum[r] = T(0);
  }
  // U_0 dtopg/dx + V_0 dtopg/dy of the output rows (compute_gradient_tf of topg)
#pragma unroll
  for (int r = 1; r <= kVfRows; ++r) {
    const T tl = __shfl_up_sync(0xffffffffu, tg[r], 1), tr = __shfl_down_sync(0xffffffffu, tg[r], 1);
    base[r] = ddx(tl, tg[r], tr) * uc[r] + ddy(j0 - 1 + r, tg[r - 1], tg[r], tg[r + 1]) * vc[r];
  }
  for (int k = 0; k < nz; ++k) {
    T un[R], vn[R];
    const bool more = k + 1 < nz;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      un[r] = (more && in[r]) ? a.U[(size_t)(k + 1) * plane + off[r]] : T(0);
      vn[r] = (more && in[r]) ? a.V[(size_t)(k + 1) * plane + off[r]] : T(0);
    }
    const T ddz = k > 0 ? a.lev[k] - a.lev[k - 1] : T(0);
    const T wk = a.w[k];
    T z[R], dz[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      dz[r] = k > 0 ? th[r] * ddz : T(0);
      zc[r] = k == 0 ? dz[r] : zc[r] + dz[r];
      z[r] = zc[r] + tg[r];
    }
#pragma unroll
    for (int r = 1; r <= kVfRows; ++r) {
      const int j = j0 - 1 + r;
      const T zl = __shfl_up_sync(0xffffffffu, z[r], 1), zr = __shfl_down_sync(0xffffffffu, z[r], 1);
      const T ul = __shfl_up_sync(0xffffffffu, uc[r], 1), ur = __shfl_down_sync(0xffffffffu, uc[r], 1);
      if (!out_lane || j >= ny) continue;
      // du/dz, dv/dz between this layer's faces, zero off the ice
      const T ufh = more ? h * (uc[r] + un[r]) : uc[r];
      const T vfh = more ? h * (vc[r] + vn[r]) : vc[r];
      const T hw = wk * th[r];
      const bool ice = th[r] > T(0);
      const T dudz = ice ? ieee_div(ufh - ufl[r], hw) : T(0);
      const T dvdz = ice ? ieee_div(vfh - vfl[r], hw) : T(0);
      const T dudx = ddx(ul, uc[r], ur) - ddx(zl, z[r], zr) * dudz;
      const T dvdy = ddy(j, vc[r - 1], vc[r], vc[r + 1]) - ddy(j, z[r - 1], z[r], z[r + 1]) * dvdz;
      const T term = dz[r] * (dudx + dvdy);
      cum[r] = k == 0 ? term : cum[r] + term;
      a.W[(size_t)k * plane + off[r]] = base[r] - cum[r];
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      ufl[r] = more ? h * (uc[r] + un[r]) : uc[r];
      vfl[r] = more ? h * (vc[r] + vn[r]) : vc[r];
      uc[r] = un[r];
      vc[r] = vn[r];
    }
  }
}

// compute_divflux (igm/utils/gradient/compute_divflux.py:6-51): upwind (face
// velocities with edge copies at the border, the upwind thickness, zero
// outside) or centered (face averages of u h, edge copies), then the
// divergence; bit-identical to the reference.
template <typename T, int METHOD>
__global__ void divflux_kernel(int ny, int nx, T dx, T rdx, const T* u, const T* v, const T* h, T* out) {
  const size_t n = (size_t)ny * nx;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(o / nx), i = (int)(o - (size_t)j * nx);
    auto hh = [&](int jj, int ii) { return (jj < 0 || jj >= ny || ii < 0 || ii >= nx) ? T(0) : h[(size_t)jj * nx + ii]; };
    auto uu = [&](int ii) { return u[(size_t)j * nx + ii]; };
    auto vv = [&](int jj) { return v[(size_t)jj * nx + i]; };
    T qw, qe, qs, qn;
    if (METHOD == IGM_DIVFLUX_UPWIND) {
      // x faces i (west) and i+1 (east)
      const T uw = i == 0 ? uu(0) : T(0.5) * (uu(i - 1) + uu(i));
      const T ue = i == nx - 1 ? uu(nx - 1) : T(0.5) * (uu(i) + uu(i + 1));
      qw = uw * (uw > T(0) ? hh(j, i - 1) : hh(j, i));
      qe = ue * (ue > T(0) ? hh(j, i) : hh(j, i + 1));
      const T vs = j == 0 ? vv(0) : T(0.5) * (vv(j - 1) + vv(j));
      const T vn = j == ny - 1 ? vv(ny - 1) : T(0.5) * (vv(j) + vv(j + 1));
      qs = vs * (vs > T(0) ? hh(j - 1, i) : hh(j, i));
      qn = vn * (vn > T(0) ? hh(j, i) : hh(j + 1, i));
    } else {
      // centered: the face averages of u h and v h, edge copies at the border
      auto qx = [&](int ii) { return uu(ii) * hh(j, ii); };
      auto qy = [&](int jj) { return vv(jj) * hh(jj, i); };
      qw = i == 0 ? qx(0) : T(0.5) * (qx(i - 1) + qx(i));
      qe = i == nx - 1 ? qx(nx - 1) : T(0.5) * (qx(i) + qx(i + 1));
      qs = j == 0 ? qy(0) : T(0.5) * (qy(j - 1) + qy(j));
      qn = j == ny - 1 ? qy(ny - 1) : T(0.5) * (qy(j) + qy(j + 1));
    }
    out[o] = div_dx(qe - qw, dx, rdx) + div_dx(qn - qs, dx, rdx);
  }
}

template <typename T>
static int vert_flow_t(int nz, int ny, int nx, double dx, const void* U, const void* V, const void* topg,
                       const void* thk, const double* levels, const double* vert_weight, void* W, bool incomp,
                       cudaStream_t st) {
  VertFlowArgs<T> a{};
  a.nz = nz; a.ny = ny; a.nx = nx;
  a.dx = (T)dx;
  a.rdx = T(1) / a.dx;
  for (int k = 0; k < nz; ++k) {
    a.lev[k] = (T)levels[k];
    a.w[k] = (T)vert_weight[k];
  }
  a.U = (const T*)U; a.V = (const T*)V; a.topg = (const T*)topg; a.thk = (const T*)thk; a.W = (T*)W;
  const int n_strips = (nx + kVfCols - 1) / kVfCols;
  const long long warps = (long long)n_strips * ((ny + kVfRows - 1) / kVfRows);
  const int grid = (int)((warps + kVfWarps - 1) / kVfWarps);
  if (incomp) {
    vert_flow_incomp_kernel<T><<<grid, kVfWarps * 32, 0, st>>>(a, n_strips);
    return launch_status("vert_flow_incomp_kernel");
  }
  vert_flow_kernel<T><<<grid, kVfWarps * 32, 0, st>>>(a, n_strips);
  return launch_status("vert_flow_kernel");
}

}  // namespace igm

using namespace igm;

extern "C" int igm_velocity_reduce(int dtype, int batch, int nz, int ny, int nx, void* U, void* V, const void* thk,
                                   int mask, const double* vert_weight, void* ubar, void* vbar, void* uvelbase,
                                   void* vvelbase, void* uvelsurf, void* vvelsurf, float* velomax, void* stream) {
  IGM_CHECK_ARG(batch >= 1 && nz >= 1 && nz <= IGM_MAX_NZ && ny >= 1 && nx >= 1, IGM_ERR_BAD_SHAPE,
                "igm_velocity_reduce: bad shape");
  IGM_CHECK_ARG(U && V && vert_weight && (thk || !mask), IGM_ERR_BAD_ARGUMENT, "igm_velocity_reduce: NULL argument");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    return velocity_t<float>(batch, nz, ny, nx, U, V, thk, mask, vert_weight, ubar, vbar, uvelbase, vvelbase,
                             uvelsurf, vvelsurf, velomax, st);
  if (dtype == IGM_F64)
    return velocity_t<double>(batch, nz, ny, nx, U, V, thk, mask, vert_weight, ubar, vbar, uvelbase, vvelbase,
                              uvelsurf, vvelsurf, velomax, st);
  set_error("igm_velocity_reduce: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_transport_step(int dtype, int ny, int nx, double dx, const void* ubar, const void* vbar,
                                  const void* thk_in, void* thk_out, const void* topg, const void* smb,
                                  void* usurf_out, void* lsurf_out, void* divflux_out, double dt,
                                  const float* dt_device, int slope_type, double ratio_density, double sealevel,
                                  void* stream) {
  IGM_CHECK_ARG(ny >= 1 && nx >= 1, IGM_ERR_BAD_SHAPE, "igm_transport_step: bad shape %dx%d", ny, nx);
  IGM_CHECK_ARG(ubar && vbar && thk_in && thk_out && topg && usurf_out, IGM_ERR_BAD_ARGUMENT,
                "igm_transport_step: NULL argument");
  IGM_CHECK_ARG(thk_in != thk_out, IGM_ERR_BAD_ARGUMENT, "igm_transport_step: thk_out must not alias thk_in");
  IGM_CHECK_ARG(slope_type >= IGM_GODUNOV && slope_type <= IGM_SUPERBEE, IGM_ERR_BAD_ARGUMENT,
                "igm_transport_step: unknown slope_type %d", slope_type);
  IGM_CHECK_ARG(dx > 0, IGM_ERR_BAD_ARGUMENT, "igm_transport_step: dx must be positive");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    return transport_t<float>(ny, nx, dx, ubar, vbar, thk_in, thk_out, topg, smb, usurf_out, lsurf_out, divflux_out,
                              dt, dt_device, slope_type, ratio_density, sealevel, st);
  if (dtype == IGM_F64)
    return transport_t<double>(ny, nx, dx, ubar, vbar, thk_in, thk_out, topg, smb, usurf_out, lsurf_out, divflux_out,
                               dt, dt_device, slope_type, ratio_density, sealevel, st);
  set_error("igm_transport_step: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_thk_surfaces(int dtype, int n, const void* thk, const void* topg, void* lsurf, void* usurf,
                                double ratio_density, double sealevel, void* stream) {
  IGM_CHECK_ARG(n >= 0 && thk && topg && usurf, IGM_ERR_BAD_ARGUMENT, "igm_thk_surfaces: bad argument");
  cudaStream_t st = as_stream(stream);
  if (n == 0) return IGM_OK;
  if (dtype == IGM_F32)
    surfaces_kernel<float><<<grid1d(n), 256, 0, st>>>(n, (const float*)thk, (const float*)topg, (float*)lsurf,
                                                     (float*)usurf, (float)ratio_density, (float)sealevel);
  else if (dtype == IGM_F64)
    surfaces_kernel<double><<<grid1d(n), 256, 0, st>>>(n, (const double*)thk, (const double*)topg, (double*)lsurf,
                                                       (double*)usurf, ratio_density, sealevel);
  else {
    set_error("igm_thk_surfaces: unknown dtype %d", dtype);
    return IGM_ERR_BAD_ARGUMENT;
  }
  return launch_status("surfaces_kernel");
}

extern "C" int igm_smb_simple(int dtype, int n, const void* usurf, const void* icemask, void* smb, double gradabl,
                              double gradacc, double ela, double maxacc, void* stream) {
  IGM_CHECK_ARG(n >= 0 && usurf && smb, IGM_ERR_BAD_ARGUMENT, "igm_smb_simple: bad argument");
  cudaStream_t st = as_stream(stream);
  if (n == 0) return IGM_OK;
  if (dtype == IGM_F32)
    smb_kernel<float><<<grid1d(n), 256, 0, st>>>(n, (const float*)usurf, (const float*)icemask, (float*)smb,
                                                 (float)gradabl, (float)gradacc, (float)ela, (float)maxacc);
  else if (dtype == IGM_F64)
    smb_kernel<double><<<grid1d(n), 256, 0, st>>>(n, (const double*)usurf, (const double*)icemask, (double*)smb,
                                                  gradabl, gradacc, ela, maxacc);
  else {
    set_error("igm_smb_simple: unknown dtype %d", dtype);
    return IGM_ERR_BAD_ARGUMENT;
  }
  return launch_status("smb_kernel");
}

extern "C" int igm_cfl_dt(const float* velomax, float* dt_out, double cfl, double dx, double step_max, void* stream) {
  IGM_CHECK_ARG(velomax && dt_out, IGM_ERR_BAD_ARGUMENT, "igm_cfl_dt: NULL argument");
  cfl_dt_kernel<<<1, 1, 0, as_stream(stream)>>>(velomax, dt_out, (float)(cfl * dx), (float)step_max);
  return launch_status("cfl_dt_kernel");
}

extern "C" int igm_absmax2(int dtype, int n, const void* a, const void* b, float* out, void* stream) {
  IGM_CHECK_ARG(n >= 0 && a && b && out, IGM_ERR_BAD_ARGUMENT, "igm_absmax2: bad argument");
  cudaStream_t st = as_stream(stream);
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float), st);
  if (e != cudaSuccess) {
    set_error("igm_absmax2: %s", cudaGetErrorString(e));
    return IGM_ERR_CUDA;
  }
  if (n == 0) return IGM_OK;
  if (dtype == IGM_F32)
    absmax2_kernel<float><<<grid1d(n), 256, 0, st>>>(n, (const float*)a, (const float*)b, out);
  else if (dtype == IGM_F64)
    absmax2_kernel<double><<<grid1d(n), 256, 0, st>>>(n, (const double*)a, (const double*)b, out);
  else {
    set_error("igm_absmax2: unknown dtype %d", dtype);
    return IGM_ERR_BAD_ARGUMENT;
  }
  return launch_status("absmax2_kernel");
}

extern "C" int igm_force_max_velbar(int dtype, size_t n, void* U, void* V, double cap, void* stream) {
  IGM_CHECK_ARG(U && V, IGM_ERR_BAD_ARGUMENT, "igm_force_max_velbar: NULL argument");
  IGM_CHECK_ARG(cap > 0, IGM_ERR_BAD_ARGUMENT, "igm_force_max_velbar: the cap must be positive");
  if (n == 0) return IGM_OK;
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    force_max_velbar_kernel<float><<<grid1d(n), 256, 0, st>>>(n, (float*)U, (float*)V, (float)cap);
  else if (dtype == IGM_F64)
    force_max_velbar_kernel<double><<<grid1d(n), 256, 0, st>>>(n, (double*)U, (double*)V, cap);
  else {
    set_error("igm_force_max_velbar: unknown dtype %d", dtype);
    return IGM_ERR_BAD_ARGUMENT;
  }
  return launch_status("force_max_velbar_kernel");
}

extern "C" int igm_vertical_velocity(int dtype, int nz, int ny, int nx, double dx, const void* U, const void* V,
                                     const void* topg, const void* thk, const double* levels,
                                     const double* vert_weight, void* W, void* stream) {
  IGM_CHECK_ARG(nz >= 2 && nz <= IGM_MAX_NZ && ny >= 2 && nx >= 2, IGM_ERR_BAD_SHAPE,
                "igm_vertical_velocity: bad shape %dx%dx%d (needs nz, ny, nx >= 2)", nz, ny, nx);
  IGM_CHECK_ARG(U && V && topg && thk && levels && vert_weight && W, IGM_ERR_BAD_ARGUMENT,
                "igm_vertical_velocity: NULL argument");
  IGM_CHECK_ARG(dx > 0, IGM_ERR_BAD_ARGUMENT, "igm_vertical_velocity: dx must be positive");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32) return vert_flow_t<float>(nz, ny, nx, dx, U, V, topg, thk, levels, vert_weight, W, false, st);
  if (dtype == IGM_F64) return vert_flow_t<double>(nz, ny, nx, dx, U, V, topg, thk, levels, vert_weight, W, false, st);
  set_error("igm_vertical_velocity: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_vertical_velocity_incompressibility(int dtype, int nz, int ny, int nx, double dx, const void* U,
                                                       const void* V, const void* topg, const void* thk,
                                                       const double* levels, const double* vert_weight, void* W,
                                                       void* stream) {
  IGM_CHECK_ARG(nz >= 2 && nz <= IGM_MAX_NZ && ny >= 2 && nx >= 2, IGM_ERR_BAD_SHAPE,
                "igm_vertical_velocity_incompressibility: bad shape %dx%dx%d (needs nz, ny, nx >= 2)", nz, ny, nx);
  IGM_CHECK_ARG(U && V && topg && thk && levels && vert_weight && W, IGM_ERR_BAD_ARGUMENT,
                "igm_vertical_velocity_incompressibility: NULL argument");
  IGM_CHECK_ARG(dx > 0, IGM_ERR_BAD_ARGUMENT, "igm_vertical_velocity_incompressibility: dx must be positive");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32) return vert_flow_t<float>(nz, ny, nx, dx, U, V, topg, thk, levels, vert_weight, W, true, st);
  if (dtype == IGM_F64) return vert_flow_t<double>(nz, ny, nx, dx, U, V, topg, thk, levels, vert_weight, W, true, st);
  set_error("igm_vertical_velocity_incompressibility: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_divflux(int dtype, int method, int ny, int nx, double dx, const void* u, const void* v,
                           const void* h, void* out, void* stream) {
  IGM_CHECK_ARG(ny >= 2 && nx >= 2 && dx > 0, IGM_ERR_BAD_SHAPE, "igm_divflux: bad shape or dx");
  IGM_CHECK_ARG(u && v && h && out, IGM_ERR_BAD_ARGUMENT, "igm_divflux: NULL argument");
  IGM_CHECK_ARG(method == IGM_DIVFLUX_UPWIND || method == IGM_DIVFLUX_CENTERED, IGM_ERR_BAD_ARGUMENT,
                "igm_divflux: unknown method %d", method);
  cudaStream_t st = as_stream(stream);
  const int grid = grid1d((size_t)ny * nx);
  auto run = [&](auto zero) {
    using T = decltype(zero);
    const T d = (T)dx;
    if (method == IGM_DIVFLUX_UPWIND)
      divflux_kernel<T, IGM_DIVFLUX_UPWIND><<<grid, 256, 0, st>>>(ny, nx, d, T(1) / d, (const T*)u, (const T*)v,
                                                                  (const T*)h, (T*)out);
    else
      divflux_kernel<T, IGM_DIVFLUX_CENTERED><<<grid, 256, 0, st>>>(ny, nx, d, T(1) / d, (const T*)u, (const T*)v,
                                                                    (const T*)h, (T*)out);
  };
  if (dtype == IGM_F32)
    run(0.f);
  else if (dtype == IGM_F64)
    run(0.0);
  else {
    set_error("igm_divflux: unknown dtype %d", dtype);
    return IGM_ERR_BAD_ARGUMENT;
  }
  return launch_status("divflux_kernel");
}

extern "C" int igm_divflux_upwind(int dtype, int ny, int nx, double dx, const void* u, const void* v, const void* h,
                                  void* out, void* stream) {
  return igm_divflux(dtype, IGM_DIVFLUX_UPWIND, ny, nx, dx, u, v, h, out, stream);
}
