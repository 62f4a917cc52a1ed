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
// Kernel shape.  A CTA is one warp wide (32 cells in x) and TYC warps tall.
// Its cells are [j0-1, j0-1+TYC) x [i0-1, i0+31), which covers every cell that
// touches its (TYC-1) x 31 output nodes, so the adjoint (a scatter from
// cells to their 4 corners) becomes a gather inside the CTA with no atomics.
// The kernel streams through the Nz levels: each level's node tile of U and V
// is staged in shared memory (double-buffered, next level prefetched into
// registers), each thread evaluates its cell's layer l = k-1 energy and
// adjoint, and as soon as level k-1's adjoint is complete its per-cell
// partials (S = dUs/4, P = dDx/(2dx), Q = dDy/(2dx)) are gathered into the
// node gradient and written (or fed to Adam) for that level.  Shared memory
// therefore holds two levels at a time, independent of Nz.
//
// Energy reduction: per-cell FP32 densities, FP64 block sums, per-CTA
// partials in the workspace, and the last CTA to finish sums them in a fixed
// order (deterministic) and, in solver mode, runs EarlyStopping on the device.
#include <stdarg.h>

#include <mutex>

#include "common.cuh"

namespace igm {

constexpr int kTX = 32;
// Levels of U, V (and Adam moments) kept in flight ahead of the one being
// computed.  The ring has kStages = kAhead + 2 slots: the extra slot keeps
// the level whose moments are read by the gather one iteration later.
constexpr int kAhead = 3;
constexpr int kStages = kAhead + 2;

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

enum StencilMode { kEnergyOnly = 0, kGradient = 1, kAdamStep = 2 };

template <typename T>
struct StencilArgs {
  int batch, nz, ny, nx;
  T dx, inv_dx;
  T dzeta[IGM_MAX_NZ];
  T inv_dzeta[IGM_MAX_NZ];
  // physics
  T q, inv_p, regu2, sr_lo, sr_hi, thr, Kg, inv_n, s_w, inv_sw, regw2;
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
};

template <typename T, int TYC, int MODE>
struct StencilSmem {
  static constexpr int NR = TYC + 1, NC = kTX + 1;
  static constexpr bool GRAD = MODE != kEnergyOnly;
  static constexpr bool ADAM = MODE == kAdamStep;
  T F[4][NR][NC];                        // thk, usurf, B = 2 A^(-1/n), c of the node tile
  T N[kStages][2][NR][NC];               // U, V node tiles, ring of levels
  T M[ADAM ? kStages : 1][4][TYC][kTX];  // mU, mV, vU, vV of the output nodes, ring of levels
  T Tr[GRAD ? 2 : 1][6][TYC][kTX];       // per-cell adjoint partials S, P, Q of U and V
  double red[TYC];
  unsigned int ticket;
};

template <typename T> struct MinBlocks { static constexpr int value = 3; };
template <> struct MinBlocks<double> { static constexpr int value = 2; };

template <typename T, int TYC, int MODE>
__global__ void __launch_bounds__(kTX* TYC, MinBlocks<T>::value) stencil_kernel(const StencilArgs<T> a) {
  constexpr int NT = kTX * TYC;
  constexpr int NR = TYC + 1, NC = kTX + 1;
  constexpr int NTILE = NR * NC;
  constexpr bool GRAD = MODE != kEnergyOnly;
  constexpr bool ADAM = MODE == kAdamStep;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  StencilSmem<T, TYC, MODE>& SM = *reinterpret_cast<StencilSmem<T, TYC, MODE>*>(smem_raw);
  auto& sF = SM.F;
  auto& sN = SM.N;
  auto& sM = SM.M;
  auto& sT = SM.Tr;
  double* sRed = SM.red;
  unsigned int& sTicket = SM.ticket;

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
  const int ny = a.ny, nx = a.nx, nz = a.nz;
  const int j0 = blockIdx.y * (TYC - 1), i0 = blockIdx.x * (kTX - 1);
  const size_t plane = (size_t)ny * nx;
  const size_t fbase = (size_t)blockIdx.z * plane;
  const size_t vbase = (size_t)blockIdx.z * nz * plane;

  T* Ucur = a.U0;
  T* Vcur = a.V0;
  T* Unxt = a.U1;
  T* Vnxt = a.V1;
  int iter = 0;
  T alpha = 0;
  if (MODE == kAdamStep) {
    iter = __ldcg(&a.ctl->iter);
    const int stopped = __ldcg(&a.ctl->stopped);
    if (stopped || iter >= a.max_iter) return;
    if (iter & 1) {
      Ucur = a.U1; Vcur = a.V1; Unxt = a.U0; Vnxt = a.V0;
    }
    const long long t = __ldcg(&a.ctl->adam_t0) + iter + 1;
    const T one = T(1);
    alpha = a.lr * Math<T>::sqrt(one - Math<T>::pow(a.b2, T(t))) / (one - Math<T>::pow(a.b1, T(t)));
  }

  // ---- 2-D fields of the node tile -----------------------------------------
  for (int idx = tid; idx < NTILE; idx += NT) {
    const int r = idx / NC, c = idx - r * NC;
    const int gj = j0 - 1 + r, gi = i0 - 1 + c;
    T th = 0, us = 0, Bv = 0, cv = 0;
    if (gj >= 0 && gj < ny && gi >= 0 && gi < nx) {
      const size_t o = fbase + (size_t)gj * nx + gi;
      th = a.thk[o];
      us = a.usurf[o];
      const T Av = a.A[o];
      Bv = T(2) * (a.glen3 ? Math<T>::rcbrt(Av) : Math<T>::pow(Av, -a.inv_n));
      cv = a.C[o];
    }
    sF[0][r][c] = th;
    sF[1][r][c] = us;
    sF[2][r][c] = Bv;
    sF[3][r][c] = cv;
  }

  // ---- asynchronous level loads: U, V node tile (+ Adam moments of the output nodes)
  const int own_j = j0 - 1 + ty, own_i = i0 - 1 + tx;  // this thread's node (corner a of its cell)
  const bool outnode = ty >= 1 && tx >= 1 && own_j < ny && own_i < nx;
  // each thread's share of the node tile: fixed (row, col) slots, offsets computed once
  constexpr int NSLOT = (NTILE + NT - 1) / NT;
  int slot_off[NSLOT];
  int slot_sm[NSLOT];
  bool slot_ok[NSLOT];
#pragma unroll
  for (int q = 0; q < NSLOT; ++q) {
    const int idx = tid + q * NT;
    const int r = idx / NC, c = idx - r * NC;
    const int gj = j0 - 1 + r, gi = i0 - 1 + c;
    slot_ok[q] = idx < NTILE && gj >= 0 && gj < ny && gi >= 0 && gi < nx;
    slot_off[q] = slot_ok[q] ? gj * nx + gi : 0;
    slot_sm[q] = idx < NTILE ? idx : -1;
  }
  auto issue_level = [&](int k) {
    if (k < nz) {
      const int st = k % kStages;
      const T* Ub = Ucur + vbase + (size_t)k * plane;
      const T* Vb = Vcur + vbase + (size_t)k * plane;
      T* sU = &sN[st][0][0][0];
      T* sV = &sN[st][1][0][0];
#pragma unroll
      for (int q = 0; q < NSLOT; ++q) {
        if (slot_sm[q] >= 0) {
          cp_async_elem(sU + slot_sm[q], Ub + slot_off[q], slot_ok[q]);
          cp_async_elem(sV + slot_sm[q], Vb + slot_off[q], slot_ok[q]);
        }
      }
      if (ADAM) {
        const size_t o = vbase + (size_t)k * plane + (outnode ? (size_t)own_j * nx + own_i : 0);
        cp_async_elem(&sM[ADAM ? st : 0][0][ty][tx], a.mU + o, outnode);
        cp_async_elem(&sM[ADAM ? st : 0][1][ty][tx], a.mV + o, outnode);
        cp_async_elem(&sM[ADAM ? st : 0][2][ty][tx], a.vU + o, outnode);
        cp_async_elem(&sM[ADAM ? st : 0][3][ty][tx], a.vV + o, outnode);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int k = 0; k < kAhead; ++k) issue_level(k);
  __syncthreads();

  // ---- per-cell constants -----------------------------------------------------
  const int cj = j0 - 1 + ty, ci = i0 - 1 + tx;  // this thread's cell
  const bool cell_ok = cj >= 0 && cj < ny - 1 && ci >= 0 && ci < nx - 1;
  const bool owner = cell_ok && ty >= 1 && tx >= 1;
  const T dx = a.dx;
  const T half = T(0.5), quarter = T(0.25);
  T thks, cs, Bs, sbx, sby, ssx, ssy;
  {
    const T t00 = sF[0][ty][tx], t01 = sF[0][ty][tx + 1], t10 = sF[0][ty + 1][tx], t11 = sF[0][ty + 1][tx + 1];
    const T u00 = sF[1][ty][tx], u01 = sF[1][ty][tx + 1], u10 = sF[1][ty + 1][tx], u11 = sF[1][ty + 1][tx + 1];
    thks = (((t11 + t10) + t01) + t00) / T(4);
    Bs = (((sF[2][ty + 1][tx + 1] + sF[2][ty + 1][tx]) + sF[2][ty][tx + 1]) + sF[2][ty][tx]) / T(4);
    cs = (((sF[3][ty + 1][tx + 1] + sF[3][ty + 1][tx]) + sF[3][ty][tx + 1]) + sF[3][ty][tx]) / T(4);
    const T b00 = u00 - t00, b01 = u01 - t01, b10 = u10 - t10, b11 = u11 - t11;
    const T two_dx = dx + dx;
    // compute_gradient (staggered): E = 2 ds/(dx+dx), averaged over the other axis
    sbx = half * (T(2) * (b11 - b10) / two_dx + T(2) * (b01 - b00) / two_dx);
    sby = half * (T(2) * (b11 - b01) / two_dx + T(2) * (b10 - b00) / two_dx);
    ssx = half * (T(2) * (u11 - u10) / two_dx + T(2) * (u01 - u00) / two_dx);
    ssy = half * (T(2) * (u11 - u01) / two_dx + T(2) * (u10 - u00) / two_dx);
  }
  const T hcl = thks > a.thr ? thks : a.thr;
  const T rh = T(1) / hcl;  // 1 / max(thk_s, thr)
  const T idx_ = a.inv_dx;
  const T fdamp = cs > T(0) ? T(1) : T(0.01);
  const T gshear = thks * Bs;     // d(shear density)/d(p_term_l) = thks Bs dzeta_l
  const T ggrav = a.Kg * thks;    // d(gravity density)/d(uds_l)  = Kg thks dzeta_l

  T e_shear = 0, e_grav = 0, e_slid = 0;
  // previous level's cell quantities and pending adjoints
  T pUs = 0, pVs = 0, pDxu = 0, pDyu = 0, pDxv = 0, pDyv = 0;
  T gUs = 0, gDxu = 0, gDyu = 0, gVs = 0, gDxv = 0, gDyv = 0;
  T prevUold = 0, prevVold = 0;  // this thread's node (a corner) at the previous level

  const T inv2dx = T(1) / (dx + dx);
  const T gsc = a.grad_scale;

  // writes the per-cell partials of a completed level, then gathers them
  auto flush_level = [&](int lvl, T Us_, T Dxu_, T Dyu_, T Vs_, T Dxv_, T Dyv_, T Uold, T Vold) {
    const int tb = lvl & 1;
    T S = cell_ok ? Us_ * quarter * gsc : T(0);
    T P = cell_ok ? Dxu_ * inv2dx * gsc : T(0);
    T Q = cell_ok ? Dyu_ * inv2dx * gsc : T(0);
    sT[tb][0][ty][tx] = S;
    sT[tb][1][ty][tx] = P;
    sT[tb][2][ty][tx] = Q;
    S = cell_ok ? Vs_ * quarter * gsc : T(0);
    P = cell_ok ? Dxv_ * inv2dx * gsc : T(0);
    Q = cell_ok ? Dyv_ * inv2dx * gsc : T(0);
    sT[tb][3][ty][tx] = S;
    sT[tb][4][ty][tx] = P;
    sT[tb][5][ty][tx] = Q;
    __syncthreads();
    const int nj = j0 - 1 + ty, ni = i0 - 1 + tx;
    if (ty >= 1 && tx >= 1 && nj < ny && ni < nx) {
      T g[2];
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const T (*Sv)[kTX] = sT[tb][3 * f + 0];
        const T (*Pv)[kTX] = sT[tb][3 * f + 1];
        const T (*Qv)[kTX] = sT[tb][3 * f + 2];
        g[f] = (Sv[ty][tx] - Pv[ty][tx] - Qv[ty][tx]) + (Sv[ty][tx - 1] + Pv[ty][tx - 1] - Qv[ty][tx - 1]) +
               (Sv[ty - 1][tx] - Pv[ty - 1][tx] + Qv[ty - 1][tx]) +
               (Sv[ty - 1][tx - 1] + Pv[ty - 1][tx - 1] + Qv[ty - 1][tx - 1]);
      }
      const size_t o = vbase + (size_t)lvl * plane + (size_t)nj * nx + ni;
      if (MODE == kGradient) {
        a.dU[o] = g[0];
        a.dV[o] = g[1];
      } else if (MODE == kAdamStep) {
        const T b1c = T(1) - a.b1, b2c = T(1) - a.b2;
        const int ms = ADAM ? lvl % kStages : 0;
        T m = sM[ms][0][ty][tx], v = sM[ms][2][ty][tx];
        m += (g[0] - m) * b1c;
        v += (g[0] * g[0] - v) * b2c;
        a.mU[o] = m;
        a.vU[o] = v;
        Unxt[o] = Uold - (m * alpha) / (Math<T>::sqrt(v) + a.eps);
        m = sM[ms][1][ty][tx];
        v = sM[ms][3][ty][tx];
        m += (g[1] - m) * b1c;
        v += (g[1] * g[1] - v) * b2c;
        a.mV[o] = m;
        a.vV[o] = v;
        Vnxt[o] = Vold - (m * alpha) / (Math<T>::sqrt(v) + a.eps);
      }
    }
  };

  for (int k = 0; k < nz; ++k) {
    const int nb = k % kStages;
    cp_async_wait<kAhead - 1>();  // this thread's copies of level k have landed
    __syncthreads();              // ... and everyone's; level k-2's slot is free again
    issue_level(k + kAhead);

    // level-k cell quantities
    T cUs, cVs, cDxu, cDyu, cDxv, cDyv, Uold, Vold;
    {
      const T a_ = sN[nb][0][ty][tx], b_ = sN[nb][0][ty][tx + 1], c_ = sN[nb][0][ty + 1][tx],
              d_ = sN[nb][0][ty + 1][tx + 1];
      cUs = (((d_ + c_) + b_) + a_) * quarter;
      cDxu = ((b_ - a_) * idx_ + (d_ - c_) * idx_) * half;
      cDyu = ((c_ - a_) * idx_ + (d_ - b_) * idx_) * half;
      Uold = a_;
    }
    {
      const T a_ = sN[nb][1][ty][tx], b_ = sN[nb][1][ty][tx + 1], c_ = sN[nb][1][ty + 1][tx],
              d_ = sN[nb][1][ty + 1][tx + 1];
      cVs = (((d_ + c_) + b_) + a_) * quarter;
      cDxv = ((b_ - a_) * idx_ + (d_ - c_) * idx_) * half;
      cDyv = ((c_ - a_) * idx_ + (d_ - b_) * idx_) * half;
      Vold = a_;
    }
    T hUs = 0, hDxu = 0, hDyu = 0, hVs = 0, hDxv = 0, hDyv = 0;  // pending adjoint of level k

    if (k == 0) {
      // Weertman sliding on the basal level (cost_sliding_weertman.py:23-43)
      const T tb = cUs * sbx + cVs * sby;
      const T N = (cUs * cUs + cVs * cVs) + a.regw2 + tb * tb;
      T Np, dN;  // N^(s/2) and d(N^(s/2))/dN * (1/s)*s/2 -> handled below
      if (a.weert3) {
        const T cr = Math<T>::cbrt(N);
        Np = cr * cr;                       // N^(2/3)
        dN = Math<T>::rcbrt(N);             // N^(-1/3)
      } else {
        Np = Math<T>::pow(N, a.s_w * half);
        dN = Math<T>::pow(N, a.s_w * half - T(1));
      }
      e_slid = cs * Np * a.inv_sw;
      if (GRAD) {
        const T gN = cs * half * dN;        // d(c N^(s/2) / s)/dN
        hUs += gN * (T(2) * cUs + T(2) * tb * sbx);
        hVs += gN * (T(2) * cVs + T(2) * tb * sby);
      }
      if (nz == 1) {
        pUs = cUs; pVs = cVs; pDxu = cDxu; pDyu = cDyu; pDxv = cDxv; pDyv = cDyv;
      }
    }

    if (k >= 1 || nz == 1) {
      const int l = nz == 1 ? 0 : k - 1;
      const T dz = a.dzeta[l];
      const T axu = (pDxu + cDxu) * half, ayu = (pDyu + cDyu) * half;
      const T axv = (pDxv + cDxv) * half, ayv = (pDyv + cDyv) * half;
      const T rz = (fdamp * a.inv_dzeta[l]) * rh;
      const T uz = (cUs - pUs) * rz, vz = (cVs - pVs) * rz;
      const T X = axu - uz * sbx, Y = ayu - uz * sby;
      const T Z = axv - vz * sbx, W = ayv - vz * sby;
      const T Exy = half * Z + half * Y, Ezz = -X - W;
      const T srxy = half * (X * X + Exy * Exy + Exy * Exy + W * W + Ezz * Ezz);
      const T Exz = half * uz, Eyz = half * vz;
      const T srz = half * (Exz * Exz + Eyz * Eyz + Exz * Exz + Eyz * Eyz);
      const T sr2 = srxy + srz;
      const T sc = sr2 < a.sr_lo ? a.sr_lo : (sr2 > a.sr_hi ? a.sr_hi : sr2);
      const T base = sc + a.regu2;
      const T bq = a.glen3 ? Math<T>::rcbrt(base) : Math<T>::pow(base, a.q);
      e_shear += dz * (bq * sr2 * a.inv_p);
      const T Ub = (pUs + cUs) * half, Vb = (pVs + cVs) * half;
      T uds = Ub * ssx + Vb * ssy;
      const bool gact = !a.fnge || uds < T(0);
      if (a.fnge && uds > T(0)) uds = T(0);
      e_grav += dz * uds;
      if (GRAD) {
        const bool inside = sr2 >= a.sr_lo && sr2 <= a.sr_hi;
        const T gp = (bq + (inside ? a.q * (bq / base) * sr2 : T(0))) * a.inv_p;  // d p_term / d sr2
        const T gs = gshear * dz * gp;
        const T GX = gs * (T(2) * X + W);
        const T GW = gs * (T(2) * W + X);
        const T GY = gs * Exy;
        const T Guz = gs * half * uz - GX * sbx - GY * sby;
        const T Gvz = gs * half * vz - GY * sbx - GW * sby;
        const T gg = gact ? ggrav * dz * half : T(0);
        // layer l couples level l (pending g*) and level l+1 (pending h*)
        gDxu += GX * half; hDxu += GX * half;
        gDyu += GY * half; hDyu += GY * half;
        gDxv += GY * half; hDxv += GY * half;
        gDyv += GW * half; hDyv += GW * half;
        gUs += -Guz * rz + gg * ssx; hUs += Guz * rz + gg * ssx;
        gVs += -Gvz * rz + gg * ssy; hVs += Gvz * rz + gg * ssy;
      }
    }

    if (GRAD) {
      if (nz == 1) {
        hUs += gUs; hDxu += gDxu; hDyu += gDyu; hVs += gVs; hDxv += gDxv; hDyv += gDyv;
      } else if (k >= 1) {
        flush_level(k - 1, gUs, gDxu, gDyu, gVs, gDxv, gDyv, prevUold, prevVold);
      }
      gUs = hUs; gDxu = hDxu; gDyu = hDyu; gVs = hVs; gDxv = hDxv; gDyv = hDyv;
    }
    pUs = cUs; pVs = cVs; pDxu = cDxu; pDyu = cDyu; pDxv = cDxv; pDyv = cDyv;
    prevUold = Uold;
    prevVold = Vold;
  }
  if (GRAD) {
    flush_level(nz - 1, gUs, gDxu, gDyu, gVs, gDxv, gDyv, prevUold, prevVold);
  }

  // ---- energy reduction ---------------------------------------------------------
  const T es = owner ? thks * (Bs * e_shear) : T(0);
  const T eg = owner ? a.Kg * thks * e_grav : T(0);
  const T el = owner ? e_slid : T(0);
  const int nblocks = gridDim.x * gridDim.y * gridDim.z;
  const int bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const double s0 = block_sum<NT>((double)es, sRed, tid);
  const double s1 = block_sum<NT>((double)el, sRed, tid);
  const double s2 = block_sum<NT>((double)eg, sRed, tid);
  if (tid == 0) {
    a.partials[3 * (size_t)bid + 0] = s0;
    a.partials[3 * (size_t)bid + 1] = s1;
    a.partials[3 * (size_t)bid + 2] = s2;
    __threadfence();
    sTicket = atomicAdd(a.counter, 1u);
  }
  __syncthreads();
  if (sTicket != (unsigned)(nblocks - 1)) return;
  __threadfence();
  double r[3] = {0.0, 0.0, 0.0};
  for (int i = tid; i < nblocks; i += NT) {
    r[0] += __ldcg(&a.partials[3 * (size_t)i + 0]);
    r[1] += __ldcg(&a.partials[3 * (size_t)i + 1]);
    r[2] += __ldcg(&a.partials[3 * (size_t)i + 2]);
  }
  const double t0 = block_sum<NT>(r[0], sRed, tid);
  const double t1 = block_sum<NT>(r[1], sRed, tid);
  const double t2 = block_sum<NT>(r[2], sRed, tid);
  if (tid == 0) {
    *a.counter = 0u;
    if (a.terms) {
      a.terms[0] = t0;
      a.terms[1] = t1;
      a.terms[2] = t2;
    }
    if (MODE == kAdamStep) {
      igm_solver_ctl* ctl = a.ctl;
      const double cost = (t0 + t1 + t2) * a.inv_count;
      a.costs[iter] = cost;
      ctl->last_cost = cost;
      ctl->terms[0] = t0 * a.inv_count;
      ctl->terms[1] = t1 * a.inv_count;
      ctl->terms[2] = t2 * a.inv_count;
      if (!isfinite(cost)) {
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

// Cell rows per CTA (256 threads; several CTAs per SM keep enough loads in flight).
template <typename T> struct TileRows { static constexpr int value = 8; };

static inline int grid_blocks_rows(const igm_grid* g, int tyc, dim3* grid) {
  *grid = dim3((g->nx + kTX - 2) / (kTX - 1), (g->ny + tyc - 2) / (tyc - 1), g->batch);
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

template <typename T, int MODE>
static int launch_stencil(const StencilArgs<T>& s, const igm_grid* g, cudaStream_t st) {
  constexpr int TYC = TileRows<T>::value;
  constexpr size_t smem = sizeof(StencilSmem<T, TYC, MODE>);
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(stencil_kernel<T, TYC, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) {
      set_error("stencil_kernel smem attribute: %s", cudaGetErrorString(e));
      return IGM_ERR_CUDA;
    }
    configured = true;
  }
  dim3 gr;
  grid_blocks_rows(g, TYC, &gr);
  stencil_kernel<T, TYC, MODE><<<gr, dim3(kTX, TYC), smem, st>>>(s);
  return launch_status("stencil_kernel");
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
  if (dU) return launch_stencil<T, kGradient>(s, g, st);
  return launch_stencil<T, kEnergyOnly>(s, g, st);
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
  for (int i = 0; i < n_it; ++i) {
    rc = launch_stencil<T, kAdamStep>(s, g, st);
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
