// Data assimilation (igm/processes/data_assimilation): the cost terms of the
// default configuration and their gradient, the flow direction of the
// anisotropic regularisation.  HBM-bound node stencils with deterministic
// (fixed-order) FP64 cost reductions.
#include "common.cuh"

namespace igm {

// cost indices of igm_assim_cost_grad
enum { kCVel = 0, kCThk = 1, kCIce = 2, kCPos = 3, kCReg = 4, kCUs = 5, kNCost = 6 };

template <typename T>
struct AssimArgs {
  int ny, nx;
  T dx;
  const T* thk;
  const T* usurf;
  const T* uvs;  // emulated surface velocities (already zero where thk <= 0)
  const T* vvs;
  const T* uobs;  // observations, NaN where missing
  const T* vobs;
  const T* thkobs;
  const T* dens;  // density weights of the thickness observations
  const T* icemaskobs;
  const T* fdx;   // flow directions [ny-1][nx-1] (anisotropic branch)
  const T* fdy;
  const T* usobs;  // usurfobs (misfit_usurf) or NULL
  igm_assim_params p;
  T* g_thk;  // dC/dthk (field-only mode: dC/dfield)
  T* g_u;    // dC/duvs
  T* g_v;
  T* g_us;   // dC/dusurf or NULL
  int field_only;  // the regularisation and positivity penalty of one field (thk holds it)
  T pos_thr;       // field-only: the penalty applies below this value
  // regularisation weights: 1 (half sums) or, fix_opti_normalization_issue, the means' 1/count
  T kx, ky, kcell;
  double kconv;    // the convexity term: 1, or 0.5 / (ny nx)
  int sole_mask;   // optimization.sole_mask: differences only between nodes of the observed ice
  int mask_eq1;    // ... where icemaskobs == 1 (isotropic slidingco / arrhenius) instead of > 0.5
  double* partials;  // [gridDim.x][kNCost]
};

// Scale factors of the cost sums and the gradients (host-computed once per
// call): the kernel accumulates unscaled sums, the final reduction scales.
struct AssimScales {
  double c_vel, c_thk, c_pen, c_reg, c_us;  // cost = scale * sum
  double gamma;                       // convexity weight
};

// A warp owns a strip of 30 columns (lanes 1..30; lanes 0 and 31 carry the
// columns on either side) and walks down a segment of rows.  Each lane
// evaluates the regularisation cell (j, c) to the lower right of its node
// once per row; the gradient of a node gathers its four cells: the left
// neighbour's by shuffle, the previous cell row from registers.  The node
// inputs of row j + 1 are loaded while row j is evaluated.
constexpr int kAmCols = 30;
constexpr int kAmWarps = 4;

template <typename T>
struct AssimRow {
  T th, us, uso;          // thk (field-only mode: the field), usurf, usurfobs (this lane's column)
  T uo, vo, uv, vv;       // observed / emulated surface velocities
  T to, de, im;           // thkobs, density weight, icemaskobs
  T fx, fy;               // flow direction of cell (j, c)
};

template <typename T>
__device__ __forceinline__ void assim_march(const AssimArgs<T>& a, const AssimScales& sc, int lane, int strip,
                                            int y0, int y1, double* acc) {
  const int nx = a.nx, ny = a.ny;
  const auto& p = a.p;
  const int c = strip * kAmCols - 1 + lane;
  const bool col = c >= 0 && c < nx;
  const size_t cc = col ? (size_t)c : 0;
  const bool cell_col = c >= 0 && c < nx - 1;
  const bool out = lane >= 1 && lane <= kAmCols && col;
  const bool aniso = p.aniso_factor != 1.0;
  const bool reg_thk = p.regularize_thk != 0;
  const bool fo = a.field_only != 0;
  const bool us_cost = !fo && p.usurf_cost != 0;
  const bool thk_ctl = p.no_thk_control == 0;
  const bool sole = a.sole_mask != 0, eq1 = a.mask_eq1 != 0;
  const T kus = (T)(1.0 / (p.usurfobs_std * p.usurfobs_std * (p.n_usurf > 0 ? p.n_usurf : 1.0)));
  const T rdx = T(1) / a.dx, hr = T(0.5) * rdx;
  const T w = (T)p.regu_thk;
  const T s_a = (T)(1.0 / sqrt(p.aniso_factor)), s_b = (T)sqrt(p.aniso_factor);
  const T thr = (T)p.velsurfobs_thr;
  const T kv = (T)(1.0 / (p.velsurfobs_std * p.velsurfobs_std * p.n_vel));
  const T kt = (T)(1.0 / (p.thkobs_std * p.thkobs_std * p.n_thk));
  const T kp = (T)(2e10 / ((double)ny * nx));
  const T kg = (T)(p.regu_thk * p.gamma * a.kconv);
  auto load = [&](int j, bool full) {
    AssimRow<T> r;
    const bool ok = col && j < ny;
    const size_t o = (size_t)j * nx + cc;
    r.th = ok ? a.thk[o] : T(0);
    r.us = (ok && !fo && (!reg_thk || us_cost)) ? a.usurf[o] : T(0);
    const bool okn = ok && full && !fo;
    r.uso = (okn && us_cost) ? a.usobs[o] : T(0);
    r.im = (ok && (okn || sole)) ? a.icemaskobs[o] : T(0);
    r.uo = okn ? a.uobs[o] : T(0);
    r.vo = okn ? a.vobs[o] : T(0);
    r.uv = okn ? a.uvs[o] : T(0);
    r.vv = okn ? a.vvs[o] : T(0);
    r.to = okn ? a.thkobs[o] : T(0);
    r.de = okn ? a.dens[o] : T(0);
    const bool okc = aniso && cell_col && j < ny - 1;
    const size_t q = (size_t)j * (nx - 1) + cc;
    r.fx = okc ? a.fdx[q] : T(0);
    r.fy = okc ? a.fdy[q] : T(0);
    return r;
  };
  auto field = [&](const AssimRow<T>& r) { return (reg_thk || fo) ? r.th : r.us - r.th; };
  // cell (j, c) from the fields of rows j (f0 this lane, f0r the next lane) and j + 1
  // -> P = gdx + gdy, M = gdx - gdy and its cost; the isotropic branch: the forward
  // differences of this node
  struct Cell {
    T P, M, cost, dxp, dyp;
  };
  auto cell = [&](int j, T f0, T f1, const AssimRow<T>& r, T im1) {
    Cell k{T(0), T(0), T(0), T(0), T(0)};
    const T f0r = __shfl_down_sync(0xffffffffu, f0, 1);
    const T f1r = __shfl_down_sync(0xffffffffu, f1, 1);
    // sole_mask (regu_thk.py:29-31, 47-50; regu_slidingco.py:12-14, 30-33; regu_arrhenius.py:9-11):
    // a cell needs its four corners > 0.5, an isotropic difference its two nodes (> 0.5 or == 1)
    const int g0 = r.im > T(0.5), g1 = im1 > T(0.5);
    const int e0 = eq1 ? (r.im == T(1)) : g0, e1 = eq1 ? (im1 == T(1)) : g1;
    const int g0r = __shfl_down_sync(0xffffffffu, g0, 1), g1r = __shfl_down_sync(0xffffffffu, g1, 1);
    const int e0r = __shfl_down_sync(0xffffffffu, e0, 1);
    if (aniso) {
      if (cell_col && j >= 0 && j < ny - 1 && (!sole || (g0 && g0r && g1 && g1r))) {
        const T dbdx = ((f0r - f0) + (f1r - f1)) * hr;
        const T dbdy = ((f1 - f0) + (f1r - f0r)) * hr;
        const T A = dbdx * r.fx + dbdy * r.fy, B = dbdx * r.fy - dbdy * r.fx;
        const T wc = w * a.kcell;
        const T gdx = wc * (s_a * A * r.fx + s_b * B * r.fy);
        const T gdy = wc * (s_a * A * r.fy - s_b * B * r.fx);
        k.P = gdx + gdy;
        k.M = gdx - gdy;
        k.cost = (s_a * A * A * T(0.5) + s_b * B * B * T(0.5)) * a.kcell;
      }
    } else if (col && j >= 0) {
      if (c + 1 < nx && (!sole || (e0 && e0r))) k.dxp = (f0r - f0) * rdx;
      if (j + 1 < ny && (!sole || (e0 && e1))) k.dyp = (f1 - f0) * rdx;
    }
    return k;
  };
  // prologue: cell row y0 - 1
  AssimRow<T> cur = load(y0, true);
  T f_cur = field(cur);
  Cell prev{T(0), T(0), T(0), T(0), T(0)};
  if (y0 >= 1) {
    const AssimRow<T> up = load(y0 - 1, false);
    prev = cell(y0 - 1, field(up), f_cur, up, cur.im);
  }
  for (int j = y0; j < y1; ++j) {
    const AssimRow<T> nxt = load(j + 1, j + 1 < y1);
    const T f_nxt = field(nxt);
    const Cell k = cell(j, f_cur, f_nxt, cur, nxt.im);
    T gf;
    if (aniso) {
      const T Ml = __shfl_up_sync(0xffffffffu, k.M, 1);
      const T Pl = __shfl_up_sync(0xffffffffu, prev.P, 1);
      gf = hr * ((Ml - k.P) + (Pl - prev.M));
    } else {
      const T dxm = __shfl_up_sync(0xffffffffu, k.dxp, 1);
      gf = w * rdx * (a.kx * (dxm - k.dxp) + a.ky * (prev.dyp - k.dyp));
    }
    if (out && fo) {
      // one control field (regu_slidingco.py:8-52, regu_arrhenius.py:5-24, total_cost.py:45-54):
      // its regularisation and positivity penalty
      const size_t o = (size_t)j * nx + cc;
      const T f = cur.th;
      T g = gf;
      if (p.penalty && !(f >= a.pos_thr)) {
        acc[kCPos] += (double)(f * f);
        g += kp * f;
      }
      acc[kCReg] += aniso ? (double)k.cost
                          : 0.5 * ((double)a.kx * k.dxp * k.dxp + (double)a.ky * k.dyp * k.dyp);
      a.g_thk[o] = g;
    } else if (out) {
      const size_t o = (size_t)j * nx + cc;
      const T th = cur.th;
      // surface-velocity misfit (misfit_velsurf.py:8-19)
      const T nrm = sqrt(cur.uo * cur.uo + cur.vo * cur.vo);
      const bool rel = nrm >= thr;  // false when a component is NaN
      T gu = T(0), gv = T(0);
      if (rel && !isnan(cur.uo)) {
        const T d = cur.uo - cur.uv;
        acc[kCVel] += (double)(d * d);
        gu = -d * kv;
      }
      if (rel && !isnan(cur.vo)) {
        const T d = cur.vo - cur.vv;
        acc[kCVel] += (double)(d * d);
        gv = -d * kv;
      }
      if (p.mask_velsurf && !(th > T(0))) {
        gu = T(0);
        gv = T(0);
      }
      a.g_u[o] = gu;
      a.g_v[o] = gv;
      T g = T(0);
      // thickness misfit (misfit_thk.py:8-16)
      if (!isnan(cur.to)) {
        const T d = cur.to - th;
        acc[kCThk] += (double)(cur.de * d * d);
        g -= cur.de * d * kt;
      }
      // penalties (total_cost.py:36-46)
      if (p.penalty) {
        if (p.icemask_cost && !(cur.im > T(0.5))) {
          acc[kCIce] += (double)(th * th);
          g += kp * th;
        }
        if (thk_ctl && !(th >= T(0))) {
          acc[kCPos] += (double)(th * th);
          g += kp * th;
        }
      }
      // regularisation (regu_thk.py:8-70): smoothness cost of cell (j, c) or of this node's
      // forward differences, the convexity term
      const double rc = aniso ? (double)k.cost
                              : 0.5 * ((double)a.kx * k.dxp * k.dxp + (double)a.ky * k.dyp * k.dyp);
      if (thk_ctl) {
        acc[kCReg] += rc - sc.gamma * a.kconv * (double)th;
        g += (reg_thk ? gf : -gf) - kg;
      }
      a.g_thk[o] = g;
      if (a.g_us) {
        // dC/dusurf: misfit_usurf (misfit_usurf.py:5-15) and the bed usurf - thk of regu_thk
        T gs = (reg_thk || !thk_ctl) ? T(0) : gf;
        if (us_cost && cur.im > T(0.5)) {
          const T d = cur.us - cur.uso;
          acc[kCUs] += (double)(d * d);
          gs += d * kus;
        }
        a.g_us[o] = gs;
      } else if (us_cost && cur.im > T(0.5)) {
        const T d = cur.us - cur.uso;
        acc[kCUs] += (double)(d * d);
      }
    }
    prev = k;
    cur = nxt;
    f_cur = f_nxt;
  }
}

template <typename T>
__global__ void __launch_bounds__(kAmWarps * 32) assim_cost_grad_kernel(const AssimArgs<T> a, const AssimScales sc,
                                                                       int n_strips, int rows, int n_tasks) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double acc[kNCost] = {0, 0, 0, 0, 0, 0};
  for (int t = blockIdx.x * kAmWarps + warp; t < n_tasks; t += gridDim.x * kAmWarps) {
    const int strip = t % n_strips, seg = t / n_strips;
    const int y0 = seg * rows, y1 = min(y0 + rows, a.ny);
    assim_march<T>(a, sc, lane, strip, y0, y1, acc);
  }
  // deterministic block reduction: fixed xor trees, warps in order
  __shared__ double red[kAmWarps][kNCost];
#pragma unroll
  for (int c = 0; c < kNCost; ++c) {
    double v = acc[c];
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNCost) {
    double v = 0.0;
    for (int w = 0; w < kAmWarps; ++w) v += red[w][threadIdx.x];
    a.partials[(size_t)blockIdx.x * kNCost + threadIdx.x] = v;
  }
}

// one warp per cost: lanes stride over the partials, then a fixed xor tree
__global__ void assim_sum_kernel(const double* partials, int n_parts, AssimScales sc, double* costs) {
  const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (c >= kNCost) return;  // uniform per warp
  double v = 0.0;
  for (int b = lane; b < n_parts; b += 32) v += partials[(size_t)b * kNCost + c];
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
  const double f = c == kCVel ? sc.c_vel : c == kCThk ? sc.c_thk : c == kCReg ? sc.c_reg : c == kCUs ? sc.c_us
                                                                                                   : sc.c_pen;
  if (lane == 0) costs[c] = f * v;
}

// ---- flow direction (utils.py:86-110) --------------------------------------
// the separable Gaussian of sigma 3 cells (scipy's gaussian_filter, truncate 4)
constexpr int kGaussR = 12;  // int(4 sigma + 0.5), sigma = 3
struct GaussW { double w[2 * kGaussR + 1]; };

// The whole flow direction in one kernel: a CTA produces a TY x TX tile of
// cells.  Per component, the cell averages of the tile and a 12-cell halo
// (zero outside the domain) go to shared memory, then the y pass over the
// halo columns and the x pass, each accumulated in double and stored in T as
// scipy's gaussian_filter does between its passes; the x component waits in
// registers for the y component, then both are normalised and stored.
template <typename T, int TY, int TX>
__global__ void __launch_bounds__(256) flow_direction_kernel(int ny, int nx, GaussW g, const T* u, const T* v, T* fx,
                                                             T* fy) {
  constexpr int HY = TY + 2 * kGaussR, HX = TX + 2 * kGaussR;
  constexpr int PER = TY * TX / 256;  // outputs per thread: PER consecutive columns of one row
  constexpr int RB = 4;               // rows per thread in the y pass
  static_assert(TY % RB == 0 && TX % PER == 0, "tile");
  const int xr = threadIdx.x / (TX / PER), xc0 = (threadIdx.x % (TX / PER)) * PER;
  // the staged values are T-rounded, held in double so the taps need no conversion
  __shared__ double A[HY][HX];
  __shared__ double Bs[TY][HX];
  const int cy = ny - 1, cx = nx - 1;
  const int y0 = blockIdx.y * TY, x0 = blockIdx.x * TX;
  T res[2][PER];
#pragma unroll
  for (int comp = 0; comp < 2; ++comp) {
    const T* f = comp == 0 ? u : v;
    auto z = [](T x) { return isnan(x) ? T(0) : x; };
    for (int i = threadIdx.x; i < HY * HX; i += 256) {
      const int hy = i / HX, hx = i - hy * HX;
      const int j = y0 - kGaussR + hy, k = x0 - kGaussR + hx;
      T val = T(0);
      if (j >= 0 && j < cy && k >= 0 && k < cx) {
        const size_t a = (size_t)j * nx + k;
        val = (((z(f[a + nx + 1]) + z(f[a + 1])) + z(f[a + nx])) + z(f[a])) / T(4);
      }
      A[hy][hx] = (double)val;
    }
    __syncthreads();
    // y pass: a thread takes RB consecutive rows of one column (RB + 24 reads for RB outputs);
    // each output adds its 25 taps in the order of the single-output loop
    for (int it = threadIdx.x; it < (TY / RB) * HX; it += 256) {
      const int rb = it / HX, hx = it - rb * HX, r0 = rb * RB;
      double sacc[RB];
#pragma unroll
      for (int q = 0; q < RB; ++q) sacc[q] = 0.0;
#pragma unroll
      for (int k = 0; k < 2 * kGaussR + RB; ++k) {
        const double v = A[r0 + k][hx];
#pragma unroll
        for (int q = 0; q < RB; ++q)
          if (k - q >= 0 && k - q <= 2 * kGaussR) sacc[q] += g.w[k - q] * v;
      }
#pragma unroll
      for (int q = 0; q < RB; ++q) Bs[r0 + q][hx] = (double)(T)sacc[q];
    }
    __syncthreads();
    // x pass: a thread takes PER consecutive columns of one row
    {
      double sacc[PER];
#pragma unroll
      for (int q = 0; q < PER; ++q) sacc[q] = 0.0;
#pragma unroll
      for (int k = 0; k < 2 * kGaussR + PER; ++k) {
        const double v = Bs[xr][xc0 + k];
#pragma unroll
        for (int q = 0; q < PER; ++q)
          if (k - q >= 0 && k - q <= 2 * kGaussR) sacc[q] += g.w[k - q] * v;
      }
#pragma unroll
      for (int q = 0; q < PER; ++q) res[comp][q] = (T)sacc[q];
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int r = xr, c = xc0 + q;
    const int j = y0 + r, k = x0 + c;
    if (j >= cy || k >= cx) continue;
    T x = res[0][q], y = res[1][q];
    x = x / sqrt(x * x + y * y);
    y = y / sqrt(x * x + y * y);
    const size_t o = (size_t)j * cx + k;
    fx[o] = isnan(x) ? T(0) : x;
    fy[o] = isnan(y) ? T(0) : y;
  }
}

static int grid_n(size_t n) {
  size_t b = (n + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  return (int)(b < 1 ? 1 : b);
}

template <typename T>
static void set_norm(AssimArgs<T>& a, int fix_normalization) {
  const double ny = a.ny, nx = a.nx;
  a.kx = fix_normalization ? (T)(1.0 / (ny * (nx - 1))) : T(1);
  a.ky = fix_normalization ? (T)(1.0 / ((ny - 1) * nx)) : T(1);
  a.kcell = fix_normalization ? (T)(1.0 / ((ny - 1) * (nx - 1))) : T(1);
  a.kconv = fix_normalization ? 0.5 / (ny * nx) : 1.0;
}

template <typename T>
static int march_launch(AssimArgs<T>& a, const AssimScales& sc, int n_parts, double* costs, cudaStream_t st) {
  // segments of rows sized for about 32 resident warps per SM, at least 8 rows; the
  // warps stride over the (strip, segment) tasks so the grid fits the partials
  const int ny = a.ny, nx = a.nx;
  const int n_strips = (nx + kAmCols - 1) / kAmCols;
  const long long target = 148LL * 32;
  int rows = (int)((n_strips * (long long)ny + target - 1) / target);
  rows = rows < 8 ? 8 : rows;
  const long long tasks = (long long)n_strips * ((ny + rows - 1) / rows);
  long long grid = (tasks + kAmWarps - 1) / kAmWarps;
  if (grid > n_parts) grid = n_parts;
  assim_cost_grad_kernel<T><<<(int)grid, kAmWarps * 32, 0, st>>>(a, sc, n_strips, rows, (int)tasks);
  int rc = launch_status("assim_cost_grad_kernel");
  if (rc) return rc;
  assim_sum_kernel<<<1, 32 * kNCost, 0, st>>>(a.partials, (int)grid, sc, costs);
  return launch_status("assim_sum_kernel");
}

template <typename T>
static int cost_grad_t(int ny, int nx, double dx, const void* thk, const void* usurf, const void* uvs,
                       const void* vvs, const void* uobs, const void* vobs, const void* thkobs, const void* dens,
                       const void* icemaskobs, const void* fdx, const void* fdy, const void* usobs,
                       const igm_assim_params* p, void* g_thk, void* g_u, void* g_v, void* g_us, double* partials,
                       int n_parts, double* costs, cudaStream_t st) {
  AssimArgs<T> a{};
  a.ny = ny; a.nx = nx; a.dx = (T)dx;
  a.thk = (const T*)thk; a.usurf = (const T*)usurf; a.uvs = (const T*)uvs; a.vvs = (const T*)vvs;
  a.uobs = (const T*)uobs; a.vobs = (const T*)vobs; a.thkobs = (const T*)thkobs; a.dens = (const T*)dens;
  a.icemaskobs = (const T*)icemaskobs; a.fdx = (const T*)fdx; a.fdy = (const T*)fdy; a.usobs = (const T*)usobs;
  a.p = *p;
  a.g_thk = (T*)g_thk; a.g_u = (T*)g_u; a.g_v = (T*)g_v; a.g_us = (T*)g_us;
  a.partials = partials;
  AssimScales sc{};
  sc.c_vel = 0.5 / (p->velsurfobs_std * p->velsurfobs_std * p->n_vel);
  sc.c_thk = 0.5 / (p->thkobs_std * p->thkobs_std * p->n_thk);
  sc.c_pen = 1e10 / ((double)ny * nx);
  sc.c_reg = p->regu_thk;
  sc.c_us = p->usurf_cost ? 0.5 / (p->usurfobs_std * p->usurfobs_std * (p->n_usurf > 0 ? p->n_usurf : 1.0)) : 0.0;
  sc.gamma = p->gamma;
  set_norm(a, p->fix_normalization);
  a.sole_mask = p->sole_mask;
  return march_launch<T>(a, sc, n_parts, costs, st);
}

template <typename T>
static int field_regu_t(int ny, int nx, double dx, const void* field, const void* fdx, const void* fdy, double regu,
                        double aniso, int penalty, double pos_thr, int fix_normalization, const void* icemaskobs,
                        int sole_mask, void* grad, double* partials, int n_parts, double* costs, cudaStream_t st) {
  AssimArgs<T> a{};
  a.ny = ny; a.nx = nx; a.dx = (T)dx;
  a.thk = (const T*)field; a.fdx = (const T*)fdx; a.fdy = (const T*)fdy;
  a.p.regu_thk = regu;
  a.p.aniso_factor = aniso;
  a.p.penalty = penalty;
  a.p.velsurfobs_std = a.p.thkobs_std = a.p.usurfobs_std = 1.0;
  a.p.n_vel = a.p.n_thk = a.p.n_usurf = 1.0;
  a.field_only = 1;
  a.pos_thr = (T)pos_thr;
  a.g_thk = (T*)grad;
  a.partials = partials;
  a.icemaskobs = (const T*)icemaskobs;
  a.sole_mask = sole_mask;
  a.mask_eq1 = 1;
  AssimScales sc{};
  sc.c_pen = 1e10 / ((double)ny * nx);
  sc.c_reg = regu;
  set_norm(a, fix_normalization);
  return march_launch<T>(a, sc, n_parts, costs, st);
}

template <typename T>
static int flow_t(int ny, int nx, const void* u, const void* v, void* fx, void* fy, void* scratch, cudaStream_t st) {
  (void)scratch;
  const int cy = ny - 1, cx = nx - 1;
  GaussW g{};
  double sum = 0.0;
  for (int k = -kGaussR; k <= kGaussR; ++k) sum += (g.w[k + kGaussR] = exp(-0.5 * k * k / 9.0));
  for (int k = 0; k < 2 * kGaussR + 1; ++k) g.w[k] /= sum;
  constexpr int TY = sizeof(T) == 4 ? 32 : 16, TX = 32;
  const dim3 grid((cx + TX - 1) / TX, (cy + TY - 1) / TY);
  flow_direction_kernel<T, TY, TX><<<grid, 256, 0, st>>>(ny, nx, g, (const T*)u, (const T*)v, (T*)fx, (T*)fy);
  return launch_status("flow_direction_kernel");
}

// Control update of optimize_update (optimize/update.py:22-42, 56-98) for one
// control x with scaling sc (see igm_assim_control): mode 0 before the
// forward (the variable, x from it, zero moments), mode 1 the gradient of the
// variable with the control's mask, mode 2 x from the variable and the
// reprojection.
template <typename T>
__global__ void assim_control_kernel(size_t n, igm_assim_control_params p, const T* g_direct, const float* g_emul,
                                     const T* icemaskobs, T* x, float* var, float* grad, float* m, float* v) {
  const T sc = (T)p.scale;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    if (p.mode == 0) {
      const float w = p.transform ? (float)sqrt(x[o] / sc) : (float)(x[o] / sc);
      var[o] = w;
      x[o] = p.transform ? ((T)w * (T)w) * sc : (T)w * sc;
      m[o] = 0.f;
      v[o] = 0.f;
    } else if (p.mode == 1) {
      bool on = true;
      if (p.mask == 1) on = icemaskobs[o] > T(0.5);
      if (p.mask == 2) on = icemaskobs[o] == T(1);
      const T g = g_direct[o] + (g_emul ? (T)g_emul[o] : T(0));
      const T dxdw = p.transform ? T(2) * (T)var[o] * sc : sc;
      grad[o] = on ? (float)(g * dxdw) : 0.f;
    } else if (p.mode == 3) {
      if (!(icemaskobs[o] > T(0.5))) x[o] = T(0);
    } else {
      const T w = (T)var[o];
      T t = p.transform ? (w * w) * sc : w * sc;
      if (p.reproject == 1) {
        if (p.reproject_mask && !(icemaskobs[o] > T(0.5))) t = T(0);
        if (t < T(0)) t = T(0);
      } else if (p.reproject == 2) {
        if (t < (T)p.lower) t = (T)p.lower;
      }
      x[o] = t;
    }
  }
}

// compute_rms_std_optimization (data_assimilation/utils.py:10-66): count, sum
// and sum of squares of the misfits thk - thkobs (at the thickness
// observations), |velsurf| - |velsurfobs| (inside icemaskobs > 0.5 where the
// observed speed is defined), divfluxobs - divflux and usurf - usurfobs (inside
// the mask), and the sum of thk; per-block FP64 partials, then one warp turns
// them into the nine record entries.
constexpr int kNStat = 13;

template <typename T>
struct StatArgs {
  size_t n;
  const T *thk, *thkobs, *uvs, *vvs, *uobs, *vobs, *im, *div, *divobs, *us, *usobs;
  double* partials;
};

template <typename T>
__global__ void __launch_bounds__(256) assim_stats_kernel(const StatArgs<T> a) {
  double acc[kNStat];
#pragma unroll
  for (int k = 0; k < kNStat; ++k) acc[k] = 0.0;
  auto add = [&](int k, T d) {
    acc[k] += 1.0;
    acc[k + 1] += (double)d;
    acc[k + 2] += (double)d * (double)d;
  };
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < a.n; o += (size_t)gridDim.x * blockDim.x) {
    const T th = a.thk[o];
    acc[12] += (double)th;
    if (a.thkobs) {
      const T to = a.thkobs[o];
      if (!isnan(to)) add(0, th - to);
    }
    const bool in = a.im[o] > T(0.5);
    if (in && a.uobs) {
      const T uo = a.uobs[o], vo = a.vobs[o];
      const T mo = sqrt(uo * uo + vo * vo);
      if (!isnan(mo)) {
        const T u = a.uvs[o], v = a.vvs[o];
        add(3, sqrt(u * u + v * v) - mo);
      }
    }
    if (in && a.divobs) add(6, a.divobs[o] - a.div[o]);
    if (in && a.usobs) add(9, a.us[o] - a.usobs[o]);
  }
  __shared__ double red[8][kNStat];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kNStat; ++k) {
    double v = acc[k];
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNStat) {
    double v = 0.0;
    for (int w = 0; w < 8; ++w) v += red[w][threadIdx.x];
    a.partials[(size_t)blockIdx.x * kNStat + threadIdx.x] = v;
  }
}

// out[9]: rmsthk, stdthk, rmsvel, stdvel, rmsdiv, stddiv, rmsusurf, stdusurf, vol
// (means and population standard deviations; a term without data is 0, an empty
// mask gives NaN as numpy's mean of an empty selection)
__global__ void assim_stats_finish_kernel(const double* partials, int n_parts, double dx2, int have_thk,
                                          int have_vel, int have_div, int have_us, double* out) {
  // warp k adds up statistic k (lane-strided, fixed xor tree); then thread 0 forms the record
  __shared__ double tot[kNStat];
  const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k < kNStat) {
    double v = 0.0;
    for (int b = lane; b < n_parts; b += 32) v += partials[(size_t)b * kNStat + k];
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    if (lane == 0) tot[k] = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const int have[4] = {have_thk, have_vel, have_div, have_us};
  for (int t = 0; t < 4; ++t) {
    const double c = tot[3 * t], s1 = tot[3 * t + 1], s2 = tot[3 * t + 2];
    double mean = 0.0, sd = 0.0;
    if (have[t]) {
      if (t == 0 && c == 0.0) {
        mean = sd = 0.0;  // no thickness observation: the reference records 0
      } else {
        mean = s1 / c;
        const double var = s2 / c - mean * mean;
        sd = sqrt(var > 0.0 ? var : 0.0);
      }
    }
    out[2 * t] = mean;
    out[2 * t + 1] = sd;
  }
  out[8] = tot[12] * dx2 / 1e9;
}

// ---- flux-divergence cost terms --------------------------------------------
// cost_divfluxobs (cost_terms/cost_divfluxobs.py:9-29): 0.5 mean over the
// observed nodes of ((obs - D) / std)^2 + regu 0.5 (mean (dD/dx)^2 + mean
// (dD/dy)^2); cost_divfluxfcz (cost_terms/cost_divfluxfcz.py:10-38): the
// target intercept + slope usurf, 0.5 mean over icemaskobs > 0.5 of
// ((target - D) / std)^2; both + 0.5 1000 mean_mask(D / std)^2 with
// force_zero_sum.  D = compute_divflux(ubar, vbar, thk).  Four launches: the
// global sums (counts, sum of D in the mask), dC/dD per node, the adjoint of
// compute_divflux into dC/dthk and dC/dU, dC/dV of every level (velbar =
// sum_k w_k U_k, zero where the thk mask is off), the cost.
template <typename T>
struct DivCostArgs {
  int ny, nx, nz, kind, method, fzs;
  T dx, rdx;
  double sd, regu, slope, intercept;
  const T *ubar, *vbar, *thk, *D, *obs, *usurf, *im, *mask;
  T *g_thk, *dU, *dV, *gD;
  T w[IGM_MAX_NZ];
  double* partials;  // [n_parts][3] sums, then [n_parts][3] cost sums
  int n_parts;
  double* scal;      // count_act, count_mask, sum_mask D
  double* cost;
};

template <typename T>
__device__ __forceinline__ void block_reduce3(double v0, double v1, double v2, double* out) {
  __shared__ double red[8][3];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v[3] = {v0, v1, v2};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    for (int s = 16; s > 0; s >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], s);
    if (lane == 0) red[warp][c] = v[c];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
    out[(size_t)blockIdx.x * 3 + threadIdx.x] = t;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) divcost_sums_kernel(const DivCostArgs<T> a) {
  const size_t n = (size_t)a.ny * a.nx;
  double c_act = 0.0, c_m = 0.0, s_m = 0.0;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const bool in = a.im[o] > T(0.5);
    if (a.kind == 0) c_act += isnan(a.obs[o]) ? 0.0 : 1.0;
    if (in) {
      c_m += 1.0;
      s_m += (double)a.D[o];
    }
  }
  block_reduce3<T>(c_act, c_m, s_m, a.partials);
}

// fixed-order sums of n_parts rows of 3 (one warp per column)
__global__ void divcost_finish3_kernel(const double* partials, int n_parts, double* out) {
  const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (c >= 3) return;
  double v = 0.0;
  for (int b = lane; b < n_parts; b += 32) v += partials[(size_t)b * 3 + c];
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
  if (lane == 0) out[c] = v;
}

template <typename T>
__global__ void __launch_bounds__(256) divcost_gradD_kernel(const DivCostArgs<T> a) {
  const int ny = a.ny, nx = a.nx;
  const size_t n = (size_t)ny * nx;
  const double n_act = a.kind == 0 ? a.scal[0] : a.scal[1];
  const double n_m = a.scal[1];
  const T kd = (T)(1.0 / (a.sd * a.sd * n_act));
  const T ksx = (T)(a.regu / ((double)ny * (nx - 1))), ksy = (T)(a.regu / ((double)(ny - 1) * nx));
  const T kz = a.fzs ? (T)(1000.0 * (a.scal[2] / (a.sd * n_m)) / (a.sd * n_m)) : T(0);
  const T rdx = a.rdx;
  double c_r = 0.0, c_x = 0.0, c_y = 0.0;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(o / nx), i = (int)(o - (size_t)j * nx);
    const T D0 = a.D[o];
    const bool in = a.im[o] > T(0.5);
    T g = T(0);
    if (a.kind == 0) {
      const T ob = a.obs[o];
      if (!isnan(ob)) {
        const T r = ob - D0;
        c_r += (double)r * (double)r;
        g -= r * kd;
      }
      // smoothness of D: forward differences owned by this node, backward ones from the neighbours
      if (i + 1 < nx) {
        const T d = (a.D[o + 1] - D0) * rdx;
        c_x += (double)d * (double)d;
        g -= ksx * d * rdx;
      }
      if (i >= 1) g += ksx * ((D0 - a.D[o - 1]) * rdx) * rdx;
      if (j + 1 < ny) {
        const T d = (a.D[o + nx] - D0) * rdx;
        c_y += (double)d * (double)d;
        g -= ksy * d * rdx;
      }
      if (j >= 1) g += ksy * ((D0 - a.D[o - nx]) * rdx) * rdx;
    } else if (in) {
      const T r = (T)(a.intercept + a.slope * (double)a.usurf[o]) - D0;
      c_r += (double)r * (double)r;
      g -= r * kd;
    }
    if (in) g += kz;
    a.gD[o] = g;
  }
  block_reduce3<T>(c_r, c_x, c_y, a.partials + (size_t)a.n_parts * 3);
}

// the adjoint of compute_divflux at node (j, i): the faces i, i+1 (x) and j, j+1 (y)
template <typename T, int METHOD>
__global__ void __launch_bounds__(256) divcost_adjoint_kernel(const DivCostArgs<T> a) {
  const int ny = a.ny, nx = a.nx;
  const size_t n = (size_t)ny * nx;
  const T rdx = a.rdx;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(o / nx), i = (int)(o - (size_t)j * nx);
    auto gd = [&](int jj, int ii) {
      return (jj < 0 || jj >= ny || ii < 0 || ii >= nx) ? T(0) : a.gD[(size_t)jj * nx + ii];
    };
    auto hh = [&](int jj, int ii) {
      return (jj < 0 || jj >= ny || ii < 0 || ii >= nx) ? T(0) : a.thk[(size_t)jj * nx + ii];
    };
    // d C / d Q of the faces: Q(f) enters D(f - 1) with + 1/dx and D(f) with - 1/dx
    const T gqw = (gd(j, i - 1) - gd(j, i)) * rdx, gqe = (gd(j, i) - gd(j, i + 1)) * rdx;
    const T gqs = (gd(j - 1, i) - gd(j, i)) * rdx, gqn = (gd(j, i) - gd(j + 1, i)) * rdx;
    const T cw = i == 0 ? T(1) : T(0.5), ce = i == nx - 1 ? T(1) : T(0.5);
    const T cs = j == 0 ? T(1) : T(0.5), cn = j == ny - 1 ? T(1) : T(0.5);
    const T u0 = a.ubar[o], v0 = a.vbar[o], h0 = a.thk[o];
    T gu, gv, gh;
    if (METHOD == IGM_DIVFLUX_UPWIND) {
      auto uu = [&](int ii) { return a.ubar[(size_t)j * nx + ii]; };
      auto vv = [&](int jj) { return a.vbar[(size_t)jj * nx + i]; };
      const T uw = i == 0 ? uu(0) : T(0.5) * (uu(i - 1) + u0);
      const T ue = i == nx - 1 ? uu(nx - 1) : T(0.5) * (u0 + uu(i + 1));
      const T vs = j == 0 ? vv(0) : T(0.5) * (vv(j - 1) + v0);
      const T vn = j == ny - 1 ? vv(ny - 1) : T(0.5) * (v0 + vv(j + 1));
      const T hw = uw > T(0) ? hh(j, i - 1) : h0, he = ue > T(0) ? h0 : hh(j, i + 1);
      const T hs = vs > T(0) ? hh(j - 1, i) : h0, hn = vn > T(0) ? h0 : hh(j + 1, i);
      gu = gqw * hw * cw + gqe * he * ce;
      gv = gqs * hs * cs + gqn * hn * cn;
      // this node's thickness is the upwind value of face i when uw <= 0, of face i+1 when ue > 0
      gh = (uw > T(0) ? T(0) : gqw * uw) + (ue > T(0) ? gqe * ue : T(0)) + (vs > T(0) ? T(0) : gqs * vs) +
           (vn > T(0) ? gqn * vn : T(0));
    } else {
      // centered: Q(f) averages q = u h of its two nodes (an edge copy at the border)
      const T gqx = gqw * cw + gqe * ce, gqy = gqs * cs + gqn * cn;
      gu = gqx * h0;
      gv = gqy * h0;
      gh = gqx * u0 + gqy * v0;
    }
    a.g_thk[o] += gh;
    const bool on = a.mask == nullptr || a.mask[o] > T(0);
    const size_t plane = n;
    for (int k = 0; k < a.nz; ++k) {
      const T du = on ? a.w[k] * gu : T(0), dv = on ? a.w[k] * gv : T(0);
      const size_t q = (size_t)k * plane + o;
      if (k == a.nz - 1) {
        a.dU[q] += du;
        a.dV[q] += dv;
      } else {
        a.dU[q] = du;
        a.dV[q] = dv;
      }
    }
  }
}

template <typename T>
__global__ void divcost_cost_kernel(const DivCostArgs<T> a) {
  __shared__ double t[3];
  const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (c < 3) {
    double v = 0.0;
    const double* p = a.partials + (size_t)a.n_parts * 3;
    for (int b = lane; b < a.n_parts; b += 32) v += p[(size_t)b * 3 + c];
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    if (lane == 0) t[c] = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double n_act = a.kind == 0 ? a.scal[0] : a.scal[1];
  double cst = 0.5 * t[0] / (a.sd * a.sd * n_act);
  if (a.kind == 0)
    cst += a.regu * 0.5 * (t[1] / ((double)a.ny * (a.nx - 1)) + t[2] / ((double)(a.ny - 1) * a.nx));
  if (a.fzs) {
    const double m = a.scal[2] / (a.sd * a.scal[1]);
    cst += 0.5 * 1000.0 * m * m;
  }
  *a.cost = cst;
}

// include_low_speed_term of misfit_velsurf (cost_terms/misfit_velsurf.py:21-28):
// 0.5 100 log((|vs| + 1) / (|obs| + 1))^2 with |.| the norm of all observed
// components (the reference selects velsurf[ACT], a 1-D vector).  Sums of the
// squares per block, then one warp forms the norms, adds the term to the
// velsurf cost and stores the gradient factor c = 100 L / ((|vs| + 1) |vs|),
// then dC/dvs += c vs on the observed components.
template <typename T>
__global__ void __launch_bounds__(256) low_speed_sums_kernel(size_t n, const T* uvs, const T* vvs, const T* uobs,
                                                             const T* vobs, double* partials) {
  double s_v = 0.0, s_o = 0.0;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const T uo = uobs[o], vo = vobs[o];
    if (!isnan(uo)) {
      s_v += (double)uvs[o] * (double)uvs[o];
      s_o += (double)uo * (double)uo;
    }
    if (!isnan(vo)) {
      s_v += (double)vvs[o] * (double)vvs[o];
      s_o += (double)vo * (double)vo;
    }
  }
  block_reduce3<T>(s_v, s_o, 0.0, partials);
}

__global__ void low_speed_finish_kernel(const double* partials, int n_parts, double* cost, double* factor) {
  const int lane = threadIdx.x;
  double sv = 0.0, so = 0.0;
  for (int b = lane; b < n_parts; b += 32) {
    sv += partials[(size_t)b * 3];
    so += partials[(size_t)b * 3 + 1];
  }
  for (int s = 16; s > 0; s >>= 1) {
    sv += __shfl_xor_sync(0xffffffffu, sv, s);
    so += __shfl_xor_sync(0xffffffffu, so, s);
  }
  if (lane != 0) return;
  const double nv = sqrt(sv), no = sqrt(so);
  const double L = log((nv + 1.0) / (no + 1.0));
  *cost += 0.5 * 100.0 * L * L;
  *factor = nv > 0.0 ? 100.0 * L / ((nv + 1.0) * nv) : 0.0;
}

template <typename T>
__global__ void low_speed_grad_kernel(size_t n, const T* uvs, const T* vvs, const T* uobs, const T* vobs,
                                      const double* factor, T* g_u, T* g_v) {
  const T c = (T)*factor;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    if (!isnan(uobs[o])) g_u[o] += c * uvs[o];
    if (!isnan(vobs[o])) g_v[o] += c * vvs[o];
  }
}

}  // namespace igm

using namespace igm;

extern "C" int igm_assim_cost_grad(int dtype, int ny, int nx, double dx, const void* thk, const void* usurf,
                                   const void* uvelsurf, const void* vvelsurf, const void* uvelsurfobs,
                                   const void* vvelsurfobs, const void* thkobs, const void* dens_thkobs,
                                   const void* icemaskobs, const void* flowdirx, const void* flowdiry,
                                   const void* usurfobs, const igm_assim_params* params, void* grad_thk,
                                   void* grad_uvelsurf, void* grad_vvelsurf, void* grad_usurf, double* partials,
                                   int n_parts, double* costs, void* stream) {
  IGM_CHECK_ARG(ny >= 2 && nx >= 2, IGM_ERR_BAD_SHAPE, "igm_assim_cost_grad: bad shape %dx%d", ny, nx);
  IGM_CHECK_ARG(thk && usurf && uvelsurf && vvelsurf && uvelsurfobs && vvelsurfobs && thkobs && dens_thkobs &&
                    icemaskobs && params && grad_thk && grad_uvelsurf && grad_vvelsurf && partials && costs,
                IGM_ERR_BAD_ARGUMENT, "igm_assim_cost_grad: NULL argument");
  IGM_CHECK_ARG(params->aniso_factor == 1.0 || (flowdirx && flowdiry), IGM_ERR_BAD_ARGUMENT,
                "igm_assim_cost_grad: the anisotropic regularisation needs flowdirx, flowdiry");
  IGM_CHECK_ARG(!params->usurf_cost || (usurfobs && params->usurfobs_std > 0), IGM_ERR_BAD_ARGUMENT,
                "igm_assim_cost_grad: misfit_usurf needs usurfobs and usurfobs_std > 0");
  IGM_CHECK_ARG(params->aniso_factor > 0 && params->n_vel >= 1 && params->n_thk >= 1 && n_parts >= 1 && dx > 0,
                IGM_ERR_BAD_ARGUMENT, "igm_assim_cost_grad: bad parameter");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    return cost_grad_t<float>(ny, nx, dx, thk, usurf, uvelsurf, vvelsurf, uvelsurfobs, vvelsurfobs, thkobs,
                              dens_thkobs, icemaskobs, flowdirx, flowdiry, usurfobs, params, grad_thk,
                              grad_uvelsurf, grad_vvelsurf, grad_usurf, partials, n_parts, costs, st);
  if (dtype == IGM_F64)
    return cost_grad_t<double>(ny, nx, dx, thk, usurf, uvelsurf, vvelsurf, uvelsurfobs, vvelsurfobs, thkobs,
                               dens_thkobs, icemaskobs, flowdirx, flowdiry, usurfobs, params, grad_thk,
                               grad_uvelsurf, grad_vvelsurf, grad_usurf, partials, n_parts, costs, st);
  set_error("igm_assim_cost_grad: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_assim_field_regu(int dtype, int ny, int nx, double dx, const void* field, const void* flowdirx,
                                    const void* flowdiry, double regu, double aniso_factor, int penalty,
                                    double penalty_threshold, int fix_normalization, const void* icemaskobs,
                                    int sole_mask, void* grad, double* partials, int n_parts, double* costs,
                                    void* stream) {
  IGM_CHECK_ARG(ny >= 2 && nx >= 2 && dx > 0, IGM_ERR_BAD_SHAPE, "igm_assim_field_regu: bad shape %dx%d", ny, nx);
  IGM_CHECK_ARG(field && grad && partials && costs && n_parts >= 1 && aniso_factor > 0, IGM_ERR_BAD_ARGUMENT,
                "igm_assim_field_regu: bad argument");
  IGM_CHECK_ARG(aniso_factor == 1.0 || (flowdirx && flowdiry), IGM_ERR_BAD_ARGUMENT,
                "igm_assim_field_regu: the anisotropic regularisation needs flowdirx, flowdiry");
  IGM_CHECK_ARG(!sole_mask || icemaskobs, IGM_ERR_BAD_ARGUMENT, "igm_assim_field_regu: sole_mask needs icemaskobs");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    return field_regu_t<float>(ny, nx, dx, field, flowdirx, flowdiry, regu, aniso_factor, penalty, penalty_threshold,
                               fix_normalization, icemaskobs, sole_mask, grad, partials, n_parts, costs, st);
  if (dtype == IGM_F64)
    return field_regu_t<double>(ny, nx, dx, field, flowdirx, flowdiry, regu, aniso_factor, penalty,
                                penalty_threshold, fix_normalization, icemaskobs, sole_mask, grad, partials, n_parts,
                                costs, st);
  set_error("igm_assim_field_regu: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_assim_flow_direction(int dtype, int ny, int nx, const void* uvelsurf, const void* vvelsurf,
                                        void* flowdirx, void* flowdiry, void* scratch, void* stream) {
  IGM_CHECK_ARG(ny >= 2 && nx >= 2, IGM_ERR_BAD_SHAPE, "igm_assim_flow_direction: bad shape %dx%d", ny, nx);
  IGM_CHECK_ARG(uvelsurf && vvelsurf && flowdirx && flowdiry, IGM_ERR_BAD_ARGUMENT,
                "igm_assim_flow_direction: NULL argument");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32) return flow_t<float>(ny, nx, uvelsurf, vvelsurf, flowdirx, flowdiry, scratch, st);
  if (dtype == IGM_F64) return flow_t<double>(ny, nx, uvelsurf, vvelsurf, flowdirx, flowdiry, scratch, st);
  set_error("igm_assim_flow_direction: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_assim_control(int dtype, size_t n, const igm_assim_control_params* params, void* x,
                                 const void* grad_direct, const float* grad_emulator, const void* icemaskobs,
                                 float* variable, float* grad, float* m, float* v, void* stream) {
  IGM_CHECK_ARG(params && n >= 1 && params->scale > 0 && params->mode >= 0 && params->mode <= 3,
                IGM_ERR_BAD_ARGUMENT, "igm_assim_control: bad mode, size or scale");
  const igm_assim_control_params& p = *params;
  IGM_CHECK_ARG(x && (variable || p.mode == 3) && (p.mode != 0 || (m && v)) &&
                    (p.mode != 1 || (grad_direct && grad)) &&
                    ((p.mode == 1 && p.mask != 0) || (p.mode == 2 && p.reproject == 1 && p.reproject_mask) ||
                             p.mode == 3
                         ? icemaskobs != nullptr
                         : true),
                IGM_ERR_BAD_ARGUMENT, "igm_assim_control: NULL argument");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    assim_control_kernel<float><<<grid_n(n), 256, 0, st>>>(n, p, (const float*)grad_direct, grad_emulator,
                                                           (const float*)icemaskobs, (float*)x, variable, grad, m, v);
  else if (dtype == IGM_F64)
    assim_control_kernel<double><<<grid_n(n), 256, 0, st>>>(n, p, (const double*)grad_direct, grad_emulator,
                                                            (const double*)icemaskobs, (double*)x, variable, grad, m,
                                                            v);
  else {
    set_error("igm_assim_control: unknown dtype %d", dtype);
    return IGM_ERR_BAD_ARGUMENT;
  }
  return launch_status("assim_control_kernel");
}

extern "C" int igm_assim_stats(int dtype, int ny, int nx, double dx, const void* thk, const void* thkobs,
                               const void* uvelsurf, const void* vvelsurf, const void* uvelsurfobs,
                               const void* vvelsurfobs, const void* icemaskobs, const void* divflux,
                               const void* divfluxobs, const void* usurf, const void* usurfobs, double* partials,
                               int n_parts, double* out, void* stream) {
  IGM_CHECK_ARG(ny >= 1 && nx >= 1, IGM_ERR_BAD_SHAPE, "igm_assim_stats: bad shape %dx%d", ny, nx);
  IGM_CHECK_ARG(thk && icemaskobs && partials && out && n_parts >= 1, IGM_ERR_BAD_ARGUMENT,
                "igm_assim_stats: NULL argument");
  IGM_CHECK_ARG(!uvelsurfobs || (vvelsurfobs && uvelsurf && vvelsurf), IGM_ERR_BAD_ARGUMENT,
                "igm_assim_stats: velocity observations need both components and the emulated velocities");
  IGM_CHECK_ARG(!divfluxobs || divflux, IGM_ERR_BAD_ARGUMENT, "igm_assim_stats: divfluxobs needs divflux");
  IGM_CHECK_ARG(!usurfobs || usurf, IGM_ERR_BAD_ARGUMENT, "igm_assim_stats: usurfobs needs usurf");
  cudaStream_t st = as_stream(stream);
  const size_t n = (size_t)ny * nx;
  int grid = grid_n(n);
  if (grid > n_parts) grid = n_parts;
  auto run = [&](auto zero) {
    using T = decltype(zero);
    StatArgs<T> a{n, (const T*)thk, (const T*)thkobs, (const T*)uvelsurf, (const T*)vvelsurf,
                  (const T*)uvelsurfobs, (const T*)vvelsurfobs, (const T*)icemaskobs, (const T*)divflux,
                  (const T*)divfluxobs, (const T*)usurf, (const T*)usurfobs, partials};
    assim_stats_kernel<T><<<grid, 256, 0, st>>>(a);
  };
  if (dtype == IGM_F32)
    run(0.f);
  else if (dtype == IGM_F64)
    run(0.0);
  else {
    set_error("igm_assim_stats: unknown dtype %d", dtype);
    return IGM_ERR_BAD_ARGUMENT;
  }
  int rc = launch_status("assim_stats_kernel");
  if (rc) return rc;
  assim_stats_finish_kernel<<<1, 32 * kNStat, 0, st>>>(partials, grid, dx * dx, thkobs != nullptr, uvelsurfobs != nullptr,
                                              divfluxobs != nullptr, usurfobs != nullptr, out);
  return launch_status("assim_stats_finish_kernel");
}

extern "C" int igm_assim_divflux_cost_grad(int dtype, int ny, int nx, double dx, int nz, const double* vert_weight,
                                           const void* ubar, const void* vbar, const void* thk, const void* divflux,
                                           const void* divfluxobs, const void* usurf, const void* icemaskobs,
                                           const void* mask_thk, const igm_divflux_cost_params* params,
                                           void* grad_thk, void* dU, void* dV, void* scratch, double* partials,
                                           int n_parts, double* cost, void* stream) {
  IGM_CHECK_ARG(ny >= 2 && nx >= 2 && dx > 0 && nz >= 1 && nz <= IGM_MAX_NZ, IGM_ERR_BAD_SHAPE,
                "igm_assim_divflux_cost_grad: bad shape");
  IGM_CHECK_ARG(params && vert_weight && ubar && vbar && thk && divflux && icemaskobs && grad_thk && dU && dV &&
                    scratch && partials && cost && n_parts >= 1,
                IGM_ERR_BAD_ARGUMENT, "igm_assim_divflux_cost_grad: NULL argument");
  IGM_CHECK_ARG((params->kind == 0 && divfluxobs) || (params->kind == 1 && usurf), IGM_ERR_BAD_ARGUMENT,
                "igm_assim_divflux_cost_grad: kind 0 needs divfluxobs, kind 1 needs usurf");
  IGM_CHECK_ARG(params->method == IGM_DIVFLUX_UPWIND || params->method == IGM_DIVFLUX_CENTERED,
                IGM_ERR_BAD_ARGUMENT, "igm_assim_divflux_cost_grad: unknown method");
  IGM_CHECK_ARG(params->divfluxobs_std > 0, IGM_ERR_BAD_ARGUMENT, "igm_assim_divflux_cost_grad: std <= 0");
  cudaStream_t st = as_stream(stream);
  const size_t n = (size_t)ny * nx;
  int grid = grid_n(n);
  if (grid > n_parts) grid = n_parts;
  auto run = [&](auto zero) -> int {
    using T = decltype(zero);
    DivCostArgs<T> a{};
    a.ny = ny; a.nx = nx; a.nz = nz;
    a.kind = params->kind; a.method = params->method; a.fzs = params->force_zero_sum;
    a.dx = (T)dx; a.rdx = T(1) / a.dx;
    a.sd = params->divfluxobs_std; a.regu = params->regu_divflux; a.slope = params->slope;
    a.intercept = params->intercept;
    a.ubar = (const T*)ubar; a.vbar = (const T*)vbar; a.thk = (const T*)thk; a.D = (const T*)divflux;
    a.obs = (const T*)divfluxobs; a.usurf = (const T*)usurf; a.im = (const T*)icemaskobs; a.mask = (const T*)mask_thk;
    a.g_thk = (T*)grad_thk; a.dU = (T*)dU; a.dV = (T*)dV; a.gD = (T*)scratch;
    for (int k = 0; k < nz; ++k) a.w[k] = (T)vert_weight[k];
    a.partials = partials; a.n_parts = grid; a.scal = partials + (size_t)6 * grid; a.cost = cost;
    divcost_sums_kernel<T><<<grid, 256, 0, st>>>(a);
    int rc = launch_status("divcost_sums_kernel");
    if (rc) return rc;
    divcost_finish3_kernel<<<1, 96, 0, st>>>(partials, grid, a.scal);
    if ((rc = launch_status("divcost_finish3_kernel"))) return rc;
    divcost_gradD_kernel<T><<<grid, 256, 0, st>>>(a);
    if ((rc = launch_status("divcost_gradD_kernel"))) return rc;
    if (a.method == IGM_DIVFLUX_UPWIND)
      divcost_adjoint_kernel<T, IGM_DIVFLUX_UPWIND><<<grid_n(n), 256, 0, st>>>(a);
    else
      divcost_adjoint_kernel<T, IGM_DIVFLUX_CENTERED><<<grid_n(n), 256, 0, st>>>(a);
    if ((rc = launch_status("divcost_adjoint_kernel"))) return rc;
    divcost_cost_kernel<T><<<1, 96, 0, st>>>(a);
    return launch_status("divcost_cost_kernel");
  };
  if (dtype == IGM_F32) return run(0.f);
  if (dtype == IGM_F64) return run(0.0);
  set_error("igm_assim_divflux_cost_grad: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" size_t igm_assim_divflux_partials_len(int n_parts) { return (size_t)6 * n_parts + 3; }

extern "C" int igm_assim_low_speed(int dtype, int ny, int nx, const void* uvelsurf, const void* vvelsurf,
                                   const void* uvelsurfobs, const void* vvelsurfobs, void* grad_uvelsurf,
                                   void* grad_vvelsurf, double* partials, int n_parts, double* cost, void* stream) {
  IGM_CHECK_ARG(ny >= 1 && nx >= 1, IGM_ERR_BAD_SHAPE, "igm_assim_low_speed: bad shape");
  IGM_CHECK_ARG(uvelsurf && vvelsurf && uvelsurfobs && vvelsurfobs && grad_uvelsurf && grad_vvelsurf && partials &&
                    cost && n_parts >= 1,
                IGM_ERR_BAD_ARGUMENT, "igm_assim_low_speed: NULL argument");
  cudaStream_t st = as_stream(stream);
  const size_t n = (size_t)ny * nx;
  int grid = grid_n(n);
  if (grid > n_parts) grid = n_parts;
  double* factor = partials + (size_t)3 * grid;
  auto run = [&](auto zero) -> int {
    using T = decltype(zero);
    low_speed_sums_kernel<T><<<grid, 256, 0, st>>>(n, (const T*)uvelsurf, (const T*)vvelsurf,
                                                   (const T*)uvelsurfobs, (const T*)vvelsurfobs, partials);
    int rc = launch_status("low_speed_sums_kernel");
    if (rc) return rc;
    low_speed_finish_kernel<<<1, 32, 0, st>>>(partials, grid, cost, factor);
    if ((rc = launch_status("low_speed_finish_kernel"))) return rc;
    low_speed_grad_kernel<T><<<grid_n(n), 256, 0, st>>>(n, (const T*)uvelsurf, (const T*)vvelsurf,
                                                        (const T*)uvelsurfobs, (const T*)vvelsurfobs, factor,
                                                        (T*)grad_uvelsurf, (T*)grad_vvelsurf);
    return launch_status("low_speed_grad_kernel");
  };
  if (dtype == IGM_F32) return run(0.f);
  if (dtype == IGM_F64) return run(0.0);
  set_error("igm_assim_low_speed: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}
