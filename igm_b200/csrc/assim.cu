// Data assimilation (igm/processes/data_assimilation): the cost terms of the
// default configuration and their gradient, the flow direction of the
// anisotropic regularisation.  HBM-bound node stencils with deterministic
// (fixed-order) FP64 cost reductions.
#include "common.cuh"

namespace igm {

// cost indices of igm_assim_cost_grad
enum { kCVel = 0, kCThk = 1, kCIce = 2, kCPos = 3, kCReg = 4, kNCost = 5 };

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
  igm_assim_params p;
  T* g_thk;  // dC/dthk
  T* g_u;    // dC/duvs
  T* g_v;
  double* partials;  // [gridDim.x][kNCost]
};

// regularisation of one cell (cj, ci): its cost and d cost / d(dbdx), d(dbdy)
template <typename T>
__device__ __forceinline__ void cell_regu(const AssimArgs<T>& a, int cj, int ci, T s_a, T s_b, double* cost,
                                          T* gdx, T* gdy) {
  const int nx = a.nx;
  auto fld = [&](int j, int i) -> T {
    const size_t o = (size_t)j * nx + i;
    return a.p.regularize_thk ? a.thk[o] : a.usurf[o] - a.thk[o];
  };
  const T f00 = fld(cj, ci), f01 = fld(cj, ci + 1), f10 = fld(cj + 1, ci), f11 = fld(cj + 1, ci + 1);
  const T dx = a.dx;
  const T dbdx = ((f01 - f00) / dx + (f11 - f10) / dx) / T(2);
  const T dbdy = ((f10 - f00) / dx + (f11 - f01) / dx) / T(2);
  const size_t c = (size_t)cj * (nx - 1) + ci;
  const T fx = a.fdx[c], fy = a.fdy[c];
  const T A = dbdx * fx + dbdy * fy, Bv = dbdx * fy - dbdy * fx;
  const T w = (T)a.p.regu_thk;
  if (cost) *cost = (double)w * ((double)s_a * (double)A * (double)A / 2.0 + (double)s_b * (double)Bv * (double)Bv / 2.0);
  *gdx = w * (s_a * A * fx + s_b * Bv * fy);
  *gdy = w * (s_a * A * fy - s_b * Bv * fx);
}

template <typename T>
__global__ void __launch_bounds__(256) assim_cost_grad_kernel(const AssimArgs<T> a) {
  const int ny = a.ny, nx = a.nx;
  const size_t n = (size_t)ny * nx;
  const auto& p = a.p;
  const T inv_n = T(1) / (T)n;
  const T s_a = (T)(1.0 / sqrt(p.aniso_factor)), s_b = (T)sqrt(p.aniso_factor);
  double acc[kNCost] = {0, 0, 0, 0, 0};
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(o / nx), i = (int)(o - (size_t)j * nx);
    const T th = a.thk[o];
    // surface-velocity misfit (misfit_velsurf.py:8-19): components with an observation,
    // at nodes whose observed speed reaches the threshold
    const T uo = a.uobs[o], vo = a.vobs[o];
    const T nrm = sqrt(uo * uo + vo * vo);
    const bool rel = nrm >= (T)p.velsurfobs_thr;  // false when either component is NaN
    const T sv = (T)p.velsurfobs_std;
    T gu = T(0), gv = T(0);
    if (rel && !isnan(uo)) {
      const T r = (uo - a.uvs[o]) / sv;
      acc[kCVel] += 0.5 * (double)r * (double)r / p.n_vel;
      gu = -r / sv / (T)p.n_vel;
    }
    if (rel && !isnan(vo)) {
      const T r = (vo - a.vvs[o]) / sv;
      acc[kCVel] += 0.5 * (double)r * (double)r / p.n_vel;
      gv = -r / sv / (T)p.n_vel;
    }
    // the emulated surface velocities are where(thk > 0, U, 0): no gradient off the ice
    if (p.mask_velsurf && !(th > T(0))) {
      gu = T(0);
      gv = T(0);
    }
    a.g_u[o] = gu;
    a.g_v[o] = gv;
    T g = T(0);
    // thickness misfit (misfit_thk.py:8-16)
    const T to = a.thkobs[o];
    if (!isnan(to)) {
      const T st = (T)p.thkobs_std;
      const T r = (to - th) / st;
      acc[kCThk] += 0.5 * (double)a.dens[o] * (double)r * (double)r / p.n_thk;
      g += -a.dens[o] * r / st / (T)p.n_thk;
    }
    // penalties (total_cost.py:36-46)
    if (p.penalty) {
      if (p.icemask_cost && !(a.icemaskobs[o] > T(0.5))) {
        acc[kCIce] += 1e10 * (double)th * (double)th / (double)n;
        g += T(2e10) * th * inv_n;
      }
      if (!(th >= T(0))) {
        acc[kCPos] += 1e10 * (double)th * (double)th / (double)n;
        g += T(2e10) * th * inv_n;
      }
    }
    // regularisation (regu_thk.py:8-70): convexity term, then the smoothness terms
    acc[kCReg] -= p.regu_thk * p.gamma * (double)th;
    T gf = T(0);  // d cost / d field at this node
    const T dx = a.dx, inv2dx = T(0.5) / dx;
    if (p.aniso_factor != 1.0) {
      // the four cells around the node; the cost of cell (j, i) is counted at this node
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int di = 0; di < 2; ++di) {
          const int cj = j - 1 + dj, ci = i - 1 + di;
          if (cj < 0 || ci < 0 || cj >= ny - 1 || ci >= nx - 1) continue;
          double cc = 0.0;
          T gdx, gdy;
          cell_regu(a, cj, ci, s_a, s_b, (dj == 1 && di == 1) ? &cc : nullptr, &gdx, &gdy);
          acc[kCReg] += cc;
          // this node is corner (1 - dj, 1 - di) of the cell
          gf += gdx * ((di == 0) ? inv2dx : -inv2dx) + gdy * ((dj == 0) ? inv2dx : -inv2dx);
        }
    } else {
      auto fld = [&](int jj, int ii) -> T {
        const size_t q = (size_t)jj * nx + ii;
        return p.regularize_thk ? a.thk[q] : a.usurf[q] - a.thk[q];
      };
      const T w = (T)p.regu_thk, fc = fld(j, i);
      if (i + 1 < nx) {
        const T d = (fld(j, i + 1) - fc) / dx;
        acc[kCReg] += (double)w * (double)d * (double)d / 2.0;
        gf += -w * d / dx;
      }
      if (i >= 1) gf += w * ((fc - fld(j, i - 1)) / dx) / dx;
      if (j + 1 < ny) {
        const T d = (fld(j + 1, i) - fc) / dx;
        acc[kCReg] += (double)w * (double)d * (double)d / 2.0;
        gf += -w * d / dx;
      }
      if (j >= 1) gf += w * ((fc - fld(j - 1, i)) / dx) / dx;
    }
    g += (p.regularize_thk ? gf : -gf) - (T)(p.regu_thk * p.gamma);
    a.g_thk[o] = g;
  }
  // deterministic block reduction: fixed xor trees, warps in order
  __shared__ double red[8][kNCost];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < kNCost; ++c) {
    double v = acc[c];
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNCost) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    a.partials[(size_t)blockIdx.x * kNCost + threadIdx.x] = v;
  }
}

__global__ void assim_sum_kernel(const double* partials, int n_parts, double* costs) {
  const int c = threadIdx.x;
  if (c >= kNCost) return;
  double v = 0.0;
  for (int b = 0; b < n_parts; ++b) v += partials[(size_t)b * kNCost + c];
  costs[c] = v;
}

// ---- flow direction (utils.py:86-110) --------------------------------------
// cell averages of the surface velocity (NaN as 0)
template <typename T>
__global__ void flow_avg_kernel(int ny, int nx, const T* u, const T* v, T* fx, T* fy) {
  const int cy = ny - 1, cx = nx - 1;
  const size_t n = (size_t)cy * cx;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(o / cx), i = (int)(o - (size_t)j * cx);
    auto z = [](T x) { return isnan(x) ? T(0) : x; };
    const size_t a = (size_t)j * nx + i;
    fx[o] = (((z(u[a + nx + 1]) + z(u[a + 1])) + z(u[a + nx])) + z(u[a])) / T(4);
    fy[o] = (((z(v[a + nx + 1]) + z(v[a + 1])) + z(v[a + nx])) + z(v[a])) / T(4);
  }
}

// one pass of the separable Gaussian (zero outside), along y (axis 0) or x (axis 1),
// accumulated in double and stored in T as each pass of scipy's gaussian_filter
constexpr int kGaussR = 12;  // int(4 sigma + 0.5), sigma = 3
struct GaussW { double w[2 * kGaussR + 1]; };

template <typename T>
__global__ void gauss_pass_kernel(int ny, int nx, int axis, GaussW g, const T* in, T* out) {
  const size_t n = (size_t)ny * nx;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(o / nx), i = (int)(o - (size_t)j * nx);
    double s = 0.0;
    for (int k = -kGaussR; k <= kGaussR; ++k) {
      const int jj = axis == 0 ? j + k : j, ii = axis == 0 ? i : i + k;
      if (jj < 0 || jj >= ny || ii < 0 || ii >= nx) continue;
      s += g.w[k + kGaussR] * (double)in[(size_t)jj * nx + ii];
    }
    out[o] = (T)s;
  }
}

// normalisation, the y component with the already normalised x, as the reference
template <typename T>
__global__ void flow_norm_kernel(size_t n, T* fx, T* fy) {
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    T x = fx[o], y = fy[o];
    x = x / sqrt(x * x + y * y);
    y = y / sqrt(x * x + y * y);
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
static int cost_grad_t(int ny, int nx, double dx, const void* thk, const void* usurf, const void* uvs,
                       const void* vvs, const void* uobs, const void* vobs, const void* thkobs, const void* dens,
                       const void* icemaskobs, const void* fdx, const void* fdy, const igm_assim_params* p,
                       void* g_thk, void* g_u, void* g_v, double* partials, int n_parts, double* costs,
                       cudaStream_t st) {
  AssimArgs<T> a{};
  a.ny = ny; a.nx = nx; a.dx = (T)dx;
  a.thk = (const T*)thk; a.usurf = (const T*)usurf; a.uvs = (const T*)uvs; a.vvs = (const T*)vvs;
  a.uobs = (const T*)uobs; a.vobs = (const T*)vobs; a.thkobs = (const T*)thkobs; a.dens = (const T*)dens;
  a.icemaskobs = (const T*)icemaskobs; a.fdx = (const T*)fdx; a.fdy = (const T*)fdy;
  a.p = *p;
  a.g_thk = (T*)g_thk; a.g_u = (T*)g_u; a.g_v = (T*)g_v;
  a.partials = partials;
  int grid = grid_n((size_t)ny * nx);
  if (grid > n_parts) grid = n_parts;
  assim_cost_grad_kernel<T><<<grid, 256, 0, st>>>(a);
  int rc = launch_status("assim_cost_grad_kernel");
  if (rc) return rc;
  assim_sum_kernel<<<1, 32, 0, st>>>(partials, grid, costs);
  return launch_status("assim_sum_kernel");
}

template <typename T>
static int flow_t(int ny, int nx, const void* u, const void* v, void* fx, void* fy, void* scratch, cudaStream_t st) {
  const int cy = ny - 1, cx = nx - 1;
  const size_t n = (size_t)cy * cx;
  T* X = (T*)fx;
  T* Y = (T*)fy;
  T* S = (T*)scratch;
  flow_avg_kernel<T><<<grid_n(n), 256, 0, st>>>(ny, nx, (const T*)u, (const T*)v, X, Y);
  int rc = launch_status("flow_avg_kernel");
  if (rc) return rc;
  GaussW g{};
  double sum = 0.0;
  for (int k = -kGaussR; k <= kGaussR; ++k) sum += (g.w[k + kGaussR] = exp(-0.5 * k * k / 9.0));
  for (int k = 0; k < 2 * kGaussR + 1; ++k) g.w[k] /= sum;
  for (T* f : {X, Y}) {
    gauss_pass_kernel<T><<<grid_n(n), 256, 0, st>>>(cy, cx, 0, g, f, S);
    if ((rc = launch_status("gauss_pass_kernel"))) return rc;
    gauss_pass_kernel<T><<<grid_n(n), 256, 0, st>>>(cy, cx, 1, g, S, f);
    if ((rc = launch_status("gauss_pass_kernel"))) return rc;
  }
  flow_norm_kernel<T><<<grid_n(n), 256, 0, st>>>(n, X, Y);
  return launch_status("flow_norm_kernel");
}

// Control update of optimize_update (optimize/update.py:23-27, 38-42,
// 56-68, 77-98) for control thk with scaling sc, at the three points where
// the reference touches the control:
//   mode 0, before the forward: the optimizer's variable thk / sc, then
//     thk = variable * sc, and zero moments (the reference wraps the control
//     in a new tf.Variable at every iteration, so Adam's slots are new);
//   mode 1, the gradient: sc (dC/dthk direct + through the emulator) where
//     icemaskobs > 0.5, zero elsewhere;
//   mode 2, after the step: thk = variable * sc, then the reprojection onto
//     the ice mask and thk >= 0.
template <typename T>
__global__ void assim_control_kernel(size_t n, int mode, T sc, int reproject_mask, int reproject_pos, T* thk,
                                     const T* g_direct, const float* g_emul, const T* icemaskobs, float* var,
                                     float* grad, float* m, float* v) {
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    if (mode == 0) {
      const float x = (float)(thk[o] / sc);
      var[o] = x;
      thk[o] = (T)x * sc;
      m[o] = 0.f;
      v[o] = 0.f;
    } else if (mode == 1) {
      const T g = g_direct[o] + (g_emul ? (T)g_emul[o] : T(0));
      grad[o] = icemaskobs[o] > T(0.5) ? (float)(g * sc) : 0.f;
    } else {
      T t = (T)var[o] * sc;
      if (reproject_mask && !(icemaskobs[o] > T(0.5))) t = T(0);
      if (reproject_pos && t < T(0)) t = T(0);
      thk[o] = t;
    }
  }
}

}  // namespace igm

using namespace igm;

extern "C" int igm_assim_cost_grad(int dtype, int ny, int nx, double dx, const void* thk, const void* usurf,
                                   const void* uvelsurf, const void* vvelsurf, const void* uvelsurfobs,
                                   const void* vvelsurfobs, const void* thkobs, const void* dens_thkobs,
                                   const void* icemaskobs, const void* flowdirx, const void* flowdiry,
                                   const igm_assim_params* params, void* grad_thk, void* grad_uvelsurf,
                                   void* grad_vvelsurf, double* partials, int n_parts, double* costs, void* stream) {
  IGM_CHECK_ARG(ny >= 2 && nx >= 2, IGM_ERR_BAD_SHAPE, "igm_assim_cost_grad: bad shape %dx%d", ny, nx);
  IGM_CHECK_ARG(thk && usurf && uvelsurf && vvelsurf && uvelsurfobs && vvelsurfobs && thkobs && dens_thkobs &&
                    icemaskobs && params && grad_thk && grad_uvelsurf && grad_vvelsurf && partials && costs,
                IGM_ERR_BAD_ARGUMENT, "igm_assim_cost_grad: NULL argument");
  IGM_CHECK_ARG(params->aniso_factor == 1.0 || (flowdirx && flowdiry), IGM_ERR_BAD_ARGUMENT,
                "igm_assim_cost_grad: the anisotropic regularisation needs flowdirx, flowdiry");
  IGM_CHECK_ARG(params->aniso_factor > 0 && params->n_vel >= 1 && params->n_thk >= 1 && n_parts >= 1 && dx > 0,
                IGM_ERR_BAD_ARGUMENT, "igm_assim_cost_grad: bad parameter");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    return cost_grad_t<float>(ny, nx, dx, thk, usurf, uvelsurf, vvelsurf, uvelsurfobs, vvelsurfobs, thkobs,
                              dens_thkobs, icemaskobs, flowdirx, flowdiry, params, grad_thk, grad_uvelsurf,
                              grad_vvelsurf, partials, n_parts, costs, st);
  if (dtype == IGM_F64)
    return cost_grad_t<double>(ny, nx, dx, thk, usurf, uvelsurf, vvelsurf, uvelsurfobs, vvelsurfobs, thkobs,
                               dens_thkobs, icemaskobs, flowdirx, flowdiry, params, grad_thk, grad_uvelsurf,
                               grad_vvelsurf, partials, n_parts, costs, st);
  set_error("igm_assim_cost_grad: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_assim_flow_direction(int dtype, int ny, int nx, const void* uvelsurf, const void* vvelsurf,
                                        void* flowdirx, void* flowdiry, void* scratch, void* stream) {
  IGM_CHECK_ARG(ny >= 2 && nx >= 2, IGM_ERR_BAD_SHAPE, "igm_assim_flow_direction: bad shape %dx%d", ny, nx);
  IGM_CHECK_ARG(uvelsurf && vvelsurf && flowdirx && flowdiry && scratch, IGM_ERR_BAD_ARGUMENT,
                "igm_assim_flow_direction: NULL argument");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32) return flow_t<float>(ny, nx, uvelsurf, vvelsurf, flowdirx, flowdiry, scratch, st);
  if (dtype == IGM_F64) return flow_t<double>(ny, nx, uvelsurf, vvelsurf, flowdirx, flowdiry, scratch, st);
  set_error("igm_assim_flow_direction: unknown dtype %d", dtype);
  return IGM_ERR_BAD_ARGUMENT;
}

extern "C" int igm_assim_control(int dtype, int mode, size_t n, double scale, int reproject_mask, int reproject_pos,
                                 void* thk, const void* grad_direct, const float* grad_emulator, const void* icemaskobs,
                                 float* variable, float* grad, float* m, float* v, void* stream) {
  IGM_CHECK_ARG(mode >= 0 && mode <= 2 && n >= 1 && scale > 0, IGM_ERR_BAD_ARGUMENT,
                "igm_assim_control: bad mode, size or scale");
  IGM_CHECK_ARG(thk && (mode != 0 || (variable && m && v)) && (mode != 1 || (grad_direct && icemaskobs && grad)) &&
                    (mode != 2 || (variable && (icemaskobs || !reproject_mask))),
                IGM_ERR_BAD_ARGUMENT, "igm_assim_control: NULL argument");
  cudaStream_t st = as_stream(stream);
  if (dtype == IGM_F32)
    assim_control_kernel<float><<<grid_n(n), 256, 0, st>>>(n, mode, (float)scale, reproject_mask, reproject_pos,
                                                           (float*)thk, (const float*)grad_direct,
                                                           grad_emulator, (const float*)icemaskobs,
                                                           variable, grad, m, v);
  else if (dtype == IGM_F64)
    assim_control_kernel<double><<<grid_n(n), 256, 0, st>>>(n, mode, scale, reproject_mask, reproject_pos,
                                                            (double*)thk, (const double*)grad_direct,
                                                            grad_emulator, (const double*)icemaskobs,
                                                            variable, grad, m, v);
  else {
    set_error("igm_assim_control: unknown dtype %d", dtype);
    return IGM_ERR_BAD_ARGUMENT;
  }
  return launch_status("assim_control_kernel");
}
