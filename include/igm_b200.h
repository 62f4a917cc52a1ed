/*
 * igm_b200.h - C ABI of libigmb200.so, the B200 (sm_100a) implementation of
 * IGM's iceflow process and the thk transport step it drives.
 *
 * Conventions
 *  - Every entry point returns an int status (igm_status); 0 is success.
 *    igm_status_string() names a code, igm_last_error() returns the detail
 *    of the most recent failure on the calling thread.
 *  - All array arguments are DEVICE pointers (cudaMalloc'd or torch CUDA
 *    storage) unless the comment says "host".  `stream` is a cudaStream_t
 *    passed as void* (NULL = legacy default stream).  Every call is
 *    asynchronous with respect to the host.
 *  - dtype selects the arithmetic: IGM_F32 (the product path) or IGM_F64
 *    (the double-precision judge used to measure the FP32 error).
 *  - 2-D fields are [batch][ny][nx], 3-D velocity fields are
 *    [batch][nz][ny][nx], C order (x fastest), as the reference stores
 *    state.U (igm/processes/iceflow/utils.py:31-32).
 *  - Scratch: calls that reduce over the grid take a caller-owned
 *    workspace of igm_workspace_size() bytes.  It must be zero-filled once
 *    before its first use; every kernel leaves it zeroed again.  Calls that
 *    share one workspace must be ordered (same stream).
 *
 * Reference paths below are relative to the IGM 3.0.0 source tree.
 */
#ifndef IGM_B200_H
#define IGM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define IGM_API __attribute__((visibility("default")))
#else
#define IGM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define IGM_MAX_NZ 64
#define IGM_MAX_WINDOWS 64 /* patches per emulator batch */
#define IGM_MAX_VARS 80    /* trainable tensors handled by one Adam call */

typedef enum igm_status {
  IGM_OK = 0,
  IGM_ERR_BAD_SHAPE = 1,
  IGM_ERR_BAD_ARGUMENT = 2,
  IGM_ERR_NAN_DETECTED = 3,
  IGM_ERR_NOT_CONVERGED = 4,
  IGM_ERR_CUDA = 5,
  IGM_ERR_UNSUPPORTED = 6,
  IGM_ERR_WORKSPACE = 7
} igm_status;

typedef enum igm_dtype { IGM_F32 = 0, IGM_F64 = 1 } igm_dtype;

typedef enum igm_slope_type { IGM_GODUNOV = 0, IGM_MINMOD = 1, IGM_SUPERBEE = 2 } igm_slope_type;
typedef enum igm_divflux_method { IGM_DIVFLUX_UPWIND = 0, IGM_DIVFLUX_CENTERED = 1 } igm_divflux_method;

typedef enum igm_conv_mode {
  IGM_CONV_FWD_LEAKY = 0, /* y = LeakyReLU(conv3x3(x) + bias) */
  IGM_CONV_DGRAD = 1      /* y = conv3x3_flipped(x) * LeakyReLU'(act_mask) (+ bias-gradient partials) */
} igm_conv_mode;

/* cfg.processes.iceflow.physics.* (igm/conf/processes/iceflow.yaml:4-21) */
typedef struct igm_physics {
  double exp_glen;       /* n */
  double exp_weertman;   /* m */
  double regu_glen;
  double regu_weertman;
  double thr_ice_thk;
  double min_sr;
  double max_sr;
  double ice_density;
  double gravity_cst;
  int32_t force_negative_gravitational_energy;
  int32_t reserved;
} igm_physics;

/* Grid and vertical discretisation.  dzeta[0..nz-2] are the layer weights of
 * compute_zeta_dzeta (igm/processes/iceflow/vert_disc.py:27-35); with nz == 1
 * dzeta[0] = 1.  dx is the uniform spacing dX (m). */
typedef struct igm_grid {
  int32_t batch;
  int32_t nz;
  int32_t ny;
  int32_t nx;
  double dx;
  double dzeta[IGM_MAX_NZ];
} igm_grid;

/* The 2-D inputs of the energy (cfg.processes.iceflow.emulator.fieldin minus
 * dX), each [batch][ny][nx] of the call's dtype. */
typedef struct igm_fields {
  const void* thk;
  const void* usurf;
  const void* arrhenius;
  const void* slidingco;
} igm_fields;

/* Keras legacy Adam hyper-parameters (solve.py:11-20 uses the defaults with
 * learning_rate = solver.step_size). */
typedef struct igm_adam {
  double lr;
  double beta_1;
  double beta_2;
  double epsilon;
} igm_adam;

/* EarlyStopping(relative_min_delta, patience) (iceflow/utils.py:80-110). */
typedef struct igm_early_stop {
  double relative_min_delta;
  int32_t patience;
  int32_t enabled;
} igm_early_stop;

/* Device-resident control block of one solve (caller allocates
 * sizeof(igm_solver_ctl) bytes of device memory).  Written by the kernels;
 * read back by the host once per solve. */
typedef struct igm_solver_ctl {
  int32_t iter;       /* iterations completed in this solve */
  int32_t stopped;    /* early stopping fired (or an error stopped the solve) */
  int32_t status;     /* IGM_OK or IGM_ERR_NAN_DETECTED */
  int32_t wait;       /* EarlyStopping.wait */
  int64_t adam_t0;    /* optimizer.iterations before this solve */
  double best;        /* EarlyStopping.best_loss */
  double last_cost;   /* COST of the last completed iteration */
  double terms[3];    /* its shear, sliding, gravity means */
} igm_solver_ctl;

IGM_API const char* igm_status_string(int status);
IGM_API const char* igm_last_error(void);
IGM_API int igm_version(void);
/* Number of kernels this library has launched in the process (all threads). */
IGM_API long long igm_launch_count(void);

/* Bytes of scratch the energy / solver / reduction calls need for this grid. */
IGM_API size_t igm_workspace_size(const igm_grid* grid);

/* ---------------------------------------------------------------------------
 * Blatter-Pattyn energy and its adjoint.
 * Replaces iceflow_energy (igm/processes/iceflow/energy/energy.py:12-22 with
 * cost_shear.py:55-209, cost_sliding_weertman.py:23-43, cost_gravity.py:24-69,
 * staggered grid, Lagrange basis) followed by the per-term reduce_mean of
 * solve.py:57-59, and its tf.GradientTape gradient (solve.py:77,
 * emulate.py:252).
 *   terms (device double[3]): sums over all staggered cells of all batch
 *     entries of the shear, sliding and gravity densities (MPa m/a); the
 *     reference's COST is (terms[0]+terms[1]+terms[2]) / (batch*(ny-1)*(nx-1)).
 *   dU, dV: NULL for the energy only; otherwise they receive
 *     grad_scale * d(sum of all densities)/d(U,V), same layout as U, V.
 * ------------------------------------------------------------------------- */
IGM_API int igm_energy(int dtype, const igm_grid* grid, const igm_physics* phys, const igm_fields* fields,
               const void* U, const void* V, void* dU, void* dV, double grad_scale, double* terms,
               void* workspace, size_t workspace_bytes, void* stream);

/* Same computation and results as igm_energy, for callers that cannot
 * allocate device memory: a host model that has already handed all device
 * memory to its own pool, or code that must not call cudaMalloc/cudaFree
 * because those calls may synchronise the device.  No counterpart in the
 * reference (its TensorFlow ops allocate their temporaries).
 *  - No workspace argument and no allocation: the reduction scratch is a fixed
 *    2 MiB array compiled into the library, held by every device that loads
 *    the library until the process exits.  A grid needing more scratch than
 *    that (roughly more than 87,000 CTAs of 31 x 7 nodes, e.g. 4096 x 4096 with
 *    batch 2) is rejected with IGM_ERR_WORKSPACE and no launch.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture.  The address is kept for the life of the
 *    process: the library does not survive a cudaDeviceReset (or a reset of
 *    the primary context) -- reload it after one.
 *  - All calls share the one array, which keeps the last call's contents;
 *    each call clears the counter it needs at zero on its stream.  Calls that
 *    overlap on the GPU (other streams, other host threads) race on the array:
 *    order them on one stream. */
IGM_API int igm_energy_noalloc(int dtype, const igm_grid* grid, const igm_physics* phys, const igm_fields* fields,
                               const void* U, const void* V, void* dU, void* dV, double grad_scale, double* terms,
                               void* stream);

/* ---------------------------------------------------------------------------
 * Plain solver: n_iterations fused iterations of
 *   COST, grad = energy_and_gradient(U, V); Adam.apply_gradients;
 *   EarlyStopping.should_stop(COST)
 * (igm/processes/iceflow/solve/solve.py:45-114), each ONE kernel: stencil
 * energy + adjoint + Adam + the FP64 reduction + the early-stopping update
 * on the device, no host synchronisation.  Iteration i reads (U0,V0) when
 * ctl->iter is even and (U1,V1) when odd, and writes the other pair; after
 * the solve the result is in pair (ctl->iter % 2).  Iterations after early
 * stopping (or after max_iter) return at once.  mU..vV are the Adam moments
 * (zero-filled by the caller at the start of a solve, as the reference's
 * fresh tf.Variables get fresh slots).  costs (device double[max_iter])
 * receives the COST history.
 * igm_solver_begin resets ctl for a new solve whose optimizer has already
 * taken adam_iterations steps (Keras' global optimizer.iterations).
 * ------------------------------------------------------------------------- */
IGM_API int igm_solver_begin(igm_solver_ctl* ctl, int64_t adam_iterations, void* stream);
IGM_API int igm_solver_iterate(int dtype, const igm_grid* grid, const igm_physics* phys, const igm_fields* fields,
                       void* U0, void* V0, void* U1, void* V1, void* mU, void* mV, void* vU, void* vV,
                       const igm_adam* adam, const igm_early_stop* early_stop, int n_iterations, int max_iter,
                       igm_solver_ctl* ctl, double* costs, void* workspace, size_t workspace_bytes,
                       void* stream);

/* ---------------------------------------------------------------------------
 * Velocity post-processing: optional mask U,V = where(thk > 0, U, 0)
 * (solve.py:116-117, emulate.py:143-144), then velbase = U[0],
 * velsurf = U[nz-1], velbar = sum_k U[k] * vert_weight[k]
 * (igm/processes/iceflow/utils.py:21-51) and, fused, the CFL maximum
 * max(max|ubar|, max|vbar|) of time.update (igm/processes/time/time.py:36-39).
 * vert_weight: host double[nz] (define_vertical_weight, vert_disc.py:43-47).
 * Any of the 2-D outputs and velomax (device float, overwritten) may be NULL.
 * ------------------------------------------------------------------------- */
IGM_API int igm_velocity_reduce(int dtype, int batch, int nz, int ny, int nx, void* U, void* V, const void* thk,
                        int mask, const double* vert_weight, void* ubar, void* vbar, void* uvelbase,
                        void* vvelbase, void* uvelsurf, void* vvelsurf, float* velomax, void* stream);

/* ---------------------------------------------------------------------------
 * Thickness transport step (igm/processes/thk/thk.py:27-54 with
 * compute_divflux_slope_limiter, igm/utils/gradient/
 * compute_divflux_slope_limiter.py:11-65):
 *   divflux = div(q) slope-limited upwind; thk_out = max(thk + dt (smb - divflux), 0);
 *   lsurf = max(topg, -ratio_density thk_out + sealevel); usurf = lsurf + thk_out.
 * smb may be NULL (zero, thk.py:41-42).  lsurf_out and divflux_out may be NULL.
 * dt is taken from dt_device (device float) when it is not NULL, else from dt.
 * thk_out must not alias thk_in.
 * ------------------------------------------------------------------------- */
IGM_API int igm_transport_step(int dtype, int ny, int nx, double dx, const void* ubar, const void* vbar,
                       const void* thk_in, void* thk_out, const void* topg, const void* smb, void* usurf_out,
                       void* lsurf_out, void* divflux_out, double dt, const float* dt_device, int slope_type,
                       double ratio_density, double sealevel, void* stream);

/* ---------------------------------------------------------------------------
 * Vertical velocity, vert_flow version 2, kinematic method (the vert_flow
 * process's default): replaces compute_vertical_velocity_kinematic_v2 /
 * compute_w_kinematic_tf (igm/processes/vert_flow/vert_flow_v2.py:17-37,
 * with compute_gradient_layers_tf :62-87, compute_divflux_layers :126-147 and
 * compute_dz, igm/processes/iceflow/vert_disc.py:17-23).  For each layer k,
 * z_k = sum_{l<k} thk (levels[l+1] - levels[l]), the layer surface topg + z_k,
 * its centred slopes (sx, sy) with extrapolated border faces, the running
 * weighted means ub_k = sum_{l<=k} w_l U_l / sum_{l<=k} w_l (and vb_k), and
 *   W_k = -(d(ub_k z_k)/dx + d(vb_k z_k)/dy) + U_k sx + V_k sy.
 * U, V, W: [nz][ny][nx]; topg, thk: [ny][nx]; levels, vert_weight: host
 * double[nz] (compute_levels and define_vertical_weight, vert_disc.py:10-13,
 * 43-47).  nz, ny, nx >= 2.  wvelbase and wvelsurf of the process are W_0 and
 * W_{nz-1} (vert_flow.py:55-56).  Bit-identical to the reference in FP32/FP64.
 * ------------------------------------------------------------------------- */
IGM_API int igm_vertical_velocity(int dtype, int nz, int ny, int nx, double dx, const void* U, const void* V,
                          const void* topg, const void* thk, const double* levels, const double* vert_weight,
                          void* W, void* stream);

/* Vertical velocity, vert_flow version 2, incompressibility method: replaces
 * compute_vertical_velocity_incompressibility_v2 (igm/processes/vert_flow/
 * vert_flow_v2.py:40-57, with gradx/grady_non_flat_layers_tf :168-199 and
 * compute_gradient_tf, igm/utils/gradient/compute_gradient_tf.py:6-35) for a
 * uniform spacing dX = dx.  With z_k = sum_{l<k} thk (levels[l+1] - levels[l])
 * and the layer surface Z_k = topg + z_k, the terrain-following derivatives
 *   du/dx_k = (dU_k/dx) - (dZ_k/dx) (U_{k+1/2} - U_{k-1/2}) / (vert_weight_k thk)
 * (layer faces U_{-1/2} = U_0, U_{Nz-1/2} = U_{Nz-1}, zero where thk = 0), the
 * same for dv/dy, and
 *   W_k = U_0 dtopg/dx + V_0 dtopg/dy - sum_{l<=k} (z_l - z_{l-1}) (du/dx + dv/dy)_l.
 * Arguments and layouts as igm_vertical_velocity.  Bit-identical to the
 * reference in FP32/FP64. */
IGM_API int igm_vertical_velocity_incompressibility(int dtype, int nz, int ny, int nx, double dx, const void* U,
                                            const void* V, const void* topg, const void* thk, const double* levels,
                                            const double* vert_weight, void* W, void* stream);

/* ---------------------------------------------------------------------------
 * Data assimilation (igm/processes/data_assimilation), default configuration:
 * control thk, costs velsurf + thk + icemask, penalty obstacle constraint,
 * thickness regularisation.
 * ------------------------------------------------------------------------- */
typedef struct igm_assim_params {
  double velsurfobs_std;   /* fitting.velsurfobs_std */
  double velsurfobs_thr;   /* fitting.velsurfobs_thr */
  double thkobs_std;       /* fitting.thkobs_std */
  double regu_thk;         /* regularization.thk */
  double gamma;            /* convexity_weight * areaicemask^(convexity_power - 2) */
  double aniso_factor;     /* regularization.smooth_anisotropy_factor (1: isotropic branch) */
  double n_vel;            /* number of observed velocity components used (the mean's count) */
  double n_thk;            /* number of thickness observations */
  int32_t penalty;         /* "penalty" in optimization.obstacle_constraint */
  int32_t icemask_cost;    /* "icemask" in cost_list */
  int32_t regularize_thk;  /* regularization.to_regularize == "thk" (else "topg": usurf - thk) */
  int32_t mask_velsurf;    /* the surface velocities are where(thk > 0, U, 0): no gradient off the ice */
  double usurfobs_std;     /* fitting.usurfobs_std (misfit_usurf) */
  double n_usurf;          /* number of nodes inside icemaskobs > 0.5 (misfit_usurf's count) */
  int32_t usurf_cost;      /* "usurf" in cost_list */
  int32_t no_thk_control;  /* thk not in control_list: no thk_positive penalty, no regu_thk */
  int32_t fix_normalization; /* optimization.fix_opti_normalization_issue: regularisation means, not sums */
  int32_t sole_mask;       /* optimization.sole_mask: regu_thk's differences only inside icemaskobs > 0.5 */
} igm_assim_params;

/* The cost terms of total_cost (cost_terms/total_cost.py:13-70) that depend
 * on thk and usurf -- misfit_velsurf.py:8-19, misfit_thk.py:8-16, the icemask
 * and positive-thickness penalties (:36-46), regu_thk.py:8-70 (with
 * fix_normalization: fix_opti_normalization_issue's means) and, with
 * usurf_cost, misfit_usurf.py:5-15
 * -- and their gradients w.r.t. thk, the emulated surface velocities
 * (uvelsurf, vvelsurf, zero where thk <= 0) and, when grad_usurf is given,
 * usurf (misfit_usurf and regu_thk's bed usurf - thk).  Observations are NaN
 * where missing; flowdirx/y [ny-1][nx-1] (anisotropic branch only, else NULL);
 * usurfobs only with usurf_cost.  costs (device double[6]): velsurf, thk,
 * icemask, thk_positive, thk_regu, usurf; partials: device double[n_parts * 6]
 * scratch.  All 2-D arrays [ny][nx] of the dtype. */
IGM_API int igm_assim_cost_grad(int dtype, int ny, int nx, double dx, const void* thk, const void* usurf,
                        const void* uvelsurf, const void* vvelsurf, const void* uvelsurfobs,
                        const void* vvelsurfobs, const void* thkobs, const void* dens_thkobs,
                        const void* icemaskobs, const void* flowdirx, const void* flowdiry, const void* usurfobs,
                        const igm_assim_params* params, void* grad_thk, void* grad_uvelsurf, void* grad_vvelsurf,
                        void* grad_usurf, double* partials, int n_parts, double* costs, void* stream);

/* The regularisation and positivity penalty of another control field:
 * regu_slidingco (cost_terms/regu_slidingco.py:8-52; isotropic, or anisotropic
 * with aniso_factor = smooth_anisotropy_factor_sl and the flow directions),
 * regu_arrhenius (cost_terms/regu_arrhenius.py:5-24; isotropic), both with
 * weight regu (fix_normalization: 0.5 regu times the means
 * of the squared differences instead of their half sums, as
 * fix_opti_normalization_issue), and with penalty the 1e10 mean(field^2
 * where field < penalty_threshold) of
 * total_cost.py:45-54 (threshold 0 for slidingco, 1 for arrhenius).  With
 * sole_mask (icemaskobs given) only the differences between two nodes with
 * icemaskobs == 1 (isotropic) or the cells whose four corners are > 0.5
 * (anisotropic) count, as regu_slidingco / regu_arrhenius mask them.  grad:
 * dC/dfield [ny][nx]; costs (device double[6], the layout of
 * igm_assim_cost_grad): [3] the penalty, [4] the regularisation, the others 0. */
IGM_API int igm_assim_field_regu(int dtype, int ny, int nx, double dx, const void* field, const void* flowdirx,
                                 const void* flowdiry, double regu, double aniso_factor, int penalty,
                                 double penalty_threshold, int fix_normalization, const void* icemaskobs,
                                 int sole_mask, void* grad, double* partials, int n_parts, double* costs,
                                 void* stream);

/* The control update of optimize_update (data_assimilation/optimize/update.py:
 * 22-42, 56-98) for one control x (thk, usurf, slidingco or arrhenius) with
 * scaling `scale`, at the three points where the reference touches it:
 *   mode 0 (before the emulator forward): variable = x / scale (transform 1,
 *     fitting.log_slidingco: sqrt(x / scale)), then x from the variable, and
 *     m = v = 0 (the reference re-creates the control tf.Variable at every
 *     iteration, so its Adam slots start at zero);
 *   mode 1 (the gradient): grad = dx/dvariable (grad_direct + grad_emulator),
 *     zero where the mask is off (mask 1: icemaskobs > 0.5, as for thk, usurf
 *     and arrhenius; 2: icemaskobs == 1, slidingco with sole_mask; 0: none);
 *   mode 2 (after igm_adam_clipnorm): x from the variable, then the
 *     reprojection (reproject 1, thk: 0 outside icemaskobs > 0.5 when
 *     reproject_mask, then x >= 0; 2: x >= lower, 0 for slidingco, 1 for
 *     arrhenius; 0: none);
 *   mode 3 (after mode 2, for a thk that is not a control): x = 0 outside
 *     icemaskobs > 0.5 -- the reference's reprojection applies this whenever
 *     "reproject" is an obstacle constraint and "icemask" is in cost_list
 *     (optimize/update.py:84-88); reads only x and icemaskobs.
 * variable, grad, m, v and grad_emulator (the emulator's input-field gradient,
 * igm_cnn_input_gradient) are device float[n], x, grad_direct and icemaskobs
 * [n] of the dtype; grad_emulator may be NULL; arguments a mode does not read
 * may be NULL. */
typedef struct igm_assim_control_params {
  int32_t mode;            /* 0, 1, 2, 3 as above */
  int32_t transform;       /* 0: x = variable scale; 1: x = variable^2 scale */
  int32_t mask;            /* 0 none, 1 icemaskobs > 0.5, 2 icemaskobs == 1 */
  int32_t reproject;       /* 0 none, 1 thk, 2 lower bound */
  int32_t reproject_mask;  /* reproject 1: zero outside the mask ("icemask" in cost_list) */
  int32_t reserved;
  double scale;            /* scaling.<control> */
  double lower;            /* reproject 2 */
} igm_assim_control_params;
IGM_API int igm_assim_control(int dtype, size_t n, const igm_assim_control_params* params, void* x,
                              const void* grad_direct, const float* grad_emulator, const void* icemaskobs,
                              float* variable, float* grad, float* m, float* v, void* stream);

/* compute_rms_std_optimization (data_assimilation/utils.py:10-66): out
 * (device double[9]) = rmsthk, stdthk, rmsvel, stdvel, rmsdiv, stddiv,
 * rmsusurf, stdusurf, vol -- the mean and population standard deviation of
 * thk - thkobs at the thickness observations, of |velsurf| - |velsurfobs|
 * inside icemaskobs > 0.5 where the observed speed is defined, of divfluxobs -
 * divflux and usurf - usurfobs inside the mask, and sum(thk) dx^2 / 1e9.  An
 * observation field passed as NULL gives 0 for its pair (the reference's
 * "no such observation"); an empty selection gives NaN (numpy's mean of an
 * empty array), except thk, which the reference records as 0.
 * partials: device double[n_parts * 13] scratch. */
IGM_API int igm_assim_stats(int dtype, int ny, int nx, double dx, const void* thk, const void* thkobs,
                            const void* uvelsurf, const void* vvelsurf, const void* uvelsurfobs,
                            const void* vvelsurfobs, const void* icemaskobs, const void* divflux,
                            const void* divfluxobs, const void* usurf, const void* usurfobs, double* partials,
                            int n_parts, double* out, void* stream);

/* include_low_speed_term of misfit_velsurf (cost_terms/misfit_velsurf.py:
 * 21-28): adds 0.5 100 log((|vs| + 1) / (|obs| + 1))^2 to *cost (device
 * double: the velsurf entry of igm_assim_cost_grad's costs) and its gradient
 * to grad_uvelsurf / grad_vvelsurf, where |.| is the norm of all components
 * with an observation (the reference's velsurf[ACT] is a 1-D selection; no
 * speed threshold here).  partials: device double[3 n_parts + 1] scratch. */
IGM_API int igm_assim_low_speed(int dtype, int ny, int nx, const void* uvelsurf, const void* vvelsurf,
                                const void* uvelsurfobs, const void* vvelsurfobs, void* grad_uvelsurf,
                                void* grad_vvelsurf, double* partials, int n_parts, double* cost, void* stream);

/* Parameters of the flux-divergence cost terms. */
typedef struct igm_divflux_cost_params {
  int32_t kind;            /* 0: cost_divfluxobs, 1: cost_divfluxfcz */
  int32_t method;          /* igm_divflux_method: divflux.method */
  int32_t force_zero_sum;  /* divflux.force_zero_sum */
  int32_t reserved;
  double divfluxobs_std;   /* fitting.divfluxobs_std */
  double regu_divflux;     /* regularization.divflux (kind 0: weight of the smoothness of divflux) */
  double slope, intercept; /* kind 1: the regression of divflux on usurf (a constant of the gradient) */
} igm_divflux_cost_params;

/* The flux-divergence cost terms of data assimilation and their gradient:
 * cost_divfluxobs (cost_terms/cost_divfluxobs.py:9-29): 0.5 mean over the
 * observed nodes of ((divfluxobs - D) / std)^2 + regu 0.5 (mean (dD/dx)^2 +
 * mean (dD/dy)^2); cost_divfluxfcz (cost_terms/cost_divfluxfcz.py:10-38): the
 * target intercept + slope usurf inside icemaskobs > 0.5, 0.5 mean over the
 * mask of ((target - D) / std)^2; both + 0.5 1000 mean_mask(D / std)^2 with
 * force_zero_sum.  divflux = D = igm_divflux(ubar, vbar, thk) of the same
 * method.  Writes *cost (device double) and the gradient: grad_thk[n] +=
 * dC/dthk (through the flux's thickness), dU, dV [nz][ny][nx] = vert_weight[k]
 * dC/dubar (velbar = sum_k vert_weight[k] U_k), zero where mask_thk <= 0
 * (NULL: no mask), ADDED to the top level nz - 1 (which holds dC/dvelsurf of
 * igm_assim_cost_grad) and assigned to the others.  vert_weight: host
 * double[nz]; scratch: device [n] of the dtype; partials: device
 * double[igm_assim_divflux_partials_len(n_parts)]. */
IGM_API int igm_assim_divflux_cost_grad(int dtype, int ny, int nx, double dx, int nz, const double* vert_weight,
                                        const void* ubar, const void* vbar, const void* thk, const void* divflux,
                                        const void* divfluxobs, const void* usurf, const void* icemaskobs,
                                        const void* mask_thk, const igm_divflux_cost_params* params,
                                        void* grad_thk, void* dU, void* dV, void* scratch, double* partials,
                                        int n_parts, double* cost, void* stream);
IGM_API size_t igm_assim_divflux_partials_len(int n_parts);

/* compute_flow_direction_for_anisotropic_smoothing (data_assimilation/utils.py:
 * 86-110): cell averages of the surface velocity (NaN as 0), a Gaussian of
 * sigma 3 cells (radius 12, zero outside; y then x, as scipy.ndimage), then
 * x /= |(x, y)|, y /= |(x_normalised, y)|, NaN as 0, in one tiled kernel.
 * Outputs [ny-1][nx-1]; scratch is not used (kept for callers that pass it). */
IGM_API int igm_assim_flow_direction(int dtype, int ny, int nx, const void* uvelsurf, const void* vvelsurf,
                             void* flowdirx, void* flowdiry, void* scratch, void* stream);

/* compute_divflux (igm/utils/gradient/compute_divflux.py:6-51), as data
 * assimilation computes state.divflux after each update and in its
 * flux-divergence costs: method IGM_DIVFLUX_UPWIND (face velocities with edge
 * copies at the border, upwind thickness, zero outside) or
 * IGM_DIVFLUX_CENTERED (face averages of u h, edge copies), then
 * d(u h)/dx + d(v h)/dy.  Bit-identical to the reference in FP32/FP64.
 * igm_divflux_upwind is igm_divflux with IGM_DIVFLUX_UPWIND. */
IGM_API int igm_divflux(int dtype, int method, int ny, int nx, double dx, const void* u, const void* v, const void* h,
                        void* out, void* stream);
IGM_API int igm_divflux_upwind(int dtype, int ny, int nx, double dx, const void* u, const void* v, const void* h,
                       void* out, void* stream);

/* Surfaces from thickness (thk.py:11-24): lsurf = max(topg, -r thk + sealevel),
 * usurf = lsurf + thk.  lsurf may be NULL. */
IGM_API int igm_thk_surfaces(int dtype, int n, const void* thk, const void* topg, void* lsurf, void* usurf,
                     double ratio_density, double sealevel, void* stream);

/* ELA mass balance (igm/processes/smb_simple/smb_simple.py:39-46):
 * smb = clip((usurf - ela) * (usurf < ela ? gradabl : gradacc), -100, maxacc),
 * then, when icemask is not NULL, smb = (smb < 0 || icemask > 0.5) ? smb : -10. */
IGM_API int igm_smb_simple(int dtype, int n, const void* usurf, const void* icemask, void* smb, double gradabl,
                   double gradacc, double ela, double maxacc, void* stream);

/* max(max|a|, max|b|) over n elements into the device float *out
 * (time.py:36-39 when ubar/vbar did not come from igm_velocity_reduce). */
IGM_API int igm_absmax2(int dtype, int n, const void* a, const void* b, float* out, void* stream);

/* force_max_velbar (igm/processes/iceflow/utils.py:182-194, Lagrange basis;
 * applied by emulate.py:147-148 and solve.py:178-179 when the option is > 0):
 * in place over n nodes of U and V ([nz, ny, nx] flattened), where
 * mag = sqrt(U^2 + V^2) >= cap: U = cap (U / mag), V = cap (V / mag).
 * Bit-identical to the reference graph (no fused multiply-add, IEEE division
 * and square root). */
IGM_API int igm_force_max_velbar(int dtype, size_t n, void* U, void* V, double cap, void* stream);

/* CFL step on the device (time.py:36-50, without the save-time snapping):
 * dt_out = velomax > 0 ? min(cfl dx / velomax, step_max) : step_max. */
IGM_API int igm_cfl_dt(const float* velomax, float* dt_out, double cfl, double dx, double step_max, void* stream);

/* ===========================================================================
 * CNN emulator (igm/processes/iceflow/emulate/neural_network.py:9-66:
 * nb_layers x [Conv2D 3x3 "same", 32 filters, bias, LeakyReLU(alpha)] and a
 * 1x1 Conv2D head to 2 Nz outputs), BF16 tensor-core convolutions with FP32
 * accumulation.
 *
 * Activations use the row-chunked layout bf16 [batch][H][C/8][W][8]
 * ("channels in groups of 8, innermost"); the input tensor has C = 16 (the
 * fieldin channels, zero-padded), hidden activations C = 32.
 * Parameters are one fp32 vector in Keras order: per 3x3 layer the kernel
 * [3][3][cin][32] then the bias [32]; then the head kernel [32][nout] and bias
 * [nout] (igm_cnn_param_offset gives each offset).
 * ========================================================================= */

/* 3x3 convolution on the tensor cores.  cin = 16 or 32 (C of x); 32 outputs.
 *  IGM_CONV_FWD_LEAKY: y = LeakyReLU_alpha(conv(x, wpack) + bias).
 *  IGM_CONV_DGRAD: x is the gradient w.r.t. a layer's pre-activation, wpack the
 *    layer's dgrad pack; y = (dL/d input of the layer) * (act_mask > 0 ? 1 : alpha),
 *    i.e. the gradient w.r.t. the previous layer's pre-activation.  When
 *    db_partials is not NULL it receives per-CTA sums of y over the pixels
 *    ([db_slots][32]; slots beyond the CTAs used are zeroed, so every slot is
 *    written and a fixed-order reduction over all db_slots needs no clearing).
 * err (device int, may be NULL) is set non-zero if a pipeline wait timed out. */
IGM_API int igm_conv3x3(int mode, int batch, int height, int width, int cin, const void* x, const void* wpack,
                        const float* bias, const void* act_mask, void* y, float* db_partials, int db_slots,
                        float alpha, int* err, void* stream);

/* Weight gradient of a 3x3 convolution: per-CTA partial sums of X^T G over all
 * pixels (G = gradient w.r.t. the pre-activation, 32 channels), laid out
 * partials[n_parts][3 (kw)][128 (r * cin + ci)][jn * 32 (jj * 32 + co)] with
 * jn = 2 for cin 32 and 4 for cin 16; entry (r, jj) belongs to kernel row
 * kh = r - jj.  Each part holds igm_conv3x3_wgrad_partial_len(cin) floats.
 * Reduce them with igm_cnn_wgrad_finish. */
IGM_API int igm_conv3x3_wgrad(int batch, int height, int width, int cin, const void* x, const void* g,
                              float* partials, int n_parts, int* err, void* stream);
IGM_API size_t igm_conv3x3_wgrad_partial_len(int cin);
/* The centre tap alone of igm_conv3x3_wgrad (cin 32): the partials of kw = 1 bit
 * for bit as igm_conv3x3_wgrad writes them (the weight gradient of the 1x1
 * head, igm_cnn_head_wgrad_finish), a third of the MMAs; the kw = 0, 2 slots of
 * the partial buffer hold no defined values. */
IGM_API int igm_conv1x1_wgrad(int batch, int height, int width, const void* x, const void* g, float* partials,
                              int n_parts, int* err, void* stream);
/* nlayers (1..16) forward 3x3 convolutions of 32 -> 32 channels in one launch,
 * as nlayers calls of igm_conv3x3(IGM_CONV_FWD_LEAKY) would compute them: layer
 * k reads x (k = 0) or outs[k-1] and writes outs[k] = LeakyReLU(conv(., wpacks[k])
 * + biases[k]); outs may alternate between two buffers (outs[k] == outs[k-2]).
 * The tiles of a layer start as soon as the tiles of the previous layer they
 * read are stored (a cooperative launch with per-tile flags).  flags: a device
 * int buffer of igm_conv3x3_stack_flags_len ints holding no value equal to
 * epoch (a zeroed buffer and a per-call counter from 1 serve).  outs, wpacks,
 * biases: host arrays of nlayers device pointers. */
IGM_API int igm_conv3x3_stack(int batch, int height, int width, int nlayers, const void* x, void* const* outs,
                              const void* const* wpacks, const float* const* biases, int* flags, int epoch,
                              float alpha, int* err, void* stream);
IGM_API size_t igm_conv3x3_stack_flags_len(int batch, int height, int width, int nlayers);
/* Both gradients of a 32 -> 32 channel layer in one pass over its inputs
 * (replaces igm_conv3x3(IGM_CONV_DGRAD) + igm_conv3x3_wgrad for the hidden
 * layers; the Keras GradientTape of emulate.py:252 through Conv2D(3x3) +
 * LeakyReLU): from g, the gradient w.r.t. the layer's pre-activation, the
 * layer's dgrad pack and x, the layer's input activation (which is also the
 * LeakyReLU mask of the data gradient):
 *   g_prev      = (dL/dx) * (x > 0 ? 1 : alpha), as IGM_CONV_DGRAD writes it;
 *   db_partials = per-CTA sums of g_prev over the pixels, [n_parts][32];
 *   w_partials  = the igm_conv3x3_wgrad(cin 32) partials of (x, g), [n_parts]
 *                 x igm_conv3x3_wgrad_partial_len(32) floats, for igm_cnn_wgrad_finish.
 * Every slot of both partial buffers is written.  err as for igm_conv3x3.
 * With prev_w_partials, prev_db_partials (the partial buffers of the previous
 * call, the layer above, n_parts parts each; not this call's buffers) the call
 * also finishes them: prev_w_out = igm_cnn_wgrad_finish(prev_w_partials, cin 32)
 * and prev_db_out = igm_reduce_partials(prev_db_partials, 32), bit for bit as
 * those calls compute them.  All four prev_* NULL: nothing is finished. */
IGM_API int igm_conv3x3_backward(int batch, int height, int width, const void* g, const void* wpack_bwd,
                                 const void* x, void* g_prev, float* db_partials, float* w_partials, int n_parts,
                                 float alpha, int* err, const float* prev_w_partials, const float* prev_db_partials,
                                 float* prev_w_out, float* prev_db_out, void* stream);
IGM_API int igm_conv_sm_count(void);

IGM_API size_t igm_cnn_param_count(int nb_layers, int cin, int nout);
IGM_API size_t igm_cnn_param_offset(int nb_layers, int cin, int nout, int layer, int bias);

/* fp32 parameters -> bf16 UMMA operand packs: wpack_fwd (layer 0: 9*2*32*8,
 * layers >= 1: 9*4*32*8 elements each), ordered [kw][ci/8][kh][co][ci%8], and
 * wpack_bwd (layers >= 1, flipped and transposed for dgrad, 9*4*32*8 each),
 * ordered [2-kw][co/8][2-kh][ci][co%8]. */
IGM_API int igm_cnn_pack_weights(int nb_layers, int cin, int nout, const float* params, void* wpack_fwd,
                                 void* wpack_bwd, void* stream);

/* Emulator input (fieldin_to_X, iceflow/utils.py:147-158, with split_into_patches
 * windows, emulate.py:283-308): X[b] = scaled (thk, usurf, arrhenius, slidingco, dx)
 * of the window at host (win_y0[b], win_x0[b]) of size h x w of the [ny][nx]
 * fields, and fp32 copies of the windowed fields ([batch][h][w], each may be
 * NULL).  X (may be NULL) is the row-chunked bf16 [batch][h][2][w][8] tensor of
 * the first layer: each scaled field x in three channels (x_h, x_l, x_h) with
 * x_h = bf16(x), x_l = bf16(x - x_h) -- with the layer-0 weight pack (W_h, W_h,
 * W_l) the tensor-core convolution then sums x_h W_h + x_l W_h + x_h W_l, about
 * 16 significant bits of x W, enough for the metre-scale steps of a ~3000 m
 * surface.  scales: host float[5]. */
IGM_API int igm_cnn_input(int batch, int h, int w, int ny, int nx, const float* thk, const float* usurf,
                          const float* arrhenius, const float* slidingco, double dx, const float* scales,
                          const int* win_y0, const int* win_x0, void* X, float* thk_out, float* usurf_out,
                          float* arrhenius_out, float* slidingco_out, void* stream);

/* First 3x3 layer in FP32 on CUDA cores, from the windowed FP32 fields
 * (thk, usurf, arrhenius, slidingco [batch][h][w]) and the constant dX
 * channel, scaled by host scales[5]: act = LeakyReLU(conv(X, w1) + b1), bf16
 * row-chunked with 32 channels.  w1 is the Keras kernel [3][3][cin][32].
 * BF16 inputs would lose the surface slope (metres on a ~3000 m surface). */
IGM_API int igm_cnn_layer1_forward(int batch, int h, int w, int cin, const float* thk, const float* usurf,
                                   const float* arrhenius, const float* slidingco, double dx, const float* scales,
                                   const float* w1, const float* b1, float alpha, void* act, void* stream);
/* Its weight gradient: per-block partials [n_parts][9 * cin * 32] of
 * X^T G (G = gradient w.r.t. the layer's pre-activation, bf16 row-chunked). */
IGM_API int igm_cnn_layer1_wgrad(int batch, int h, int w, int cin, const float* thk, const float* usurf,
                                 const float* arrhenius, const float* slidingco, double dx, const float* scales,
                                 const void* g, float* partials, int n_parts, void* stream);

/* 1x1 head: Y = out_scale (A Wh + bh); U[b][k] = Y[..., k], V[b][k] =
 * Y[..., nz + k] (Y_to_UV, iceflow/utils.py:133-139), planar fp32
 * [batch][nz][h][w]; zero where thk_mask <= 0 when thk_mask is not NULL
 * (emulate.py:143-144).  out_scale = 1 is the reference network. */
IGM_API int igm_cnn_head_forward(int batch, int h, int w, int nz, const void* act, const float* head_w,
                                 const float* head_b, float out_scale, float* U, float* V, const float* thk_mask,
                                 void* stream);

/* Backward of the head and of the last LeakyReLU: dpre (bf16 row-chunked) and
 * per-block partials [n_parts][igm_cnn_head_partial_len(nz)] = dWh [32][2nz],
 * dbh [2nz], db_last [32]. */
IGM_API size_t igm_cnn_head_partial_len(int nz);
IGM_API int igm_cnn_head_backward(int batch, int h, int w, int nz, const void* act, const float* head_w,
                                  const float* dU, const float* dV, float out_scale, float alpha, void* dpre,
                                  float* partials, int n_parts, void* stream);

/* Head backward for 2 nz <= 32 outputs, with its kernel gradient on the tensor
 * cores: writes dpre as igm_cnn_head_backward does, the output gradient
 * dY = out_scale * (dU, dV) as a row-chunked bf16 [batch][h][4][w][8] tensor
 * (dy_bf16; outputs beyond 2 nz zero) and per-CTA partials
 * [n_parts][2 nz + 32] of dbh and of the last conv layer's bias gradient.
 * The head kernel gradient is then igm_conv3x3_wgrad(act, dy_bf16) reduced by
 * igm_cnn_head_wgrad_finish.  With dy_bf16 and partials both NULL only dpre is
 * written (the data gradient, as the input-field gradient of data
 * assimilation needs). */
IGM_API int igm_cnn_head_backward_tc(int batch, int h, int w, int nz, const void* act, const float* head_w,
                                     const float* dU, const float* dV, float out_scale, float alpha, void* dpre,
                                     void* dy_bf16, float* partials, int n_parts, void* stream);
/* igm_conv3x3_wgrad partials over (act, dy_bf16) -> head kernel gradient [32][nout]
 * (the centre tap), nout <= 32. */
IGM_API int igm_cnn_head_wgrad_finish(const float* partials, int n_parts, int nout, float* out, void* stream);

/* Gradient of the emulator's output with respect to its raw input fields
 * (the gradient tf.GradientTape takes through the Keras model to the fields
 * in data assimilation, igm/processes/data_assimilation/optimize/update.py:
 * 37-70): from dpre0, the gradient of the first layer's pre-activation (bf16
 * [batch][h][4][w][8], as the second layer's dgrad of igm_conv3x3 leaves it),
 * and the first layer's FP32 kernel w0 [3][3][cin][32] (Keras layout),
 *   out[b][c][y][x] = scales[c] sum_{kh,kw,co} dpre0[b][y-kh+1][x-kw+1][co] w0[kh][kw][c][co]
 * (zero "same" padding) for the first n_grad (1..cin) fields, out
 * [batch][n_grad][h][w]; scales: host double[n_grad], the fixed input scales.
 * (Data assimilation with control thk needs the first field only.) */
IGM_API int igm_cnn_input_gradient(int batch, int h, int w, int cin, int n_grad, const void* dpre0, const float* w0,
                                   const double* scales, float* out, void* stream);

/* out[i] (+)= sum_p partials[p * stride + i], i < len, fixed summation order. */
IGM_API int igm_reduce_partials(const float* partials, int n_parts, int len, int stride, float* out,
                                int accumulate, void* stream);

/* igm_conv3x3_wgrad partials -> kernel gradient [3][3][cin][32]; cin_tensor is
 * the C of the layer's input tensor (16 or 32). */
IGM_API int igm_cnn_wgrad_finish(const float* partials, int n_parts, int cin, int cin_tensor, float* out,
                                 void* stream);
/* igm_conv3x3_wgrad partials of the first layer over the split input of
 * igm_cnn_input -> its kernel gradient [3][3][cin][32] (cin <= 5 fields): the
 * x_h and x_l channel gradients of each field added. */
IGM_API int igm_cnn_wgrad_finish_split(const float* partials, int n_parts, int cin, float* out, void* stream);

/* Keras legacy Adam with per-variable clip_by_norm (emulate.py:22-35, :267):
 * for each variable v (elements [var_offsets[v], var_offsets[v+1]) of the
 * vectors): g = g * c / max(|g|, c) when clipnorm c > 0, then the Adam update
 * at step `iteration` (1-based).  var_offsets: host size_t[n_vars + 1];
 * norms: device double[igm_adam_norms_len(n_vars, var_offsets)] scratch (the
 * variables' norms in the first n_vars entries, then per-chunk partial sums of
 * the squares: the norms are reduced deterministically across the GPU). */
IGM_API size_t igm_adam_norms_len(int n_vars, const size_t* var_offsets);
IGM_API int igm_adam_clipnorm(int n_vars, const size_t* var_offsets, float* params, const float* grads, float* m,
                              float* v, double* norms, double lr, double beta_1, double beta_2, double epsilon,
                              double clipnorm, int64_t iteration, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IGM_B200_H */
