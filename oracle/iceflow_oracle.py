"""CPU oracle for IGM's iceflow + thk hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``igm_b200``) imports this
module; it is imported by ``tests/``, by ``__graft_entry__.smoke()`` as the
checker, and by ``bench.py``'s CPU-baseline leg.

It restates, op by op and in the same evaluation order, the reference's
TensorFlow code for the path (all paths relative to the reference project):

* Blatter-Pattyn energy, staggered grid, Lagrange vertical basis
  - ``igm/processes/iceflow/energy/cost_shear.py:55-209``
  - ``igm/processes/iceflow/energy/cost_gravity.py:24-69``
  - ``igm/processes/iceflow/energy/cost_sliding_weertman.py:23-43``
  - ``igm/processes/iceflow/energy/utils.py:11-25`` (stag2, stag2v, stag4h)
  - ``igm/utils/gradient/compute_gradient.py:3-16`` (staggered branch)
  - the per-term ``reduce_mean`` + ``add_n`` of ``igm/processes/iceflow/solve/solve.py:57-59``
* vertical discretisation ``igm/processes/iceflow/vert_disc.py:10-47``
* velbase / velsurf / velbar ``igm/processes/iceflow/utils.py:21-51``
* vertical velocity, vert_flow version 2, kinematic and incompressibility
  methods ``igm/processes/vert_flow/vert_flow_v2.py:17-60,62-87,126-147``
  with ``compute_dz`` of ``igm/processes/iceflow/vert_disc.py:17-23``
* EarlyStopping ``igm/processes/iceflow/utils.py:80-110``
* the plain solver loop ``igm/processes/iceflow/solve/solve.py:22-119``
* Keras legacy Adam (TF 2.15.1, third party, not vendored): the published
  Adam update of Kingma & Ba (2015, Algorithm 1 with the "epsilon hat"
  variant), in the form ``m += (g-m)(1-b1); v += (g^2-v)(1-b2);
  x -= lr*sqrt(1-b2^t)/(1-b1^t) * m/(sqrt(v)+eps)``, with optional
  per-variable clip-by-norm ``g*c/max(|g|,c)``.
* slope-limited upwind transport
  ``igm/utils/gradient/compute_divflux_slope_limiter.py:3-65`` and the thk
  update ``igm/processes/thk/thk.py:11-54``
* CFL time step ``igm/processes/time/time.py:28-65``
* ELA mass balance ``igm/processes/smb_simple/smb_simple.py:24-50``
* the CNN emulator ``igm/processes/iceflow/emulate/neural_network.py:9-66``
  (Conv2D 3x3 "same" + bias + LeakyReLU(0.01), 1x1 head), with the NHWC
  layout conversions of ``igm/processes/iceflow/utils.py:133-158``; its
  retraining loop ``igm/processes/iceflow/emulate/emulate.py:155-328``
  (patches, pertubate_X)
* data assimilation ``igm/processes/data_assimilation``: the cost terms of
  ``cost_terms/*.py`` (misfit_velsurf with the low-speed term, misfit_thk,
  misfit_usurf, regu_thk, regu_slidingco, regu_arrhenius, cost_divfluxobs,
  cost_divfluxfcz, the penalties of total_cost), ``compute_divflux``
  (``igm/utils/gradient/compute_divflux.py:6-51``), the flow direction and
  density weights and the rms/std record of ``utils.py``, and one ADAM
  iteration of ``optimize/update.py:15-103`` over the controls.

All functions take and return ``torch`` CPU tensors; the dtype of the inputs
(float32 or float64) is the arithmetic precision.  Gradients of the energy are
obtained with torch autograd of this restatement, the stand-in for the
reference's ``tf.GradientTape`` (``solve.py:77``).

Parity pin: ``tests/golden/make_golden.py`` executes the reference's own
source files for these functions (under a TF-API shim over torch, because
TensorFlow cannot be installed here) and stores the results as fixtures;
``tests/test_oracle_golden.py`` checks this module against them.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

# --------------------------------------------------------------------------
# physical parameters (defaults of igm/conf/processes/iceflow.yaml:4-21)
# --------------------------------------------------------------------------


@dataclass
class Physics:
    exp_glen: float = 3.0
    exp_weertman: float = 3.0
    regu_glen: float = 1.0e-5
    regu_weertman: float = 1.0e-10
    thr_ice_thk: float = 0.1
    min_sr: float = 1.0e-20
    max_sr: float = 1.0e20
    ice_density: float = 910.0
    gravity_cst: float = 9.81
    force_negative_gravitational_energy: bool = False


def sqrt_ieee(t):
    """Correctly rounded square root of a CPU tensor (numpy's, IEEE 754):
    torch's vectorised CPU sqrt is not correctly rounded in every element,
    while the reference's arithmetic and the device kernels are.  No
    autograd through it."""
    return torch.from_numpy(np.asarray(np.sqrt(t.detach().numpy()))).to(t.dtype)


def _t(x, dtype=None):
    if isinstance(x, torch.Tensor):
        return x if dtype is None else x.to(dtype)
    return torch.as_tensor(np.asarray(x), dtype=dtype)


# --------------------------------------------------------------------------
# vertical discretisation  (vert_disc.py:10-13, 27-35, 43-47)
# --------------------------------------------------------------------------


def compute_levels(Nz: int, vert_spacing: float, dtype=torch.float32):
    """vert_disc.py:10-13: zeta_k = k/(Nz-1), level = zeta/s * (1 + (s-1) zeta)."""
    zeta = (torch.arange(Nz, dtype=torch.float64) / (Nz - 1)).to(dtype) if Nz > 1 else torch.zeros(1, dtype=dtype)
    return (zeta / vert_spacing) * (1.0 + (vert_spacing - 1.0) * zeta)


def compute_zeta_dzeta(levels):
    """vert_disc.py:27-35: midpoints and differences of the levels."""
    if levels.shape[0] > 1:
        return (levels[1:] + levels[:-1]) / 2, levels[1:] - levels[:-1]
    return 0.5 * torch.ones(1, dtype=levels.dtype), torch.ones(1, dtype=levels.dtype)


def define_vertical_weight(Nz: int, vert_spacing: float, dtype=torch.float32):
    """vert_disc.py:43-47: weights from Nz+1 equispaced points through the same map."""
    zeta = (torch.arange(Nz + 1, dtype=torch.float64) / Nz).to(dtype)
    w = (zeta / vert_spacing) * (1.0 + (vert_spacing - 1.0) * zeta)
    return (w[1:] - w[:-1])[:, None, None]


# --------------------------------------------------------------------------
# staggered-grid primitives  (energy/utils.py:11-25, compute_gradient.py:3-16)
# --------------------------------------------------------------------------


def stag2v(B):
    if B.shape[-3] > 1:
        B = (B[..., :-1, :, :] + B[..., 1:, :, :]) / 2
    return B


def stag4h(B):
    return (B[..., 1:, 1:] + B[..., 1:, :-1] + B[..., :-1, 1:] + B[..., :-1, :-1]) / 4


def compute_gradient_stag(s, dx):
    """compute_gradient.py:3-16 with a uniform dX field equal to ``dx``."""
    E = 2.0 * (s[..., :, 1:] - s[..., :, :-1]) / (dx + dx)
    diffx = 0.5 * (E[..., 1:, :] + E[..., :-1, :])
    EE = 2.0 * (s[..., 1:, :] - s[..., :-1, :]) / (dx + dx)
    diffy = 0.5 * (EE[..., :, 1:] + EE[..., :, :-1])
    return diffx, diffy


# --------------------------------------------------------------------------
# energy  (cost_shear.py, cost_gravity.py, cost_sliding_weertman.py)
# U, V : [B, Nz, Ny, Nx]   thk, usurf, arrhenius, slidingco : [B, Ny, Nx]
# --------------------------------------------------------------------------


def _horizontal_derivatives(U, V, dx):
    """cost_shear.py:25-38 (staggered branch)."""
    dUdx = (U[..., :, :, 1:] - U[..., :, :, :-1]) / dx
    dVdx = (V[..., :, :, 1:] - V[..., :, :, :-1]) / dx
    dUdy = (U[..., :, 1:, :] - U[..., :, :-1, :]) / dx
    dVdy = (V[..., :, 1:, :] - V[..., :, :-1, :]) / dx
    dUdx = (dUdx[..., :, :-1, :] + dUdx[..., :, 1:, :]) / 2
    dVdx = (dVdx[..., :, :-1, :] + dVdx[..., :, 1:, :]) / 2
    dUdy = (dUdy[..., :, :, :-1] + dUdy[..., :, :, 1:]) / 2
    dVdy = (dVdy[..., :, :, :-1] + dVdy[..., :, :, 1:]) / 2
    return dUdx, dVdx, dUdy, dVdy


def cost_shear(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, ph: Physics):
    """cost_shear.py:103-179, Lagrange basis, staggered grid."""
    B = 2.0 * arrhenius ** (-1.0 / ph.exp_glen)
    B = B[:, None, :, :]
    p = 1.0 + 1.0 / ph.exp_glen
    dUdx, dVdx, dUdy, dVdy = _horizontal_derivatives(U, V, dx)
    sloptopgx, sloptopgy = compute_gradient_stag(usurf - thk, dx)
    U = stag4h(U)
    V = stag4h(V)
    slidingco = stag4h(slidingco)
    thk = stag4h(thk)
    B = stag4h(B)
    dUdx = stag2v(dUdx)
    dVdx = stag2v(dVdx)
    dUdy = stag2v(dUdy)
    dVdy = stag2v(dVdy)
    B = stag2v(B)
    if U.shape[-3] > 1:
        h = torch.clamp(thk, min=ph.thr_ice_thk)[:, None]
        dUdz = (U[:, 1:] - U[:, :-1]) / (dzeta[None, :, None, None] * h)
        dVdz = (V[:, 1:] - V[:, :-1]) / (dzeta[None, :, None, None] * h)
    else:
        dUdz = torch.zeros_like(U)
        dVdz = torch.zeros_like(V)
    fl = slidingco[:, None] > 0
    dUdz = torch.where(fl, dUdz, 0.01 * dUdz)
    dVdz = torch.where(fl, dVdz, 0.01 * dVdz)
    sx = sloptopgx[:, None]
    sy = sloptopgy[:, None]
    dUdx = dUdx - dUdz * sx
    dUdy = dUdy - dUdz * sy
    dVdx = dVdx - dVdz * sx
    dVdy = dVdy - dVdz * sy
    Exx = dUdx
    Eyy = dVdy
    Ezz = -dUdx - dVdy
    Exy = 0.5 * dVdx + 0.5 * dUdy
    srxy2 = 0.5 * (Exx**2 + Exy**2 + Exy**2 + Eyy**2 + Ezz**2)
    Exz = 0.5 * dUdz
    Eyz = 0.5 * dVdz
    srz2 = 0.5 * (Exz**2 + Eyz**2 + Exz**2 + Eyz**2)
    sr2 = srxy2 + srz2
    # TF converts the clip bounds to the tensor's dtype: in float32, 1e40 -> +inf
    npdt = np.float32 if sr2.dtype == torch.float32 else np.float64
    with np.errstate(over="ignore"):
        lo = torch.as_tensor(npdt(ph.min_sr**2), dtype=sr2.dtype)
        hi = torch.as_tensor(npdt(ph.max_sr**2), dtype=sr2.dtype)
    sr2capped = torch.clamp(sr2, lo, hi)
    p_term = ((sr2capped + ph.regu_glen**2) ** ((p - 2) / 2)) * sr2 / p
    return thk * torch.sum(B * dzeta[None, :, None, None] * p_term, dim=1)


def cost_gravity(U, V, thk, usurf, dx, dzeta, ph: Physics):
    """cost_gravity.py:24-69, Lagrange basis, staggered grid."""
    slopsurfx, slopsurfy = compute_gradient_stag(usurf, dx)
    U = stag4h(U)
    V = stag4h(V)
    thk = stag4h(thk)
    U = stag2v(U)
    V = stag2v(V)
    uds = U * slopsurfx[:, None] + V * slopsurfy[:, None]
    if ph.force_negative_gravitational_energy:
        uds = torch.clamp(uds, max=0.0)
    return ph.ice_density * ph.gravity_cst * 10 ** (-6) * thk * torch.sum(dzeta[None, :, None, None] * uds, dim=1)


def cost_sliding_weertman(U, V, thk, usurf, slidingco, dx, ph: Physics):
    """cost_sliding_weertman.py:23-43, staggered grid."""
    C = 1.0 * slidingco
    s = 1.0 + 1.0 / ph.exp_weertman
    sloptopgx, sloptopgy = compute_gradient_stag(usurf - thk, dx)
    U = stag4h(U)
    V = stag4h(V)
    C = stag4h(C)
    ub = U[:, 0]
    vb = V[:, 0]
    N = (ub**2 + vb**2) + ph.regu_weertman**2 + (ub * sloptopgx + vb * sloptopgy) ** 2
    return C * N ** (s / 2) / s


def energy_terms(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, ph: Physics | None = None):
    """Per-cell energy densities [shear, sliding, gravity], each [B, Ny-1, Nx-1].

    Order follows ``energy_components: [shear, sliding_weertman, gravity]``
    (iceflow.yaml:5) as dispatched by energy.py:12-22.  4-D U/V expected
    (batch first, as solve.py:51 passes ``U[None]``); 3-D inputs get a batch
    dimension added.
    """
    ph = ph or Physics()
    if U.dim() == 3:
        U, V = U[None], V[None]
        thk, usurf, arrhenius, slidingco = thk[None], usurf[None], arrhenius[None], slidingco[None]
    return [
        cost_shear(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, ph),
        cost_sliding_weertman(U, V, thk, usurf, slidingco, dx, ph),
        cost_gravity(U, V, thk, usurf, dx, dzeta, ph),
    ]


def energy(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, ph: Physics | None = None):
    """COST = sum of reduce_mean of each term (solve.py:57-59).  Returns (cost, [means])."""
    terms = energy_terms(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, ph)
    means = [t.mean() for t in terms]
    return means[0] + means[1] + means[2], means


def energy_and_grad(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, ph: Physics | None = None):
    """COST and dCOST/dU, dCOST/dV by autograd (stand-in for tape.gradient, solve.py:77)."""
    U = U.detach().clone().requires_grad_(True)
    V = V.detach().clone().requires_grad_(True)
    cost, means = energy(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, ph)
    gU, gV = torch.autograd.grad(cost, [U, V])
    return cost.detach(), [m.detach() for m in means], gU, gV


# --------------------------------------------------------------------------
# optimiser, early stopping, solver
# --------------------------------------------------------------------------


class KerasLegacyAdam:
    """Adam as Keras' legacy optimizer applies it (see module docstring).

    ``iterations`` is global to the optimizer object and survives across
    solves, exactly as ``state.optimizer`` does in the reference
    (solve.py:11-20, 84); moment slots are per variable object.
    """

    def __init__(self, lr=1.0, beta_1=0.9, beta_2=0.999, epsilon=1e-7, clipnorm=None):
        self.lr, self.b1, self.b2, self.eps, self.clipnorm = lr, beta_1, beta_2, epsilon, clipnorm
        self.iterations = 0
        self.slots: dict[int, tuple[torch.Tensor, torch.Tensor, torch.Tensor]] = {}

    def apply_gradients(self, grads_and_vars):
        t = self.iterations + 1
        dt = None
        for g, x in grads_and_vars:
            dt = x.dtype
            if self.clipnorm is not None:
                n = sqrt_ieee(torch.sum(g.to(torch.float64) ** 2)).to(g.dtype)
                g = g * self.clipnorm / torch.maximum(n, torch.tensor(self.clipnorm, dtype=g.dtype))
            # slots are keyed by the variable object; holding the variable in its
            # slot keeps its id from being reused by a later variable (TF variables
            # have unique handles, so a new variable always gets fresh slots)
            key = id(x)
            if key not in self.slots or self.slots[key][0] is not x:
                self.slots[key] = (x, torch.zeros_like(x), torch.zeros_like(x))
            _, m, v = self.slots[key]
            one = torch.tensor(1.0, dtype=dt)
            b1p = torch.tensor(self.b1, dtype=dt) ** t
            b2p = torch.tensor(self.b2, dtype=dt) ** t
            alpha = self.lr * sqrt_ieee(one - b2p) / (one - b1p)
            m += (g - m) * (1 - self.b1)
            v += (g * g - v) * (1 - self.b2)
            x -= (m * alpha) / (sqrt_ieee(v) + self.eps)
        self.iterations += 1


class EarlyStopping:
    """utils.py:80-110."""

    def __init__(self, relative_min_delta=1e-3, patience=10):
        self.relative_min_delta = relative_min_delta
        self.patience = patience
        self.wait = 0
        self.best_loss = None

    def should_stop(self, current_loss):
        if self.best_loss is None:
            self.best_loss = current_loss
            return False
        rel = (self.best_loss - current_loss) / abs(self.best_loss)
        if rel > self.relative_min_delta:
            self.best_loss = current_loss
            self.wait = 0
            return False
        self.wait += 1
        return self.wait >= self.patience


def solve_iceflow(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, optimizer: KerasLegacyAdam,
                  nbitmax=100, ph: Physics | None = None, early_stopping=True,
                  relative_min_delta=0.0002, patience=10):
    """solve.py:22-119 (Adam branch, no sliding_law, no plotting).

    U, V [Nz, Ny, Nx] are copied (the reference wraps them in new
    tf.Variables, so the optimizer creates fresh moment slots).  Returns
    (U, V, cost_history) with U, V masked to zero where thk == 0.
    """
    U = U.detach().clone()
    V = V.detach().clone()
    es = EarlyStopping(relative_min_delta=relative_min_delta, patience=patience)
    costs = []
    for _ in range(nbitmax):
        cost, _, gU, gV = energy_and_grad(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, ph)
        costs.append(float(cost))
        optimizer.apply_gradients([(gU, U), (gV, V)])
        if early_stopping and es.should_stop(np.float32(cost) if U.dtype == torch.float32 else float(cost)):
            break
    mask = (thk > 0)[None]
    U = torch.where(mask, U, torch.zeros_like(U))
    V = torch.where(mask, V, torch.zeros_like(V))
    return U, V, costs


def force_max_velbar(U, V, cap):
    """utils.py:182-194 (Lagrange basis): where |(U, V)| >= cap, both
    components scaled to that speed; the magnitude as tf.norm of the stacked
    pair, sqrt(U U + V V)."""
    mag = sqrt_ieee(U * U + V * V)
    c = torch.tensor(cap, dtype=U.dtype)
    return torch.where(mag >= c, c * (U / mag), U), torch.where(mag >= c, c * (V / mag), V)


def get_velbase(U, V):
    return U[..., 0, :, :], V[..., 0, :, :]


def get_velsurf(U, V):
    return U[..., -1, :, :], V[..., -1, :, :]


def get_velbar(U, V, vert_weight):
    return torch.sum(U * vert_weight, dim=-3), torch.sum(V * vert_weight, dim=-3)


# --------------------------------------------------------------------------
# vertical velocity (vert_flow, version 2, kinematic method)
# --------------------------------------------------------------------------


def cumsum0(x):
    """``tf.cumsum(x, axis=0)``: an inclusive scan accumulated in the tensor's
    own dtype, level after level (``torch.cumsum`` on CPU accumulates float32
    in double, which rounds differently)."""
    out = [x[0]]
    for k in range(1, x.shape[0]):
        out.append(out[-1] + x[k])
    return torch.stack(out)


def compute_dz(thk, levels):
    """vert_disc.py:17-23: layer thicknesses thk * (level[k+1] - level[k])."""
    ddz = levels[1:] - levels[:-1]
    return thk[None] * ddz[:, None, None]


def gradient_layers(s, dx):
    """compute_gradient_layers_tf (vert_flow_v2.py:62-87): centred differences
    of face values, with the faces on the domain border extrapolated
    (1.5 s0 - 0.5 s1); s : [L, Ny, Nx]."""
    EX = torch.cat([1.5 * s[:, :, 0:1] - 0.5 * s[:, :, 1:2], 0.5 * s[:, :, :-1] + 0.5 * s[:, :, 1:],
                    1.5 * s[:, :, -1:] - 0.5 * s[:, :, -2:-1]], 2)
    EY = torch.cat([1.5 * s[:, 0:1, :] - 0.5 * s[:, 1:2, :], 0.5 * s[:, :-1, :] + 0.5 * s[:, 1:, :],
                    1.5 * s[:, -1:, :] - 0.5 * s[:, -2:-1, :]], 1)
    return (EX[:, :, 1:] - EX[:, :, :-1]) / dx, (EY[:, 1:, :] - EY[:, :-1, :]) / dx


def divflux_layers(u, v, h, dx):
    """compute_divflux_layers (vert_flow_v2.py:126-147): centred divergence of
    (u h, v h) per layer, border faces taking the border cell's flux."""
    Qx = u * h
    Qy = v * h
    fx = torch.cat([Qx[:, :, 0:1], 0.5 * (Qx[:, :, :-1] + Qx[:, :, 1:]), Qx[:, :, -1:]], 2)
    fy = torch.cat([Qy[:, 0:1, :], 0.5 * (Qy[:, :-1, :] + Qy[:, 1:, :]), Qy[:, -1:, :]], 1)
    return (fx[:, :, 1:] - fx[:, :, :-1]) / dx + (fy[:, 1:, :] - fy[:, :-1, :]) / dx


def vertical_velocity_kinematic(U, V, topg, thk, levels, vert_weight, dx):
    """compute_vertical_velocity_kinematic_v2 / compute_w_kinematic_tf
    (vert_flow_v2.py:17-37): the layer surfaces z_k = topg + sum_{l<k} dz_l,
    their slopes, the running vertical means of U, V from the bed up to layer
    k (weights vert_weight), and W = -div(mean * z-height) + U dz/dx + V dz/dy.
    U, V : [Nz, Ny, Nx]; vert_weight : [Nz, 1, 1]; returns W [Nz, Ny, Nx]."""
    dz = compute_dz(thk, levels)
    cumdz = torch.cat([torch.zeros_like(thk)[None], cumsum0(dz)], 0)
    sx, sy = gradient_layers(topg + cumdz, dx)
    ub = cumsum0(vert_weight * U) / cumsum0(vert_weight)
    vb = cumsum0(vert_weight * V) / cumsum0(vert_weight)
    div = divflux_layers(ub, vb, cumdz, dx)
    return -div + U * sx + V * sy


def _faces_mean_z(U):
    """[U_0, (U_k + U_{k+1})/2, U_{Nz-1}]: the layer-face values of
    gradx/grady_non_flat_layers_tf (vert_flow_v2.py:175, 192)."""
    return torch.cat([U[0:1], 0.5 * (U[:-1] + U[1:]), U[-1:]], 0)


def vertical_velocity_incompressibility(U, V, topg, thk, levels, vert_weight, dx):
    """compute_vertical_velocity_incompressibility_v2 (vert_flow_v2.py:40-57)
    with gradx/grady_non_flat_layers_tf (:168-199), compute_gradx/grady_layers_tf
    (:90-123) and compute_gradient_tf (utils/gradient/compute_gradient_tf.py:6-35)
    for a uniform spacing dX = dx: terrain-following horizontal derivatives
    du/dx = (du/dx)_flat - dZ/dx du/dz on the layer surfaces Z, and
    W_k = U_0 dtopg/dx + V_0 dtopg/dy - sum_{l<=k} dz_l (du/dx + dv/dy)_l."""
    dz = torch.cat([torch.zeros_like(thk)[None], compute_dz(thk, levels)], 0)
    Z = cumsum0(dz) + topg
    sx_b, sy_b = gradient_layers(topg[None], dx)
    sx, sy = gradient_layers(Z, dx)
    gUx, _ = gradient_layers(U, dx)
    _, gVy = gradient_layers(V, dx)
    h = vert_weight * thk
    Uf, Vf = _faces_mean_z(U), _faces_mean_z(V)
    dUdz = torch.where(thk > 0, (Uf[1:] - Uf[:-1]) / h, torch.zeros_like(h))
    dVdz = torch.where(thk > 0, (Vf[1:] - Vf[:-1]) / h, torch.zeros_like(h))
    dudx = gUx - sx * dUdz
    dvdy = gVy - sy * dVdz
    intdwdz = cumsum0(dz * (dudx + dvdy))
    return sx_b[0] * U[0] + sy_b[0] * V[0] - intdwdz


# --------------------------------------------------------------------------
# transport, time step, mass balance
# --------------------------------------------------------------------------


def _minmod(a, b):
    z = torch.zeros_like(a)
    return torch.where((a.abs() < b.abs()) & (a * b > 0.0), a,
                       torch.where((a.abs() > b.abs()) & (a * b > 0.0), b, z))


def _maxmod(a, b):
    z = torch.zeros_like(a)
    return torch.where((a.abs() < b.abs()) & (a * b > 0.0), b,
                       torch.where((a.abs() > b.abs()) & (a * b > 0.0), a, z))


def compute_divflux_slope_limiter(u, v, h, dx, dy, dt, slope_type="superbee"):
    """compute_divflux_slope_limiter.py:11-65.  u, v, h : [Ny, Nx]."""
    u = torch.cat([u[:, 0:1], 0.5 * (u[:, :-1] + u[:, 1:]), u[:, -1:]], 1)
    v = torch.cat([v[0:1, :], 0.5 * (v[:-1, :] + v[1:, :]), v[-1:, :]], 0)
    Hx = torch.nn.functional.pad(h, (2, 2, 0, 0))
    Hy = torch.nn.functional.pad(h, (0, 0, 2, 2))
    sigpx = (Hx[:, 2:] - Hx[:, 1:-1]) / dx
    sigmx = (Hx[:, 1:-1] - Hx[:, :-2]) / dx
    sigpy = (Hy[2:, :] - Hy[1:-1, :]) / dy
    sigmy = (Hy[1:-1, :] - Hy[:-2, :]) / dy
    if slope_type == "godunov":
        slopex = torch.zeros_like(sigpx)
        slopey = torch.zeros_like(sigpy)
    elif slope_type == "minmod":
        slopex = _minmod(sigmx, sigpx)
        slopey = _minmod(sigmy, sigpy)
    elif slope_type == "superbee":
        slopex = _maxmod(_minmod(sigpx, 2.0 * sigmx), _minmod(sigmx, 2.0 * sigpx))
        slopey = _maxmod(_minmod(sigpy, 2.0 * sigmy), _minmod(sigmy, 2.0 * sigpy))
    else:
        raise ValueError(f"unknown slope_type {slope_type}")
    w = Hx[:, 1:-2] + 0.5 * dx * (1.0 - u * dt / dx) * slopex[:, :-1]
    e = Hx[:, 2:-1] - 0.5 * dx * (1.0 + u * dt / dx) * slopex[:, 1:]
    s = Hy[1:-2, :] + 0.5 * dy * (1.0 - v * dt / dy) * slopey[:-1, :]
    n = Hy[2:-1, :] - 0.5 * dy * (1.0 + v * dt / dy) * slopey[1:, :]
    Qx = u * torch.where(u > 0, w, e)
    Qy = v * torch.where(v > 0, s, n)
    return (Qx[:, 1:] - Qx[:, :-1]) / dx + (Qy[1:, :] - Qy[:-1, :]) / dy


def thk_update(thk, topg, ubar, vbar, smb, dx, dt, slope_type="superbee",
               ratio_density=0.910, sealevel=0.0):
    """thk.py:27-54.  Returns (thk, lsurf, usurf, divflux)."""
    divflux = compute_divflux_slope_limiter(ubar, vbar, thk, dx, dx, dt, slope_type)
    thk = torch.clamp(thk + dt * (smb - divflux), min=0)
    lsurf = torch.maximum(topg, -ratio_density * thk + sealevel)
    usurf = lsurf + thk
    return thk, lsurf, usurf, divflux


def thk_surfaces(thk, topg, ratio_density=0.910, sealevel=0.0):
    """thk.py:11-24 (initialize)."""
    lsurf = torch.maximum(topg, -ratio_density * thk + sealevel)
    return lsurf, lsurf + thk


def cfl_dt(ubar, vbar, dx, cfl=0.3, step_max=1.0):
    """time.py:36-50 (without the save-time snapping, done by the caller)."""
    velomax = float(torch.maximum(ubar.abs().max(), vbar.abs().max()))
    if cfl > 0 and velomax > 0:
        return min(cfl * dx / velomax, step_max), velomax
    return step_max, velomax


def smb_simple(usurf, gradabl, gradacc, ela, maxacc):
    """smb_simple.py:39-41."""
    smb = usurf - ela
    smb = smb * torch.where(smb < 0, torch.tensor(gradabl, dtype=smb.dtype), torch.tensor(gradacc, dtype=smb.dtype))
    return torch.clamp(smb, -100, maxacc)


def interp1d(xs, ys, x):
    """interp1d_tf.py: piecewise-linear, clamped to the table's range."""
    return float(np.interp(np.clip(x, np.min(xs), np.max(xs)), xs, ys))


# --------------------------------------------------------------------------
# CNN emulator (neural_network.py:9-66) and layout helpers (utils.py:133-158)
# --------------------------------------------------------------------------


def cnn_forward(X, weights, biases, alpha=0.01, bf16=False, return_acts=False, bf16_first=True, out_scale=1.0):
    """Stack of Conv2D(3x3, same) + LeakyReLU, then a 1x1 Conv2D head.

    X : [B, H, W, Cin] (NHWC, as fieldin_to_X builds it);
    weights[l] : [3, 3, Cin_l, Cout_l] (Keras kernel layout), biases[l] : [Cout_l].
    The last entry is the 1x1 head ([1, 1, 32, 2Nz]).  With ``bf16`` the
    inputs of every 3x3 conv and their weights are rounded to bfloat16 and the
    products accumulated in float32 (the emulator kernels' arithmetic); the
    head and everything else stay float32.
    Returns Y : [B, H, W, 2Nz].
    """
    x = X.permute(0, 3, 1, 2)
    acts = []
    nl = len(weights) - 1
    for l in range(nl):
        w = weights[l].permute(3, 2, 0, 1)
        if bf16 and (l > 0 or bf16_first):
            xin = x.to(torch.bfloat16).to(torch.float32)
            w = w.to(torch.bfloat16).to(torch.float32)
        else:
            xin = x
        x = torch.nn.functional.conv2d(xin, w, biases[l], padding=1)
        x = torch.nn.functional.leaky_relu(x, alpha)
        if bf16:
            x = x.to(torch.bfloat16).to(torch.float32)
        acts.append(x)
    w = weights[-1].permute(3, 2, 0, 1)
    y = torch.nn.functional.conv2d(x, w, biases[-1]) * out_scale
    y = y.permute(0, 2, 3, 1)
    return (y, acts) if return_acts else y


def Y_to_UV(Y, Nz):
    """utils.py:133-139: channels [0,Nz) are U levels, [Nz,2Nz) V levels."""
    return Y[..., :Nz].movedim(-1, 1), Y[..., Nz:].movedim(-1, 1)


def fieldin_to_X(fields):
    """utils.py:147-158 for 2-D fields: stack on a trailing channel axis, add batch."""
    return torch.stack(fields, dim=-1)[None]


def split_into_patches(X, nbmax):
    """emulate.py:283-308 ("sequential"): X [1, ny, nx, C] -> [P, 1, ly, lx, C]."""
    ny, nx = X.shape[1], X.shape[2]
    sy = ny // nbmax + 1
    sx = nx // nbmax + 1
    ly = int(ny / sy)
    lx = int(nx / sx)
    XX = []
    for i in range(sx):
        for j in range(sy):
            XX.append(X[:, j * ly:(j + 1) * ly, i * lx:(i + 1) * lx, :])
    return torch.stack(XX, dim=0)


# --------------------------------------------------------------------------
# synthetic glaciers: the input generators live in the package and are
# re-exported here for the tests
# --------------------------------------------------------------------------
from igm_b200.synthetic import box_filter, ridge_glacier, valley_glacier  # noqa: E402,F401


# --------------------------------------------------------------------------
# emulator retraining loop (emulate.py:155-281) and the clock (time.py:11-65)
# --------------------------------------------------------------------------


@dataclass
class EmulatorTraining:
    retrain_freq: int = 10
    lr: float = 2.0e-5
    lr_init: float = 1.0e-4
    lr_decay: float = 0.95
    warm_up_it: float = -1e10
    nbit_init: int = 1
    nbit: int = 1
    framesizemax: int = 750


def pertubate_X(X, channels):
    """pertubate_X (emulate.py:310-328): X and, for each channel in
    ``channels``, copies with that channel scaled by 1.2 and 0.8, along the
    batch axis."""
    XX = [X]
    for c in channels:
        vec = torch.zeros(X.shape[-1], dtype=X.dtype)
        vec[c] = 1.0
        XX.append(X + X * vec * 0.2)
        XX.append(X - X * vec * 0.2)
    return torch.cat(XX, 0)


def emulator_retrain(weights, biases, optimizer: KerasLegacyAdam, X, it, tr: EmulatorTraining,
                     Nz, dzeta, ph: Physics | None = None, bf16=False, pertubate_channels=None,
                     input_scales=None, out_scale=1.0):
    """emulate.py:155-281 ("sequential" patches, no borders).

    ``weights``/``biases`` are leaf tensors updated in place; X is
    [1, ny, nx, 5] (thk, usurf, arrhenius, slidingco, dX).  Returns the list
    of per-epoch summed costs, or None when this iteration does not retrain.
    ``pertubate_channels``: the channels pertubate_X scales (the retraining
    batch then holds 1 + 2 len(channels) samples per patch; each sample's
    energy uses its own fields -- the reference's cost_shear.py:75-76
    broadcasts dzeta[None, :, None, None] against thk [B, ny, nx], which
    fails for a batch B > 1 other than Nz - 1, so this restates the intent).
    ``input_scales`` multiply the network input only.
    """
    run_it = tr.retrain_freq > 0 and (it % tr.retrain_freq == 0)
    warm_up = int(it <= tr.warm_up_it)
    if not (warm_up or run_it):
        return None
    if pertubate_channels:
        X = pertubate_X(X, pertubate_channels)
    Xp = split_into_patches(X, tr.framesizemax)
    nbit, lr = (tr.nbit_init, tr.lr_init) if warm_up else (tr.nbit, tr.lr)
    optimizer.lr = lr
    params = []
    for w, b in zip(weights, biases):
        params += [w, b]
    costs = []
    for _ in range(nbit):
        total = 0.0
        for i in range(Xp.shape[0]):
            if tr.lr_decay < 1:
                optimizer.lr = lr * (tr.lr_decay ** (i / 1000))
            Xi = Xp[i]
            ps = [p.detach().clone().requires_grad_(True) for p in params]
            Xin = Xi * torch.tensor(input_scales, dtype=Xi.dtype) if input_scales is not None else Xi
            Y = cnn_forward(Xin, ps[0::2], ps[1::2], bf16=bf16, bf16_first=input_scales is None,
                            out_scale=out_scale)
            U, V = Y_to_UV(Y, Nz)
            cost, _ = energy(U, V, Xi[..., 0], Xi[..., 1], Xi[..., 2], Xi[..., 3], Xi[0, 0, 0, 4], dzeta, ph)
            grads = torch.autograd.grad(cost, ps)
            with torch.no_grad():
                optimizer.apply_gradients(list(zip(grads, params)))
            total = total + float(cost.detach())
        costs.append(total)
    return costs


class Clock:
    """time.py:11-65: CFL time step snapped to the save times."""

    def __init__(self, start=2000.0, end=2100.0, save=10.0, cfl=0.3, step_max=1.0):
        self.t = np.float32(start)
        self.end, self.cfl, self.step_max = end, cfl, step_max
        self.itsave = -1
        ts = list(np.arange(start, end, save)) + [end]
        self.time_save = np.asarray(ts, dtype=np.float32)
        self.dt = np.float32(step_max)
        self.saveresult = False
        self.continue_run = True

    def update(self, ubar, vbar, dx, it):
        if self.cfl > 0:
            velomax = np.float32(max(float(ubar.abs().max()), float(vbar.abs().max())))
            if velomax > 0:
                dt = np.float32(min(np.float32(self.cfl * dx) / velomax, self.step_max))
            else:
                dt = np.float32(self.step_max)
        else:
            dt = np.float32(self.step_max)
        self.dt = dt
        if self.time_save[self.itsave + 1] <= self.t + self.dt:
            self.dt = np.float32(self.time_save[self.itsave + 1] - self.t)
            self.saveresult = True
            self.itsave += 1
        else:
            self.saveresult = False
        if it >= 0:
            self.t = np.float32(self.t + self.dt)
        self.continue_run = bool(self.t < self.end)


# --------------------------------------------------------------------------
# data assimilation: cost terms of the default configuration
# (igm/processes/data_assimilation/cost_terms/*.py, utils.py)
# --------------------------------------------------------------------------


@dataclass
class AssimParams:
    velsurfobs_std: float = 1.0
    velsurfobs_thr: float = 0.0
    thkobs_std: float = 3.0
    regu_thk: float = 10.0
    convexity_weight: float = 0.002
    convexity_power: float = 1.3
    smooth_anisotropy_factor: float = 0.2
    to_regularize: str = "topg"
    penalty: bool = True
    icemask_cost: bool = True
    fix_normalization: bool = False  # optimization.fix_opti_normalization_issue
    low_speed: bool = False          # fitting.include_low_speed_term
    sole_mask: bool = False          # optimization.sole_mask


def getmag(u, v):
    """igm/utils/math/getmag.py: the Euclidean norm of (u, v)."""
    return torch.sqrt(u * u + v * v)


def da_flow_direction(uvelsurf, vvelsurf):
    """compute_flow_direction_for_anisotropic_smoothing (utils.py:86-110): the
    cell average of the surface velocity, smoothed by a Gaussian of 3 cells
    (scipy, zero outside), normalised -- the y component with the already
    normalised x component, as in the reference -- zero where undefined.
    Returns float32 [Ny-1, Nx-1] tensors (constants of the gradient)."""
    from scipy.ndimage import gaussian_filter
    u = torch.where(torch.isnan(uvelsurf), torch.zeros_like(uvelsurf), uvelsurf)
    v = torch.where(torch.isnan(vvelsurf), torch.zeros_like(vvelsurf), vvelsurf)
    fx = (u[1:, 1:] + u[:-1, 1:] + u[1:, :-1] + u[:-1, :-1]) / 4.0
    fy = (v[1:, 1:] + v[:-1, 1:] + v[1:, :-1] + v[:-1, :-1]) / 4.0
    fx = torch.as_tensor(gaussian_filter(fx.detach().numpy(), 3, mode="constant"))
    fy = torch.as_tensor(gaussian_filter(fy.detach().numpy(), 3, mode="constant"))
    fx = fx / getmag(fx, fy)
    fy = fy / getmag(fx, fy)
    fx = torch.where(torch.isnan(fx), torch.zeros_like(fx), fx)
    fy = torch.where(torch.isnan(fy), torch.zeros_like(fy), fy)
    return fx, fy


def da_misfit_velsurf(uvelsurf, vvelsurf, uobs, vobs, std, thr, low_speed=False):
    """misfit_velsurf (cost_terms/misfit_velsurf.py:8-30): 0.5 mean over the
    observed components at nodes whose observed speed reaches thr of
    ((obs - vs) / std)^2; with include_low_speed_term + 0.5 100
    log((|vs| + 1) / (|obs| + 1))^2, where -- velsurf[ACT] being the 1-D
    selection of the observed components, without the threshold -- |.| is the
    norm of all of them."""
    vs = torch.stack([uvelsurf, vvelsurf], -1)
    vo = torch.stack([uobs, vobs], -1)
    rel = (torch.linalg.vector_norm(vo, dim=-1) >= thr)[..., None]
    m = ~torch.isnan(vo) & rel
    c = 0.5 * torch.mean(((vo[m] - vs[m]) / std) ** 2)
    if low_speed:
        # the reference selects with ACT alone here (no speed threshold)
        act = ~torch.isnan(vo)
        c = c + 0.5 * 100 * torch.log((torch.linalg.vector_norm(vs[act]) + 1) /
                                      (torch.linalg.vector_norm(vo[act]) + 1)) ** 2
    return c


def da_costs(thk, usurf, uvelsurf, vvelsurf, uobs, vobs, thkobs, dens_thkobs, icemaskobs, icemask, flowdir, dx,
             p: AssimParams, thk_control=True):
    """The cost terms of total_cost (cost_terms/total_cost.py:13-70) for
    control ``thk``, costs velsurf + thk + icemask and the penalty
    constraint: misfit_velsurf.py:8-19, misfit_thk.py:8-16, the icemask and
    positive-thickness penalties (total_cost.py:36-46) and regu_thk.py:8-70
    (to_regularize topg or thk, fix_opti_normalization_issue off).  Returns a
    dict of scalar tensors."""
    cost = {"velsurf": da_misfit_velsurf(uvelsurf, vvelsurf, uobs, vobs, p.velsurfobs_std, p.velsurfobs_thr,
                                         p.low_speed)}
    a = ~torch.isnan(thkobs)
    cost["thk"] = 0.5 * torch.mean(dens_thkobs[a] * ((thkobs[a] - thk[a]) / p.thkobs_std) ** 2)
    z = torch.zeros_like(thk)
    if p.penalty:
        if p.icemask_cost:
            cost["icemask"] = 10 ** 10 * torch.mean(torch.where(icemaskobs > 0.5, z, thk ** 2))
        if thk_control:
            cost["thk_positive"] = 10 ** 10 * torch.mean(torch.where(thk >= 0, z, thk ** 2))
    if not thk_control:
        return cost
    area = torch.sum(torch.where(icemask > 0.5, 1.0, 0.0)) * dx ** 2
    gamma = p.convexity_weight * area ** (p.convexity_power - 2.0)
    field = usurf - thk if p.to_regularize == "topg" else thk
    f = p.smooth_anisotropy_factor
    if f == 1:
        dbdx = (field[:, 1:] - field[:, :-1]) / dx
        dbdy = (field[1:, :] - field[:-1, :]) / dx
        if p.sole_mask:
            im = icemaskobs > 0.5
            dbdx = torch.where(im[:, 1:] & im[:, :-1], dbdx, torch.zeros_like(dbdx))
            dbdy = torch.where(im[1:, :] & im[:-1, :], dbdy, torch.zeros_like(dbdy))
        if p.fix_normalization:
            cost["thk_regu"] = p.regu_thk * 0.5 * (torch.mean(dbdx ** 2) + torch.mean(dbdy ** 2)
                                                   - gamma * torch.mean(thk))
        else:
            cost["thk_regu"] = p.regu_thk * (torch.sum(dbdx ** 2) / 2 + torch.sum(dbdy ** 2) / 2
                                             - gamma * torch.sum(thk))
    else:
        fx, fy = flowdir
        dbdx = (field[:, 1:] - field[:, :-1]) / dx
        dbdx = (dbdx[1:, :] + dbdx[:-1, :]) / 2.0
        dbdy = (field[1:, :] - field[:-1, :]) / dx
        dbdy = (dbdy[:, 1:] + dbdy[:, :-1]) / 2.0
        if p.sole_mask:
            im = icemaskobs > 0.5
            cm = im[1:, 1:] & im[1:, :-1] & im[:-1, 1:] & im[:-1, :-1]
            dbdx = torch.where(cm, dbdx, torch.zeros_like(dbdx))
            dbdy = torch.where(cm, dbdy, torch.zeros_like(dbdy))
        if p.fix_normalization:
            cost["thk_regu"] = p.regu_thk * 0.5 * (
                (1.0 / np.sqrt(f)) * torch.mean((dbdx * fx + dbdy * fy) ** 2)
                + np.sqrt(f) * torch.mean((dbdx * fy - dbdy * fx) ** 2)
                - torch.mean(gamma * thk))
        else:
            cost["thk_regu"] = p.regu_thk * (
                (1.0 / np.sqrt(f)) * torch.sum((dbdx * fx + dbdy * fy) ** 2) / 2
                + np.sqrt(f) * torch.sum((dbdx * fy - dbdy * fx) ** 2) / 2
                - torch.sum(gamma * thk))
    return cost


def divflux_upwind(u, v, h, dx):
    """compute_divflux, method upwind (utils/gradient/compute_divflux.py:17-33,
    45-46): face velocities (edge copies at the border), upwind thickness with
    zero outside, divergence."""
    uf = torch.cat([u[:, 0:1], 0.5 * (u[:, :-1] + u[:, 1:]), u[:, -1:]], 1)
    vf = torch.cat([v[0:1, :], 0.5 * (v[:-1, :] + v[1:, :]), v[-1:, :]], 0)
    Hx = torch.nn.functional.pad(h, (1, 1, 0, 0))
    Hy = torch.nn.functional.pad(h, (0, 0, 1, 1))
    Qx = uf * torch.where(uf > 0, Hx[:, :-1], Hx[:, 1:])
    Qy = vf * torch.where(vf > 0, Hy[:-1, :], Hy[1:, :])
    return (Qx[:, 1:] - Qx[:, :-1]) / dx + (Qy[1:, :] - Qy[:-1, :]) / dx


# --------------------------------------------------------------------------
# data assimilation loop (igm/processes/data_assimilation): density weights,
# one ADAM iteration of optimize_update for control thk, the rms/std record
# --------------------------------------------------------------------------


def create_density_matrix(data, kernel_size=5):
    """utils.py:68-82: the number of non-NaN entries of ``data`` in the
    kernel_size x kernel_size window around each node ('SAME', zero
    outside)."""
    m = (~torch.isnan(data)).to(data.dtype)[None, None]
    k = torch.ones((1, 1, kernel_size, kernel_size), dtype=data.dtype)
    return torch.nn.functional.conv2d(m, k, padding=kernel_size // 2)[0, 0]


def da_density_weights(thkobs, uniformize=True):
    """optimize/initialize.py:40-46: inverse observation density, zero where
    thkobs is NaN, normalised by its mean over the positive entries."""
    if not uniformize:
        return torch.ones_like(thkobs)
    d = create_density_matrix(thkobs, 5)
    d = torch.where(d > 0, 1.0 / d, torch.zeros_like(d))
    d = torch.where(torch.isnan(thkobs), torch.zeros_like(d), d)
    return d / torch.mean(d[d > 0])


@dataclass
class AssimControl:
    """The optimisation keys of optimize_update for control thk
    (conf/processes/data_assimilation.yaml, optimization / scaling)."""
    step_size: float = 1.0
    step_size_decay: float = 0.9
    scaling_thk: float = 2.0
    reproject: bool = True
    icemask_cost: bool = True


@dataclass
class AssimControls:
    """The controls of optimize_update and the keys of their cost terms
    (conf/processes/data_assimilation.yaml: control_list, scaling,
    fitting.log_slidingco, regularization.slidingco / arrhenius /
    smooth_anisotropy_factor_sl, fitting.usurfobs_std)."""
    controls: list = field(default_factory=lambda: ["thk"])
    scaling: dict = field(default_factory=lambda: {"thk": 2.0, "usurf": 0.5, "slidingco": 1e-4, "arrhenius": 0.1})
    log_slidingco: bool = False
    regu_slidingco: float = 1.0
    regu_arrhenius: float = 10.0
    aniso_sl: float = 1.0
    usurfobs_std: float = 2.0


def da_optimize_step(fields, dx, weights, biases, Nz, vert_weight, obs, p: AssimParams, ctl: AssimControl,
                     optimizer: KerasLegacyAdam, i, mc: AssimControls, bf16=True, out_scale=1.0, input_scales=None,
                     divflux_cost=None):
    """One ADAM iteration of optimize_update (optimize/update.py:15-103) over
    the controls of ``mc``: each control becomes a new variable x / scale
    (sqrt(x / scale) for slidingco with log_slidingco: fresh Adam slots, the
    optimizer's iteration count carries on), the fields are rebuilt from the
    variables, the emulator forward is masked where thk == 0
    (emulate.py:116-152), the flow directions come from the emulated surface
    velocities (constants of the gradient: they pass through scipy), then
    total_cost (total_cost.py:13-71: the costs of da_costs, misfit_usurf with
    "usurfobs" in obs, the flux-divergence term of ``divflux_cost``, the
    slidingco / arrhenius penalties and regularisations), its gradient w.r.t.
    the variables (zero outside icemaskobs > 0.5 except for slidingco), one
    Adam step at step_size decay^(i/100), the fields from the variables, the
    reprojection (thk: mask and >= 0; slidingco >= 0; arrhenius >= 1), the
    flux divergence of the emulated depth-averaged velocity.

    ``fields``: dict thk, usurf, arrhenius, slidingco.  Returns (new fields,
    costs dict, dict of uvelsurf, vvelsurf, ubar, vbar, divflux and the
    variables' gradients under "gradient_<control>")."""
    sc = mc.scaling
    var, x = {}, dict(fields)
    for c in mc.controls:
        if c == "slidingco" and mc.log_slidingco:
            var[c] = torch.sqrt(fields[c] / sc[c]).detach().clone().requires_grad_(True)
            x[c] = (var[c] ** 2) * sc[c]
        else:
            var[c] = (fields[c] / sc[c]).detach().clone().requires_grad_(True)
            x[c] = var[c] * sc[c]
    th, us, ar, sl = x["thk"], x["usurf"], x["arrhenius"], x["slidingco"]
    dX = torch.full_like(th, dx)
    X = fieldin_to_X([th, us, ar, sl, dX])
    if input_scales is not None:
        X = X * torch.tensor(input_scales, dtype=X.dtype)
    Y = cnn_forward(X, weights, biases, bf16=bf16, bf16_first=False, out_scale=out_scale)
    U, V = Y_to_UV(Y, Nz)
    U = torch.where(th > 0, U[0], torch.zeros_like(U[0]))
    V = torch.where(th > 0, V[0], torch.zeros_like(V[0]))
    uvs, vvs = U[-1], V[-1]
    flow = None
    if p.smooth_anisotropy_factor != 1 or ("slidingco" in mc.controls and mc.aniso_sl != 1):
        flow = da_flow_direction(uvs.detach(), vvs.detach())
    cost = da_costs(th, us, uvs, vvs, obs["uobs"], obs["vobs"], obs["thkobs"], obs["dens"], obs["icemaskobs"],
                    obs["icemask"], flow if p.smooth_anisotropy_factor != 1 else None, dx, p,
                    thk_control="thk" in mc.controls)
    if divflux_cost is not None:
        dc = divflux_cost
        ub_g, vb_g = torch.sum(U * vert_weight, 0), torch.sum(V * vert_weight, 0)
        if dc["kind"] == "fcz" and (i % 10 == 0 or "slope" not in dc):
            act = obs["icemaskobs"] > 0.5
            D0 = compute_divflux(ub_g.detach(), vb_g.detach(), th.detach(), dx, dc["method"])
            dc["slope"], dc["intercept"] = linregress(us[act].detach().numpy(), D0[act].numpy())
        cost["divflux"] = da_cost_divflux(dc["kind"], ub_g, vb_g, th, dx, obs["icemaskobs"],
                                          divfluxobs=dc.get("divfluxobs"), usurf=us.detach(), slope=dc.get("slope"),
                                          intercept=dc.get("intercept"), std=dc["std"], regu=dc["regu"],
                                          force_zero_sum=dc["force_zero_sum"], method=dc["method"])
    if "usurfobs" in obs:
        cost["usurf"] = da_misfit_usurf(us, obs["usurfobs"], obs["icemaskobs"], mc.usurfobs_std)
    if p.penalty:
        if "slidingco" in mc.controls and not mc.log_slidingco:
            cost["slidingco_positive"] = da_penalty(sl, 0.0)
        if "arrhenius" in mc.controls:
            cost["arrhenius_positive"] = da_penalty(ar, 1.0)
    smask = obs["icemaskobs"] if p.sole_mask else None
    if "slidingco" in mc.controls:
        cost["slid_regu"] = da_regu_field(sl, dx, mc.regu_slidingco, mc.aniso_sl, flow, normalize=p.fix_normalization,
                                          icemaskobs=smask)
    if "arrhenius" in mc.controls:
        cost["arrh_regu"] = da_regu_field(ar, dx, mc.regu_arrhenius, normalize=p.fix_normalization,
                                          icemaskobs=smask)
    total = sum(cost.values())
    grads = torch.autograd.grad(total, [var[c] for c in mc.controls])
    inside = obs["icemaskobs"] > 0.5
    # update.py:58-68: slidingco's gradient unmasked, or (sole_mask) where icemaskobs == 1
    sl_mask = obs["icemaskobs"] == 1
    grads = [(torch.where(sl_mask, g, torch.zeros_like(g)) if p.sole_mask else g) if c == "slidingco"
             else torch.where(inside, g, torch.zeros_like(g)) for c, g in zip(mc.controls, grads)]
    if ctl.step_size_decay < 1:
        optimizer.lr = ctl.step_size * (ctl.step_size_decay ** (i / 100))
    new_vars = [var[c].detach().clone() for c in mc.controls]
    optimizer.apply_gradients(list(zip(grads, new_vars)))
    out = dict(fields)
    for c, w in zip(mc.controls, new_vars):
        out[c] = (w ** 2) * sc[c] if (c == "slidingco" and mc.log_slidingco) else w * sc[c]
    if ctl.reproject:
        # update.py:84-91: the icemask reprojection of thk applies whenever "icemask" is a cost, thk a control
        # or not; the bound thk >= 0 only when thk is a control
        if ctl.icemask_cost:
            out["thk"] = torch.where(inside, out["thk"], torch.zeros_like(out["thk"]))
        if "thk" in mc.controls:
            t = out["thk"]
            out["thk"] = torch.where(t < 0, torch.zeros_like(t), t)
        if "slidingco" in mc.controls:
            out["slidingco"] = torch.where(out["slidingco"] < 0, torch.zeros_like(out["slidingco"]), out["slidingco"])
        if "arrhenius" in mc.controls:
            out["arrhenius"] = torch.where(out["arrhenius"] < 1.0, torch.ones_like(out["arrhenius"]),
                                           out["arrhenius"])
    U, V = U.detach(), V.detach()
    ubar = torch.sum(U * vert_weight, 0)
    vbar = torch.sum(V * vert_weight, 0)
    method = divflux_cost["method"] if divflux_cost is not None else "upwind"
    aux = {"uvelsurf": uvs.detach(), "vvelsurf": vvs.detach(), "ubar": ubar, "vbar": vbar,
           "divflux": compute_divflux(ubar, vbar, out["thk"], dx, method)}
    aux.update({f"gradient_{c}": g for c, g in zip(mc.controls, grads)})
    return out, {k: v.detach() for k, v in cost.items()}, aux


def da_optimize_update(thk, usurf, arrhenius, slidingco, dx, weights, biases, Nz, vert_weight, obs, p: AssimParams,
                       ctl: AssimControl, optimizer: KerasLegacyAdam, i, bf16=True, out_scale=1.0, input_scales=None,
                       divflux_cost=None):
    """da_optimize_step for control_list [thk] with scaling ctl.scaling_thk:
    returns (thk, costs dict, aux with the gradient of thk's variable under
    "gradient")."""
    mc = AssimControls(controls=["thk"], scaling={"thk": ctl.scaling_thk})
    out, cost, aux = da_optimize_step({"thk": thk, "usurf": usurf, "arrhenius": arrhenius, "slidingco": slidingco},
                                      dx, weights, biases, Nz, vert_weight, obs, p, ctl, optimizer, i, mc, bf16=bf16,
                                      out_scale=out_scale, input_scales=input_scales, divflux_cost=divflux_cost)
    aux["gradient"] = aux["gradient_thk"]
    return out["thk"], cost, aux


def da_rms_std(thk, thkobs, uvelsurf, vvelsurf, uobs, vobs, icemaskobs, dx, divflux=None, divfluxobs=None,
               usurf=None, usurfobs=None):
    """compute_rms_std_optimization (utils.py:10-66): mean and population
    standard deviation of thk - thkobs at the thickness observations (0 when
    there are none), of the speed misfit inside the observed mask where the
    observed speed is defined, of divfluxobs - divflux and usurf - usurfobs
    inside the mask (0 when the observation is absent), the volume in km^3."""
    def ms(d):
        d = d.double()
        return (float(d.mean()), float(d.std(unbiased=False))) if d.numel() else (float("nan"), float("nan"))
    I = icemaskobs > 0.5
    out = {}
    if thkobs is not None:
        a = ~torch.isnan(thkobs)
        out["rmsthk"], out["stdthk"] = ms(thk[a] - thkobs[a]) if a.any() else (0.0, 0.0)
    else:
        out["rmsthk"], out["stdthk"] = 0.0, 0.0
    if uobs is not None:
        vs, vo = getmag(uvelsurf, vvelsurf), getmag(uobs, vobs)
        m = I & ~torch.isnan(vo)
        out["rmsvel"], out["stdvel"] = ms(vs[m] - vo[m])
    else:
        out["rmsvel"], out["stdvel"] = 0.0, 0.0
    out["rmsdiv"], out["stddiv"] = ms(divfluxobs[I] - divflux[I]) if divfluxobs is not None else (0.0, 0.0)
    out["rmsusurf"], out["stdusurf"] = ms(usurf[I] - usurfobs[I]) if usurfobs is not None else (0.0, 0.0)
    out["vol"] = float(thk.double().sum() * dx * dx / 1e9)
    return out


def compute_divflux(u, v, h, dx, method="upwind"):
    """compute_divflux (utils/gradient/compute_divflux.py:6-51): upwind (the
    face velocity carries the upwind thickness, zero outside) or centered (the
    face average of u h, edge copies at the border)."""
    if method == "upwind":
        return divflux_upwind(u, v, h, dx)
    if method != "centered":
        raise ValueError(method)
    qx, qy = u * h, v * h
    Qx = torch.cat([qx[:, 0:1], 0.5 * (qx[:, :-1] + qx[:, 1:]), qx[:, -1:]], 1)
    Qy = torch.cat([qy[0:1, :], 0.5 * (qy[:-1, :] + qy[1:, :]), qy[-1:, :]], 0)
    return (Qx[:, 1:] - Qx[:, :-1]) / dx + (Qy[1:, :] - Qy[:-1, :]) / dx


def linregress(x, y):
    """Least-squares line y = intercept + slope x (scipy.stats.linregress's
    slope and intercept), in float64."""
    x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
    xm, ym = x.mean(), y.mean()
    sxx = ((x - xm) ** 2).mean()
    sxy = ((x - xm) * (y - ym)).mean()
    slope = sxy / sxx
    return slope, ym - slope * xm


def da_cost_divflux(kind, ubar, vbar, thk, dx, icemaskobs, divfluxobs=None, usurf=None, slope=None,
                    intercept=None, std=1.0, regu=1.0, force_zero_sum=False, method="upwind"):
    """cost_divfluxobs (cost_terms/cost_divfluxobs.py:9-29, kind "obs"):
    0.5 mean(((obs - D) / std)^2) over the observed nodes + regu 0.5
    (mean(dD/dx^2) + mean(dD/dy^2)); cost_divfluxfcz
    (cost_terms/cost_divfluxfcz.py:10-38, kind "fcz"): the target intercept +
    slope usurf inside icemaskobs > 0.5 (the regression is a constant of the
    gradient), 0.5 mean(((target - D) / std)^2) over the mask; both plus
    0.5 1000 mean(D / std)^2 over the mask with force_zero_sum."""
    D = compute_divflux(ubar, vbar, thk, dx, method)
    act_m = icemaskobs > 0.5
    if kind == "obs":
        act = ~torch.isnan(divfluxobs)
        c = 0.5 * torch.mean(((divfluxobs[act] - D[act]) / std) ** 2)
        dddx = (D[:, 1:] - D[:, :-1]) / dx
        dddy = (D[1:, :] - D[:-1, :]) / dx
        c = c + regu * 0.5 * (torch.mean(dddx ** 2) + torch.mean(dddy ** 2))
    else:
        tar = torch.where(act_m, intercept + slope * usurf, torch.zeros_like(usurf))
        c = 0.5 * torch.mean(((tar[act_m] - D[act_m]) / std) ** 2)
    if force_zero_sum:
        c = c + 0.5 * 1000 * torch.mean(D[act_m] / std) ** 2
    return c


def da_regu_field(f, dx, weight, aniso=1.0, flowdir=None, normalize=False, icemaskobs=None):
    """regu_slidingco (cost_terms/regu_slidingco.py:8-52) and regu_arrhenius
    (cost_terms/regu_arrhenius.py:5-24) with sole_mask and
    fix_opti_normalization_issue off: weight (l2_loss(df/dx) + l2_loss(df/dy))
    on the node differences (aniso == 1), or the cell-centred differences
    split along and across the flow direction weighted 1/sqrt(aniso) and
    sqrt(aniso); with ``normalize`` (fix_opti_normalization_issue) weight 0.5
    times the means instead of the half sums."""
    red = (lambda x: 0.5 * torch.mean(x)) if normalize else (lambda x: torch.sum(x) / 2)
    if aniso == 1.0:
        dadx = (f[:, 1:] - f[:, :-1]) / dx
        dady = (f[1:, :] - f[:-1, :]) / dx
        if icemaskobs is not None:  # sole_mask: both nodes with icemaskobs == 1
            m = icemaskobs == 1
            dadx = torch.where(m[:, 1:] & m[:, :-1], dadx, torch.zeros_like(dadx))
            dady = torch.where(m[1:, :] & m[:-1, :], dady, torch.zeros_like(dady))
        return weight * (red(dadx ** 2) + red(dady ** 2))
    dadx = (f[:, 1:] - f[:, :-1]) / dx
    dadx = (dadx[1:, :] + dadx[:-1, :]) / 2.0
    dady = (f[1:, :] - f[:-1, :]) / dx
    dady = (dady[:, 1:] + dady[:, :-1]) / 2.0
    if icemaskobs is not None:  # sole_mask: the four corners with icemaskobs > 0.5
        m = icemaskobs > 0.5
        cm = m[1:, 1:] & m[1:, :-1] & m[:-1, 1:] & m[:-1, :-1]
        dadx = torch.where(cm, dadx, torch.zeros_like(dadx))
        dady = torch.where(cm, dady, torch.zeros_like(dady))
    fx, fy = flowdir
    return weight * ((1.0 / np.sqrt(aniso)) * red((dadx * fx + dady * fy) ** 2)
                     + np.sqrt(aniso) * red((dadx * fy - dady * fx) ** 2))


def da_penalty(f, threshold):
    """The positivity penalties of total_cost.py:40-54: 1e10 mean of f^2
    where f < threshold (0 for thk and slidingco, 1 for arrhenius)."""
    return 1e10 * torch.mean(torch.where(f >= threshold, torch.zeros_like(f), f ** 2))


def da_misfit_usurf(usurf, usurfobs, icemaskobs, std):
    """misfit_usurf (cost_terms/misfit_usurf.py:5-15): 0.5 mean over
    icemaskobs > 0.5 of ((usurf - usurfobs) / std)^2."""
    act = icemaskobs > 0.5
    return 0.5 * torch.mean(((usurf[act] - usurfobs[act]) / std) ** 2)
