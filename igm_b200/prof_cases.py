"""One launch of each hot kernel on a case larger than L2, for profiling
(``python -m igm_b200.prof_cases``; run it under ncu with -k and -c).

Stencil (energy, energy + adjoint, one fused Adam iteration), transport and
the vertical velocity at 1500 x 1500 x Nz 10 in FP32; the data-assimilation
cost/gradient, flow direction and upwind divergence at 1500 x 1500 in FP32;
the tensor-core convolution (forward, dgrad, wgrad, the fused backward) at
batch 2 x 1000 x 1000 x 32 channels, and the forward stack of 15 such layers
at batch 1.

``python -m igm_b200.prof_cases assimilation_iteration`` instead sets up the
data-assimilation loop on the 1000 x 1000 x Nz 10 glacier tongue (default
configuration, 16-layer emulator), runs 5 iterations, then one more between
cudaProfilerStart and cudaProfilerStop (for ncu --profile-from-start off).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from . import kernels as K
from .solver import DeviceAdamSolver
from .synthetic import valley_glacier
from .vertical import compute_levels, compute_zeta_dzeta, define_vertical_weight


def assimilation_inputs(N, thk, uvs, vvs, seed=0):
    """Observations for the data-assimilation kernels: surface velocities
    with 10% missing, thickness profiles on every 50th column, the ice mask
    of thk > 0, uniform density weights."""
    rng = np.random.default_rng(seed)
    hole = torch.as_tensor(rng.random((N, N)) < 0.1, device=thk.device)
    nan = torch.full_like(thk, float("nan"))
    uobs = torch.where(hole, nan, uvs + 1.0)
    vobs = torch.where(hole, nan, vvs - 1.0)
    thkobs = nan.clone()
    thkobs[:, ::50] = thk[:, ::50]
    mask = (thk > 0).float()
    p = L.AssimParams()
    p.velsurfobs_std, p.velsurfobs_thr, p.thkobs_std, p.regu_thk = 1.0, 0.0, 3.0, 10.0
    p.gamma, p.aniso_factor = 1e-8, 0.2
    p.n_vel = float((~torch.isnan(uobs)).sum().item() * 2)
    p.n_thk = float((~torch.isnan(thkobs)).sum().item())
    p.penalty, p.icemask_cost, p.regularize_thk, p.mask_velsurf = 1, 1, 0, 1
    return dict(uobs=uobs, vobs=vobs, thkobs=thkobs, dens=torch.ones_like(thk), mask=mask, params=p)


def assimilation(N, f, uvs, vvs):
    """One launch each of the data-assimilation kernels."""
    a = assimilation_inputs(N, f[0], uvs, vvs)
    flow = K.assim_flow_direction(uvs, vvs)                       # flow direction (3 kernels)
    K.assim_cost_grad(f[0], f[1], uvs, vvs, a["uobs"], a["vobs"], a["thkobs"], a["dens"], a["mask"], flow, 50.0,
                      a["params"])                                # cost terms + gradient
    K.divflux_upwind(uvs, vvs, f[0], 50.0)                        # upwind flux divergence


def main():
    N, nz = 1500, 10
    st = valley_glacier(N, N, 50.0, seed=0, varying_coeffs=True)
    f = [torch.as_tensor(st[k]).cuda() for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    dz = compute_zeta_dzeta(compute_levels(nz, 4.0))[1]
    rng = np.random.default_rng(0)
    U = torch.as_tensor(rng.normal(30, 20, (nz, N, N)).astype(np.float32)).cuda()
    V = torch.as_tensor(rng.normal(0, 20, (nz, N, N)).astype(np.float32)).cuda()
    K.energy(U, V, *f, 50.0, dz)                                  # stencil: energy
    K.energy(U, V, *f, 50.0, dz, grad=True)                       # stencil: energy + adjoint
    DeviceAdamSolver().solve(U, V, *f, 50.0, dz, nbitmax=1, early_stopping=False, mask=False)  # fused Adam step
    ub, vb = U[0].contiguous(), V[0].contiguous()
    K.transport_step(ub, vb, f[0], f[1], None, 50.0, 0.01)       # transport
    topg = torch.as_tensor(st["topg"]).cuda()
    K.vertical_velocity(U, V, topg, f[0], compute_levels(nz, 4.0), define_vertical_weight(nz, 4.0), 50.0)  # vert_flow
    K.vertical_velocity(U, V, topg, f[0], compute_levels(nz, 4.0), define_vertical_weight(nz, 4.0), 50.0,
                        method="incompressibility")
    assimilation(N, f, U[-1].contiguous(), V[-1].contiguous())
    B, H, W = 2, 1000, 1000                                       # 2 x 64 MB activations (> L2)
    x = torch.randn(B, H, 4, W, 8, device="cuda").to(torch.bfloat16)
    y = torch.empty_like(x)
    y2 = torch.empty_like(x)
    wp = (torch.randn(9 * 4 * 32 * 8, device="cuda") * 0.05).to(torch.bfloat16)
    bias = torch.zeros(32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib, s = L.lib(), L.stream_ptr()
    L.check(lib.igm_conv3x3(0, B, H, W, 32, x.data_ptr(), wp.data_ptr(), bias.data_ptr(), None, y.data_ptr(), None,
                            0, 0.01, err.data_ptr(), s), "conv forward")
    dbp = torch.zeros(148, 32, device="cuda")
    L.check(lib.igm_conv3x3(1, B, H, W, 32, y.data_ptr(), wp.data_ptr(), None, x.data_ptr(), y2.data_ptr(),
                            dbp.data_ptr(), 148, 0.01, err.data_ptr(), s), "conv dgrad")
    part = torch.empty(148, int(lib.igm_conv3x3_wgrad_partial_len(32)), device="cuda")
    L.check(lib.igm_conv3x3_wgrad(B, H, W, 32, x.data_ptr(), y.data_ptr(), part.data_ptr(), 148, err.data_ptr(), s),
            "conv wgrad")
    L.check(lib.igm_conv3x3_backward(B, H, W, y.data_ptr(), wp.data_ptr(), x.data_ptr(), y2.data_ptr(),
                                     dbp.data_ptr(), part.data_ptr(), 148, 0.01, err.data_ptr(), None, None, None, None,
                                     s), "conv backward")
    # the forward stack: 15 layers of batch 1 x 1000 x 1000, outputs alternating between two buffers
    import ctypes as C
    nl = 15
    outs = (C.c_void_p * nl)(*[(y if k % 2 == 0 else y2).data_ptr() for k in range(nl)])
    wps = (C.c_void_p * nl)(*([wp.data_ptr()] * nl))
    bss = (C.c_void_p * nl)(*([bias.data_ptr()] * nl))
    flags = torch.zeros(int(lib.igm_conv3x3_stack_flags_len(1, H, W, nl)), dtype=torch.int32, device="cuda")
    L.check(lib.igm_conv3x3_stack(1, H, W, nl, x.data_ptr(), outs, wps, bss, flags.data_ptr(), 1, 0.01,
                                  err.data_ptr(), s), "conv stack")
    torch.cuda.synchronize()
    if int(err.item()) != 0:
        raise RuntimeError(f"kernel error flag {int(err.item())}")
    print("ok")


def assimilation_iteration(N=1000, nz=10, warm=5):
    """One data-assimilation iteration (optimize_update + the rms/std
    record) bracketed for the profiler, after ``warm`` iterations."""
    from .config import default_cfg
    from .processes import data_assimilation as DA
    from .processes import iceflow as P
    from .state import State
    from .synthetic import tongue_glacier
    g = tongue_glacier(N, N, 50.0, seed=0)
    scales = [1 / 300.0, 1 / 3000.0, 1 / 100.0, 10.0, 1 / 50.0]
    cfg = default_cfg({"iceflow": {"numerics": {"Nz": nz},
                                   "emulator": {"pretrained": False, "input_scales": scales, "seed": 0,
                                                "output_scale": 50.0,
                                                "network": {"weight_initialization": "he_normal"}}},
                       "data_assimilation": {"output": {"save_iterat_in_ncdf": False}}})
    st = State()
    for k in ("thk", "usurf", "topg", "arrhenius", "slidingco"):
        setattr(st, k, torch.as_tensor(g[k]).cuda())
    st.dx = 50.0
    st.icemask = (st.thk > 0).float()
    st.icemaskobs = st.icemask.clone()
    P.initialize(cfg, st)
    obs = assimilation_inputs(N, st.thk, st.uvelsurf.contiguous(), st.vvelsurf.contiguous())
    st.uvelsurfobs, st.vvelsurfobs, st.thkobs = obs["uobs"], obs["vobs"], obs["thkobs"]
    DA.optimize_initialize(cfg, st)
    a = st._igm_assim

    def it(i):
        DA.optimize_update(cfg, st, {}, i)
        DA._record_rms(a, st, i)

    for i in range(warm):
        it(i)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    it(warm)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    st.iceflow_model.check_errors()
    print("ok")


if __name__ == "__main__":
    import sys
    if len(sys.argv) > 1 and sys.argv[1] == "assimilation_iteration":
        assimilation_iteration()
    else:
        main()
