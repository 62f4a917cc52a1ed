"""The plain solver on the device (igm/processes/iceflow/solve/solve.py:11-119).

One fused kernel per iteration (energy + adjoint + Keras-legacy Adam +
FP64 reduction + EarlyStopping); the whole solve is enqueued without host
synchronisation and the host reads the 64-byte control block once at the end.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .kernels import fields_struct, workspace


class DeviceAdamSolver:
    """Minimises the Blatter-Pattyn energy over (U, V) with Adam.

    ``iterations`` mirrors Keras' ``optimizer.iterations``: it is global to the
    solver object and carries over between solves (the bias correction uses
    it), while the moment slots start from zero at every solve, as the
    reference's fresh ``tf.Variable(U)`` get fresh slots (solve.py:27-28)."""

    def __init__(self, lr=1.0, beta_1=0.9, beta_2=0.999, epsilon=1e-7):
        self.adam = L.Adam()
        self.adam.lr, self.adam.beta_1, self.adam.beta_2, self.adam.epsilon = lr, beta_1, beta_2, epsilon
        self.iterations = 0
        self.last_costs = np.zeros(0)
        self.last_status = 0

    def solve(self, U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, nbitmax=100, phys=None,
              relative_min_delta=0.0002, patience=10, early_stopping=True, mask=True):
        """Returns (U, V, costs) with U, V [Nz, Ny, Nx] (or [B, Nz, Ny, Nx])
        masked to zero where thk == 0 (solve.py:116-117) when ``mask``."""
        batched = U.dim() == 4
        U4 = U if batched else U[None]
        V4 = V if batched else V[None]
        f2 = [t if batched else t[None] for t in (thk, usurf, arrhenius, slidingco)]
        B, nz, ny, nx = U4.shape
        dev = U.device
        g = L.make_grid(B, nz, ny, nx, dx, dzeta)
        ph = phys if isinstance(phys, L.Physics) else L.make_physics(phys)
        U0, V0 = U4.clone(), V4.clone()
        U1, V1 = torch.empty_like(U0), torch.empty_like(V0)
        mU, mV, vU, vV = (torch.zeros_like(U0) for _ in range(4))
        ctl = torch.zeros(C.sizeof(L.SolverCtl), dtype=torch.uint8, device=dev)
        costs = torch.zeros(max(int(nbitmax), 1), dtype=torch.float64, device=dev)
        es = L.EarlyStop()
        es.relative_min_delta, es.patience, es.enabled = float(relative_min_delta), int(patience), int(bool(early_stopping))
        wp, wn = workspace(dev).get(g, dev)
        f = fields_struct(*f2)
        st = L.stream_ptr()
        lib = L.lib()
        L.check(lib.igm_solver_begin(L.ptr(ctl), int(self.iterations), st), "igm_solver_begin")
        if nbitmax > 0:
            rc = lib.igm_solver_iterate(L.dtype_code(U.dtype), C.byref(g), C.byref(ph), C.byref(f),
                                        L.ptr(U0), L.ptr(V0), L.ptr(U1), L.ptr(V1), L.ptr(mU), L.ptr(mV), L.ptr(vU),
                                        L.ptr(vV), C.byref(self.adam), C.byref(es), int(nbitmax), int(nbitmax),
                                        L.ptr(ctl), L.ptr(costs), wp, wn, st)
            L.check(rc, "igm_solver_iterate")
        hc = L.SolverCtl.from_buffer_copy(ctl.cpu().numpy().tobytes())
        n = int(hc.iter)
        self.iterations += n
        self.last_status = int(hc.status)
        self.last_costs = costs[:n].cpu().numpy()
        if hc.status != 0:
            raise L.IgmError(hc.status, f"solver stopped at iteration {n}: non-finite energy")
        Ur, Vr = (U0, V0) if n % 2 == 0 else (U1, V1)
        if mask:
            w = (C.c_double * nz)(*([0.0] * nz))
            rc = lib.igm_velocity_reduce(L.dtype_code(U.dtype), B, nz, ny, nx, L.ptr(Ur), L.ptr(Vr), L.ptr(f2[0]), 1, w,
                                         None, None, None, None, None, None, None, st)
            L.check(rc, "igm_velocity_reduce(mask)")
        if not batched:
            Ur, Vr = Ur[0], Vr[0]
        return Ur, Vr, self.last_costs
