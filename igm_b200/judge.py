"""The yardstick the emulator and the plain solver are judged against: the
FP64 minimiser of the Blatter-Pattyn energy of a state, converged.

This is measurement infrastructure (bench.py, tests), not a process of the
drop-in path: the iceflow process minimises the energy with the reference's
own Adam solver (igm/processes/iceflow/solve/solve.py:22-119).

Why a different optimiser here.  On steep, fast-sliding glaciers the
energy is very flat along large-scale, depth-coherent velocity modes (the
plug flow of thick ice held back by lateral drag and weak Weertman
friction: the curvature of |u|^(4/3) falls off as |u|^(-2/3)).  Adam moves
each velocity by about its step size per iteration, and a single-grid
quasi-Newton method needs thousands of iterations to move such a mode, so
both stop several percent (in velocity) away from the minimiser while the
energy has converged to a fraction of a percent.  Grid sequencing fixes
this: the state is coarsened by factors of two (2 x 2 cell averages of thk,
usurf, A and c; dx doubled), the energy is minimised on the coarsest grid,
where the large-scale modes are few cells wide, and each solution is
interpolated (bilinearly) to the next finer grid as the starting point of
its own minimisation.  Each level runs L-BFGS (two-loop recursion, memory
m, Armijo backtracking) on the device energy and its hand-written adjoint
(igm_energy, FP64).

``converged_velocity`` returns the fine-grid minimiser and a record of each
level (iterations, energy per cell, gradient norm); ``agreement`` compares
two solutions the way the bench reports velocity errors (relative L2 of the
staggered velocities over ice cells).
"""

from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

from . import kernels as K


def staggered(X):
    """stag4h: the 4-corner average of [..., ny, nx] -> [..., ny-1, nx-1]."""
    return 0.25 * (X[..., 1:, 1:] + X[..., 1:, :-1] + X[..., :-1, 1:] + X[..., :-1, :-1])


def velocity_rel_l2(U, V, Ur, Vr, thk):
    """Relative L2 of the staggered velocities over cells touching ice (the
    staggered grid leaves a checkerboard mode of the node values that the
    energy does not see; stag4h removes it)."""
    m = staggered((thk > 0).double()[None])[0] > 0
    su, sv, sur, svr = (staggered(X.double()) for X in (U, V, Ur, Vr))
    num = ((su - sur)[:, m] ** 2).sum() + ((sv - svr)[:, m] ** 2).sum()
    den = (sur[:, m] ** 2).sum() + (svr[:, m] ** 2).sum()
    return float(torch.sqrt(num / den.clamp_min(1e-300)))


def _coarsen(f):
    """2 x 2 averages (a trailing odd row / column averaged with itself)."""
    ny, nx = f.shape
    g = f[None, None]
    if ny % 2:
        g = torch.cat([g, g[..., -1:, :]], 2)
    if nx % 2:
        g = torch.cat([g, g[..., :, -1:]], 3)
    return F.avg_pool2d(g, 2)[0, 0]


def _refine(X, shape):
    """Bilinear interpolation of [nz, ny, nx] node values onto the finer grid."""
    return F.interpolate(X[None], size=shape, mode="bilinear", align_corners=True)[0]


class _Energy:
    def __init__(self, fields, dx, dzeta, phys):
        self.f = [t.double().contiguous() for t in fields]
        self.dx, self.dz, self.ph = float(dx), np.asarray(dzeta, np.float64), phys
        ny, nx = self.f[0].shape
        self.ns = (ny - 1) * (nx - 1)
        self.nz = len(self.dz) + 1
        self.shape = (self.nz, ny, nx)

    def __call__(self, x):
        n = int(np.prod(self.shape))
        U, V = x[:n].view(self.shape), x[n:].view(self.shape)
        t, dU, dV = K.energy(U, V, *self.f, self.dx, self.dz, self.ph, grad=True, grad_scale=1.0 / self.ns)
        return float(t.sum()) / self.ns, torch.cat([dU.reshape(-1), dV.reshape(-1)])


def lbfgs(fg, x, iters, mem=20, gtol=0.0):
    """L-BFGS with Armijo backtracking; returns (x, energy, gradient norm,
    iterations run)."""
    S, Y, R = [], [], []
    e, g = fg(x)
    it = 0
    for it in range(1, iters + 1):
        q = g.clone()
        al = []
        for s, y, rho in zip(reversed(S), reversed(Y), reversed(R)):
            a = rho * float(torch.dot(s, q))
            q.add_(y, alpha=-a)
            al.append(a)
        gam = float(torch.dot(S[-1], Y[-1]) / torch.dot(Y[-1], Y[-1])) if S else 1.0 / max(float(g.norm()), 1e-300)
        q.mul_(gam)
        for (s, y, rho), a in zip(zip(S, Y, R), reversed(al)):
            b = rho * float(torch.dot(y, q))
            q.add_(s, alpha=a - b)
        d = q.neg_()
        gd = float(torch.dot(g, d))
        if gd >= 0:  # not a descent direction: restart from steepest descent
            S.clear(), Y.clear(), R.clear()
            d = -g * gam
            gd = float(torch.dot(g, d))
        step, ok = 1.0, False
        for _ in range(40):
            xn = x + step * d
            en, gn = fg(xn)
            if np.isfinite(en) and en <= e + 1e-4 * step * gd:
                ok = True
                break
            step *= 0.5
        if not ok:
            break
        s, y = xn - x, gn - g
        sy = float(torch.dot(s, y))
        if sy > 1e-12 * float(s.norm()) * float(y.norm()):
            S.append(s), Y.append(y), R.append(1.0 / sy)
            if len(S) > mem:
                S.pop(0), Y.pop(0), R.pop(0)
        x, e, g = xn, en, gn
        if gtol > 0 and float(g.norm()) < gtol:
            break
    return x, e, float(g.norm()), it


def converged_velocity(thk, usurf, arrhenius, slidingco, dx, dzeta, phys=None, levels=4, iters=(3000, 2000, 1500, 1500),
                       U0=None, V0=None, mem=20):
    """FP64 minimiser of the energy of the state (fields [ny, nx] on the
    device).  ``levels`` grids (the finest the state's); ``iters[l]`` L-BFGS
    iterations on level l, coarsest first.  U0, V0: optional start on the
    finest grid (then only the finest level runs).  Returns (U, V, record)
    with U, V float64 [nz, ny, nx]."""
    fine = [t.double() for t in (thk, usurf, arrhenius, slidingco)]
    pyr = [(fine, float(dx))]
    for _ in range(levels - 1):
        f, h = pyr[-1]
        if min(f[0].shape) < 16:
            break
        pyr.append(([_coarsen(t) for t in f], 2 * h))
    pyr = pyr[::-1]
    nz = len(dzeta) + 1
    record = []
    x = None
    start = 0
    if U0 is not None:
        start = len(pyr) - 1
        x = torch.cat([U0.double().reshape(-1), V0.double().reshape(-1)])
    for lvl in range(start, len(pyr)):
        f, h = pyr[lvl]
        fg = _Energy(f, h, dzeta, phys)
        ny, nx = f[0].shape
        if x is None:
            x = torch.zeros(2 * nz * ny * nx, dtype=torch.float64, device=f[0].device)
        elif x.numel() != 2 * nz * ny * nx:
            pny, pnx = pyr[lvl - 1][0][0].shape
            n = nz * pny * pnx
            U = _refine(x[:n].view(nz, pny, pnx), (ny, nx))
            V = _refine(x[n:].view(nz, pny, pnx), (ny, nx))
            x = torch.cat([U.reshape(-1), V.reshape(-1)])
        k = iters[min(lvl, len(iters) - 1)] if U0 is None else iters[-1]
        x, e, gn, done = lbfgs(fg, x, k, mem=mem)
        record.append({"grid": [ny, nx], "dx": h, "iterations": done, "energy_per_cell": e, "grad_norm": gn})
    ny, nx = fine[0].shape
    n = nz * ny * nx
    return x[:n].view(nz, ny, nx).clone(), x[n:].view(nz, ny, nx).clone(), record
