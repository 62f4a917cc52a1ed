"""pretraining process (igm/processes/pretraining/pretraining.py:25-494):
physics-informed offline training of the iceflow emulator on a library of
glacier geometries, on the device.

The reference's loop, kept step for step: the training and test sets are the
sub-directories of ``data_dir/train`` and ``data_dir/test``, each holding an
``ex.nc`` with ``thk``, ``usurf`` (time, y, x) and ``x``; the test cases
(``state.PAR``: time slice 3, the middle arrhenius and slidingco of the
configured ranges, the finest coarsening, plus the quarter points of each
range and the next coarsening) are solved once with the plain solver
(``compute_solutions``); every epoch visits the training sets in random
order, each at a random time slice, with a random rot90 / flip / transpose
(``_aug``) and -- after ``soft_begining`` epochs -- a random coarsening
2^k and random uniform arrhenius and slidingco, and takes one Adam step on
the Blatter-Pattyn energy of the network's output (the emulator's
retraining step); the learning rate decays by 0.9^(epoch % restart / 100);
the model is saved every epochs / 5 epochs and the test misfits are
written every ``freq_test`` epochs; ``initialize`` ends the program, as the
reference's does.

Differences, each forced by what is available here: the sets are read with
scipy's netCDF reader, so ``ex.nc`` must be netCDF-3 (the format the output
writer ``igm_b200.outputs`` produces; a netCDF-4 file raises
NotImplementedError naming the conversion); the draws use a seeded numpy
generator (``pretraining.seed``) where the reference draws unseeded; the
models are written as the reference's Keras ``model-<epoch>.h5`` /
``model.h5`` and, beside them, as ``.npz`` (the exact parameters with their
scales and the Adam state, which this package's loader reads); the misfit
plots are not drawn
(no matplotlib).  Every computation on the fields -- the solves, the
network's forward and backward passes, the energy and its adjoint, Adam --
runs in the device kernels; the host prepares the inputs (slicing,
augmentation) and the diagnostics.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

from .. import kernels as K
from ..cnn import CNN
from ..emulator import EmulatorOptimizer, train_step
from ..solver import DeviceAdamSolver
from ..vertical import compute_levels, compute_zeta_dzeta, define_vertical_weight
from . import iceflow as P


def _direct_name(cfg) -> str:
    """pretraining.py:26-45."""
    ic = cfg.processes.iceflow
    net = ic.emulator.network
    return (f"pinnbp_{ic.numerics.Nz}_{int(ic.numerics.vert_spacing)}_{net.architecture}_{net.nb_layers}_"
            f"{net.nb_out_filter}_{ic.physics.dim_arrhenius}_1")


def _findsubdata(folder):
    """pretraining.py:539-547: the sub-directories of ``folder``, sorted."""
    paths = [f.path for f in os.scandir(folder) if f.is_dir()]
    paths.sort(key=lambda x: (os.path.isdir(x), x))
    return [p.split("/")[-1] for p in paths], paths


def _read_ex(path):
    """thk, usurf (time, y, x) and x of ``path/ex.nc`` as float32 arrays."""
    fn = os.path.join(path, "ex.nc")
    with open(fn, "rb") as fh:
        head = fh.read(8)
    if head[:4] == b"\x89HDF":
        raise NotImplementedError(f"{fn} is netCDF-4 (HDF5); convert it to netCDF-3 (e.g. nccopy -k classic)")
    from scipy.io import netcdf_file
    with netcdf_file(fn, "r", mmap=False) as nc:
        thk = np.array(nc.variables["thk"][:], dtype=np.float32)
        usurf = np.array(nc.variables["usurf"][:], dtype=np.float32)
        x = np.array(nc.variables["x"][:], dtype=np.float64)
    if thk.ndim == 2:
        thk, usurf = thk[None], usurf[None]
    return thk, usurf, x


def _aug(M, ri):
    """pretraining.py:550-559 on [batch, y, x]: ri[0] quarter turns
    counter-clockwise (tf.image.rot90), then a left-right flip, an up-down
    flip and a transpose where ri[1], ri[2], ri[3] are 1."""
    for _ in range(int(ri[0])):
        M = np.rot90(M, 1, axes=(1, 2))
    if ri[1] == 1:
        M = M[:, :, ::-1]
    if ri[2] == 1:
        M = M[:, ::-1, :]
    if ri[3] == 1:
        M = np.swapaxes(M, 1, 2)
    return np.ascontiguousarray(M)


def par_list(pt, test_paths):
    """state.PAR of pretraining.py:55-73: [path, time slice, arrhenius,
    slidingco, coarsening exponent] per test case."""
    par = []
    mid_a = 0.5 * pt.min_arrhenius + 0.5 * pt.max_arrhenius
    mid_c = 0.5 * pt.min_slidingco + 0.5 * pt.max_slidingco
    for p in test_paths:
        par.append([p, 3, mid_a, mid_c, pt.min_coarsen])
        if pt.min_arrhenius < pt.max_arrhenius:
            par.append([p, 3, 0.25 * pt.min_arrhenius + 0.75 * pt.max_arrhenius, mid_c, pt.min_coarsen])
            par.append([p, 3, 0.75 * pt.min_arrhenius + 0.25 * pt.max_arrhenius, mid_c, pt.min_coarsen])
        if pt.min_slidingco < pt.max_slidingco:
            par.append([p, 3, mid_a, 0.25 * pt.min_slidingco + 0.75 * pt.max_slidingco, pt.min_coarsen])
            par.append([p, 3, mid_a, 0.75 * pt.min_slidingco + 0.25 * pt.max_slidingco, pt.min_coarsen])
        if pt.min_coarsen < pt.max_coarsen:
            par.append([p, 3, mid_a, mid_c, pt.min_coarsen + 1])
    return par


def learning_rate(cfg, epoch):
    """The rate set after epoch ``epoch`` (pretraining.py:341-345)."""
    lr = float(cfg.processes.iceflow.emulator.lr)
    restart = int(cfg.processes.pretraining.train_iceflow_emulator_restart_lr)
    if restart > 0:
        return lr * 0.9 ** ((epoch % restart) / 100)
    return lr * 0.9 ** (epoch / 100)


def _code(par):
    p, it, a, c, r = par
    return f"{p.split('/')[-1]}_{it}_A{int(a)}_C{int(c * 100) / 100}_R{int(r)}"


def _device_fields(thk, usurf, val_a, val_c, device):
    t = torch.as_tensor(np.ascontiguousarray(thk, dtype=np.float32), device=device)
    u = torch.as_tensor(np.ascontiguousarray(usurf, dtype=np.float32), device=device)
    return [t, u, torch.full_like(t, float(val_a)), torch.full_like(t, float(val_c))]


def compute_solutions(cfg, state):
    """pretraining.py:108-195: the plain solver's velocities of every test
    case (from zero, the solver's own settings), with its cost history in
    <direct_name>/<case>/costs-stokes.dat."""
    ic = cfg.processes.iceflow
    state.solutions, state.solutions_cost = [], []
    solver = DeviceAdamSolver(lr=float(ic.solver.step_size))
    phys = P.physics(cfg)
    dev = torch.device("cuda", torch.cuda.current_device())
    for par in state.PAR:
        p, it, val_a, val_c, val_r = par
        co = int(2 ** val_r)
        thk, usurf, x = _read_ex(p)
        f = _device_fields(thk[it, ::co, ::co], usurf[it, ::co, ::co], val_a, val_c, dev)
        resol = float((x[1] - x[0]) * co)
        Z = torch.zeros((ic.numerics.Nz,) + tuple(f[0].shape), dtype=torch.float32, device=dev)
        U, V, costs = solver.solve(Z, Z, *f, resol, state.dzeta, nbitmax=int(ic.solver.nbitmax), phys=phys,
                                   relative_min_delta=0.0002, patience=10,
                                   early_stopping=bool(ic.solver.get("early_stopping", True)))
        path = os.path.join(state.direct_name, _code(par))
        os.makedirs(path, exist_ok=True)
        np.savetxt(os.path.join(path, "costs-stokes.dat"), np.stack(costs), fmt="%.5f")
        state.solutions.append([(f, resol), (U, V)])
        state.solutions_cost.append(float(costs[-1]))


def _normp(dz, u, v, p):
    """_computenormp (pretraining.py:496-499)."""
    return float(np.sum(dz * (np.abs(u) ** p + np.abs(v) ** p))) ** (1 / p)


def misfits(cfg, state, thk, U, V, Up, Vp):
    """_computemisfitall (pretraining.py:502-536): relative L1 and L2 of the
    layer-averaged velocities weighted by the layer thickness, and the L1
    velbar misfit where thk > 1 (returned twice, as the reference does)."""
    nz = cfg.processes.iceflow.numerics.Nz
    sp = cfg.processes.iceflow.numerics.vert_spacing
    zeta = np.arange(nz) / (nz - 1)
    temp = (zeta / sp) * (1.0 + (sp - 1.0) * zeta)
    temp = temp[1:] - temp[:-1]
    th = thk.astype(np.float64)
    dz = np.stack([th * z for z in temp])
    w = np.asarray(state.vert_weight, np.float64)
    du, dv = (U - Up).astype(np.float64), (V - Vp).astype(np.float64)
    ub, vb = (du * w).sum(0), (dv * w).sum(0)
    ma = (th > 1).astype(np.float64)
    nb = ma.sum()
    l1bar = float((ma * np.abs(ub)).sum() + (ma * np.abs(vb)).sum()) / max(2 * nb, 1.0)
    av = lambda a: 0.5 * (a[1:] + a[:-1])  # noqa: E731
    ut, up, vt, vp = av(U.astype(np.float64)), av(Up.astype(np.float64)), av(V.astype(np.float64)), av(
        Vp.astype(np.float64))
    n1 = _normp(dz, ut - up, vt - vp, 1.0) / max(_normp(dz, ut, vt, 1.0), 1e-300)
    n2 = _normp(dz, ut - up, vt - vp, 2.0) / max(_normp(dz, ut, vt, 2.0), 1e-300)
    return n1, n2, l1bar, l1bar


def _save(net, path, init="glorot_uniform"):
    """The network at ``path`` (``.npz``: the exact parameters with their
    input and output scales and the Adam state, which this package's loader
    reads) and beside it, under the same name with ``.h5``, the Keras model
    file the reference writes (pretraining.py:350-351, 491-492): the network
    on raw fields, which the reference's emulator loads."""
    from ..emulator import keras_variables
    from ..keras_h5 import write_keras_cnn
    np.savez(path, params=net.params.cpu().numpy(), adam_m=net.m.cpu().numpy(), adam_v=net.v.cpu().numpy(),
             iterations=np.array(net.opt_iterations), nb_layers=np.array(net.L), nout=np.array(net.nout),
             cin=np.array(net.cin), scales=net.scales, out_scale=np.array(net.out_scale))
    write_keras_cnn(os.path.splitext(path)[0] + ".h5", keras_variables(net), net.L, net.cin, net.nout,
                    alpha=net.alpha, init=init)


def train_iceflow_emulator(cfg, state, trainingset, augmentation=True):
    """pretraining.py:198-494."""
    ic = cfg.processes.iceflow
    pt = cfg.processes.pretraining
    e = ic.emulator
    nz = int(ic.numerics.Nz)
    init = str(e.network.weight_initialization)
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(int(pt.get("seed", 0)))
    net = CNN(nb_layers=int(e.network.nb_layers), cin=len(e.fieldin), nout=2 * nz,
              init=e.network.weight_initialization, seed=int(e.get("seed", 0)),
              scales=list(e.get("input_scales", [1.0] * 5)), nb_out_filter=int(e.network.nb_out_filter),
              out_scale=float(e.get("output_scale", 1.0)), device=dev)
    if os.path.exists("model0.h5"):
        from ..keras_h5 import cnn_params_from_keras, read_keras_weights
        net.set_params(cnn_params_from_keras(read_keras_weights("model0.h5"), net.L, net.cin, net.nout))
        net.scales = np.ones(5, np.float32)
        net.out_scale = 1.0
    # the reference's optimizer here is a plain Adam (no clipnorm)
    opt = EmulatorOptimizer(float(e.lr), 1e-7, 0.0)
    lr = float(e.lr)
    phys = P.physics(cfg)
    state.MISFIT, state.MISFIT_CO = [], []
    epochs = int(pt.epochs)
    save_every = max(1, epochs // 5)
    for epoch in range(epochs):
        nsub = list(trainingset)
        rng.shuffle(nsub)
        for p in nsub:
            thk, usurf, x = _read_ex(p)
            rec = thk.shape[0]
            bs = int(pt.batch_size)
            st = max(rec // bs, 1)
            it = int(rng.integers(0, st))
            ri = rng.integers(0, [4, 2, 2, 2]) if augmentation else np.zeros(4, int)
            if pt.soft_begining > 0 and pt.soft_begining < epoch:
                co = int(2 ** int(rng.integers(int(pt.min_coarsen), max(int(pt.max_coarsen), int(pt.min_coarsen) + 1))))
                val_a = float(rng.uniform(pt.min_arrhenius, pt.max_arrhenius))
                val_c = float(rng.uniform(pt.min_slidingco, pt.max_slidingco))
            else:
                co = int(2 ** int(pt.min_coarsen))
                val_a = 0.5 * (pt.min_arrhenius + pt.max_arrhenius)
                val_c = 0.5 * (pt.min_slidingco + pt.max_slidingco)
            tb = _aug(thk[it::st, ::co, ::co], ri)[:bs]
            ub = _aug(usurf[it::st, ::co, ::co], ri)[:bs]
            f = _device_fields(tb[0], ub[0], val_a, val_c, dev)
            ny, nx = f[0].shape
            train_step(net, f, float((x[1] - x[0]) * co), [(0, 0)], ny, nx, state.dzeta, phys, lr, opt)
        lr = learning_rate(cfg, epoch)
        if epoch % save_every == 0:
            _save(net, os.path.join(state.direct_name, f"model-{epoch}.npz"), init)
        if epoch % int(pt.freq_test) == 0:
            mis, mis_co = [], []
            for par, (fx, (U, V)), cost0 in zip(state.PAR, state.solutions, state.solutions_cost):
                (f, resol) = fx
                ny, nx = f[0].shape
                buf = net.buffers(1, ny, nx, train=False)
                net.prepare_input(f, resol, [(0, 0)], ny, nx, buf)
                Up, Vp = net.forward(buf, 1, ny, nx)
                Up, Vp = Up[0].clone(), Vp[0].clone()
                terms = K.energy(Up, Vp, *f, resol, state.dzeta, phys)[0]
                cost = float(terms.sum().item()) / ((ny - 1) * (nx - 1))
                n1, n2, nb1, nb1a = misfits(cfg, state, f[0].cpu().numpy(), U.cpu().numpy(), V.cpu().numpy(),
                                            Up.cpu().numpy(), Vp.cpu().numpy())
                mis.append(nb1)
                mis_co.append(cost - cost0)
                print(" TEST :", epoch, _code(par), n1, n2, nb1, nb1a, mis_co[-1], lr)
                path = os.path.join(state.direct_name, _code(par))
                with open(os.path.join(path, "misfit-pinn.dat"), "a") as fid:
                    fid.write("%.0f %.4f %.4f %.4f %.4f %.4f \n" % (epoch, n1, n2, nb1, nb1a, mis_co[-1]))
            state.MISFIT.append(mis)
            state.MISFIT_CO.append(mis_co)
    net.check_errors()
    state.MISFIT = np.stack(state.MISFIT) if state.MISFIT else np.zeros((0, len(state.PAR)))
    state.MISFIT_CO = np.stack(state.MISFIT_CO) if state.MISFIT_CO else np.zeros((0, len(state.PAR)))
    _save(net, os.path.join(state.direct_name, "model.npz"), init)
    state.iceflow_model = net


def initialize(cfg, state):
    """pretraining.py:25-97 (Lagrange basis)."""
    ic = cfg.processes.iceflow
    if ic.numerics.vert_basis != "Lagrange":
        raise NotImplementedError(f"vert_basis={ic.numerics.vert_basis!r}: only the Lagrange basis is supported")
    pt = cfg.processes.pretraining
    state.direct_name = _direct_name(cfg)
    os.makedirs(state.direct_name, exist_ok=True)
    _, train_paths = _findsubdata(os.path.join(pt.data_dir, "train"))
    _, test_paths = _findsubdata(os.path.join(pt.data_dir, "test"))
    state.PAR = par_list(pt, test_paths)
    levels = compute_levels(ic.numerics.Nz, ic.numerics.vert_spacing)
    state.zeta, state.dzeta = compute_zeta_dzeta(levels)
    state.vert_weight = define_vertical_weight(ic.numerics.Nz, ic.numerics.vert_spacing)
    state.Leg_P, state.Leg_dPdz, state.Leg_I = None, None, None
    state.it = 0
    compute_solutions(cfg, state)
    train_iceflow_emulator(cfg, state, train_paths)
    print("pretraining done, the code stop here, as the emulator is trained")
    print("pretraining can not be followed with a run now.")
    sys.exit()


def update(cfg, state):
    pass


def finalize(cfg, state):
    pass
