"""What the trained network gains over the method without it.

On a small valley glacier (48 x 64 cells, dx 100 m, Nz 6, log-uniform A and
c) the converged FP64 minimiser of the energy (igm_b200.judge, grid-sequenced
L-BFGS) is the yardstick.  An emulator network (8 layers of 3x3 x 32
filters, He-initialised) is trained physics-informed on the state --
whole-domain Adam steps on the Blatter-Pattyn energy, the loss of
update_iceflow_emulator (igm/processes/iceflow/emulate/emulate.py:155-281).

* Training gain: after 400 steps the network's velocity error against the
  yardstick (relative L2 of the staggered velocities over ice cells) is at
  most a quarter of the untrained network's, and its energy gap to the
  minimum at most a tenth (measured: about a twentieth; the trajectory
  depends on the reduction order of the bias gradients, hence the margin).
* Gain over the plain method: the reference's solver (Adam at lr 1,
  solve.py:22-119) run for 30 iterations from the trained network's
  velocities ends at an energy gap at most a fifth of the one it reaches in
  30 iterations from zero velocities, the start the plain method has without
  an emulator -- and at a smaller velocity error.
"""

import numpy as np
import pytest
import torch

from igm_b200 import judge as J
from igm_b200 import kernels as K
from igm_b200.cnn import CNN
from igm_b200.emulator import EmulatorOptimizer, train_step
from igm_b200.solver import DeviceAdamSolver
from igm_b200.vertical import compute_levels, compute_zeta_dzeta
from oracle import iceflow_oracle as O

pytestmark = pytest.mark.gpu

NZ, DX = 6, 100.0
SCALES = [1 / 300.0, 1 / 3000.0, 1 / 100.0, 10.0, 1 / 100.0]


def test_training_and_warm_start_gain():
    g = O.valley_glacier(48, 64, DX, seed=3, varying_coeffs=True)
    f = [torch.as_tensor(g[k]).cuda() for k in ("thk", "usurf", "arrhenius", "slidingco")]
    ny, nx = f[0].shape
    dz = compute_zeta_dzeta(compute_levels(NZ, 4.0))[1]
    ns = (ny - 1) * (nx - 1)
    Ur, Vr, rec = J.converged_velocity(*f, DX, dz, levels=3, iters=(3000, 3000, 3000))
    f64 = [t.double() for t in f]

    def energy(U, V):
        return float(K.energy(U.double(), V.double(), *f64, DX, dz)[0].sum()) / ns

    e_min = energy(Ur, Vr)

    def judge(U, V):
        return J.velocity_rel_l2(U, V, Ur, Vr, f[0]), (energy(U, V) - e_min) / abs(e_min)

    net = CNN(nb_layers=8, cin=5, nout=2 * NZ, init="he_normal", seed=4, scales=SCALES, out_scale=100.0)
    net.init_weights("he_normal", 4, head_gain=0.1)

    def emulate():
        buf = net.buffers(1, ny, nx, train=False)
        net.prepare_input(f, DX, [(0, 0)], ny, nx, buf)
        U, V = net.forward(buf, 1, ny, nx, thk_mask=f[0])
        return U[0].clone(), V[0].clone()

    err0, gap0 = judge(*emulate())
    opt = EmulatorOptimizer(1e-3, 1e-7, 1.0)
    for i in range(400):
        train_step(net, f, DX, [(0, 0)], ny, nx, dz, None, 1e-3 if i < 300 else 3e-4, opt)
    net.check_errors()
    Ue, Ve = emulate()
    err1, gap1 = judge(Ue, Ve)
    print(f"yardstick: {rec}")
    print(f"untrained: vel err {err0:.3e}, energy gap {gap0:.3e}; trained: vel err {err1:.3e}, gap {gap1:.3e}")
    assert err1 <= 0.25 * err0, (err0, err1)
    assert gap1 <= 0.1 * gap0, (gap0, gap1)

    Z = torch.zeros_like(Ue)
    Us, Vs, _ = DeviceAdamSolver(lr=1.0).solve(Ue, Ve, *f, DX, dz, nbitmax=30, early_stopping=False)
    Uz, Vz, _ = DeviceAdamSolver(lr=1.0).solve(Z, Z, *f, DX, dz, nbitmax=30, early_stopping=False)
    err_s, gap_s = judge(Us, Vs)
    err_z, gap_z = judge(Uz, Vz)
    print(f"30 solver iterations from the emulator: err {err_s:.3e}, gap {gap_s:.3e}; "
          f"from zero: err {err_z:.3e}, gap {gap_z:.3e}")
    assert gap_s <= 0.2 * gap_z, (gap_s, gap_z)
    assert err_s < err_z, (err_s, err_z)
