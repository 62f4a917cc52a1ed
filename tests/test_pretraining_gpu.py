"""The pretraining process end to end on the device (igm_b200/processes/
pretraining.py against igm/processes/pretraining/pretraining.py:25-494), on
a small library of synthetic valley glaciers written as netCDF-3 ex.nc
files: the test cases are solved by the plain solver (their cost histories
written), the emulator trains for 12 epochs over two training sets with
augmentation, coarsening and random arrhenius / slidingco after the soft
beginning, the test misfits are written every 4 epochs, the models are
saved, and initialize ends the program as the reference's does.  The
training must lower the emulator's energy gap to the solved test cases."""

import os

import numpy as np
import pytest
import torch

from igm_b200.config import default_cfg
from igm_b200.state import State
from igm_b200.synthetic import valley_glacier

pytestmark = pytest.mark.gpu


def write_ex(path, seed, ny=40, nx=48, nt=5):
    from scipy.io import netcdf_file
    os.makedirs(path, exist_ok=True)
    thk, usurf = [], []
    for t in range(nt):
        g = valley_glacier(ny, nx, 100.0, seed=seed)
        s = 1.0 - 0.08 * t  # a thinning glacier
        thk.append(g["thk"] * s)
        usurf.append(g["topg"] + g["thk"] * s)
    with netcdf_file(os.path.join(path, "ex.nc"), "w") as nc:
        nc.createDimension("time", nt)
        nc.createDimension("y", ny)
        nc.createDimension("x", nx)
        nc.createVariable("x", "f4", ("x",))[:] = np.arange(nx) * 100.0
        nc.createVariable("y", "f4", ("y",))[:] = np.arange(ny) * 100.0
        nc.createVariable("thk", "f4", ("time", "y", "x"))[:] = np.stack(thk)
        nc.createVariable("usurf", "f4", ("time", "y", "x"))[:] = np.stack(usurf)


def test_pretraining_process(tmp_path, monkeypatch):
    from igm_b200.processes import pretraining as PT
    monkeypatch.chdir(tmp_path)
    for i, sub in enumerate(["train/g1", "train/g2", "test/t1"]):
        write_ex(str(tmp_path / "lib" / sub), seed=i)
    cfg = default_cfg({"iceflow": {"numerics": {"Nz": 4}, "solver": {"nbitmax": 300},
                                   "emulator": {"lr": 1e-3, "network": {"nb_layers": 3,
                                                                        "weight_initialization": "he_normal"},
                                                "input_scales": [1 / 300.0, 1 / 3000.0, 1 / 100.0, 10.0, 1 / 100.0],
                                                "output_scale": 50.0}},
                       "pretraining": {"data_dir": str(tmp_path / "lib"), "epochs": 12, "freq_test": 4,
                                       "soft_begining": 4, "min_arrhenius": 50.0, "max_arrhenius": 100.0,
                                       "min_slidingco": 0.02, "max_slidingco": 0.06, "min_coarsen": 0,
                                       "max_coarsen": 1}})
    st = State()
    with pytest.raises(SystemExit):
        PT.initialize(cfg, st)
    d = tmp_path / st.direct_name
    assert st.direct_name == "pinnbp_4_4_cnn_3_32_2_1"
    assert len(st.PAR) == 6 and len(st.solutions) == 6
    for par in st.PAR:
        case = d / PT._code(par)
        assert (case / "costs-stokes.dat").exists()
        rows = np.loadtxt(case / "misfit-pinn.dat", ndmin=2)
        assert rows.shape == (3, 6) and list(rows[:, 0]) == [0, 4, 8]
    for f in ("model", "model-0", "model-2", "model-10"):
        assert (d / (f + ".npz")).exists() and (d / (f + ".h5")).exists(), f
    assert st.MISFIT.shape == (3, 6) and st.MISFIT_CO.shape == (3, 6)
    # the energy gap of the emulator to the solved test cases shrinks with training
    gap = st.MISFIT_CO.mean(1)
    print("mean energy gap at the tests:", gap, "velbar L1 misfit:", st.MISFIT.mean(1))
    assert np.all(np.isfinite(st.MISFIT)) and gap[-1] < gap[0]
    saved = np.load(d / "model.npz")
    assert torch.equal(torch.as_tensor(saved["params"]), st.iceflow_model.params.cpu())
