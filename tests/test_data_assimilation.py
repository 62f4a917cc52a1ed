"""Host side of the data_assimilation process: the observation-density
weights of optimize_initialize against the oracle, and the configurations
that raise."""

import numpy as np
import pytest
import torch

from igm_b200.config import default_cfg
from igm_b200.processes import data_assimilation as DA
from oracle import iceflow_oracle as O


def _glacier(ny=40, nx=70, dx=100.0):
    x, y = np.arange(nx) * dx, np.arange(ny) * dx
    X, Y = np.meshgrid(x, y)
    return np.maximum(0.0, 180.0 * (1 - ((Y - 2000.0) / 1500.0) ** 2) * (1 - X / 7500.0)).astype(np.float32)


@pytest.mark.parametrize("seed,frac", [(0, 0.07), (1, 0.0), (2, 1.0)])
def test_density_weights_match_oracle(seed, frac):
    thk = _glacier()
    tob = np.full_like(thk, np.nan)
    rng = np.random.default_rng(seed)
    pick = rng.random(tob.shape) < frac
    tob[pick] = thk[pick]
    tob[:, 12] = thk[:, 12]
    ours = DA._density_weights(tob, True)
    ref = O.da_density_weights(torch.as_tensor(tob)).numpy()
    np.testing.assert_allclose(ours, ref, rtol=1e-6, atol=1e-7)
    np.testing.assert_array_equal(DA._density_weights(tob, False), np.ones_like(tob))


def test_density_matrix_counts():
    m = np.full((6, 9), np.nan, dtype=np.float32)
    m[0, 0] = 1.0
    m[3, 4] = 2.0
    c = DA.create_density_matrix(m, 5)
    ref = O.create_density_matrix(torch.as_tensor(m), 5).numpy()
    np.testing.assert_array_equal(c, ref)
    assert c[0, 0] == 1 and c[2, 2] == 2 and c[5, 8] == 0


def test_unsupported_configurations_raise():
    for over in ({"control_list": ["thk", "topg"]}, {"control_list": ["thk", "thk"]}, {"cost_list": ["velsurf", "vol"]}, {"divflux": {"method": "flux-limiter"}},
                 {"optimization": {"method": "L-BFGS"}}, {"cook": {"infer_params": True}}):
        cfg = default_cfg({"data_assimilation": over})
        with pytest.raises(NotImplementedError):
            DA._check_supported(cfg)


def _fake(**kw):
    import types
    return types.SimpleNamespace(**kw)


def test_control_update_settings_per_control():
    """Transform, gradient mask and reprojection of each control
    (optimize/update.py:23-27, 58-68, 84-98)."""
    a = _fake(reproject=True, log_slidingco=False, params=_fake(sole_mask=0), cost_list=["velsurf", "icemask"])
    kw = lambda c: DA._Assim.control_kw(a, c)  # noqa: E731
    assert kw("thk") == dict(transform=0, mask=1, reproject=1, lower=0.0, reproject_mask=True)
    assert kw("slidingco") == dict(transform=0, mask=0, reproject=2, lower=0.0, reproject_mask=True)
    assert kw("arrhenius") == dict(transform=0, mask=1, reproject=2, lower=1.0, reproject_mask=True)
    assert kw("usurf") == dict(transform=0, mask=1, reproject=0, lower=0.0, reproject_mask=True)
    a.log_slidingco, a.params.sole_mask, a.reproject, a.cost_list = True, 1, False, ["velsurf"]
    assert kw("slidingco") == dict(transform=1, mask=2, reproject=0, lower=0.0, reproject_mask=False)
    assert kw("thk")["reproject"] == 0


def test_cost_table_follows_total_cost_order():
    """costs.dat columns: total_cost.py's dictionary order over the terms present."""
    n = 3
    hist = torch.arange(n * 6, dtype=torch.float64).reshape(n, 6)  # velsurf thk icemask thk_positive thk_regu usurf
    field = torch.zeros((n, 6), dtype=torch.float64)
    field[:, 3], field[:, 4] = 100.0, 200.0
    present = {"velsurf": True, "thk": True, "usurf": True, "icemask": True, "thk_positive": True,
               "slidingco_positive": True, "arrhenius_positive": False, "thk_regu": True, "slid_regu": True,
               "arrh_regu": False}
    a = _fake(cost_hist=hist, present=present, div_kind="obs", div_hist=torch.full((n,), 7.0, dtype=torch.float64),
              field_hist={"slidingco": field})
    keys, table = DA._cost_table(a, n)
    assert keys == ["velsurf", "thk", "divflux", "usurf", "icemask", "thk_positive", "slidingco_positive",
                    "thk_regu", "slid_regu"]
    np.testing.assert_array_equal(table[1], [6, 7, 7.0, 11, 8, 9, 100.0, 10, 200.0])
