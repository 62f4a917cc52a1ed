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
