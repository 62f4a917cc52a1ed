"""Host side of the emulator's retraining: the patch split of
split_into_patches and pertubate_X's choice of fields and copies."""

import numpy as np
import torch

from igm_b200.config import default_cfg
from oracle import iceflow_oracle as O


def test_pertubate_field_selection():
    """pertubate_X's copies: thk and usurf without data assimilation, the
    controls with it; each scaled copy stacked along y."""
    from igm_b200 import emulator as E
    f = [torch.full((2, 3), float(k + 1)) for k in range(4)]
    st, n = E._pertubate_fields(default_cfg(), f)
    assert n == 5 and st[0].shape == (10, 3)
    np.testing.assert_allclose(st[0][:, 0].numpy(), [1, 1, 1.2, 1.2, 0.8, 0.8, 1, 1, 1, 1])
    np.testing.assert_allclose(st[1][:, 0].numpy(), [2, 2, 2, 2, 2, 2, 2.4, 2.4, 1.6, 1.6])
    st, n = E._pertubate_fields(default_cfg({"data_assimilation": {"control_list": ["slidingco"]}}), f)
    assert n == 3
    np.testing.assert_allclose(st[3][:, 0].numpy(), [4, 4, 4.8, 4.8, 3.2, 3.2])
    np.testing.assert_allclose(st[0][:, 0].numpy(), [1] * 6)


def test_patch_windows_follow_split_into_patches():
    """The retraining's patch origins and sizes are those of the oracle's
    split_into_patches (emulate.py:283-308: sy = ny // nbmax + 1 patches of
    int(ny / sy) rows, column-major), for several grid / frame sizes."""
    from igm_b200.emulator import _patch_windows
    for ny, nx, nbmax in ((40, 70, 1000), (1000, 1000, 750), (301, 999, 128), (64, 64, 64), (17, 5, 4)):
        wins, ly, lx = _patch_windows(ny, nx, nbmax)
        X = torch.arange(ny * nx, dtype=torch.float64).reshape(1, ny, nx, 1)
        P = O.split_into_patches(X, nbmax)
        assert P.shape[0] == len(wins) and P.shape[2:4] == (ly, lx)
        for k, (y0, x0) in enumerate(wins):
            np.testing.assert_array_equal(P[k, 0, :, :, 0].numpy(), X[0, y0:y0 + ly, x0:x0 + lx, 0].numpy())
