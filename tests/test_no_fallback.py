"""The product path has no CPU fallback: without the built library every
kernel call raises, and host (CPU) tensors are refused before any launch."""

import pytest
import torch

from igm_b200 import _lib as L
from igm_b200 import kernels as K


def test_missing_library_raises(monkeypatch, tmp_path):
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "libigmb200.so"))
    monkeypatch.setattr(L, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        L.lib()
    h = torch.ones(8, 8)
    with pytest.raises(RuntimeError, match="not found"):
        K.divflux(h, h, h, 100.0)


def test_host_tensors_are_refused():
    from igm_b200.build import build
    build()
    h = torch.ones(8, 8)
    with pytest.raises(ValueError, match="CUDA tensor"):
        K.divflux(h, h, h, 100.0)
    with pytest.raises(ValueError, match="CUDA tensor"):
        K.transport_step(h, h, h, torch.zeros(8, 8), torch.zeros(8, 8), 100.0, 1.0)
