"""Vertical discretisation (igm/processes/iceflow/vert_disc.py:10-47), float32
on the host: a handful of numbers per run."""

from __future__ import annotations

import numpy as np


def compute_levels(Nz: int, vert_spacing: float) -> np.ndarray:
    """zeta_k = k/(Nz-1); level = zeta/s (1 + (s-1) zeta)   (vert_disc.py:10-13)."""
    if Nz > 1:
        zeta = (np.arange(Nz, dtype=np.float64) / (Nz - 1)).astype(np.float32)
    else:
        zeta = np.zeros(1, dtype=np.float32)
    s = np.float32(vert_spacing)
    return (zeta / s) * (np.float32(1.0) + (s - np.float32(1.0)) * zeta)


def compute_zeta_dzeta(levels: np.ndarray):
    """Layer midpoints and thicknesses (vert_disc.py:27-35); (0.5, 1) for Nz = 1."""
    if levels.shape[0] > 1:
        return (levels[1:] + levels[:-1]) / np.float32(2), levels[1:] - levels[:-1]
    return np.full(1, 0.5, np.float32), np.ones(1, np.float32)


def define_vertical_weight(Nz: int, vert_spacing: float) -> np.ndarray:
    """velbar weights from Nz+1 equispaced points through the same map
    (vert_disc.py:43-47), shape [Nz, 1, 1]."""
    zeta = (np.arange(Nz + 1, dtype=np.float64) / Nz).astype(np.float32)
    s = np.float32(vert_spacing)
    w = (zeta / s) * (np.float32(1.0) + (s - np.float32(1.0)) * zeta)
    return (w[1:] - w[:-1])[:, None, None]
