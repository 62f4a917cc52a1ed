"""Synthetic glaciers with the shapes and value distributions of the
benchmark workloads: inputs for the benchmark, the tests and the smoke run.
(Input generators only; nothing here is part of the ice-flow computation.)"""

from __future__ import annotations

import numpy as np


def box_filter(a: np.ndarray, k: int = 5) -> np.ndarray:
    """k x k moving average with edge replication."""
    r = k // 2
    p = np.pad(a, r, mode="edge")
    c = np.cumsum(np.cumsum(p, 0), 1)
    c = np.pad(c, ((1, 0), (1, 0)))
    return (c[k:, k:] - c[:-k, k:] - c[k:, :-k] + c[:-k, :-k]) / (k * k)


def valley_glacier(ny=100, nx=100, dx=100.0, seed=0, noise_sigma=5.0, varying_coeffs=False):
    """Synthetic valley glacier.

    The 10 km x 10 km valley of the 100x100 / dx=100 m case; larger grids map
    their domain onto the same shape (coordinates scaled to 10 km), and the
    bed noise is scaled with dx/100 m so its slope stays the same.
    Bed: 3000 - 0.1 X + 0.002 (Y-5000)^2 + N(0, sigma^2);
    thk = max(0, 300 (1-((Y-5000)/2500)^2) (1-X/10000)); usurf = topg + thk.
    A = 78, c = 0.045 uniform, or (``varying_coeffs``) log-uniform per cell
    in [20,150] and [0.01,0.1], smoothed with a 5-cell box filter.
    Returns float32 numpy arrays.
    """
    rng = np.random.default_rng(seed)
    Lx, Ly = nx * dx, ny * dx
    x = np.arange(nx) * dx * (10000.0 / Lx)
    y = np.arange(ny) * dx * (10000.0 / Ly)
    X, Y = np.meshgrid(x, y)
    sigma = noise_sigma * (dx / 100.0) if (nx, ny) != (100, 100) else noise_sigma
    topg = 3000.0 - 0.1 * X + 0.002 * (Y - 5000.0) ** 2 + rng.normal(0.0, sigma, size=(ny, nx))
    thk = np.maximum(0.0, 300.0 * (1.0 - ((Y - 5000.0) / 2500.0) ** 2) * (1.0 - X / 10000.0))
    usurf = topg + thk
    if varying_coeffs:
        A = np.exp(rng.uniform(np.log(20.0), np.log(150.0), size=(ny, nx)))
        c = np.exp(rng.uniform(np.log(0.01), np.log(0.1), size=(ny, nx)))
        A = box_filter(A, 5)
        c = box_filter(c, 5)
    else:
        A = np.full((ny, nx), 78.0)
        c = np.full((ny, nx), 0.045)
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return dict(topg=f(topg), thk=f(thk), usurf=f(usurf), arrhenius=f(A), slidingco=f(c), dx=float(dx))


def ridge_glacier(n=4096, dx=25.0, seed=0, n_ridges=12):
    """Multi-valley bed: a 0.05-slope plane plus seeded Gaussian ridges
    (height 500-1500 m, sigma 2-8 km).  thk starts at zero (the caller spins
    it up).  A, c log-uniform per cell as in ``valley_glacier``."""
    rng = np.random.default_rng(seed)
    x = np.arange(n) * dx
    X, Y = np.meshgrid(x, x)
    topg = 3500.0 - 0.05 * X
    for _ in range(n_ridges):
        cx, cy = rng.uniform(0, n * dx, size=2)
        h = rng.uniform(500.0, 1500.0)
        s = rng.uniform(2000.0, 8000.0)
        topg = topg + h * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    A = box_filter(np.exp(rng.uniform(np.log(20.0), np.log(150.0), size=(n, n))), 5)
    c = box_filter(np.exp(rng.uniform(np.log(0.01), np.log(0.1), size=(n, n))), 5)
    thk = np.zeros((n, n))
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return dict(topg=f(topg), thk=f(thk), usurf=f(topg), arrhenius=f(A), slidingco=f(c), dx=float(dx))


def tongue_glacier(ny=40, nx=70, dx=100.0, seed=3):
    """Glacier tongue for thickness inversions: a 0.05-slope plane bed with a
    transverse undulation (amplitude 20 m, wavelength 1.41 Ly) and a
    parabolic-in-y, linearly thinning-in-x tongue centred on the domain, half
    width 0.375 Ly, vanishing at 1.07 Lx, maximum thickness 180 sqrt(Ly / 4 km)
    m (Lx = nx dx, Ly = ny dx).  A, c log-uniform per cell in [20, 150] and
    [0.01, 0.1], smoothed with a 5-cell box filter.  Returns float32 arrays
    plus x, y coordinates."""
    x, y = np.arange(nx) * dx, np.arange(ny) * dx
    X, Y = np.meshgrid(x, y)
    Lx, Ly = nx * dx, ny * dx
    topg = 2000.0 - 0.05 * X + 20.0 * np.sin(Y * (4000.0 / 900.0) / Ly)
    hmax = 180.0 * np.sqrt(Ly / 4000.0)
    thk = np.maximum(0.0, hmax * (1 - ((Y - 0.5 * Ly) / (0.375 * Ly)) ** 2) * (1 - X / (Lx * 7500.0 / 7000.0)))
    rng = np.random.default_rng(seed)
    A = box_filter(np.exp(rng.uniform(np.log(20.0), np.log(150.0), (ny, nx))), 5)
    c = box_filter(np.exp(rng.uniform(np.log(0.01), np.log(0.1), (ny, nx))), 5)
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return dict(topg=f(topg), thk=f(thk), usurf=f(topg + thk), arrhenius=f(A), slidingco=f(c), dx=float(dx), x=f(x),
                y=f(y))
