"""The transport and vertical-velocity kernels divide with Markstein's step
from the divisor's correctly rounded reciprocal (q = RN(a y), r = a - d q
exact, RN(q + r y)); the reference divides in IEEE arithmetic.  Checked here
on the CPU with exact rational arithmetic for the two fused steps, against
numpy's IEEE division, for the grid spacings and the per-layer weight sums in
use and numerators across the range the kernels see."""

from fractions import Fraction

import numpy as np
import pytest


def rn32(x: Fraction) -> np.float32:
    """Round an exact rational to the nearest float32, ties to even."""
    c = np.float32(float(x))  # within one float32 ulp of x
    best = None
    for cand in (np.nextafter(c, np.float32(-np.inf)), c, np.nextafter(c, np.float32(np.inf))):
        d = abs(Fraction(float(cand)) - x)
        key = (d, int(np.frombuffer(np.float32(cand).tobytes(), np.uint32)[0]) & 1)
        if best is None or key < best[0]:
            best = (key, np.float32(cand))
    return best[1]


def markstein_div(a: np.float32, dx: np.float32, rdx: np.float32) -> np.float32:
    if a == 0:
        return a
    q = np.float32(a * rdx)
    r = rn32(Fraction(float(a)) - Fraction(float(dx)) * Fraction(float(q)))
    return rn32(Fraction(float(q)) + Fraction(float(r)) * Fraction(float(rdx)))


@pytest.mark.parametrize("dx", [25.0, 50.0, 100.0, 250.0, 37.5, 1000.0 / 3.0])
def test_markstein_division_matches_ieee(dx):
    rng = np.random.default_rng(int(dx * 7))
    dx32 = np.float32(dx)
    rdx = np.float32(np.float32(1.0) / dx32)
    mag = 10.0 ** rng.uniform(-20, 6, size=4000)
    a = (mag * rng.choice([-1.0, 1.0], size=mag.size)).astype(np.float32)
    # thickness differences and small integers as well
    a = np.concatenate([a, np.arange(-300, 301, dtype=np.float32), (np.float32(dx) * np.arange(1, 50)).astype(np.float32)])
    for v in a:
        want = np.float32(v) / dx32
        got = markstein_div(np.float32(v), dx32, rdx)
        assert np.float32(got).tobytes() == np.float32(want).tobytes(), (v, dx, got, want)


def test_zero_numerator_keeps_sign():
    dx32 = np.float32(50.0)
    rdx = np.float32(1.0) / dx32
    for z in (np.float32(0.0), np.float32(-0.0)):
        assert np.float32(markstein_div(z, dx32, rdx)).tobytes() == (z / dx32).tobytes()


def markstein_div64(a: float, b: float, rb: float) -> float:
    """The same three steps in float64 (Fraction -> float rounds to nearest)."""
    if a == 0:
        return a
    q = a * rb
    r = float(Fraction(a) - Fraction(b) * Fraction(q))
    return float(Fraction(q) + Fraction(r) * Fraction(rb))


@pytest.mark.parametrize("nz,spacing", [(2, 1.0), (5, 1.0), (10, 4.0), (16, 4.0), (30, 2.0), (64, 4.0)])
def test_markstein_division_by_cumulative_weights(nz, spacing):
    """The vertical-velocity kernel divides the running weighted sums of U, V
    by the running sum of the vertical weights (one divisor per layer) with the
    same step from that divisor's correctly rounded reciprocal; checked against
    IEEE division in float32 and float64 for those divisors."""
    from igm_b200.vertical import define_vertical_weight
    w = define_vertical_weight(nz, spacing)[:, 0, 0]
    sums32, s = [], np.float32(0)
    for k in range(nz):
        s = w[0] if k == 0 else np.float32(s + w[k])
        sums32.append(np.float32(s))
    rng = np.random.default_rng(nz)
    mag = 10.0 ** rng.uniform(-8, 6, size=1500)
    a = mag * rng.choice([-1.0, 1.0], size=mag.size)
    for b32 in sums32:
        rb32 = np.float32(np.float32(1.0) / b32)
        b64 = float(b32)
        rb64 = 1.0 / b64
        for v in a:
            v32 = np.float32(v)
            got = markstein_div(v32, b32, rb32)
            assert np.float32(got).tobytes() == np.float32(v32 / b32).tobytes(), (v32, b32)
            assert markstein_div64(float(v), b64, rb64) == float(v) / b64, (v, b64)
