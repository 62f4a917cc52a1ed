"""The transport kernel divides by dx with Markstein's step from the correctly
rounded reciprocal (q = RN(a y), r = a - dx q exact, RN(q + r y)); the
reference divides in IEEE float32.  Checked here on the CPU with exact rational
arithmetic for the two fused steps, against numpy's IEEE float32 division, for
the grid spacings in use and numerators across the range the transport sees."""

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
