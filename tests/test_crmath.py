"""The correctly rounded sin/cos shared by the device kernels and the oracle's CR flavour."""
import math
import random

import pytest

mpmath = pytest.importorskip("mpmath")


def _cr(f, x):
    with mpmath.workprec(300):
        return float(f(mpmath.mpf(x)))


def test_sincos_correctly_rounded(oracle):
    rng = random.Random(20261203)
    xs = [rng.uniform(-12.0, 12.0) for _ in range(3000)]
    xs += [rng.uniform(-3e5, 3e5) for _ in range(500)]
    xs += [rng.uniform(-1e-7, 1e-7) for _ in range(200)]
    for k in range(-60, 61):          # arguments next to multiples of pi/2
        v = k * math.pi / 2
        xs += [v, math.nextafter(v, math.inf), math.nextafter(v, -math.inf)]
    xs += [0.0, 1e-300, 5e-324, 1.0, math.pi, 2.0 ** 20]
    bad = []
    for x in xs:
        s, c = oracle.cr_sincos(x)
        if s != _cr(mpmath.sin, x) or c != _cr(mpmath.cos, x):
            bad.append(x)
    assert not bad, f"{len(bad)} misrounded, e.g. {bad[:3]}"


def test_sincos_signed_zero_and_fallback(oracle):
    s, c = oracle.cr_sincos(-0.0)
    assert math.copysign(1.0, s) == -1.0 and c == 1.0
    s, c = oracle.cr_sincos(1e10)          # beyond the reduction range: platform libm
    assert s == math.sin(1e10) and c == math.cos(1e10)
    s, c = oracle.cr_sincos(float("nan"))
    assert math.isnan(s) and math.isnan(c)
