"""sfx_pow (shared by the GPU pass and the oracle) against exact decimal
arithmetic and the C99 special cases."""
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest


def test_sfx_pow_is_correctly_rounded_on_samples(oracle):
    getcontext().prec = 50
    rng = np.random.Generator(np.random.PCG64(42))
    gam = 5.0 / 3.0
    exps = [0.5 * (gam - 1) / gam, -0.5 * (gam + 1) / gam, 2 / (gam - 1), 2 * gam / (gam - 1),
            1 / gam, 0.2, -0.8, 3.0]
    bad = 0
    for i in range(3000):
        x = math.exp(rng.uniform(-30, 30))
        y = exps[i % len(exps)] if i % 2 else rng.uniform(-8, 8)
        got = oracle.pow(x, y)
        exact = Decimal(x) ** Decimal(y)
        err = abs(Decimal(got) - exact) / Decimal(math.ulp(got))
        if err > Decimal("0.5000001"):
            bad += 1
    assert bad == 0


@pytest.mark.parametrize("x,y", [(0.0, -0.8), (0.0, 0.2), (-0.0, -3.0), (-0.0, 3.0), (-2.0, 3.0),
                                 (-2.0, 0.5), (math.inf, -1.0), (-math.inf, 3.0), (1.0, math.nan),
                                 (math.nan, 0.0), (0.5, math.inf), (2.0, -math.inf),
                                 (-1.0, math.inf), (2.0, 1024.0), (10.0, 308.3), (4.0, 0.5),
                                 (1e-310, 0.5), (2.0, -1074.0)])
def test_sfx_pow_special_values_follow_c99(oracle, x, y):
    got = oracle.pow(x, y)
    with np.errstate(all="ignore"):
        want = float(np.power(np.float64(x), np.float64(y)))  # libm pow
    if math.isnan(want):
        assert math.isnan(got)
    else:
        assert got == want and math.copysign(1, got) == math.copysign(1, want)


def test_sfx_pow_fast_error_bound(oracle):
    """the split pass's plain-double pow: within 1.5 (2 + |y log2 x|) ulp of
    the exact power on the exponents of the exact solver and random ones"""
    getcontext().prec = 50
    rng = np.random.Generator(np.random.PCG64(7))
    gam = 5.0 / 3.0
    exps = [0.5 * (gam - 1) / gam, -0.5 * (gam + 1) / gam, 2 / (gam - 1), 2 * gam / (gam - 1),
            1 / gam]
    worst = 0.0
    for i in range(4000):
        x = math.exp(rng.uniform(-70, 10))
        y = exps[i % len(exps)] if i % 3 else rng.uniform(-5, 5)
        got = oracle.pow_fast(x, y)
        exact = Decimal(x) ** Decimal(y)
        ulps = float(abs(Decimal(got) - exact) / Decimal(math.ulp(float(exact))))
        worst = max(worst, ulps / (2 + abs(y * math.log2(x))))
    assert worst <= 1.5, worst


@pytest.mark.parametrize("x,y", [(0.0, 0.2), (0.0, -0.8), (1e-310, 0.5), (-2.0, 3.0),
                                 (math.inf, 0.2), (2.0, 2000.0), (1.0, 0.2), (4.0, 0.5)])
def test_sfx_pow_fast_outside_its_domain_is_sfx_pow(oracle, x, y):
    a, b = oracle.pow_fast(x, y), oracle.pow(x, y)
    if x == 1.0 or x == 4.0:
        assert abs(a - b) <= 4 * math.ulp(b)
    else:
        assert (math.isnan(a) and math.isnan(b)) or a == b
