"""Known answer: the exact Riemann problem with vacuum (Toro, "Riemann Solvers
and Numerical Methods for Fluid Dynamics", section 4.6), the solution the
reference's rundir/testsuite/vacuum/vacuum.py plots its simulations against.
The oracle's exact solver, sampled at the interface (x/t = 0), must give the
analytic state: a left state next to vacuum, a right state next to vacuum,
and two states that move apart fast enough to open a vacuum between them,
with the interface in the constant state, in the rarefaction fan or in the
vacuum.  The oracle equals the reference's solver bit for bit on its Riemann
fixtures; this pins both against the closed form."""
import math

import numpy as np
import pytest

from oracle.oracle import Params

GAMMA = 5.0 / 3.0


def _left_next_to_vacuum(r, u, p, x, g):
    """the left state r, u, p with vacuum on its right, sampled at x/t = x"""
    a = math.sqrt(g * p / r)
    if x <= u - a:
        return r, u, p
    if x < u + 2.0 * a / (g - 1.0):
        f = 2.0 / (g + 1.0) + (g - 1.0) / ((g + 1.0) * a) * (u - x)
        return (r * f ** (2.0 / (g - 1.0)), 2.0 / (g + 1.0) * (a + 0.5 * (g - 1.0) * u + x),
                p * f ** (2.0 * g / (g - 1.0)))
    return 0.0, 0.0, 0.0


def _right_next_to_vacuum(r, u, p, x, g):
    """the right state with vacuum on its left: the mirror image of the left case"""
    rr, uu, pp = _left_next_to_vacuum(r, -u, p, -x, g)
    return rr, -uu, pp


def vacuum_solution(WL, WR, g, x=0.0):
    (rL, uL, pL), (rR, uR, pR) = WL, WR
    if rR == 0.0:
        return _left_next_to_vacuum(rL, uL, pL, x, g)
    if rL == 0.0:
        return _right_next_to_vacuum(rR, uR, pR, x, g)
    aL, aR = math.sqrt(g * pL / rL), math.sqrt(g * pR / rR)
    assert uR - uL >= 2.0 * (aL + aR) / (g - 1.0)   # the two fans do not meet
    if x <= uL + 2.0 * aL / (g - 1.0):
        return _left_next_to_vacuum(rL, uL, pL, x, g)
    if x >= uR - 2.0 * aR / (g - 1.0):
        return _right_next_to_vacuum(rR, uR, pR, x, g)
    return 0.0, 0.0, 0.0


def _cases(kind, n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    g = GAMMA
    out = []
    for _ in range(n):
        rL, rR = np.exp(rng.normal(0, 1, 2))
        pL, pR = np.exp(rng.normal(0, 1, 2))
        aL, aR = math.sqrt(g * pL / rL), math.sqrt(g * pR / rR)
        if kind == "right vacuum":
            uL = rng.normal(0, 2) * aL
            out.append(((rL, uL, pL), (0.0, 0.0, 0.0)))
        elif kind == "left vacuum":
            uR = rng.normal(0, 2) * aR
            out.append(((0.0, 0.0, 0.0), (rR, uR, pR)))
        else:
            gap = 2.0 * (aL + aR) / (g - 1.0) * (1.0 + abs(rng.normal(0, 1)))
            shift = rng.normal(0, 1.5) * gap
            out.append(((rL, shift - 0.5 * gap, pL), (rR, shift + 0.5 * gap, pR)))
    return out


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kind", ["right vacuum", "left vacuum", "vacuum generation"])
def test_exact_solver_matches_the_vacuum_solution(oracle, dim, kind):
    cases = _cases(kind, 300, {"right vacuum": 1, "left vacuum": 2,
                               "vacuum generation": 3}[kind] + 10 * dim)
    S = dim + 2
    WL = np.zeros((len(cases), S))
    WR = np.zeros((len(cases), S))
    for i, (l, r) in enumerate(cases):
        WL[i, [0, 1, S - 1]] = l
        WR[i, [0, 1, S - 1]] = r
    nrm = np.zeros((len(cases), dim))
    nrm[:, 0] = 1.0
    half, _, code = oracle.riemann(dim, Params(solver="Exact", gamma=GAMMA), WL, WR, nrm)
    assert np.all(code >= 0)
    regions = set()
    for i, (l, r) in enumerate(cases):
        rho, u, p = vacuum_solution(l, r, GAMMA)
        regions.add("vacuum" if rho == 0.0 else ("state" if rho in (l[0], r[0]) else "fan"))
        got = half[i, [0, 1, S - 1]]
        np.testing.assert_allclose(got, [rho, u, p], rtol=1e-12, atol=1e-300,
                                   err_msg=f"{kind} case {i}: {l} | {r}")
        assert np.all(half[i, 2:S - 1] == 0.0)       # no transverse velocity appears
    # the sample point falls in every region the kind has
    assert regions == {"state", "fan", "vacuum"}
