"""Properties of the two Riemann solvers that hold for any states (the
oracle restatement, pinned bit for bit against the reference's solvers):
equal states on both sides give the physical Euler flux through the face
(consistency), and swapping the sides while reversing the normal negates
the flux (the face seen from the other cell)."""
import numpy as np
import pytest

from oracle.oracle import Params

GAMMA = 5.0 / 3.0


def _states(dim, n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    S = dim + 2
    W = np.zeros((n, S))
    W[:, 0] = np.exp(rng.normal(0, 1, n))
    W[:, 1:dim + 1] = rng.normal(0, 1, (n, dim))
    W[:, S - 1] = np.exp(rng.normal(0, 1, n))
    nrm = rng.normal(0, 1, (n, dim))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    return W, nrm


def euler_flux(W, nrm, g):
    D = nrm.shape[1]
    rho, v, p = W[:, 0], W[:, 1:D + 1], W[:, D + 1]
    vn = (v * nrm).sum(1)
    E = p / (g - 1.0) + 0.5 * rho * (v * v).sum(1)
    F = np.zeros_like(W)
    F[:, 0] = rho * vn
    F[:, 1:D + 1] = rho[:, None] * v * vn[:, None] + p[:, None] * nrm
    F[:, D + 1] = (E + p) * vn
    return F


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("solver", ["Exact", "HLLC"])
def test_equal_states_give_the_physical_flux(oracle, dim, solver):
    W, nrm = _states(dim, 500, 40 + dim)
    _, flux, code = oracle.riemann(dim, Params(solver=solver, gamma=GAMMA), W, W, nrm)
    assert np.all(code >= 0)
    F = euler_flux(W, nrm, GAMMA)
    scale = np.abs(F).max(1, keepdims=True)
    assert np.all(np.abs(flux - F) <= 1e-12 * scale)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("solver", ["Exact", "HLLC"])
def test_swapping_the_sides_negates_the_flux(oracle, dim, solver):
    WL, nrm = _states(dim, 500, 50 + dim)
    WR, _ = _states(dim, 500, 60 + dim)
    p = Params(solver=solver, gamma=GAMMA)
    _, f1, c1 = oracle.riemann(dim, p, WL, WR, nrm)
    _, f2, c2 = oracle.riemann(dim, p, WR, WL, -nrm)
    assert np.all(c1 >= 0) and np.all(c2 >= 0)
    scale = np.abs(f1).max(1, keepdims=True)
    assert np.all(np.abs(f1 + f2) <= 1e-10 * scale)
