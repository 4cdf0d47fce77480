"""The CPU oracle against the reference's own results (golden fixtures made
by running the unmodified reference flux pass, tests/golden/make_golden.py)
and against the reference's Riemann-solver unit-test vectors."""
import numpy as np
import pytest

from golden_util import (GAMMA_CASES, GOLDEN, MESH_CASES, MOVING_CASES, MOVING_FAILS,
                         TORO_HALF_STATES, assert_values_equal, load_case, load_riemann,
                         toro_pairs)
from oracle.oracle import Params


@pytest.mark.parametrize("name", MESH_CASES)
@pytest.mark.parametrize("powk", ["sfxpow", "libm"])
def test_oracle_matches_reference_bitwise(oracle, name, powk):
    mesh, meta, ref = load_case(name)
    p = Params(solver=meta["solver"], gamma=meta["gamma"], use_libm_pow=(powk == "libm"))
    out = oracle.run(mesh, p, meta["dt"], meta["nsteps"], meta["W0"])
    assert out["status"] == 0 and out["steps"] == meta["nsteps"]
    for key in ("W", "Q", "grad", "dQ"):
        np.testing.assert_array_equal(out[key], ref[f"ref_{powk}_{key}"], err_msg=key)


@pytest.mark.parametrize("name", GAMMA_CASES)
@pytest.mark.parametrize("powk", ["sfxpow", "libm"])
def test_oracle_matches_reference_at_another_gamma(oracle, name, powk):
    """gamma = 1.4: the solvers' gamma-dependent constants and get_Q/get_W's
    energy, step by step as the reference forms them"""
    mesh, meta, ref = load_case(name)
    assert meta["gamma"] == 1.4
    p = Params(solver=meta["solver"], gamma=meta["gamma"], use_libm_pow=(powk == "libm"))
    out = oracle.run(mesh, p, meta["dt"], meta["nsteps"], meta["W0"])
    assert out["status"] == 0 and out["steps"] == meta["nsteps"]
    for key in ("W", "Q", "grad", "dQ"):
        np.testing.assert_array_equal(out[key], ref[f"ref_{powk}_{key}"], err_msg=key)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("solver", ["Exact", "HLLC"])
@pytest.mark.parametrize("powk", ["sfxpow", "libm"])
def test_oracle_riemann_matches_reference_at_another_gamma(oracle, dim, solver, powk):
    z = np.load(GOLDEN / f"riemann_gamma14_{dim}d.npz")
    p = Params(solver=solver, gamma=float(z["gamma"]), use_libm_pow=(powk == "libm"))
    half, flux, code = oracle.riemann(dim, p, z["WL"], z["WR"], z["normal"])
    assert np.all(code >= 0) and np.all(z[f"{solver}_{powk}_status"] == 0)
    np.testing.assert_array_equal(flux, z[f"{solver}_{powk}_flux"])
    if solver == "Exact":
        np.testing.assert_array_equal(half, z[f"{solver}_{powk}_half"])


@pytest.mark.parametrize("powk", ["sfxpow", "libm"])
def test_oracle_matches_reference_at_another_tolerance(oracle, powk):
    """the exact solver at tolerance 1e-6 and cutoff -2 (defaults 1e-8, -5)"""
    mesh, meta, ref = load_case("tol6_random3d_exact")
    z = np.load(GOLDEN / "tol6_random3d_exact.npz")
    p = Params(solver="Exact", gamma=meta["gamma"], tolerance=float(z["tolerance"]),
               cutoff=float(z["cutoff"]), use_libm_pow=(powk == "libm"))
    out = oracle.run(mesh, p, meta["dt"], meta["nsteps"], meta["W0"])
    assert out["status"] == 0 and out["steps"] == meta["nsteps"]
    for key in ("W", "Q", "grad", "dQ"):
        np.testing.assert_array_equal(out[key], ref[f"ref_{powk}_{key}"], err_msg=key)
    # the parameters matter: the defaults end elsewhere
    out0 = oracle.run(mesh, Params(solver="Exact", gamma=meta["gamma"],
                                   use_libm_pow=(powk == "libm")),
                      meta["dt"], meta["nsteps"], meta["W0"])
    assert np.any(out0["Q"] != out["Q"])


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("powk", ["sfxpow", "libm"])
def test_oracle_riemann_matches_reference_at_another_tolerance(oracle, dim, powk):
    z = np.load(GOLDEN / f"riemann_tol6_{dim}d.npz")
    p = Params(solver="Exact", tolerance=float(z["tolerance"]), cutoff=float(z["cutoff"]),
               use_libm_pow=(powk == "libm"))
    half, flux, code = oracle.riemann(dim, p, z["WL"], z["WR"], z["normal"])
    assert np.all(code >= 0) and np.all(z[f"Exact_{powk}_status"] == 0)
    np.testing.assert_array_equal(flux, z[f"Exact_{powk}_flux"])
    np.testing.assert_array_equal(half, z[f"Exact_{powk}_half"])
    # the parameters matter: the defaults give other fluxes on some pairs
    _, flux0, _ = oracle.riemann(dim, Params(solver="Exact", use_libm_pow=(powk == "libm")),
                                 z["WL"], z["WR"], z["normal"])
    assert np.any(flux0 != flux)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("solver", ["Exact", "HLLC"])
@pytest.mark.parametrize("powk", ["sfxpow", "libm"])
def test_oracle_riemann_matches_reference(oracle, dim, solver, powk):
    z = load_riemann(dim)
    p = Params(solver=solver, use_libm_pow=(powk == "libm"))
    half, flux, code = oracle.riemann(dim, p, z["WL"], z["WR"], z["normal"])
    assert np.all(code >= 0)
    np.testing.assert_array_equal(flux, z[f"{solver}_{powk}_flux"])
    if solver == "Exact":
        np.testing.assert_array_equal(half, z[f"{solver}_{powk}_half"])
    half, flux, code = oracle.riemann(dim, Params(solver=solver), z["WL"], z["WR"], z["normal"],
                                      reflective=True)
    np.testing.assert_array_equal(flux, z[f"{solver}_reflective_flux"])


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_toro_half_states(oracle, dim):
    WL, WR, nrm, exp = toro_pairs(dim)
    half, flux, code = oracle.riemann(dim, Params(solver="Exact", gamma=1.66667), WL, WR, nrm)
    assert np.all(code >= 0)
    for i in range(len(TORO_HALF_STATES)):
        assert_values_equal(half[i, 0], exp[i, 0])
        assert_values_equal(half[i, 1], exp[i, 1])
        assert_values_equal(half[i, dim + 1], exp[i, 2])


def test_branch_coverage_of_riemann_fixture(oracle):
    """the fixture exercises vacuum, Newton-only, Newton, Brent and every
    sampled region"""
    seen = set()
    for dim in (2, 3):
        z = load_riemann(dim)
        _, _, code = oracle.riemann(dim, Params(solver="Exact"), z["WL"], z["WR"], z["normal"])
        for c in code:
            seen.add(("vac", int(c) & 7))
            seen.add(("it", (int(c) >> 3) & 3))
            seen.add(("s", (int(c) >> 5) & 15))
    for v in range(1, 5):
        assert ("vac", v) in seen
    for it in (1, 2, 3):
        assert ("it", it) in seen
    for s in (1, 3, 4, 6, 8, 9, 11):
        assert ("s", s) in seen, s


@pytest.mark.parametrize("name", MOVING_CASES)
@pytest.mark.parametrize("powk", ["sfxpow", "libm"])
def test_oracle_moving_step_matches_reference(oracle, name, powk):
    """one step with moving generators (generator velocities, face
    velocities, fluxes in the faces' frames, drift) against the reference
    built without -DSTATIC: bit for bit with sfx_pow/sfx_cbrt, within 1e-12
    per field with glibc's pow and cbrt"""
    mesh, meta, ref = load_case(name)
    p = Params(solver=meta["solver"], gamma=meta["gamma"], use_libm_pow=powk == "libm")
    W, Q, st, pos = oracle.run_moving(mesh, p, meta["dt"], meta["W0"], mesh.periodic)
    assert st == 0
    if powk == "sfxpow":
        np.testing.assert_array_equal(pos, ref["ref_sfxpow_pos"])
        np.testing.assert_array_equal(Q, ref["ref_sfxpow_Q"])
        np.testing.assert_array_equal(W, ref["ref_sfxpow_W"])
    else:
        b = ref["ref_libm_Q"]
        for k in range(b.shape[1]):
            lim = 1e-12 * np.abs(b[:, k]) + 1e-15 * np.abs(b[:, k]).max()
            assert np.all(np.abs(Q[:, k] - b[:, k]) <= lim), k
        assert np.allclose(pos, ref["ref_libm_pos"], rtol=0, atol=1e-14)
    # the generators did move (a fair fraction of a cell in 2D)
    assert np.abs(pos - mesh.cell_pos).max() > 1e-3


def test_oracle_moving_step_fails_where_the_reference_fails(oracle):
    """two generators 2e-4 apart: their face moves at ~50 and the HLLC step
    drives a cell to negative energy; the reference throws UpdateQException"""
    mesh, meta, ref = load_case(MOVING_FAILS)
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    _, _, st, _ = oracle.run_moving(mesh, p, meta["dt"], meta["W0"], mesh.periodic)
    assert int(ref["ref_sfxpow_status"]) == 11          # UpdateQException in the harness
    assert st == 5                                       # SFX_ERR_NEG_STATE
