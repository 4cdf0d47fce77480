"""GPU flux pass (through the C ABI) against the CPU oracle and the
reference's own results: bit-identical in plain FP64."""
import numpy as np
import pytest

from golden_util import MESH_CASES, REFTESS_CASES, TORO_HALF_STATES, assert_values_equal, \
    load_case, load_riemann, toro_pairs
from oracle.oracle import Params

pytestmark = pytest.mark.gpu


def _ctx(dim, solver, gamma=5 / 3, precision=0):
    from shadowfax_b200.hydro import Context, RiemannSolverFactory
    return Context(dim, RiemannSolverFactory.generate(solver, gamma), precision)


def _pass(mesh, meta):
    from shadowfax_b200.hydro import FluxPass
    ctx = _ctx(mesh.dim, meta["solver"], meta["gamma"])
    fp = FluxPass(ctx, mesh)
    fp.set_primitive(meta["W0"])
    return ctx, fp


def assert_close_per_field(a, b, rtol=1e-12, atol_scale=1e-15):
    """per conserved field and per cell: |a - b| <= rtol |b| + atol_scale *
    max|b| over the field.  The absolute term only matters for values at the
    round-off level of their field (e.g. a y-momentum that is zero in exact
    arithmetic in a 1D problem)."""
    for k in range(b.shape[1]):
        scale = np.max(np.abs(b[:, k]))
        err = np.abs(a[:, k] - b[:, k])
        lim = rtol * np.abs(b[:, k]) + atol_scale * scale
        assert np.all(err <= lim), (k, float(np.max(err / np.maximum(lim, 1e-300))))


@pytest.mark.parametrize("name", MESH_CASES)
def test_single_pass_bitwise_vs_oracle(cuda_ok, oracle, name):
    mesh, meta, _ = load_case(name)
    ctx, fp = _pass(mesh, meta)
    W, Q = fp.state()
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    Qo = oracle.init_Q(mesh, p, meta["W0"])
    np.testing.assert_array_equal(Q, Qo)
    np.testing.assert_array_equal(W, meta["W0"])
    grad, dQ, br, rc, bad = fp.flux_pass(meta["dt"])
    og, odQ, ocode, orc, obad = oracle.flux_pass(mesh, p, meta["dt"], meta["W0"], Qo)
    assert rc == orc == 0
    np.testing.assert_array_equal(grad, og)
    np.testing.assert_array_equal(dQ, odQ)
    np.testing.assert_array_equal(br, ocode)   # branch choices bit-exact on every face


@pytest.mark.parametrize("name", ["sod2d_exact", "sedov3d_hllc", "random2d_periodic_exact"])
def test_face_off_its_right_cell_bitwise_vs_oracle(cuda_ok, oracle, name):
    """a local face whose right position is not bit for bit its right cell's
    position: the two cells of that face see different geometry, so the
    gradients are formed cell by cell instead of from shared face terms, and
    still equal the oracle's"""
    import dataclasses
    mesh, meta, _ = load_case(name)
    rpos = mesh.face_right_pos.copy()
    f = int(np.flatnonzero(mesh.face_kind == 0)[len(rpos) // 3])
    rpos[f, 0] = np.nextafter(rpos[f, 0], np.inf)
    mesh = dataclasses.replace(mesh, face_right_pos=rpos)
    ctx, fp = _pass(mesh, meta)
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    Qo = oracle.init_Q(mesh, p, meta["W0"])
    grad, dQ, br, rc, bad = fp.flux_pass(meta["dt"])
    og, odQ, ocode, orc, obad = oracle.flux_pass(mesh, p, meta["dt"], meta["W0"], Qo)
    assert rc == orc == 0
    np.testing.assert_array_equal(grad, og)
    np.testing.assert_array_equal(dQ, odQ)
    np.testing.assert_array_equal(br, ocode)


@pytest.mark.parametrize("name", MESH_CASES + REFTESS_CASES)
def test_steps_bitwise_vs_reference(cuda_ok, name):
    """n steps on the GPU == the reference's CPU pass (sfx_pow build), bit for
    bit; and within 1e-12 relative of the reference with glibc pow.  The
    reftess cases are meshes the reference's own DelTess/VorTess built, and
    their reference results come from its step loop on that tessellation"""
    mesh, meta, ref = load_case(name)
    ctx, fp = _pass(mesh, meta)
    st = fp.step(meta["dt"], meta["nsteps"])
    assert st.status == 0 and st.steps_done == meta["nsteps"]
    W, Q = fp.state()
    np.testing.assert_array_equal(Q, ref["ref_sfxpow_Q"])
    np.testing.assert_array_equal(W, ref["ref_sfxpow_W"])
    assert_close_per_field(Q, ref["ref_libm_Q"])


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("solver", ["Exact", "HLLC"])
def test_riemann_bitwise_vs_reference(cuda_ok, oracle, dim, solver):
    z = load_riemann(dim)
    ctx = _ctx(dim, solver)
    half, flux, code = ctx.riemann(z["WL"], z["WR"], z["normal"])
    np.testing.assert_array_equal(flux, z[f"{solver}_sfxpow_flux"])
    if solver == "Exact":
        np.testing.assert_array_equal(half, z[f"{solver}_sfxpow_half"])
    _, _, ocode = oracle.riemann(dim, Params(solver=solver), z["WL"], z["WR"], z["normal"])
    np.testing.assert_array_equal(code, ocode)
    _, flux, _ = ctx.riemann(z["WL"], z["WR"], z["normal"], reflective=True)
    np.testing.assert_array_equal(flux, z[f"{solver}_reflective_flux"])


@pytest.mark.parametrize("dim", [2, 3])
def test_riemann_toro_half_states(cuda_ok, dim):
    WL, WR, nrm, exp = toro_pairs(dim)
    ctx = _ctx(dim, "Exact", 1.66667)
    half, flux, code = ctx.riemann(WL, WR, nrm)
    assert np.all(code >= 0)
    for i in range(len(TORO_HALF_STATES)):
        assert_values_equal(half[i, 0], exp[i, 0])
        assert_values_equal(half[i, 1], exp[i, 1])
        assert_values_equal(half[i, dim + 1], exp[i, 2])


def test_sod2d_c1_full_config_vs_oracle(cuda_ok, oracle):
    """the 2D Sod tube in full: 10,000 generators (seed 1), exact solver, dt 1e-4,
    100 steps; GPU == oracle (sfx_pow) bitwise, <= 1e-12 vs glibc pow"""
    from shadowfax_b200 import workloads as wl
    from shadowfax_b200.hydro import FluxPass
    pr = wl.sod2d()
    ctx = _ctx(2, "Exact")
    fp = FluxPass(ctx, pr.mesh)
    fp.set_primitive(pr.W0)
    st = fp.step(pr.dt, pr.nsteps)
    assert st.status == 0
    W, Q = fp.state()
    o = oracle.run(pr.mesh, Params(solver="Exact"), pr.dt, pr.nsteps, pr.W0)
    np.testing.assert_array_equal(Q, o["Q"])
    np.testing.assert_array_equal(W, o["W"])
    ol = oracle.run(pr.mesh, Params(solver="Exact", use_libm_pow=True), pr.dt, pr.nsteps, pr.W0)
    assert_close_per_field(Q, ol["Q"])
    # mass is conserved to round-off in the reflective box
    m0 = oracle.init_Q(pr.mesh, Params(solver="Exact"), pr.W0)[:, 0].sum()
    assert abs(st.totals[0] - m0) <= 1e-13 * m0


@pytest.mark.parametrize("maker,solver,n,steps", [("sedov3d", "HLLC", 20000, 8),
                                                  ("sedov3d", "Exact", 6000, 4),
                                                  ("random_field3d", "Exact", 20000, 1),
                                                  ("random_field3d", "HLLC", 20000, 2)])
def test_scaled_workloads_bitwise_vs_oracle(cuda_ok, oracle, maker, solver, n, steps):
    from shadowfax_b200 import workloads as wl
    from shadowfax_b200.hydro import FluxPass
    pr = getattr(wl, maker)(n=n, solver=solver, nsteps=steps)
    ctx = _ctx(3, solver)
    fp = FluxPass(ctx, pr.mesh)
    fp.set_primitive(pr.W0)
    Q0 = oracle.init_Q(pr.mesh, Params(solver=solver), pr.W0)
    grad, dQ, br, rc, _ = fp.flux_pass(pr.dt)
    og, odQ, ocode, orc, _ = oracle.flux_pass(pr.mesh, Params(solver=solver), pr.dt, pr.W0, Q0)
    assert rc == orc == 0
    np.testing.assert_array_equal(br, ocode)
    np.testing.assert_array_equal(dQ, odQ)
    st = fp.step(pr.dt, pr.nsteps)
    assert st.status == 0
    W, Q = fp.state()
    o = oracle.run(pr.mesh, Params(solver=solver), pr.dt, pr.nsteps, pr.W0)
    np.testing.assert_array_equal(Q, o["Q"])


def test_reruns_are_bitwise_identical(cuda_ok):
    mesh, meta, _ = load_case("sedov3d_hllc")
    outs = []
    for _ in range(2):
        ctx, fp = _pass(mesh, meta)
        fp.step(meta["dt"], meta["nsteps"])
        outs.append(fp.state()[1])
    np.testing.assert_array_equal(outs[0], outs[1])


@pytest.mark.parametrize("name", ["sod2d_exact", "sod2d_hllc", "sedov3d_hllc"])
def test_errors_match_the_oracle(cuda_ok, oracle, name):
    """a corrupted (NaN) cell state makes the pass fail with the same status
    (RiemannSolverException -> SFX_ERR_RIEMANN for the exact solver,
    FluxCalculationException -> SFX_ERR_NAN_FLUX for HLLC) at the same first
    face as the reference's face loop would throw at"""
    from shadowfax_b200 import _lib as L
    mesh, meta, _ = load_case(name)
    W_clean = meta["W0"].copy()
    W0 = meta["W0"].copy()
    W0[mesh.n_cells // 3, 0] = np.nan
    meta = dict(meta, W0=W0)
    ctx, fp = _pass(mesh, meta)
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    Q0 = oracle.init_Q(mesh, p, W0)
    _, _, _, orc, obad = oracle.flux_pass(mesh, p, meta["dt"], W0, Q0)
    assert orc in (L.SFX_ERR_RIEMANN, L.SFX_ERR_NAN_FLUX)
    with pytest.raises(L.SfxError) as ei:
        fp.step(meta["dt"], 1)
    assert ei.value.status == orc and ei.value.index == obad
    # a negative mass after the update is reported per cell (UpdateQException)
    W1 = W_clean
    ctx2, fp2 = _pass(mesh, dict(meta, W0=W1))
    Q1 = oracle.init_Q(mesh, p, W1)
    Q1[:, -1] = 1e-300  # every cell that loses energy goes negative
    fp2.set_state(W1, Q1)
    g, dQ, _, rc, _ = oracle.flux_pass(mesh, p, meta["dt"], W1, Q1)
    assert rc == 0
    _, _, arc, abad = oracle.apply(mesh, p, dQ, W1, Q1)
    assert arc == L.SFX_ERR_NEG_STATE
    with pytest.raises(L.SfxError) as ei:
        fp2.step(meta["dt"], 1)
    assert ei.value.status == arc and ei.value.index == abad
