"""FP32/FP64-split flux pass against the plain-FP64 pass: <= 1e-6 relative L1
per conserved field, mass and energy conserved to round-off, bitwise
identical reruns."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_L1 = 1e-6


def _run(pr, precision, nsteps=None):
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    ctx = Context(pr.mesh.dim, RiemannSolverFactory.generate(pr.solver, pr.gamma), precision)
    fp = FluxPass(ctx, pr.mesh)
    fp.set_primitive(pr.W0)
    t0 = fp.totals()
    st = fp.step(pr.dt, pr.nsteps if nsteps is None else nsteps)
    W, Q = fp.state()
    return W, Q, t0, np.array(st.totals[: pr.mesh.dim + 2])


def l1_rel(a, b):
    """relative L1 error per conserved field: mass, momentum, energy.  The
    momentum is one vector field: each component's L1 error is divided by
    the L1 norm of the momentum magnitude (a component that is zero in exact
    arithmetic, such as y-momentum in a 1D Sod tube, holds only round-off and
    has no scale of its own)."""
    D = b.shape[1] - 2
    den = np.abs(b).sum(0)
    den[1:D + 1] = np.sqrt((b[:, 1:D + 1] ** 2).sum(1)).sum()
    return np.abs(a - b).sum(0) / den


@pytest.mark.parametrize("case", ["sod2d", "sod2d_hllc", "sedov3d", "random3d_exact",
                                  "random3d_hllc"])
def test_split_within_tolerance_of_fp64(cuda_ok, case):
    from shadowfax_b200 import workloads as wl
    pr = {
        "sod2d": lambda: wl.sod2d(n=10_000, nsteps=100),
        "sod2d_hllc": lambda: wl.sod2d(n=10_000, nsteps=100, solver="HLLC"),
        "sedov3d": lambda: wl.sedov3d(n=40_000, nsteps=20),
        "random3d_exact": lambda: wl.random_field3d(n=40_000, nsteps=3),
        "random3d_hllc": lambda: wl.random_field3d(n=40_000, nsteps=3, solver="HLLC"),
    }[case]()
    W64, Q64, _, _ = _run(pr, 0)
    W32, Q32, t0, t1 = _run(pr, 1)
    err = l1_rel(Q32, Q64)
    print(case, "L1 rel per field", err)
    assert np.all(err <= TOL_L1), err
    # mass is conserved to round-off (the reflective/periodic box is closed)
    assert abs(t1[0] - t0[0]) <= 1e-12 * abs(t0[0])
    # energy too (the flux leaving one cell enters its neighbour exactly)
    assert abs(t1[-1] - t0[-1]) <= 1e-12 * abs(t0[-1])


def test_split_reruns_are_bitwise_identical(cuda_ok):
    from shadowfax_b200 import workloads as wl
    pr = wl.sedov3d(n=20_000, nsteps=10)
    a = _run(pr, 1)[1]
    b = _run(pr, 1)[1]
    np.testing.assert_array_equal(a, b)


def test_split_single_pass_face_flux_error_by_branch(cuda_ok):
    """random field: per-face flux error of the split pass vs FP64 for the
    exact solver, grouped by the FP64 branch (shock / rarefaction / vacuum)"""
    from shadowfax_b200 import workloads as wl
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    pr = wl.random_field3d(n=40_000)
    out = {}
    for prec in (0, 1):
        ctx = Context(3, RiemannSolverFactory.generate("Exact"), prec)
        fp = FluxPass(ctx, pr.mesh)
        fp.set_primitive(pr.W0)
        grad, dQ, br, rc, _ = fp.flux_pass(pr.dt)
        assert rc == 0
        out[prec] = (dQ, br)
    dQ64, br = out[0]
    dQ32 = out[1][0]
    region = (br >> 5) & 15
    shock = np.isin(region, [1, 6])
    raref = np.isin(region, [3, 4, 8, 9])
    scale = np.abs(dQ64).sum(0)
    for mask in (shock, raref):
        if mask.any():
            e = np.abs(dQ32[mask] - dQ64[mask]).sum(0) / np.maximum(np.abs(dQ64[mask]).sum(0), 1e-300)
            assert np.all(e <= 1e-5), e
    assert np.all(np.abs(dQ32 - dQ64).sum(0) / scale <= 1e-5)


@pytest.mark.parametrize("name", ["reftess_sod2d_reflective_exact", "reftess_random2d_periodic_hllc",
                                  "reftess_sedov3d_reflective_hllc",
                                  "reftess_random3d_periodic_exact"])
def test_split_on_reference_tessellation(cuda_ok, name):
    """the split pass on meshes the reference's own tessellation built
    (zero-area faces, mirrors, periodic images): within the tolerance of the
    reference's FP64 result, mass conserved"""
    from types import SimpleNamespace
    from golden_util import load_case
    mesh, meta, ref = load_case(name)
    pr = SimpleNamespace(mesh=mesh, solver=meta["solver"], gamma=meta["gamma"], W0=meta["W0"],
                         dt=meta["dt"], nsteps=meta["nsteps"])
    W32, Q32, t0, t1 = _run(pr, 1)
    err = l1_rel(Q32, ref["ref_sfxpow_Q"])
    assert np.all(err <= TOL_L1), err
    assert abs(t1[0] - t0[0]) <= 1e-12 * abs(t0[0])


def test_split_refuses_periodic_meshes_of_another_box(cuda_ok):
    """the split kernels apply a periodic image offset as +-1 per axis: a
    periodic mesh of a box of side 2 is refused by a split context and taken
    by the plain-FP64 one; the same mesh in the unit box is taken by both"""
    import dataclasses
    from golden_util import load_case
    from shadowfax_b200._lib import SfxError, SFX_ERR_UNSUPPORTED
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    mesh, meta, _ = load_case("random2d_periodic_exact")
    D = mesh.dim
    big = dataclasses.replace(
        mesh, cell_pos=mesh.cell_pos * 2., cell_centroid=mesh.cell_centroid * 2.,
        cell_volume=mesh.cell_volume * 2. ** D, cell_total_area=mesh.cell_total_area * 2. ** (D - 1),
        face_area=mesh.face_area * 2. ** (D - 1), face_midpoint=mesh.face_midpoint * 2.,
        face_right_pos=mesh.face_right_pos * 2.)
    solver = RiemannSolverFactory.generate(meta["solver"], meta["gamma"])
    for precision in (0, 1):
        FluxPass(Context(D, solver, precision), mesh)
    FluxPass(Context(D, solver, 0), big)
    with pytest.raises(SfxError) as e:
        FluxPass(Context(D, solver, 1), big)
    assert e.value.status == SFX_ERR_UNSUPPORTED
