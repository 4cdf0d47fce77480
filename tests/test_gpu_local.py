"""Local (hierarchical) time steps on the GPU (plain FP64):

* one system step [t_now, t_next) (sfx_step_window) against the reference's
  own VorFace/VorCell/GasParticle in a static build with every particle's
  step bounds and the inactive particles' stored gradients
  (tests/golden/local_*.npz): gradients of the active cells, the activity
  gates, the per-face step min(dt_L, dt_R), timefac, Q of every cell and W of
  the cells ending at t_next, bit for bit (sfx_pow), within 1e-12 per field
  (glibc pow);
* the new steps of the cells ending at t_next (sfx_timestep_bins) against
  the oracle's restatement of TimeLine::calculate_timestep, bit for bit;
* a run in which every cell takes the longest allowed step equals the same
  number of global steps bit for bit, and a run with mixed bins conserves
  mass to round-off;
* the split pass: one bin equals its own global steps bit for bit, and a
  mixed-bin run stays within the split pass's tolerance of the plain FP64
  run with the same bins, conserving mass to round-off."""
import numpy as np
import pytest

from golden_util import LOCAL_CASES, load_case

pytestmark = pytest.mark.gpu

TICKS = 1 << 60


def _pass(mesh, meta, solver=None, precision=0):
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    ctx = Context(mesh.dim, RiemannSolverFactory.generate(solver or meta["solver"],
                                                          meta["gamma"]), precision)
    fp = FluxPass(ctx, mesh)
    fp.set_primitive(meta["W0"])
    return ctx, fp


@pytest.mark.parametrize("name", LOCAL_CASES)
def test_window_step_bitwise_vs_reference(cuda_ok, oracle, name):
    from oracle.oracle import Params
    mesh, meta, ref = load_case(name)
    loc = meta["local"]
    ctx, fp = _pass(mesh, meta)
    fp.set_timesteps(loc["start"], loc["end"])
    fp.set_gradients(loc["grad0"])
    fp.step_window(float(loc["t_total"]), int(loc["t_now"]), int(loc["t_next"]), mesh.periodic)
    W, Q = fp.state()
    np.testing.assert_array_equal(fp.gradients(), ref["ref_sfxpow_grad"])
    np.testing.assert_array_equal(Q, ref["ref_sfxpow_Q"])
    np.testing.assert_array_equal(W, ref["ref_sfxpow_W"])
    b = ref["ref_libm_Q"]
    for k in range(b.shape[1]):
        lim = 1e-12 * np.abs(b[:, k]) + 1e-15 * np.abs(b[:, k]).max()
        assert np.all(np.abs(Q[:, k] - b[:, k]) <= lim), k
    # the new steps of the cells ending at t_next: the velocities the active
    # cells set in this step enter through |v - v_gen|
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    t_total, t_next = float(loc["t_total"]), int(loc["t_next"])
    smin = fp.timestep_bins(t_total, 0.4, TICKS, 0, t_next)
    s, e = fp.timesteps()
    os_, oe, osmin, rc = oracle.timestep_bins(mesh, p, ref["ref_sfxpow_W"], ref["ref_sfxpow_vel"],
                                              loc["start"], loc["end"], t_next, t_total, 0.4,
                                              TICKS, 0)
    assert rc == 0
    np.testing.assert_array_equal(s, os_)
    np.testing.assert_array_equal(e, oe)
    assert smin == osmin
    fp.close()
    ctx.close()


@pytest.mark.parametrize("solver,precision", [("Exact", 0), ("HLLC", 0), ("Exact", 1),
                                              ("HLLC", 1)])
def test_one_bin_equals_global_steps(cuda_ok, solver, precision):
    """with max_step below every cell's CFL step every cell takes max_step and
    is active in every system step: the same arithmetic as global steps of
    t_total * max_step / 2^60, in either precision"""
    from shadowfax_b200 import workloads as wl
    pr = wl.sod2d(n=2000, nsteps=6, solver=solver)
    meta = dict(solver=solver, gamma=pr.gamma, W0=pr.W0)
    max_step = TICKS >> 20
    t_total = pr.dt * (1 << 20)          # one max_step is the problem's dt
    ctx, fp = _pass(pr.mesh, meta, precision=precision)
    t = fp.run_local(t_total, pr.nsteps, max_step=max_step, periodic=False)
    assert t == pr.nsteps * max_step
    W, Q = fp.state()
    s, e = fp.timesteps()
    assert np.all(e - s == max_step)
    ctx2, fp2 = _pass(pr.mesh, meta, precision=precision)
    dt = t_total * (max_step / TICKS)
    assert dt == pr.dt
    fp2.step(dt, pr.nsteps)
    W2, Q2 = fp2.state()
    np.testing.assert_array_equal(Q, Q2)
    np.testing.assert_array_equal(W, W2)
    for x in (fp, fp2, ctx, ctx2):
        x.close()


def test_mixed_bins_conserve_mass(cuda_ok):
    """a Sedov-type blast: the hot cells take short steps, the cold ones long
    steps; after many system steps the bins are mixed and mass is conserved
    to round-off (a face exchanges the same dQ with both cells)"""
    from shadowfax_b200 import workloads as wl
    pr = wl.sedov3d(n=4000, nsteps=1, solver="HLLC")
    meta = dict(solver="HLLC", gamma=pr.gamma, W0=pr.W0)
    ctx, fp = _pass(pr.mesh, meta)
    m0 = fp.state()[1][:, 0].sum()
    t_total = 200 * pr.dt
    fp.run_local(t_total, 40, periodic=False)
    s, e = fp.timesteps()
    bins = np.unique(e - s)
    assert len(bins) >= 2, bins
    Q = fp.state()[1]
    assert abs(Q[:, 0].sum() - m0) <= 1e-13 * m0
    fp.close()
    ctx.close()


@pytest.mark.parametrize("solver", ["HLLC", "Exact"])
def test_split_mixed_bins_within_tolerance_of_fp64(cuda_ok, solver):
    """the split pass with local steps against the plain FP64 pass over the
    same system steps: the bins agree (the CFL steps come from the FP32
    states, so a cell within round-off of a power-of-two boundary may bin
    differently), Q within the split pass's tolerance, mass conserved to
    round-off"""
    from shadowfax_b200 import workloads as wl
    pr = wl.sedov3d(n=4000, nsteps=1, solver=solver)
    meta = dict(solver=solver, gamma=pr.gamma, W0=pr.W0)
    t_total = 200 * pr.dt
    out = {}
    for precision in (0, 1):
        ctx, fp = _pass(pr.mesh, meta, precision=precision)
        m0 = fp.state()[1][:, 0].sum()
        t = fp.run_local(t_total, 12, periodic=False)
        s, e = fp.timesteps()
        Q = fp.state()[1]
        assert abs(Q[:, 0].sum() - m0) <= 1e-12 * m0
        out[precision] = (t, s, e, Q)
        fp.close()
        ctx.close()
    t64, s64, e64, Q64 = out[0]
    t32, s32, e32, Q32 = out[1]
    assert len(np.unique(e64 - s64)) >= 2
    assert np.mean((e32 - s32) == (e64 - s64)) >= 0.99
    if t32 == t64 and np.array_equal(e32 - s32, e64 - s64):
        err = np.abs(Q32 - Q64).sum(0) / np.abs(Q64).sum(0)
        assert np.all(err[[0, -1]] <= 1e-6), err
