"""Local (hierarchical) time steps on the CPU: the oracle's restatement of
TimeLine::calculate_timestep (src/TimeLine.cpp:233-317; the reference's own
file needs ParticleVector, Tree and the HDF5 snapshot writers and cannot be
built here) against the rules it states, on hand-made and random states:
every new step is a power of two of ticks, never longer than the CFL step,
synchronised with the end of the timeline, within [min_step, max_step]; the
cells not ending at t_next are left alone; the smallest new step is
returned."""
import numpy as np
import pytest

from golden_util import LOCAL_CASES, load_case
from oracle.oracle import Params

TICKS = 1 << 60


def _cfl_step(mesh, W, vgen, gamma=5 / 3):
    D = mesh.dim
    V = mesh.cell_volume
    h = np.cbrt(V * 3 / 4 / np.pi) if D == 3 else np.sqrt(V / np.pi)
    v = np.sqrt(((W[:, 1:D + 1] - vgen) ** 2).sum(1))
    c = np.sqrt(gamma * W[:, D + 1] / W[:, 0])
    return h / (v + c)


@pytest.mark.parametrize("name", LOCAL_CASES)
def test_bins_follow_their_rules(oracle, name):
    mesh, meta, ref = load_case(name)
    loc = meta["local"]
    W, vel = ref["ref_sfxpow_W"], ref["ref_sfxpow_vel"]
    t_next, t_total = int(loc["t_next"]), float(loc["t_total"])
    cfl = 0.4
    start, end = loc["start"].astype(np.uint64), loc["end"].astype(np.uint64)
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    s2, e2, smin, rc = oracle.timestep_bins(mesh, p, W, vel, start, end, t_next, t_total, cfl,
                                            TICKS, 0)
    assert rc == 0
    ending = end == t_next
    assert ending.any() and not ending.all()
    np.testing.assert_array_equal(s2[~ending], start[~ending])
    np.testing.assert_array_equal(e2[~ending], end[~ending])
    np.testing.assert_array_equal(s2[ending], end[ending])
    step = (e2 - s2)[ending].astype(np.uint64)
    assert np.all(step > 0) and np.all((step & (step - np.uint64(1))) == 0)   # powers of two
    S = cfl * _cfl_step(mesh, W, vel, meta["gamma"])[ending]
    # a cell whose CFL step exceeds the longest allowed step takes that, as it
    # is (the reference does not synchronise this branch)
    longest = t_total < S
    assert np.all(step[longest] == TICKS)
    st, sv = step[~longest], S[~longest]
    assert np.all((np.uint64(TICKS) - end[ending][~longest]) % st == 0)     # synchronised
    real = t_total * (st.astype(np.float64) / TICKS)
    assert np.all(real <= sv * (1 + 1e-12))                                 # never above CFL
    # the largest synchronised power of two: doubling breaks one of the rules
    dbl = 2 * st.astype(np.float64)
    sync2 = ((np.uint64(TICKS) - end[ending][~longest]) % (2 * st)) == 0
    assert np.all((t_total * (dbl / TICKS) > sv) | ~sync2)
    assert smin == int(step.min())


def test_bins_clamps_and_the_max_step_branch(oracle):
    mesh, meta, ref = load_case(LOCAL_CASES[0])
    W = meta["W0"]
    n = mesh.n_cells
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    zero = np.zeros(n, np.uint64)
    vel = np.zeros((n, mesh.dim))
    S = 0.4 * _cfl_step(mesh, W, vel, meta["gamma"])
    # max_step shorter than every CFL step: every cell takes max_step
    t_total = 1.0
    max_step = TICKS >> 40
    assert t_total * max_step / TICKS < S.min()
    s2, e2, smin, rc = oracle.timestep_bins(mesh, p, W, vel, zero, zero, 0, t_total, 0.4,
                                            max_step, 0)
    assert rc == 0 and smin == max_step and np.all(e2 == max_step) and np.all(s2 == 0)
    # a min_step above the CFL steps is kept
    t_total = 64 * S.max()
    s2, e2, smin, rc = oracle.timestep_bins(mesh, p, W, vel, zero, zero, 0, t_total, 0.4,
                                            TICKS, TICKS >> 3)
    assert rc == 0 and np.all(e2 == TICKS >> 3)
    # a timeline so long that no tick is short enough: the reference's "Timestep 0!"
    _, _, _, rc = oracle.timestep_bins(mesh, p, W, vel, zero, zero, 0, 1e30, 0.4, TICKS, 0)
    assert rc == 15
