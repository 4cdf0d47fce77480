"""Request server (continuous batching): every request's result is the same
whether it runs alone or co-batched with others, FP64 requests equal the
plain FP64 pass bit for bit, a failing request stops only itself, and the
memory budget holds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems():
    """a mix of 2D and 3D meshes, both solvers, uneven sizes and step counts"""
    from shadowfax_b200 import workloads as wl
    return [
        wl.step_state2d(600, 51, solver="HLLC", nsteps=7),
        wl.step_state2d(2500, 52, solver="Exact", nsteps=12),
        wl.sedov3d(n=1500, seed=53, solver="HLLC", nsteps=5),
        wl.step_state2d(1200, 54, solver="HLLC", nsteps=19),
        wl.sedov3d(n=800, seed=55, solver="Exact", nsteps=9),
        wl.step_state2d(300, 56, solver="Exact", nsteps=3),
    ]


def _alone(pr, precision):
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    ctx = Context(pr.mesh.dim, RiemannSolverFactory.generate(pr.solver, pr.gamma), precision)
    fp = FluxPass(ctx, pr.mesh)
    fp.set_primitive(pr.W0)
    fp.step(pr.dt, pr.nsteps)
    return fp.state()


def _serve(probs, precision, chunk_steps=4, tuning=None, **kw):
    from shadowfax_b200.serve import Server
    srv = Server(precision=precision, chunk_steps=chunk_steps, **kw)
    try:
        for (d, solver), t in (tuning or {}).items():
            srv.set_tuning(d, solver, *t)
        ids = [srv.add_mesh(pr.mesh) for pr in probs]
        rids = [srv.submit(i, pr.W0, pr.solver, pr.dt, pr.nsteps) for i, pr in zip(ids, probs)]
        assert srv.drain(120.0)
        res = [srv.poll(r) for r in rids]
        st = srv.stats()
    finally:
        srv.shutdown()
    return res, st


@pytest.mark.parametrize("precision", [0, 1])
def test_requests_in_a_mix_equal_requests_alone(cuda_ok, precision):
    probs = _problems()
    res, st = _serve(probs, precision)
    assert st.completed == len(probs) and st.failed == 0 and st.bytes_in_use == 0
    for pr, r in zip(probs, res):
        assert r.status == 0 and r.steps_done == pr.nsteps
        W, Q = _alone(pr, precision)
        np.testing.assert_array_equal(r.Q, Q)
        np.testing.assert_array_equal(r.W, W)
        assert r.face_steps == pr.nsteps * pr.mesh.n_active_faces
        assert r.t_submit <= r.t_admit <= r.t_done


def test_tuned_server(cuda_ok):
    """kernel settings per class: the 80-register face kernels change the
    schedule only (bitwise the same results as alone); other lanes per cell
    and the gamma = 5/3 exact forms stay within the split pass's round-off;
    an FP64 server refuses tuning"""
    from shadowfax_b200._lib import SfxError
    probs = _problems()
    classes = [(d, s) for d in (2, 3) for s in ("Exact", "HLLC")]
    res, st = _serve(probs, 1, tuning={c: (0, 1) for c in classes})
    assert st.completed == len(probs) and st.failed == 0
    for pr, r in zip(probs, res):
        np.testing.assert_array_equal(r.Q, _alone(pr, 1)[1])
    res, _ = _serve(probs, 1, tuning={c: (2, 3) for c in classes})
    for pr, r in zip(probs, res):
        assert r.status == 0
        Q = _alone(pr, 1)[1]
        err = np.abs(r.Q - Q).sum(0) / np.abs(Q).sum(0)
        assert np.all(err[[0, -1]] <= 1e-6), err
    with pytest.raises(SfxError):
        _serve(probs[:1], 0, tuning={(2, "HLLC"): (0, 0)})


def test_one_request_alone_and_in_mix(cuda_ok):
    """the same request served by itself and among five others"""
    probs = _problems()
    alone, _ = _serve([probs[3]], 1)
    mixed, _ = _serve(probs, 1, chunk_steps=5)
    np.testing.assert_array_equal(alone[0].Q, mixed[3].Q)


def test_split_server_within_tolerance_of_fp64_server(cuda_ok):
    """<= 1e-6 relative L1 per conserved field.  These flows start at rest
    and run a few steps, so their momentum is still far below its natural
    scale, the momentum m c a sound wave carries: the momentum error is
    normalised by the larger of the momentum L1 norm and sum(m c)."""
    probs = _problems()
    r64, _ = _serve(probs, 0)
    r32, _ = _serve(probs, 1)
    for pr, a, b in zip(probs, r32, r64):
        D = pr.mesh.dim
        den = np.abs(b.Q).sum(0)
        c = np.sqrt(pr.gamma * b.W[:, D + 1] / b.W[:, 0])
        den[1:D + 1] = max(np.sqrt((b.Q[:, 1:D + 1] ** 2).sum(1)).sum(), (b.Q[:, 0] * c).sum())
        err = np.abs(a.Q - b.Q).sum(0) / den
        assert np.all(err <= 1e-6), err


def test_failing_request_stops_only_itself(cuda_ok):
    from shadowfax_b200.serve import Server
    probs = _problems()[:4]
    srv = Server(precision=1, chunk_steps=3)
    try:
        ids = [srv.add_mesh(pr.mesh) for pr in probs]
        rids = []
        for j, (i, pr) in enumerate(zip(ids, probs)):
            W0 = pr.W0.copy()
            if j == 1:
                W0[11, 0] = np.nan
            rids.append(srv.submit(i, W0, pr.solver, pr.dt, pr.nsteps))
        assert srv.drain(120.0)
        res = [srv.poll(r) for r in rids]
    finally:
        srv.shutdown()
    assert res[1].status != 0
    for j in (0, 2, 3):
        assert res[j].status == 0
        np.testing.assert_array_equal(res[j].Q, _alone(probs[j], 1)[1])


def test_memory_budget_admits_one_at_a_time(cuda_ok):
    """a budget below two request states: requests run one after another and
    all finish with the same results"""
    import time
    from shadowfax_b200.serve import Server
    probs = [p for p in _problems() if p.mesh.dim == 2]
    srv = Server(precision=1, memory_budget=1, chunk_steps=2)
    try:
        ids = [srv.add_mesh(pr.mesh) for pr in probs]
        rids = [srv.submit(i, pr.W0, pr.solver, pr.dt, pr.nsteps) for i, pr in zip(ids, probs)]
        peak_active = 0
        while True:
            st = srv.stats()
            peak_active = max(peak_active, st.active)
            if st.completed + st.failed == len(probs):
                break
            time.sleep(0.0005)
        res = [srv.poll(r) for r in rids]
    finally:
        srv.shutdown()
    assert peak_active <= 1
    for pr, r in zip(probs, res):
        assert r.status == 0
        np.testing.assert_array_equal(r.Q, _alone(pr, 1)[1])


def test_requests_arriving_while_others_run(cuda_ok):
    """continuous batching: requests submitted after the first rounds started
    join the running group and still equal their runs alone"""
    import time
    from shadowfax_b200.serve import Server
    probs = _problems()
    srv = Server(precision=1, chunk_steps=1)
    try:
        ids = [srv.add_mesh(pr.mesh) for pr in probs]
        rids = []
        for i, pr in zip(ids, probs):
            rids.append(srv.submit(i, pr.W0, pr.solver, pr.dt, pr.nsteps))
            time.sleep(0.002)
        assert srv.drain(120.0)
        res = [srv.poll(r) for r in rids]
        with pytest.raises(Exception):
            srv.poll(rids[0])  # collected requests are forgotten
    finally:
        srv.shutdown()
    for pr, r in zip(probs, res):
        assert r.status == 0
        np.testing.assert_array_equal(r.Q, _alone(pr, 1)[1])
