"""Launch groups (many meshes per launch): each member's result equals the
same mesh advanced alone, a failing member stops only itself."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(dim, solver, sizes, seed=40):
    from shadowfax_b200 import workloads as wl
    out = []
    for j, n in enumerate(sizes):
        if dim == 2:
            pr = wl.step_state2d(int(n), seed + j, solver=solver, nsteps=5)
        else:
            pr = wl.sedov3d(n=int(n), seed=seed + j, solver=solver, nsteps=5)
        out.append(pr)
    return out


def _alone(pr):
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    ctx = Context(pr.mesh.dim, RiemannSolverFactory.generate(pr.solver, pr.gamma), 1)
    fp = FluxPass(ctx, pr.mesh)
    fp.set_primitive(pr.W0)
    fp.step(pr.dt, pr.nsteps)
    return fp.state()


@pytest.mark.parametrize("dim,solver", [(2, "HLLC"), (2, "Exact"), (3, "HLLC")])
@pytest.mark.parametrize("graph", [False, True])
def test_group_members_match_alone(cuda_ok, dim, solver, graph):
    from shadowfax_b200.hydro import Context, FluxPass, Group, RiemannSolverFactory
    sizes = [300, 1700, 800, 4000, 150] if dim == 2 else [500, 2500, 1200]
    probs = _problems(dim, solver, sizes)
    ctx = Context(dim, RiemannSolverFactory.generate(solver), 1)
    members = []
    for pr in probs:
        fp = FluxPass(ctx, pr.mesh)
        fp.set_primitive(pr.W0)
        members.append(fp)
    g = Group(ctx, members, [pr.dt for pr in probs])
    st = g.step(probs[0].nsteps, graph=graph)
    assert np.all(st == 0)
    for pr, fp in zip(probs, members):
        W, Q = fp.state()
        Wa, Qa = _alone(pr)
        np.testing.assert_array_equal(Q, Qa)
        np.testing.assert_array_equal(W, Wa)


def test_failing_member_stops_only_itself(cuda_ok):
    from shadowfax_b200.hydro import Context, FluxPass, Group, RiemannSolverFactory
    probs = _problems(2, "HLLC", [400, 900, 600])
    ctx = Context(2, RiemannSolverFactory.generate("HLLC"), 1)
    members = []
    for j, pr in enumerate(probs):
        fp = FluxPass(ctx, pr.mesh)
        W0 = pr.W0.copy()
        if j == 1:
            W0[7, 0] = np.nan
        fp.set_primitive(W0)
        members.append(fp)
    g = Group(ctx, members, [pr.dt for pr in probs])
    st = g.step(probs[0].nsteps, graph=True)
    assert st[1] != 0 and st[0] == 0 and st[2] == 0
    for j in (0, 2):
        np.testing.assert_array_equal(members[j].state()[1], _alone(probs[j])[1])


def test_tune_picks_a_variant_and_stays_within_tolerance(cuda_ok):
    from shadowfax_b200.hydro import Context, FluxPass, Group, RiemannSolverFactory
    probs = _problems(3, "HLLC", [3000, 1500])
    ctx = Context(3, RiemannSolverFactory.generate("HLLC"), 1)
    members = [FluxPass(ctx, pr.mesh) for pr in probs]
    for fp, pr in zip(members, probs):
        fp.set_primitive(pr.W0)
    g = Group(ctx, members, [pr.dt for pr in probs])
    lanes = g.tune(2)
    assert lanes in (1, 2, 4, 8, 16)
    st = g.step(probs[0].nsteps)
    assert np.all(st == 0)
    for pr, fp in zip(probs, members):
        Q = fp.state()[1]
        Qa = _alone(pr)[1]
        err = np.abs(Q - Qa).sum(0) / np.abs(Qa).sum(0)
        assert np.all(err[[0, -1]] <= 1e-6)


@pytest.mark.parametrize("dim,solver", [(2, "Exact"), (3, "Exact"), (3, "HLLC")])
def test_face_variants_give_the_same_result(cuda_ok, dim, solver):
    """variants 0 and 1 of the face kernel differ only in their register cap:
    the same result bit for bit, and so do 2, 3 and 4 (left cells staged in
    shared memory by bulk copies) for the exact solver (HLLC: 3 is the
    48-register kernel and 4 that with staged cells, bitwise 0 too); variant 2 (HLLC: the prediction's dW/dt from the
    per-cell record; exact solver at gamma 5/3: fifth roots and integer
    powers) and the variant the face tuner keeps are within the split pass's
    round-off of 0"""
    from shadowfax_b200._lib import SfxError
    from shadowfax_b200.hydro import Context, FluxPass, Group, RiemannSolverFactory
    sizes = [2500, 900, 4000] if dim == 2 else [2000, 1200]
    probs = _problems(dim, solver, sizes)
    ctx = Context(dim, RiemannSolverFactory.generate(solver), 1)
    results = {}
    for v in (0, 1, 2, 3, 4, "tuned"):
        members = [FluxPass(ctx, pr.mesh) for pr in probs]
        for fp, pr in zip(members, probs):
            fp.set_primitive(pr.W0)
        g = Group(ctx, members, [pr.dt for pr in probs])
        if v == "tuned":
            Q0 = [fp.state()[1] for fp in members]
            assert g.tune_faces(2) in (0, 1, 2, 3, 4)
            for fp, q in zip(members, Q0):          # tuning reads the states only
                assert np.array_equal(fp.state()[1], q)
        else:
            g.set_face_variant(v)
        assert np.all(g.step(probs[0].nsteps, graph=True) == 0)
        results[v] = [fp.state()[1] for fp in members]
        g.close()
        for fp in members:
            fp.close()
    for a, b in zip(results[1], results[0]):
        np.testing.assert_array_equal(a, b)
    for v in (3, 4):       # the same arithmetic as 2 (exact) or 0 (HLLC)
        for a, b in zip(results[v], results[2 if solver == "Exact" else 0]):
            np.testing.assert_array_equal(a, b)
    for v in (2, "tuned"):
        for a, b in zip(results[v], results[0]):
            err = np.abs(a - b).sum(0) / np.abs(b).sum(0)
            assert np.all(err[[0, -1]] <= 1e-6), err
    with pytest.raises(SfxError):
        Group(ctx, [FluxPass(ctx, probs[0].mesh)], [probs[0].dt]).set_face_variant(5)
