"""One mesh split over several parts (CPU): the Hilbert order, the parts'
rings and face lists, the exchange lists, and the decomposition itself:
passes over the parts, with the ring exchange between steps, give the owned
cells the oracle's whole-mesh values bit for bit."""
import numpy as np
import pytest

from golden_util import load_case
from oracle.oracle import Params
from shadowfax_b200 import partition as P


def _grid(n, dim):
    ax = (np.arange(n) + 0.5) / n
    g = np.stack(np.meshgrid(*([ax] * dim), indexing="ij"), -1).reshape(-1, dim)
    return g, np.rint(g * n - 0.5).astype(int)


@pytest.mark.parametrize("dim,n", [(2, 32), (3, 8)])
def test_hilbert_order_steps_to_a_grid_neighbour(dim, n):
    pos, ijk = _grid(n, dim)
    order = np.argsort(P.hilbert_keys(pos))
    step = np.abs(np.diff(ijk[order], axis=0)).sum(1)
    assert np.all(step == 1)
    assert len(np.unique(P.hilbert_keys(pos))) == len(pos)


def _check_part(mesh, owner, pt):
    loc = pt.mesh
    own = owner == pt.rank
    assert pt.n_own == own.sum() and np.array_equal(np.sort(pt.cells[:pt.n_own]),
                                                    np.flatnonzero(own))
    # owned and ring-1 cells: the whole face list, in the global order
    off, goff = loc.cell_face_offset, mesh.cell_face_offset
    for c in range(pt.n_grad):
        g = pt.cells[c]
        assert np.array_equal(pt.faces[loc.cell_face_index[off[c]:off[c + 1]]],
                              mesh.cell_face_index[goff[g]:goff[g + 1]])
    # faces [0, n_flux): exactly the faces of owned cells and the other
    # copies of their periodic faces (the split pass applies one copy of a
    # pair to both cells)
    sel = np.repeat(own, np.diff(goff))
    mine = np.unique(mesh.cell_face_index[sel])
    twin = P._periodic_twins(mesh)
    want = np.union1d(mine, twin[mine][twin[mine] >= 0])
    assert np.array_equal(np.sort(pt.faces[:pt.n_flux]), want)
    # every periodic face of an owned or ring-1 cell has its twin in the part
    part_faces = set(pt.faces.tolist())
    for f in pt.faces:
        if twin[f] >= 0 and (pt.cells[:pt.n_grad] == mesh.face_left[f]).any():
            assert int(twin[f]) in part_faces
    if mesh.periodic:
        assert (twin >= 0).sum() == (mesh.face_kind == P.KIND_PERIODIC).sum()
        assert np.all(twin[twin[twin >= 0]] == np.flatnonzero(twin >= 0))
    assert np.all(loc.face_left >= 0) and np.all(loc.face_left < loc.n_cells)
    real = loc.face_kind != P.KIND_MIRROR
    assert np.all(loc.face_right[real] >= 0) and np.all(loc.face_right[real] < loc.n_cells)
    assert np.array_equal(pt.cells[loc.face_left], mesh.face_left[pt.faces])
    assert np.array_equal(pt.cells[loc.face_right[real]], mesh.face_right[pt.faces][real])


CASES = ["sod2d_exact", "random2d_periodic_exact", "sedov3d_hllc", "random3d_exact"]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("nparts", [2, 3])
def test_parts_and_exchange_lists(name, nparts):
    mesh, _, _ = load_case(name)
    owner = P.partition(mesh, nparts)
    counts = np.bincount(owner, minlength=nparts)
    assert counts.min() > 0.6 * mesh.n_cells / nparts
    parts = [P.build_part(mesh, owner, r) for r in range(nparts)]
    for pt in parts:
        _check_part(mesh, owner, pt)
    plans = [P.exchange_plan(mesh, owner, pt) for pt in parts]
    for r, pt in enumerate(parts):
        # every ring cell is received exactly once, from its owner
        got = np.concatenate([pt.cells[rv] for (_, rv) in plans[r].values()] or [[]])
        assert np.array_equal(np.sort(got), np.sort(pt.cells[pt.n_own:]))
        for p, (snd, rcv) in plans[r].items():
            assert np.all(snd < pt.n_own)
            assert np.array_equal(pt.cells[snd], parts[p].cells[plans[p][r][1]])
            assert np.all(owner[pt.cells[rcv]] == p)


def _exchange_host(parts, plans, W, Q):
    recs = {}
    for r, pt in enumerate(parts):
        for p, (snd, _) in plans[r].items():
            recs[(r, p)] = np.concatenate([W[r][snd], Q[r][snd, :1]], axis=1)
    for r, pt in enumerate(parts):
        for p, (_, rcv) in plans[r].items():
            rec = recs[(p, r)]
            W[r][rcv] = rec[:, :-1]
            Q[r][rcv, 0] = rec[:, -1]


@pytest.mark.parametrize("name", CASES)
def test_decomposed_steps_equal_the_whole_mesh(oracle, name):
    """per part: gradients, fluxes and the update over the local mesh, the
    owned cells kept; the ring cells' W and mass from their owners between
    steps.  After several steps the owned cells equal the oracle's steps
    over the whole mesh bit for bit (the per-part pass here is the oracle,
    standing in for the device)."""
    mesh, meta, _ = load_case(name)
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    dt, nsteps = meta["dt"], 4
    Wg = meta["W0"].copy()
    Qg = oracle.init_Q(mesh, p, Wg)
    owner = P.partition(mesh, 3)
    parts = [P.build_part(mesh, owner, r) for r in range(3)]
    plans = [P.exchange_plan(mesh, owner, pt) for pt in parts]
    W = [Wg[pt.cells].copy() for pt in parts]
    Q = [oracle.init_Q(pt.mesh, p, W[r]) for r, pt in enumerate(parts)]
    for r, pt in enumerate(parts):
        assert np.array_equal(Q[r], Qg[pt.cells])
    for _ in range(nsteps):
        grad, dQ, code, rc, bad = oracle.flux_pass(mesh, p, dt, Wg, Qg)
        assert rc == 0
        Wg, Qg, rc, bad = oracle.apply(mesh, p, dQ, Wg, Qg)
        assert rc == 0
        for r, pt in enumerate(parts):
            lg, ldQ, lcode, lrc, lbad = oracle.flux_pass(pt.mesh, p, dt, W[r], Q[r])
            assert np.array_equal(lg[:pt.n_grad], grad[pt.cells[:pt.n_grad]])
            assert np.array_equal(ldQ[:pt.n_flux], dQ[pt.faces[:pt.n_flux]])
            # the oracle's update runs over every local cell; the device pass
            # updates the owned cells only.  The ring cells get a mass and
            # energy far above their partial face sums here, so that they pass
            # the update's sign check, and only the owned cells are kept.
            Qt = Q[r].copy()
            Qt[pt.n_own:, [0, -1]] = 1e300
            Wn, Qn, arc, _ = oracle.apply(pt.mesh, p, ldQ, W[r], Qt)
            assert arc == 0
            W[r][:pt.n_own] = Wn[:pt.n_own]
            Q[r][:pt.n_own] = Qn[:pt.n_own]
        _exchange_host(parts, plans, W, Q)
    for r, pt in enumerate(parts):
        assert np.array_equal(W[r], Wg[pt.cells])
        assert np.array_equal(Q[r][:pt.n_own], Qg[pt.cells[:pt.n_own]])
        assert np.array_equal(Q[r][:, 0], Qg[pt.cells, 0])


def test_one_part_is_the_whole_mesh_and_bad_counts_are_refused():
    mesh, _, _ = load_case("random2d_periodic_exact")
    owner = P.partition(mesh, 1)
    assert np.all(owner == 0)
    pt = P.build_part(mesh, owner, 0)
    assert pt.n_own == pt.n_grad == mesh.n_cells == len(pt.cells)
    assert pt.n_flux == mesh.n_faces
    assert np.array_equal(pt.cells, np.arange(mesh.n_cells))
    assert np.array_equal(pt.mesh.cell_face_index, mesh.cell_face_index)
    assert P.exchange_plan(mesh, owner, pt) == {}
    for bad in (0, mesh.n_cells + 1):
        with pytest.raises(ValueError):
            P.partition(mesh, bad)
