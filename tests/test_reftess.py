"""Face lists of the reference's own tessellation (TEST of the exporter and
of the face-list conventions, CPU).

The fixtures (tests/golden/make_reftess.py) hold meshes that the reference's
own DelTess/VorTess built from seeded generators (exact predicates through
the fixed-width integer stand-in, whose arithmetic the reference's own
test/testExArith.cpp checks), exported in the library's face-list layout,
and the reference's step loop run on that tessellation:

* the oracle on the exported face list equals the reference's own pass on
  its own tessellation bit for bit (sfx_pow) and within 1e-12 per field with
  glibc pow: the exporter carries everything the pass uses, zero-area faces,
  periodic images and reflective mirrors included;
* the library's face-list builder (sfx_voronoi) makes the same mesh from the
  same generators: the same active faces between the same cells, areas,
  midpoints, volumes and centroids within round-off;
* the exported conventions: zero-area faces stay in the list (the pass skips
  them), a periodic image is the right cell shifted by whole box lengths, a
  mirror is the left cell reflected in a box wall."""
import numpy as np
import pytest

from golden_util import REFTESS_CASES, load_case


@pytest.mark.parametrize("name", REFTESS_CASES)
def test_oracle_on_reference_tessellation_bitwise(oracle, name):
    from oracle.oracle import Params
    mesh, meta, ref = load_case(name)
    p = Params(solver=meta["solver"], gamma=meta["gamma"])
    o = oracle.run(mesh, p, meta["dt"], meta["nsteps"], meta["W0"])
    np.testing.assert_array_equal(o["Q"], ref["ref_sfxpow_Q"])
    np.testing.assert_array_equal(o["W"], ref["ref_sfxpow_W"])
    ol = oracle.run(mesh, Params(solver=meta["solver"], gamma=meta["gamma"], use_libm_pow=True),
                    meta["dt"], meta["nsteps"], meta["W0"])
    b = ref["ref_libm_Q"]
    for k in range(b.shape[1]):
        lim = 1e-12 * np.abs(b[:, k]) + 1e-15 * np.abs(b[:, k]).max()
        assert np.all(np.abs(ol["Q"][:, k] - b[:, k]) <= lim), k


def _pairs(mesh):
    """active faces keyed by (left, right, kind, rounded right position)"""
    act = mesh.face_area > 0
    out = {}
    for f in np.nonzero(act)[0]:
        key = (int(mesh.face_left[f]), int(mesh.face_right[f]), int(mesh.face_kind[f]),
               tuple(np.round(mesh.face_right_pos[f], 9)))
        out[key] = f
    return out


@pytest.mark.parametrize("name", REFTESS_CASES)
def test_reference_tessellation_matches_the_builder(name):
    from shadowfax_b200.mesh import build_voronoi
    mesh, meta, _ = load_case(name)
    ours = build_voronoi(mesh.cell_pos, periodic=mesh.periodic)
    np.testing.assert_allclose(ours.cell_volume, mesh.cell_volume, rtol=1e-11)
    np.testing.assert_allclose(ours.cell_centroid, mesh.cell_centroid, rtol=0, atol=1e-12)
    np.testing.assert_allclose(ours.cell_total_area, mesh.cell_total_area, rtol=1e-11)
    a, b = _pairs(mesh), _pairs(ours)

    def canon(k):
        l, r, kind, x = k
        return (min(l, r), max(l, r), kind) if kind == 0 else k

    ca = {canon(k): f for k, f in a.items()}
    cb = {canon(k): f for k, f in b.items()}
    # faces of the reference's tessellation the builder has too (a periodic
    # face may be listed from either cell, with the image of the other)
    real_a = {k for k in ca if k[2] == 0}
    real_b = {k for k in cb if k[2] == 0}
    assert real_a == real_b
    for k in real_a:
        fa, fb = ca[k], cb[k]
        # two algorithms (the reference's Delaunay dual, the builder's cell
        # clipping): agreement to round-off of the geometry
        assert abs(mesh.face_area[fa] - ours.face_area[fb]) <= 1e-10 * mesh.face_area[fa] + 1e-14
        np.testing.assert_allclose(mesh.face_midpoint[fa], ours.face_midpoint[fb], atol=1e-12)
    for kind in (1, 2):
        assert (mesh.face_kind[mesh.face_area > 0] == kind).sum() == \
            (ours.face_kind[ours.face_area > 0] == kind).sum()
    # every cell is enclosed: its total area and volume agree, and the box is filled
    assert abs(mesh.cell_volume.sum() - 1.0) <= 1e-12


@pytest.mark.parametrize("name", REFTESS_CASES)
def test_reference_face_conventions(name):
    mesh, _, _ = load_case(name)
    F = mesh.n_faces
    zero = mesh.face_area == 0
    # zero-area faces are real or mirror faces, listed in their cells' face lists
    counts = np.bincount(mesh.cell_face_index, minlength=F)
    assert np.all(counts[mesh.face_kind == 0] == 2)
    assert np.all(counts[mesh.face_kind != 0] == 1)
    per = mesh.face_kind == 1
    if per.any():
        shift = mesh.face_right_pos[per] - mesh.cell_pos[mesh.face_right[per]]
        assert np.allclose(shift, np.round(shift), atol=1e-12)
        assert np.all(np.abs(np.round(shift)).sum(1) >= 1)
    mir = mesh.face_kind == 2
    if mir.any():
        assert np.all(mesh.face_right[mir] == -1)
        d = mesh.face_right_pos[mir] - mesh.cell_pos[mesh.face_left[mir]]
        walls = (np.abs(d) > 1e-15).sum(1)
        # a mirror face of nonzero area is the left cell reflected in one
        # wall; images in two or more walls (edges and corners of the box)
        # give the reference's degenerate, zero-area faces
        assert np.all(walls[mesh.face_area[mir] > 0] == 1)
        assert np.all(mesh.face_area[mir][walls > 1] == 0)
    if not mesh.periodic:
        assert not per.any()
    else:
        assert not mir.any()
    # the reference keeps degenerate faces (fewer than three distinct
    # vertices) with zero area (src/VorTess.cpp:253-264); none is periodic
    assert not (zero & per).any()
