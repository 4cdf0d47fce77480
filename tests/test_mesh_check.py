"""sfx_mesh_check: the checks sfx_mesh_upload makes of a face list, run on the
host alone.  Every committed mesh passes in both precisions; each kind of
defect gets the status the upload returns for it."""
import ctypes
import dataclasses
import glob
from pathlib import Path

import numpy as np
import pytest

from shadowfax_b200 import _lib as L
from shadowfax_b200.mesh import Mesh, build_voronoi, random_generators

GOLDEN = Path(__file__).resolve().parent / "golden"


def _fixture_meshes():
    out = []
    for f in sorted(glob.glob(str(GOLDEN / "*.npz"))):
        z = np.load(f)
        if not all(a in z.files for a in Mesh._ARRAYS):
            continue
        periodic = bool(int(z["periodic"])) if "periodic" in z.files else False
        out.append((Path(f).stem, Mesh(dim=int(z["dim"]), periodic=periodic,
                                       **{a: z[a] for a in Mesh._ARRAYS}).normalized()))
    return out


def _status(mesh, precision=L.PREC_FP64):
    d = mesh.desc()
    return L.lib().sfx_mesh_check(ctypes.byref(d), precision)


@pytest.fixture(scope="module")
def periodic2d():
    return build_voronoi(random_generators(400, 2, 3), periodic=True)


def test_committed_meshes_pass_in_both_precisions():
    meshes = _fixture_meshes()
    assert len(meshes) >= 10
    for name, m in meshes:
        for precision in (L.PREC_FP64, L.PREC_SPLIT):
            assert _status(m, precision) == 0, (name, precision)
            m.check(precision)


@pytest.mark.parametrize("dim,periodic", [(2, False), (2, True), (3, False), (3, True)])
def test_builder_meshes_pass(dim, periodic):
    m = build_voronoi(random_generators(300, dim, 11), periodic=periodic)
    assert _status(m, L.PREC_FP64) == 0 and _status(m, L.PREC_SPLIT) == 0


def _with(mesh, **arrays):
    return dataclasses.replace(mesh, **arrays)


def test_index_defects_are_bounds_errors(periodic2d):
    m = periodic2d
    n, F = m.n_cells, m.n_faces
    real = int(np.flatnonzero(m.face_kind == 0)[0])
    left = m.face_left.copy()
    left[5] = n
    right = m.face_right.copy()
    right[real] = -1
    kind = m.face_kind.copy()
    kind[7] = 5
    off = m.cell_face_offset.copy()
    off[0] = 1
    dec = m.cell_face_offset.copy()
    dec[3] = dec[2] - 1
    idx = m.cell_face_index.copy()
    idx[0] = F
    cases = {"left out of range": _with(m, face_left=left),
             "right of a real face out of range": _with(m, face_right=right),
             "unknown face kind": _with(m, face_kind=kind),
             "offsets not from 0": _with(m, cell_face_offset=off),
             "decreasing offsets": _with(m, cell_face_offset=dec),
             "face index out of range": _with(m, cell_face_index=idx)}
    # a cell listing a face it is not on: cell 0's first entry replaced by a
    # face that neither starts nor ends at cell 0
    foreign = int(np.flatnonzero((m.face_left != 0) & (m.face_right != 0))[0])
    idx2 = m.cell_face_index.copy()
    idx2[m.cell_face_offset[0]] = foreign
    cases["face not on the cell"] = _with(m, cell_face_index=idx2)
    # a periodic face listed by its right cell (only real faces are)
    per = int(np.flatnonzero(m.face_kind == 1)[0])
    R = int(m.face_right[per])
    idx3 = m.cell_face_index.copy()
    idx3[m.cell_face_offset[R]] = per
    if m.face_left[per] != R:
        cases["periodic face listed by its right cell"] = _with(m, cell_face_index=idx3)
    for what, bad in cases.items():
        for precision in (L.PREC_FP64, L.PREC_SPLIT):
            assert _status(bad, precision) == L.SFX_ERR_BOUNDS, what
    with pytest.raises(L.SfxError) as e:
        cases["unknown face kind"].check()
    assert e.value.status == L.SFX_ERR_BOUNDS


def test_missing_arrays_and_bad_arguments_are_invalid(periodic2d):
    d = periodic2d.desc()
    d.face_area = None
    assert L.lib().sfx_mesh_check(ctypes.byref(d), L.PREC_FP64) == L.SFX_ERR_INVALID
    d = periodic2d.desc()
    d.n_cells = 0
    assert L.lib().sfx_mesh_check(ctypes.byref(d), L.PREC_FP64) == L.SFX_ERR_INVALID
    d = periodic2d.desc()
    d.dim = 4
    assert L.lib().sfx_mesh_check(ctypes.byref(d), L.PREC_FP64) == L.SFX_ERR_INVALID
    d = periodic2d.desc()
    assert L.lib().sfx_mesh_check(ctypes.byref(d), 2) == L.SFX_ERR_INVALID
    assert L.lib().sfx_mesh_check(None, L.PREC_FP64) == L.SFX_ERR_INVALID


def test_split_takes_periodic_meshes_of_the_unit_box_only(periodic2d):
    m = periodic2d
    D = m.dim
    big = _with(m, cell_pos=m.cell_pos * 2., cell_centroid=m.cell_centroid * 2.,
                cell_volume=m.cell_volume * 2. ** D,
                cell_total_area=m.cell_total_area * 2. ** (D - 1),
                face_area=m.face_area * 2. ** (D - 1), face_midpoint=m.face_midpoint * 2.,
                face_right_pos=m.face_right_pos * 2.)
    assert _status(big, L.PREC_FP64) == 0
    assert _status(big, L.PREC_SPLIT) == L.SFX_ERR_UNSUPPORTED
    # a reflective mesh scaled the same way has no periodic image to refuse
    refl = build_voronoi(random_generators(300, 2, 5), periodic=False)
    big_refl = _with(refl, cell_pos=refl.cell_pos * 2., face_right_pos=refl.face_right_pos * 2.)
    assert _status(big_refl, L.PREC_SPLIT) == 0


def test_empty_and_ragged_face_lists():
    """no faces at all (one isolated cell, every face array empty) is a valid
    face list; so is one whose cells list very different numbers of faces"""
    one = Mesh(dim=2, periodic=False, cell_pos=np.array([[0.5, 0.5]]),
               cell_centroid=np.array([[0.5, 0.5]]), cell_volume=np.array([1.0]),
               cell_total_area=np.array([4.0]), cell_face_offset=np.array([0, 0], np.int32),
               cell_face_index=np.zeros(0, np.int32), face_area=np.zeros(0),
               face_midpoint=np.zeros((0, 2)), face_left=np.zeros(0, np.int32),
               face_right=np.zeros(0, np.int32), face_kind=np.zeros(0, np.int32),
               face_right_pos=np.zeros((0, 2))).normalized()
    for precision in (L.PREC_FP64, L.PREC_SPLIT):
        assert _status(one, precision) == 0
    m = build_voronoi(random_generators(300, 3, 9), periodic=False)
    counts = np.diff(m.cell_face_offset)
    assert counts.min() < counts.max()     # ragged by construction
    assert _status(m, L.PREC_SPLIT) == 0


def _expected_status(m, split):
    """the face-list rules, stated independently of the library"""
    n, F = m.n_cells, m.n_faces
    off, idx = m.cell_face_offset, m.cell_face_index
    if off[0] != 0 or np.any(np.diff(off) < 0):
        return L.SFX_ERR_BOUNDS
    L_, R_, K_ = m.face_left, m.face_right, m.face_kind
    if np.any((L_ < 0) | (L_ >= n)) or np.any(~np.isin(K_, [0, 1, 2])):
        return L.SFX_ERR_BOUNDS
    has_r = (K_ == 0) | (K_ == 1)
    if np.any(has_r & ((R_ < 0) | (R_ >= n))):
        return L.SFX_ERR_BOUNDS
    if off[-1] > len(idx):
        return None                        # the arrays themselves are too short: not fuzzed
    for i in range(n):
        for j in range(off[i], off[i + 1]):
            f = idx[j]
            if f < 0 or f >= F:
                return L.SFX_ERR_BOUNDS
            if L_[f] != i and not (R_[f] == i and K_[f] == 0):
                return L.SFX_ERR_BOUNDS
    if split:
        per = np.flatnonzero(K_ == 1)
        a = np.abs(m.face_right_pos[per] - m.cell_pos[R_[per]])
        if np.any(~((a <= 1e-9) | (np.abs(a - 1.0) <= 1e-9))):
            return L.SFX_ERR_UNSUPPORTED
    return 0


def test_random_corruptions_get_the_rules_status(periodic2d):
    m0 = periodic2d
    rng = np.random.Generator(np.random.PCG64(77))
    fields = ["face_left", "face_right", "face_kind", "cell_face_index", "cell_face_offset",
              "face_right_pos"]
    seen = set()
    for trial in range(150):
        arrays = {}
        for _ in range(int(rng.integers(1, 3))):
            name = fields[int(rng.integers(len(fields)))]
            a = arrays.get(name, getattr(m0, name)).copy()
            k = int(rng.integers(a.shape[0]))
            if name == "face_right_pos":
                a[k, int(rng.integers(a.shape[1]))] += rng.choice([0.5, 1.0, 1e-12, 2.0])
            elif name == "cell_face_offset":
                if k == len(a) - 1:
                    k -= 1          # the last offset sizes the index array itself
                a[k] += int(rng.integers(-3, 4))
            else:
                a[k] = int(rng.integers(-2, max(m0.n_cells, m0.n_faces) + 2))
            arrays[name] = a
        m = _with(m0, **arrays)
        for split in (False, True):
            want = _expected_status(m, split)
            if want is None:
                continue
            got = _status(m, L.PREC_SPLIT if split else L.PREC_FP64)
            assert got == want, (trial, split, sorted(arrays), got, want)
            seen.add(want)
    assert seen == {0, L.SFX_ERR_BOUNDS, L.SFX_ERR_UNSUPPORTED}
