"""The host face-list builder produces valid, deterministic tessellations."""
import numpy as np
import pytest

from shadowfax_b200.mesh import build_voronoi, random_generators


@pytest.mark.parametrize("dim,n", [(2, 800), (3, 1500)])
@pytest.mark.parametrize("periodic", [False, True])
def test_tessellation_invariants(dim, n, periodic):
    pos = random_generators(n, dim, 3)
    m = build_voronoi(pos, periodic=periodic)
    assert abs(m.cell_volume.sum() - 1.0) < 1e-12
    assert np.all(m.cell_volume > 0)
    # every face is listed by its left cell and, if real, by its right cell
    off, idx = m.cell_face_offset, m.cell_face_index
    count = np.zeros(m.n_faces, int)
    for i in range(m.n_cells):
        fs = idx[off[i]:off[i + 1]]
        assert np.all(np.diff(fs) > 0)  # ascending face order
        for f in fs:
            assert m.face_left[f] == i or (m.face_right[f] == i and m.face_kind[f] == 0)
            count[f] += 1
    assert np.all(count == np.where(m.face_kind == 0, 2, 1))
    # total area = sum of the cell's face areas in its face order
    ta = np.array([m.face_area[idx[off[i]:off[i + 1]]].sum() for i in range(m.n_cells)])
    np.testing.assert_allclose(ta, m.cell_total_area, rtol=1e-15)
    # the divergence theorem: sum_f A_f n_f = 0 for each closed cell
    for i in range(0, m.n_cells, max(1, m.n_cells // 50)):
        s = np.zeros(dim)
        for f in idx[off[i]:off[i + 1]]:
            xr = m.face_right_pos[f] if m.face_left[f] == i else m.cell_pos[m.face_left[f]]
            d = xr - m.cell_pos[i]
            s += m.face_area[f] * d / np.linalg.norm(d)
        assert np.linalg.norm(s) < 1e-9
    if periodic:
        assert np.all(m.face_kind != 2)
        # the two copies of a periodic face have the same area
        per = np.where(m.face_kind == 1)[0]
        assert len(per) % 2 == 0
    else:
        assert np.all(m.face_kind != 1)
        walls = m.face_kind == 2
        assert abs(m.face_area[walls].sum() - 2 * dim) < 1e-12


def test_build_is_deterministic_across_thread_counts():
    pos = random_generators(3000, 3, 9)
    a = build_voronoi(pos, nthreads=1)
    b = build_voronoi(pos, nthreads=5)
    for name in a._ARRAYS:
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name))
