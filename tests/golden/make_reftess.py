"""Generate the reference-tessellation fixtures tests/golden/reftess_*.npz.

Each case tessellates seeded generator positions with the reference's own
DelTess/VorTess (oracle/_ref/tessharness_*, the unmodified Shadowfax sources
with the fixed-width integer stand-in for the exact predicates), exports the
face list in the library's layout and runs the reference's step loop on that
tessellation, with the reference's pow (libm) and with the library's sfx_pow.
A fixture holds the input positions, the exported mesh (cells in the
reference's Hilbert order), the initial state in that order and both final
states.  Needs the reference tree (oracle/build.py); the tests only read the
fixtures.

    python tests/golden/make_reftess.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle.build import build_reference  # noqa: E402
from oracle.oracle import Params, reference_tessellation  # noqa: E402
from shadowfax_b200.mesh import build_voronoi, random_generators  # noqa: E402
from shadowfax_b200 import workloads as wl  # noqa: E402

DT = 1e-4
NSTEPS = 4


def cases():
    """(name, dim, n, periodic, solver, seed, state)"""
    yield "sod2d_reflective_exact", 2, 600, False, "Exact", 11, "sod"
    yield "random2d_periodic_hllc", 2, 700, True, "HLLC", 12, "random"
    yield "sedov3d_reflective_hllc", 3, 500, False, "HLLC", 13, "sedov"
    yield "random3d_periodic_exact", 3, 500, True, "Exact", 14, "random"


def initial_state(kind: str, pos: np.ndarray, periodic: bool) -> np.ndarray:
    n, dim = pos.shape
    W = np.zeros((n, dim + 2))
    if kind == "sod":
        left = pos[:, 0] < 0.5
        W[:, 0] = np.where(left, 1.0, 0.125)
        W[:, -1] = np.where(left, 1.0, 0.1)
    elif kind == "sedov":
        W[:, 0] = 1.0
        W[:, -1] = 1e-6
        hot = np.argsort(((pos - 0.5) ** 2).sum(1))[:8]
        W[hot, -1] = 1.0
    else:
        W = wl.random_field_state(build_voronoi(pos, periodic=periodic), 5)
    return W


def main():
    build_reference()
    for name, dim, n, periodic, solver, seed, state in cases():
        pos = random_generators(n, dim, seed, sort=False)
        W0 = initial_state(state, pos, periodic)
        p = Params(solver=solver)
        out = {}
        for pow_kind in ("sfxpow", "libm"):
            r = reference_tessellation(pos, periodic, p, dt=DT, nsteps=NSTEPS, W0=W0,
                                       pow_kind=pow_kind)
            assert r["status"] == 0 and r["steps"] == NSTEPS, (name, r["status"])
            out[pow_kind] = r
        m = out["sfxpow"]["mesh"]
        assert np.array_equal(out["libm"]["order"], out["sfxpow"]["order"])
        np.savez_compressed(
            HERE / f"reftess_{name}.npz",
            dim=dim, periodic=periodic, solver=solver, gamma=p.gamma, dt=DT, nsteps=NSTEPS,
            positions=pos, order=out["sfxpow"]["order"],
            cell_pos=m.cell_pos, cell_centroid=m.cell_centroid, cell_volume=m.cell_volume,
            cell_total_area=m.cell_total_area, cell_face_offset=m.cell_face_offset,
            cell_face_index=m.cell_face_index, face_area=m.face_area,
            face_midpoint=m.face_midpoint, face_left=m.face_left, face_right=m.face_right,
            face_kind=m.face_kind, face_right_pos=m.face_right_pos,
            W0=W0[out["sfxpow"]["order"]],
            ref_sfxpow_W=out["sfxpow"]["W"], ref_sfxpow_Q=out["sfxpow"]["Q"],
            ref_libm_W=out["libm"]["W"], ref_libm_Q=out["libm"]["Q"])
        print(f"{name}: {m.n_cells} cells, {m.n_faces} faces "
              f"({int((m.face_area == 0).sum())} of zero area), kinds "
              f"{np.bincount(m.face_kind, minlength=3).tolist()}")


if __name__ == "__main__":
    main()
