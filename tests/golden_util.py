"""Helpers to load the committed golden fixtures (tests/golden/*.npz)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

from shadowfax_b200.mesh import Mesh

GOLDEN = Path(__file__).resolve().parent / "golden"
MOVING_CASES = [f"moving_{d}d_{b}_{s}" for d in (2, 3) for b in ("reflective", "periodic")
                for s in ("exact", "hllc")]
MOVING_FAILS = "moving_2d_periodic_hllc_fails"
LOCAL_CASES = [f"local_{d}d_{s}" for d in (2, 3) for s in ("exact", "hllc")]
# meshes the reference's own DelTess/VorTess built (tests/golden/make_reftess.py)
REFTESS_CASES = ["reftess_sod2d_reflective_exact", "reftess_random2d_periodic_hllc",
                 "reftess_sedov3d_reflective_hllc", "reftess_random3d_periodic_exact"]
# the pass at gamma = 1.4 (the factory default is 5/3): oracle pins on the CPU
GAMMA_CASES = ["gamma14_sod2d_exact", "gamma14_random3d_hllc", "gamma14_random3d_exact"]
MESH_CASES = ["sod2d_exact", "sod2d_hllc", "sedov3d_hllc", "random3d_exact",
              "random2d_periodic_exact"]


def load_case(name: str):
    z = np.load(GOLDEN / f"{name}.npz")
    mesh = Mesh(dim=int(z["dim"]), periodic=bool(int(z["periodic"])),
                **{a: z[a] for a in Mesh._ARRAYS}).normalized()
    meta = dict(solver=str(z["solver"]), gamma=float(z["gamma"]), dt=float(z["dt"]),
                nsteps=int(z["nsteps"]), W0=z["W0"])
    ref = {k: z[k] for k in z.files if k.startswith("ref_")}
    if "local_start" in z.files:
        meta["local"] = {k[len("local_"):]: z[k] for k in z.files if k.startswith("local_")}
    return mesh, meta, ref


def load_riemann(dim: int):
    return dict(np.load(GOLDEN / f"riemann_{dim}d.npz"))


# Exact-solver half states from the reference's own unit test
# (test/testRiemannSolver.cpp:217-232, default ExactRiemannSolver, gamma
# 1.66667, normal (1,0,0)): (rhoL, vL, pL, rhoR, vR, pR) -> (rho, v, p),
# checked there at 1e-4 relative (test/myAssert.hpp assert_values_equal).
TORO_HALF_STATES = [
    ((1.0, 0.0, 1.0, 0.125, 0.0, 0.1), (0.47969, 0.841194, 0.293945)),
    ((1.0, -2.0, 0.4, 1.0, 2.0, 0.4), (0.00617903, 0.0, 8.32249e-05)),
    ((1.0, 0.0, 1000.0, 1.0, 0.0, 0.01), (0.615719, 18.2812, 445.626)),
    ((1.0, 0.0, 0.01, 1.0, 0.0, 100.0), (0.61577, -5.78011, 44.5687)),
    ((5.99924, 19.5975, 460.894, 5.99242, -6.19633, 46.0950), (12.743, 8.56045, 1841.82)),
    ((1.0, -1.0, 1.0e-6, 1.0, 1.0, 1.0005e-6), (0.0, 0.0, 0.0)),
]


def toro_pairs(dim: int):
    S = dim + 2
    n = len(TORO_HALF_STATES)
    WL = np.zeros((n, S))
    WR = np.zeros((n, S))
    exp = np.zeros((n, 3))
    for i, ((rl, vl, pl, rr, vr, pr), e) in enumerate(TORO_HALF_STATES):
        WL[i, 0], WL[i, 1], WL[i, S - 1] = rl, vl, pl
        WR[i, 0], WR[i, 1], WR[i, S - 1] = rr, vr, pr
        exp[i] = e
    nrm = np.zeros((n, dim))
    nrm[:, 0] = 1.0
    return WL, WR, nrm, exp


def assert_values_equal(a: float, b: float, tol: float = 1e-4):
    """test/myAssert.hpp assert_values_equal: relative 1e-4, absolute when
    the expected value is 0"""
    if b != 0.0:
        assert abs(a - b) / abs(b) <= tol, (a, b)
    else:
        assert abs(a - b) <= tol, (a, b)
