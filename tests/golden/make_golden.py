"""Generate the golden fixtures under tests/golden/ (run where the reference
tree and the reference harness binaries exist: ``python oracle/build.py``
first).  The fixtures hold small meshes, initial states and the REFERENCE's
own CPU flux-pass results on them (oracle/_ref/refharness_*, the unmodified
Shadowfax sources), with both glibc pow and sfx_pow, plus the reference
solvers' outputs on Riemann state pairs.  They let the CPU test suite pin the
oracle restatement on machines without the reference tree.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import Params, riemann_reference, run_reference  # noqa: E402
from shadowfax_b200 import workloads as wl  # noqa: E402
from shadowfax_b200.mesh import build_voronoi, random_generators  # noqa: E402

OUT = Path(__file__).resolve().parent


def cases():
    yield "sod2d_exact", wl.sod2d(n=600, nsteps=12, solver="Exact")
    yield "sod2d_hllc", wl.sod2d(n=600, nsteps=12, solver="HLLC")
    pr = wl.sedov3d(n=700, nsteps=6)
    yield "sedov3d_hllc", pr
    pr = wl.random_field3d(n=700, nsteps=3)
    yield "random3d_exact", pr
    pos = random_generators(500, 2, 11)
    m = build_voronoi(pos, periodic=True)
    rng = np.random.Generator(np.random.PCG64(12))
    W = np.zeros((500, 4))
    W[:, 0] = np.exp(rng.normal(-0.5, 1.5, 500))
    W[:, 1:3] = rng.normal(0, 2, (500, 2))
    W[:, 3] = np.exp(rng.normal(0, 1.5, 500))
    yield "random2d_periodic_exact", wl.Problem("r2d", m, W, "Exact", wl.cfl_dt(m, W), 6)


def riemann_pairs(dim: int, n: int, seed: int):
    """state pairs covering shocks, rarefactions, strong contrasts, vacuum
    generation and vacuum states"""
    rng = np.random.Generator(np.random.PCG64(seed))
    S = dim + 2
    WL = np.zeros((n, S))
    WR = np.zeros((n, S))
    WL[:, 0] = np.exp(rng.normal(0, 2, n))
    WR[:, 0] = np.exp(rng.normal(0, 2, n))
    WL[:, 1:dim + 1] = rng.normal(0, 3, (n, dim))
    WR[:, 1:dim + 1] = rng.normal(0, 3, (n, dim))
    WL[:, dim + 1] = np.exp(rng.normal(0, 3, n))
    WR[:, dim + 1] = np.exp(rng.normal(0, 3, n))
    k = n // 10
    WL[:k, 0] = 0.0                       # left vacuum
    WL[:k, 1:] = 0.0
    WR[k:2 * k, 0] = 0.0                  # right vacuum
    WR[k:2 * k, 1:] = 0.0
    WL[2 * k:3 * k, 1] = -20.0            # vacuum generation
    WR[2 * k:3 * k, 1] = 20.0
    WL[3 * k:3 * k + 5] = 0.0             # both sides vacuum
    WR[3 * k:3 * k + 5] = 0.0
    nrm = rng.normal(0, 1, (n, dim))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    return WL, WR, nrm


def main():
    for name, pr in cases():
        out = {}
        for powk in ("libm", "sfxpow"):
            p = Params(solver=pr.solver, gamma=pr.gamma)
            r = run_reference(pr.mesh, p, pr.dt, pr.nsteps, pr.W0, pow_kind=powk)
            assert r["status"] == 0 and r["steps"] == pr.nsteps, (name, r["status"])
            for key in ("W", "Q", "grad", "dQ"):
                out[f"ref_{powk}_{key}"] = r[key]
        m = pr.mesh
        np.savez_compressed(
            OUT / f"{name}.npz", dim=m.dim, periodic=int(m.periodic), solver=pr.solver,
            gamma=pr.gamma, dt=pr.dt, nsteps=pr.nsteps, W0=pr.W0,
            **{a: getattr(m, a) for a in m._ARRAYS}, **out)
        print("wrote", name, m.n_cells, m.n_faces)
    for dim in (2, 3):
        WL, WR, nrm = riemann_pairs(dim, 400, 100 + dim)
        out = dict(WL=WL, WR=WR, normal=nrm)
        for solver in ("Exact", "HLLC"):
            for powk in ("libm", "sfxpow"):
                r = riemann_reference(dim, Params(solver=solver), WL, WR, nrm, pow_kind=powk)
                out[f"{solver}_{powk}_status"] = r["status"]
                out[f"{solver}_{powk}_half"] = r["half"]
                out[f"{solver}_{powk}_flux"] = r["flux"]
            r = riemann_reference(dim, Params(solver=solver), WL, WR, nrm, reflective=True,
                                  pow_kind="sfxpow")
            out[f"{solver}_reflective_status"] = r["status"]
            out[f"{solver}_reflective_flux"] = r["flux"]
        np.savez_compressed(OUT / f"riemann_{dim}d.npz", **out)
        print("wrote riemann", dim)


if __name__ == "__main__":
    main()
