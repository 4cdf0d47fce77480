"""Generate the golden fixtures under tests/golden/ (run where the reference
tree and the reference harness binaries exist: ``python oracle/build.py``
first).  The fixtures hold small meshes, initial states and the REFERENCE's
own CPU flux-pass results on them (oracle/_ref/refharness_*, the unmodified
Shadowfax sources), with both glibc pow and sfx_pow, plus the reference
solvers' outputs on Riemann state pairs, and one step with moving generators
(the reference built without -DSTATIC; ``--moving`` makes only those) and
one system step of local time steps (``--local``), and the pass and solvers
at gamma = 1.4 (``--gamma``) and the exact solver at another tolerance and
cutoff (``--tolerance``).  They
let the CPU test suite pin the oracle restatement on machines without the
reference tree.
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


def jittered_lattice(k: int, dim: int, seed: int) -> np.ndarray:
    """k^dim generators: lattice points moved by up to a quarter cell"""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = np.stack(np.meshgrid(*[np.arange(k)] * dim, indexing="ij"), -1).reshape(-1, dim)
    return np.ascontiguousarray((g + 0.5 + rng.uniform(-0.25, 0.25, g.shape)) / k)


def moving_cases():
    """one step with moving generators on jittered lattices (generators far
    enough apart that the face velocities stay of the order of the flow's),
    moderate random states, both solvers, reflective and periodic.  The last
    case is a uniform random point set, where two generators 2e-4 apart give
    their face a velocity of about 50 (VorFace::set_v divides by the squared
    distance); with HLLC the reference then throws UpdateQException within
    the step (its de-boost reuses the already de-boosted momentum flux in
    the energy flux, src/riemann/HLLCRiemannSolver.cpp:392-400, adding
    v^2 F_rho more), and the GPU pass must fail the same way."""
    for dim in (2, 3):
        for periodic in (False, True):
            for solver in ("Exact", "HLLC"):
                k = 22 if dim == 2 else 8
                seed = 300 + 10 * dim + (5 if periodic else 0) + (1 if solver == "HLLC" else 0)
                m = build_voronoi(jittered_lattice(k, dim, seed), periodic=periodic)
                n = m.n_cells
                rng = np.random.Generator(np.random.PCG64(seed + 1))
                W = np.zeros((n, dim + 2))
                W[:, 0] = np.exp(rng.normal(0.0, 0.5, n))
                W[:, 1:dim + 1] = rng.normal(0.0, 0.3, (n, dim))
                W[:, dim + 1] = np.exp(rng.normal(0.0, 0.5, n))
                name = f"moving_{dim}d_{'periodic' if periodic else 'reflective'}_{solver.lower()}"
                yield name, wl.Problem(name, m, W, solver, wl.cfl_dt(m, W), 1)
    n, seed = 500, 326
    m = build_voronoi(random_generators(n, 2, seed), periodic=True)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    W = np.zeros((n, 4))
    W[:, 0] = np.exp(rng.normal(0.0, 0.5, n))
    W[:, 1:3] = rng.normal(0.0, 0.3, (n, 2))
    W[:, 3] = np.exp(rng.normal(0.0, 0.5, n))
    yield "moving_2d_periodic_hllc_fails", wl.Problem("f", m, W, "HLLC", wl.cfl_dt(m, W), 1)


TICKS = 1 << 60


def local_cases():
    """one system step of local time steps on jittered lattices: every cell
    in one of three power-of-two bins (1/4, 1/8, 1/16 of the timeline), the
    window [9/16, 10/16) of it, so the 1/16 cells are active, the 1/8 cells
    end their step (get_W) without being active, the 1/4 cells neither; the
    inactive cells keep stored gradients; t_total = 8 CFL steps, so the
    shortest bin is half a CFL step"""
    for dim in (2, 3):
        for solver in ("Exact", "HLLC"):
            periodic = dim == 3
            k = 22 if dim == 2 else 8
            seed = 400 + 10 * dim + (1 if solver == "HLLC" else 0)
            m = build_voronoi(jittered_lattice(k, dim, seed), periodic=periodic)
            n = m.n_cells
            rng = np.random.Generator(np.random.PCG64(seed + 1))
            W = np.zeros((n, dim + 2))
            W[:, 0] = np.exp(rng.normal(0.0, 0.5, n))
            W[:, 1:dim + 1] = rng.normal(0.0, 0.3, (n, dim))
            W[:, dim + 1] = np.exp(rng.normal(0.0, 0.5, n))
            steps = (TICKS >> 2) >> rng.integers(0, 3, n).astype(np.uint64)
            t_now = TICKS // 2 + TICKS // 16
            start = (t_now // steps) * steps
            local = dict(start=start.astype(np.uint64), end=(start + steps).astype(np.uint64),
                         t_now=t_now, t_next=t_now + TICKS // 16,
                         t_total=8 * wl.cfl_dt(m, W),
                         grad0=rng.normal(0.0, 0.2, (n, dim, dim + 2)))
            name = f"local_{dim}d_{solver.lower()}"
            yield name, wl.Problem(name, m, W, solver, 1.0, 1), local


def main_local():
    """tests/golden/local_*.npz: one system step of local time steps with the
    reference's own VorFace/VorCell/GasParticle (static build)"""
    for name, pr, local in local_cases():
        out = {}
        for powk in ("libm", "sfxpow"):
            p = Params(solver=pr.solver, gamma=pr.gamma)
            r = run_reference(pr.mesh, p, pr.dt, 1, pr.W0, pow_kind=powk, local=local)
            assert r["status"] == 0 and r["steps"] == 1, (name, r["status"])
            for key in ("W", "Q", "grad", "vel"):
                out[f"ref_{powk}_{key}"] = r[key]
        m = pr.mesh
        np.savez_compressed(
            OUT / f"{name}.npz", dim=m.dim, periodic=int(m.periodic), solver=pr.solver,
            gamma=pr.gamma, dt=pr.dt, nsteps=1, W0=pr.W0,
            **{a: getattr(m, a) for a in m._ARRAYS},
            **{f"local_{k}": np.asarray(v) for k, v in local.items()}, **out)
        act = int((local["start"] == local["t_now"]).sum())
        fin = int((local["end"] == local["t_next"]).sum())
        print("wrote", name, m.n_cells, m.n_faces, "active", act, "ending", fin)


def main_moving():
    """tests/golden/moving_*.npz: the reference built without -DSTATIC
    (oracle/_ref/refharness_*_moving_*), one step each"""
    for name, pr in moving_cases():
        out = {}
        for powk in ("libm", "sfxpow"):
            p = Params(solver=pr.solver, gamma=pr.gamma)
            r = run_reference(pr.mesh, p, pr.dt, 1, pr.W0, pow_kind=powk, moving=True)
            out[f"ref_{powk}_status"] = r["status"]
            if name.endswith("_fails"):
                assert r["status"] != 0, name
                continue
            assert r["status"] == 0 and r["steps"] == 1, (name, r["status"])
            for key in ("W", "Q", "pos"):
                out[f"ref_{powk}_{key}"] = r[key]
        m = pr.mesh
        np.savez_compressed(
            OUT / f"{name}.npz", dim=m.dim, periodic=int(m.periodic), solver=pr.solver,
            gamma=pr.gamma, dt=pr.dt, nsteps=1, W0=pr.W0,
            **{a: getattr(m, a) for a in m._ARRAYS}, **out)
        moved = (float(np.abs(out["ref_sfxpow_pos"] - m.cell_pos).max())
                 if "ref_sfxpow_pos" in out else None)
        print("wrote", name, m.n_cells, m.n_faces, moved)


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


GAMMA_ALT = 1.4


def gamma_cases():
    """the pass at another adiabatic index than the factory default (the
    solvers' gamma-dependent constants, get_Q/get_W's energy)"""
    import dataclasses
    yield "gamma14_sod2d_exact", dataclasses.replace(
        wl.sod2d(n=400, nsteps=8, solver="Exact"), gamma=GAMMA_ALT)
    yield "gamma14_random3d_hllc", dataclasses.replace(
        wl.random_field3d(n=300, nsteps=2, solver="HLLC"), gamma=GAMMA_ALT)
    yield "gamma14_random3d_exact", dataclasses.replace(
        wl.random_field3d(n=300, nsteps=2, solver="Exact"), gamma=GAMMA_ALT)


def main_gamma():
    """tests/golden/gamma14_*.npz and riemann_gamma14_{2,3}d.npz: the
    reference's pass and solvers at gamma = 1.4"""
    for name, pr in gamma_cases():
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
        WL, WR, nrm = riemann_pairs(dim, 200, 200 + dim)
        out = dict(WL=WL, WR=WR, normal=nrm, gamma=GAMMA_ALT)
        for solver in ("Exact", "HLLC"):
            for powk in ("libm", "sfxpow"):
                r = riemann_reference(dim, Params(solver=solver, gamma=GAMMA_ALT), WL, WR, nrm,
                                      pow_kind=powk)
                out[f"{solver}_{powk}_status"] = r["status"]
                out[f"{solver}_{powk}_half"] = r["half"]
                out[f"{solver}_{powk}_flux"] = r["flux"]
        np.savez_compressed(OUT / f"riemann_gamma14_{dim}d.npz", **out)
        print("wrote riemann gamma 1.4", dim)


TOL_ALT, CUTOFF_ALT = 1e-6, -2.0


def main_tolerance():
    """tests/golden/tol6_random3d_exact.npz and riemann_tol6_{2,3}d.npz: the
    exact solver at another tolerance and Newton-only cutoff than the factory
    defaults (1e-8, -5), which moves the Newton-only/Newton/Brent choice and
    the point where the iteration stops"""
    pr = wl.random_field3d(n=300, nsteps=2, solver="Exact")
    out = {}
    for powk in ("libm", "sfxpow"):
        p = Params(solver="Exact", gamma=pr.gamma, tolerance=TOL_ALT, cutoff=CUTOFF_ALT)
        r = run_reference(pr.mesh, p, pr.dt, pr.nsteps, pr.W0, pow_kind=powk)
        assert r["status"] == 0 and r["steps"] == pr.nsteps, r["status"]
        for key in ("W", "Q", "grad", "dQ"):
            out[f"ref_{powk}_{key}"] = r[key]
    m = pr.mesh
    np.savez_compressed(
        OUT / "tol6_random3d_exact.npz", dim=m.dim, periodic=int(m.periodic), solver="Exact",
        gamma=pr.gamma, tolerance=TOL_ALT, cutoff=CUTOFF_ALT, dt=pr.dt, nsteps=pr.nsteps,
        W0=pr.W0, **{a: getattr(m, a) for a in m._ARRAYS}, **out)
    print("wrote tol6_random3d_exact", m.n_cells, m.n_faces)
    for dim in (2, 3):
        WL, WR, nrm = riemann_pairs(dim, 200, 300 + dim)
        out = dict(WL=WL, WR=WR, normal=nrm, tolerance=TOL_ALT, cutoff=CUTOFF_ALT)
        for powk in ("libm", "sfxpow"):
            r = riemann_reference(dim, Params(solver="Exact", tolerance=TOL_ALT, cutoff=CUTOFF_ALT),
                                  WL, WR, nrm, pow_kind=powk)
            out[f"Exact_{powk}_status"] = r["status"]
            out[f"Exact_{powk}_half"] = r["half"]
            out[f"Exact_{powk}_flux"] = r["flux"]
        np.savez_compressed(OUT / f"riemann_tol6_{dim}d.npz", **out)
        print("wrote riemann tolerance 1e-6", dim)


if __name__ == "__main__":
    if "--moving" in sys.argv:
        main_moving()
    elif "--local" in sys.argv:
        main_local()
    elif "--gamma" in sys.argv:
        main_gamma()
    elif "--tolerance" in sys.argv:
        main_tolerance()
    else:
        main()
        main_moving()
        main_local()
        main_gamma()
        main_tolerance()
