"""Synthetic workloads the flux pass is measured and tested on.

Inputs are seeded synthetic stand-ins (numpy PCG64 streams): generators
uniform in the unit square/cube, tessellated by the host face-list builder,
with each workload's initial states.  Files are read only where a caller
asks for a mesh cache (serve_pool's cache_dir).

  sod2d           2D Sod tube, reflective unit square, exact solver, dt = 1e-4, 100 steps
  sedov3d         3D Sedov-type blast, reflective unit cube, HLLC, global CFL 0.4, 50 steps
  random_field3d  3D supersonic random field, periodic unit cube, exact solver, one pass
  random_field2d  the same field on a 2D periodic mesh
  batch2d         1,024 independent 2D step-state meshes, HLLC, 20 steps at own CFL dt
  serve_stream    Poisson request stream of static meshes (serving)
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .mesh import Mesh, build_voronoi, random_generators

GAMMA = 5.0 / 3.0


@dataclass
class Problem:
    name: str
    mesh: Mesh
    W0: np.ndarray      # [n, S] primitive variables
    solver: str          # "Exact" or "HLLC"
    dt: float
    nsteps: int
    gamma: float = GAMMA


def cell_h(mesh: Mesh) -> np.ndarray:
    """VorCell::get_h (src/VorCell.cpp:948-956)"""
    V = mesh.cell_volume
    if mesh.dim == 3:
        return np.cbrt(V * 3.0 / 4.0 / math.pi)
    return np.sqrt(V / math.pi)


def cfl_dt(mesh: Mesh, W: np.ndarray, gamma: float = GAMMA, cfl: float = 0.4) -> float:
    """Global CFL time step 0.4 min h / (|v| + c) (the per-cell criterion of
    src/TimeLine.cpp:254-274, taken as one global value without power-of-two
    binning)."""
    D = mesh.dim
    rho, p = W[:, 0], W[:, D + 1]
    c = np.sqrt(gamma * p / np.where(rho > 0, rho, 1.0)) * (rho > 0)
    v = np.sqrt((W[:, 1:D + 1] ** 2).sum(1))
    return float(cfl * np.min(cell_h(mesh) / (v + c)))


def sod2d(n: int = 10_000, seed: int = 1, nsteps: int = 100, dt: float = 1e-4,
          solver: str = "Exact") -> Problem:
    pos = random_generators(n, 2, seed)
    mesh = build_voronoi(pos, periodic=False)
    W = np.zeros((n, 4))
    left = pos[:, 0] < 0.5
    W[:, 0] = np.where(left, 1.0, 0.125)
    W[:, 3] = np.where(left, 1.0, 0.1)
    return Problem("sod2d", mesh, W, solver, dt, nsteps)


def sedov3d(n: int = 262_144, seed: int = 2, nsteps: int = 50, solver: str = "HLLC",
            n_hot: int = 32, energy: float = 1.0) -> Problem:
    pos = random_generators(n, 3, seed)
    mesh = build_voronoi(pos, periodic=False)
    W = np.zeros((n, 5))
    W[:, 0] = 1.0
    W[:, 4] = 1e-6
    d2 = ((pos - 0.5) ** 2).sum(1)
    hot = np.argsort(d2, kind="stable")[:n_hot]
    W[hot, 4] = (GAMMA - 1.0) * (energy / n_hot) / mesh.cell_volume[hot]
    return Problem("sedov3d", mesh, W, solver, cfl_dt(mesh, W), nsteps)


def random_field3d(n: int = 2_097_152, seed: int = 3, solver: str = "Exact",
                   nsteps: int = 1) -> Problem:
    pos = random_generators(n, 3, seed)
    mesh = build_voronoi(pos, periodic=True)
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    W = np.zeros((n, 5))
    W[:, 0] = np.exp(rng.normal(-0.5, 1.0, n))
    W[:, 1:4] = rng.normal(0.0, 1.0, (n, 3))
    W[:, 4] = 1.0
    return Problem("random3d", mesh, W, solver, cfl_dt(mesh, W), nsteps)


def random_field2d(n: int = 2_097_152, seed: int = 3, solver: str = "Exact",
                   nsteps: int = 1) -> Problem:
    """the random field on a 2D periodic mesh (the serving stream's 2D
    requests' states): ln rho ~ N(-1/2, 1), p = 1, v_k ~ N(0, 1)"""
    pos = random_generators(n, 2, seed)
    mesh = build_voronoi(pos, periodic=True)
    W = random_field_state(mesh, seed + 1000)
    return Problem("random2d", mesh, W, solver, cfl_dt(mesh, W), nsteps)


def step_state2d(n: int, seed: int, solver: str = "HLLC", nsteps: int = 20) -> Problem:
    """one mesh of batch2d: left/right constant states split by a line through the
    centre with a random normal angle"""
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = random_generators(n, 2, int(rng.integers(1 << 62)))
    mesh = build_voronoi(pos, periodic=False)
    rhoL, pL, rhoR, pR = rng.uniform(0.1, 1.0, 4)
    th = rng.uniform(0.0, 2 * math.pi)
    side = (pos - 0.5) @ np.array([math.cos(th), math.sin(th)]) < 0
    W = np.zeros((n, 4))
    W[:, 0] = np.where(side, rhoL, rhoR)
    W[:, 3] = np.where(side, pL, rhoR * 0 + pR)
    return Problem(f"step2d_{n}", mesh, W, solver, cfl_dt(mesh, W), nsteps)


def batch_sizes(count: int = 1024, lo: int = 1_000, hi: int = 100_000, seed: int = 4) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(math.log(lo), math.log(hi), count)).astype(np.int64)


def batch2d(count: int = 1024, seed: int = 4, solver: str = "HLLC", nsteps: int = 20,
            workers: int = 0) -> list[Problem]:
    """`count` independent 2D step-state meshes with generator
    counts log-uniform in [1e3, 1e5]; meshes are tessellated concurrently
    (the builder releases the interpreter lock)"""
    import os
    from concurrent.futures import ThreadPoolExecutor
    sizes = batch_sizes(count, seed=seed)
    workers = workers or max(1, min(8, (os.cpu_count() or 4) // 2))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        futs = [ex.submit(step_state2d, int(n), seed * 100_000 + j, solver, nsteps)
                for j, n in enumerate(sizes)]
        return [f.result() for f in futs]


# ---- c5: the request stream --------------------------------------------

SERVE_LO, SERVE_HI = 1_000, 1_000_000


def serve_pool_sizes(k: int = 10, lo: int = SERVE_LO, hi: int = SERVE_HI) -> np.ndarray:
    """pool mesh sizes: the geometric centres of k equal bins of log N over
    [lo, hi]; a request's log-uniform N is served by its bin's mesh, so the
    pool keeps the distribution's mean to about 2% (mean of the centres
    1.42e5 for k = 10 against 1.45e5)"""
    a, b = math.log(lo), math.log(hi)
    return np.exp(a + (b - a) * (np.arange(k) + 0.5) / k).round().astype(np.int64)


def random_field_state(mesh: Mesh, seed: int) -> np.ndarray:
    """the random_field3d state on any mesh: ln rho ~ N(-1/2, 1) (mean rho 1), p = 1,
    each velocity component ~ N(0, 1)"""
    n, D = mesh.n_cells, mesh.dim
    rng = np.random.Generator(np.random.PCG64(seed))
    W = np.zeros((n, D + 2))
    W[:, 0] = np.exp(rng.normal(-0.5, 1.0, n))
    W[:, 1:D + 1] = rng.normal(0.0, 1.0, (n, D))
    W[:, D + 1] = 1.0
    return W


@dataclass
class ServePool:
    """pre-tessellated meshes of the stream (periodic unit box) with a few
    random-field states each and their CFL-0.4 time steps; mesh (dim, bin)
    sits at index (dim - 2) * k + bin (None where not built)"""
    k: int
    meshes: list
    states: list        # states[mesh] = [W, ...]
    dts: list           # dts[mesh] = [dt, ...]


@dataclass
class ServeRequest:
    t: float            # arrival, seconds after the stream starts
    mesh: int           # pool mesh index: (dim - 2) * k + size bin
    state: int          # state index of that mesh
    solver: str
    nsteps: int


def serve_pool(k: int = 10, seed: int = 5, states_per_mesh: int = 2, only=None,
               workers: int = 0, cache_dir=None, library: bool = True) -> ServePool:
    """the pool meshes (all 2k, or the indices in `only`), tessellated
    concurrently, largest first; with `cache_dir`, each mesh is read from
    its mesh file there when present and written there after tessellation
    otherwise (sfx_meshfile_*).  library=False builds and reads the meshes
    without loading the GPU library (the standalone sfx_meshgen program and
    the numpy mesh-file reader; needs cache_dir): the same face lists, for
    CPU-only jobs."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    from pathlib import Path

    from .mesh import Mesh, build_voronoi_file
    if not library and not cache_dir:
        raise ValueError("serve_pool(library=False) needs a cache_dir for its mesh files")
    sizes = serve_pool_sizes(k)
    jobs = [j for j in range(2 * k) if only is None or j in only]
    workers = workers or max(1, min(4, (os.cpu_count() or 4) // 4))

    def one(j):
        dim, b = 2 + j // k, j % k
        n = int(sizes[b])
        gen_seed = seed * 1_000_003 + dim * 1000 + b
        path = None
        if cache_dir:
            path = Path(cache_dir) / f"pool_{dim}d_n{n}_seed{gen_seed}.sfxmesh"
        if not library:
            if not path.exists():
                build_voronoi_file(random_generators(n, dim, gen_seed), True, path)
            mesh = Mesh.read_file_numpy(path)
        elif path is not None and path.exists():
            mesh = Mesh.read_file(path)
        else:
            mesh = build_voronoi(random_generators(n, dim, gen_seed), periodic=True)
            if path is not None:
                mesh.write_file(path)
        Ws = [random_field_state(mesh, seed * 7919 + dim * 1000 + b * 10 + s)
              for s in range(states_per_mesh)]
        return mesh, Ws, [cfl_dt(mesh, W) for W in Ws]

    order = sorted(jobs, key=lambda j: -int(sizes[j % k]) * (3 if j >= k else 1))
    meshes, states, dts = [None] * (2 * k), [None] * (2 * k), [None] * (2 * k)
    with ThreadPoolExecutor(max_workers=workers) as ex:
        for j, (m, Ws, ds) in zip(order, ex.map(one, order)):
            meshes[j], states[j], dts[j] = m, Ws, ds
    return ServePool(k, meshes, states, dts)


def serve_stream(k: int = 10, rate: float = 200.0, duration: float = 60.0, seed: int = 5,
                 frac2d: float = 0.7, steps: tuple = (10, 200), states_per_mesh: int = 2,
                 count: int | None = None) -> list:
    """the serving stream: Poisson arrivals at `rate` per second for `duration`
    seconds (or the first `count` arrivals); 70% 2D / 30% 3D; N log-uniform
    in [1e3, 1e6] (served by the pool mesh of its bin); step count uniform on
    {10..200}; exact or HLLC 50/50"""
    rng = np.random.Generator(np.random.PCG64(seed))
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if (count is None and t >= duration) or (count is not None and len(out) >= count):
            break
        dim = 2 if rng.random() < frac2d else 3
        b = min(k - 1, int(rng.random() * k))    # log N uniform -> equal bins
        si = int(rng.integers(states_per_mesh))
        solver = "Exact" if rng.random() < 0.5 else "HLLC"
        nsteps = int(rng.integers(steps[0], steps[1] + 1))
        out.append(ServeRequest(t, (dim - 2) * k + b, si, solver, nsteps))
    return out
