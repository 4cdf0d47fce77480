"""The synthetic inputs follow the distributions they are described by:
request stream (arrival rate, 2D/3D mix, size bins, step counts, solver mix),
pool sizes, random-field states and time steps."""
import math

import numpy as np

from shadowfax_b200 import workloads as wl


def test_request_stream_distributions():
    reqs = wl.serve_stream(duration=60.0, seed=5)
    n = len(reqs)
    # Poisson arrivals at 200 per second for 60 s
    assert abs(n - 12_000) < 4 * math.sqrt(12_000)
    t = np.array([r.t for r in reqs])
    assert np.all(np.diff(t) > 0) and t[-1] < 60.0
    gaps = np.diff(t)
    assert abs(gaps.mean() * 200 - 1) < 0.05
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05          # exponential: cv = 1
    k = 10
    dims = np.array([2 if r.mesh < k else 3 for r in reqs])
    assert abs((dims == 2).mean() - 0.7) < 0.02
    bins = np.array([r.mesh % k for r in reqs])
    counts = np.bincount(bins, minlength=k) / n                  # log-uniform N: equal bins
    assert np.all(np.abs(counts - 0.1) < 0.015)
    steps = np.array([r.nsteps for r in reqs])
    assert steps.min() >= 10 and steps.max() <= 200
    assert abs(steps.mean() - 105) < 2
    exact = np.array([r.solver == "Exact" for r in reqs])
    assert abs(exact.mean() - 0.5) < 0.02
    assert {r.state for r in reqs} == {0, 1}


def test_stream_is_deterministic_and_seeded():
    a = wl.serve_stream(count=50, seed=5)
    b = wl.serve_stream(count=50, seed=5)
    c = wl.serve_stream(count=50, seed=1005)
    assert a == b and a != c and len(a) == 50


def test_pool_sizes_cover_the_log_range():
    sizes = wl.serve_pool_sizes(10)
    assert sizes[0] > 1_000 and sizes[-1] < 1_000_000
    ratios = sizes[1:] / sizes[:-1]
    assert np.allclose(ratios, 10 ** 0.3, rtol=1e-3)
    # the pool keeps the mean of the log-uniform draw to a few percent
    mean_logu = (1e6 - 1e3) / math.log(1e3)
    assert abs(sizes.mean() / mean_logu - 1) < 0.03


def test_random_field_state_and_cfl_dt():
    from shadowfax_b200.mesh import build_voronoi, random_generators
    m = build_voronoi(random_generators(20_000, 3, 11), periodic=True)
    W = wl.random_field_state(m, 3)
    lnrho = np.log(W[:, 0])
    assert abs(lnrho.mean() + 0.5) < 0.03 and abs(lnrho.std() - 1) < 0.03
    assert abs(W[:, 0].mean() - 1) < 0.06                        # mean density 1
    assert np.all(W[:, 4] == 1.0)
    v = W[:, 1:4]
    assert np.all(np.abs(v.mean(0)) < 0.03) and np.all(np.abs(v.std(0) - 1) < 0.03)
    dt = wl.cfl_dt(m, W)
    h = wl.cell_h(m)
    c = np.sqrt(wl.GAMMA * W[:, 4] / W[:, 0])
    assert dt == 0.4 * np.min(h / (np.sqrt((v ** 2).sum(1)) + c))
