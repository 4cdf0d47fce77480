"""The N>1 host logic on CPU ranks (gloo, world size 2): the ranks share one
request stream (whole requests, least face work first) and the whole-job
figure of bench.py is the work of all ranks over the slowest rank's time; one mesh
split over two ranks (the exchange, and PartitionedPass itself with the CPU
oracle standing in for the device pass) equals the whole-mesh pass bit for
bit, and a failing step on one rank stops both ranks with SfxError instead
of leaving one waiting in the exchange."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        class A:
            requests = 300
            duration = 60.0

        reqs = bench.serve_requests(A)
        owner = bench.shard_requests(reqs, world)
        mine = [j for j, o in enumerate(owner) if o == rank]
        work = sum(reqs[j].nsteps for j in mine)
        ms = 100.0 * (rank + 1)
        value, ms_max, total = bench.reduce_over_ranks(ms, work, "cpu", world)
        out[rank] = (value, ms_max, total, work, mine, owner.tolist())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_cpu_ranks_share_one_stream_and_reduce_work_and_time():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    w0, w1 = res[0][3], res[1][3]
    for r in range(world):
        value, ms_max, total, _, _, _ = res[r]
        assert ms_max == pytest.approx(200.0)          # the slowest rank's time
        assert total == pytest.approx(w0 + w1)          # all ranks' work
        assert value == pytest.approx((w0 + w1) / 0.2)
    # both ranks computed the same assignment; every request is served once
    assert res[0][5] == res[1][5]
    mine0, mine1 = set(res[0][4]), set(res[1][4])
    assert not (mine0 & mine1) and len(mine0 | mine1) == 300


def test_stream_sharding_balances_face_work():
    """whole requests to the least-loaded GPU in arrival order: the estimated
    face work per GPU differs by less than the largest single request"""
    import bench
    from shadowfax_b200 import workloads as wl
    reqs = wl.serve_stream(count=2000, seed=5)
    sizes = wl.serve_pool_sizes()
    work = np.array([sizes[r.mesh % 10] * (3.0 if r.mesh < 10 else 7.8) * r.nsteps
                     for r in reqs])
    for world in (1, 2, 3, 8):
        owner = bench.shard_requests(reqs, world)
        assert owner.min() >= 0 and owner.max() < world
        load = np.bincount(owner, weights=work, minlength=world)
        assert load.max() - load.min() <= work.max()
        # arrival order is kept within each GPU's share
        for q in range(world):
            ts = [reqs[j].t for j in np.flatnonzero(owner == q)]
            assert ts == sorted(ts)
    assert np.all(bench.shard_requests(reqs, 1) == 0)


def _split_mesh_rank(rank, world, port, name, nsteps, out):
    """one rank of a mesh split over `world` ranks: the oracle's pass over
    this rank's part (standing in for the device), the ring exchange through
    the product's exchange_records over gloo"""
    import datetime
    import sys

    import numpy as np
    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(__file__))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from golden_util import load_case
        from oracle.oracle import Oracle, Params
        from shadowfax_b200 import partition as P

        oracle = Oracle()
        mesh, meta, _ = load_case(name)
        p = Params(solver=meta["solver"], gamma=meta["gamma"])
        owner = P.partition(mesh, world)
        pt = P.build_part(mesh, owner, rank)
        plan = P.exchange_plan(mesh, owner, pt)
        W = meta["W0"][pt.cells].copy()
        Q = oracle.init_Q(pt.mesh, p, W)
        R = mesh.dim + 3
        recv = {q: torch.empty((len(rv), R), dtype=torch.float64) for q, (_, rv) in plan.items()}
        for _ in range(nsteps):
            _, dQ, _, rc, _ = oracle.flux_pass(pt.mesh, p, meta["dt"], W, Q)
            assert rc == 0
            Qt = Q.copy()
            Qt[pt.n_own:, [0, -1]] = 1e300
            Wn, Qn, rc, _ = oracle.apply(pt.mesh, p, dQ, W, Qt)
            assert rc == 0
            W[:pt.n_own], Q[:pt.n_own] = Wn[:pt.n_own], Qn[:pt.n_own]
            send = {q: torch.from_numpy(np.concatenate([W[s], Q[s, :1]], axis=1))
                    for q, (s, _) in plan.items()}
            P.exchange_records(send, recv)
            for q, (_, rv) in plan.items():
                rec = recv[q].numpy()
                W[rv] = rec[:, :-1]
                Q[rv, 0] = rec[:, -1]
        out[rank] = (pt.cells[:pt.n_own], W[:pt.n_own].copy(), Q[:pt.n_own].copy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["random2d_periodic_exact", "sedov3d_hllc"])
def test_split_mesh_over_two_cpu_ranks(name):
    """the owned cells of both ranks, after steps with the ring exchange over
    gloo, equal the oracle's steps over the whole mesh bit for bit"""
    import sys

    import numpy as np
    sys.path.insert(0, os.path.dirname(__file__))
    from golden_util import load_case
    from oracle.oracle import Oracle, Params

    world, nsteps = 2, 3
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_split_mesh_rank, args=(r, world, port, name, nsteps, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    oracle = Oracle()
    mesh, meta, _ = load_case(name)
    prm = Params(solver=meta["solver"], gamma=meta["gamma"])
    r = oracle.run(mesh, prm, meta["dt"], nsteps, meta["W0"])
    assert r["status"] == 0
    seen = np.zeros(mesh.n_cells, int)
    for rank in range(world):
        cells, W, Q = res[rank]
        seen[cells] += 1
        assert np.array_equal(W, r["W"][cells])
        assert np.array_equal(Q, r["Q"][cells])
    assert np.all(seen == 1)


class _OraclePass:
    """FluxPass's interface over the CPU oracle, on CPU tensors: the device
    pass's stand-in inside PartitionedPass on gloo ranks.  fail_at=k makes
    the k-th step raise the library's SfxError (a failure made on the host)."""

    def __init__(self, oracle, mesh, p, fail_at=None):
        self.oracle, self.mesh, self.p, self.fail_at, self.k = oracle, mesh, p, fail_at, 0

    def set_ranges(self, grad_cells, flux_faces, update_cells):
        self.n_own = update_cells

    def set_primitive(self, W):
        self.W = np.array(W, np.float64)
        self.Q = self.oracle.init_Q(self.mesh, self.p, self.W)

    def step(self, dt, nsteps=1, stats=True):
        from shadowfax_b200._lib import SFX_ERR_NEG_STATE, SfxError
        for _ in range(nsteps):
            self.k += 1
            if self.k == self.fail_at:
                raise SfxError(SFX_ERR_NEG_STATE, "sfx_step", 0)
            _, dQ, _, rc, _ = self.oracle.flux_pass(self.mesh, self.p, dt, self.W, self.Q)
            assert rc == 0
            Qt = self.Q.copy()
            Qt[self.n_own:, [0, -1]] = 1e300      # ring cells are not updated
            Wn, Qn, rc, _ = self.oracle.apply(self.mesh, self.p, dQ, self.W, Qt)
            assert rc == 0
            n = self.n_own
            self.W[:n], self.Q[:n] = Wn[:n], Qn[:n]

    def pack_cells(self, idx, out):
        i = idx.numpy()
        out.copy_(torch.from_numpy(np.concatenate([self.W[i], self.Q[i, :1]], axis=1)))

    def unpack_cells(self, idx, inp):
        i = idx.numpy()
        rec = inp.numpy()
        self.W[i] = rec[:, :-1]
        self.Q[i, 0] = rec[:, -1]

    def state(self):
        return self.W.copy(), self.Q.copy()


def _partitioned_rank(rank, world, port, name, nsteps, fail_rank, out):
    import datetime
    import sys
    import time

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(__file__))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    # a short timeout: a rank left waiting in the exchange ends with a
    # timeout error, not with the SfxError the test expects
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        from golden_util import load_case
        from oracle.oracle import Oracle, Params
        from shadowfax_b200 import partition as P
        from shadowfax_b200._lib import SfxError

        mesh, meta, _ = load_case(name)
        p = Params(solver=meta["solver"], gamma=meta["gamma"])
        owner = P.partition(mesh, world)
        part = P.build_part(mesh, owner, rank)
        stub = _OraclePass(Oracle(), part.mesh, p, fail_at=2 if rank == fail_rank else None)
        pp = P.PartitionedPass(None, mesh, owner, rank, flux_pass=stub)
        pp.set_primitive(meta["W0"])
        t0 = time.perf_counter()
        try:
            pp.step(meta["dt"], nsteps)
            cells, W, Q = pp.owned_state()
            out[rank] = ("ok", cells, W, Q, pp.comm_device.type)
        except SfxError as e:
            out[rank] = ("SfxError", e.status, time.perf_counter() - t0, stub.k)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run_partitioned(name, nsteps, fail_rank):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_partitioned_rank,
                             args=(r, world, port, name, nsteps, fail_rank, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        return dict(out)


@pytest.mark.parametrize("name", ["random2d_periodic_exact", "sedov3d_hllc"])
def test_partitioned_pass_over_two_cpu_ranks(name):
    """PartitionedPass itself (exchange lists, packing, the exchange, the
    per-step status agreement) on two gloo ranks: the owned cells equal the
    oracle's whole-mesh steps bit for bit"""
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from golden_util import load_case
    from oracle.oracle import Oracle, Params

    nsteps = 3
    res = _run_partitioned(name, nsteps, fail_rank=-1)
    mesh, meta, _ = load_case(name)
    r = Oracle().run(mesh, Params(solver=meta["solver"], gamma=meta["gamma"]), meta["dt"],
                     nsteps, meta["W0"])
    seen = np.zeros(mesh.n_cells, int)
    for rank in range(2):
        kind, cells, W, Q, comm = res[rank]
        assert kind == "ok" and comm == "cpu"
        seen[cells] += 1
        assert np.array_equal(W, r["W"][cells])
        assert np.array_equal(Q, r["Q"][cells])
    assert np.all(seen == 1)


@pytest.mark.parametrize("fail_rank", [0, 1])
def test_failing_step_on_one_rank_stops_both(fail_rank):
    """the second step fails on one rank (SfxError from its pass): both ranks
    raise SfxError with that status after the same step, well inside the
    process group's timeout, and neither exchanges after the failure"""
    from shadowfax_b200._lib import SFX_ERR_NEG_STATE
    res = _run_partitioned("random2d_periodic_exact", 4, fail_rank)
    for rank in range(2):
        kind, status, secs, k = res[rank]
        assert kind == "SfxError" and status == SFX_ERR_NEG_STATE
        assert k == 2            # no rank ran a step after the failing one
        assert secs < 15.0
