"""The N>1 host logic of bench.py on CPU ranks (gloo, world size 2): each rank
serves its own request stream, and the whole-job figure is the work of all
ranks over the slowest rank's time."""
import os
import socket

import pytest
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
        from shadowfax_b200 import workloads as wl

        class A:
            steps = 50
            duration = None

        reqs = bench.serve_requests(A, rank)
        work = sum(r.nsteps for r in reqs)
        ms = 100.0 * (rank + 1)
        value, ms_max, total = bench.reduce_over_ranks(ms, work, "cpu", world)
        out[rank] = (value, ms_max, total, work, [(r.mesh, r.nsteps) for r in reqs[:5]],
                     len(wl.serve_stream(count=50, seed=5 + 1000 * rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_cpu_ranks_reduce_work_and_time():
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
        value, ms_max, total, _, _, n = res[r]
        assert ms_max == pytest.approx(200.0)          # the slowest rank's time
        assert total == pytest.approx(w0 + w1)          # all ranks' work
        assert value == pytest.approx((w0 + w1) / 0.2)
        assert n == 50
    # the ranks serve different streams (no request served twice)
    assert res[0][4] != res[1][4]
