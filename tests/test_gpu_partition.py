"""One mesh split into parts, all parts on one GPU in one process (plain
FP64 and the FP32/FP64 split): each part's pass restricted to its ranges
(sfx_mesh_set_ranges) and
the ring records moved between parts through device buffers
(sfx_mesh_pack_cells / sfx_mesh_unpack_cells) give the owned cells the
values of the pass over the whole mesh, bit for bit.  On several GPUs the
same records travel through exchange_records (NCCL); that transfer is
covered by the gloo test in test_multirank.py."""
import numpy as np
import pytest

from golden_util import load_case

pytestmark = pytest.mark.gpu


def _ctx(mesh, meta, precision=0):
    from shadowfax_b200.hydro import Context, RiemannSolverFactory
    return Context(mesh.dim, RiemannSolverFactory.generate(meta["solver"], meta["gamma"]),
                   precision)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,nparts", [("sod2d_exact", 2), ("random2d_periodic_exact", 3),
                                         ("sedov3d_hllc", 2), ("random3d_exact", 3)])
def test_parts_on_one_gpu_equal_the_whole_mesh(cuda_ok, name, nparts, precision):
    import torch

    from shadowfax_b200 import partition as P
    from shadowfax_b200.hydro import FluxPass
    mesh, meta, _ = load_case(name)
    dt, nsteps = meta["dt"], 5
    ctx = _ctx(mesh, meta, precision)
    whole = FluxPass(ctx, mesh)
    whole.set_primitive(meta["W0"])
    whole.step(dt, nsteps)
    Wg, Qg = whole.state()

    owner = P.partition(mesh, nparts)
    parts = [P.build_part(mesh, owner, r) for r in range(nparts)]
    plans = [P.exchange_plan(mesh, owner, pt) for pt in parts]
    fps = []
    for pt in parts:
        fp = FluxPass(ctx, pt.mesh)
        fp.set_ranges(pt.n_grad, pt.n_flux, pt.n_own)
        fp.set_primitive(meta["W0"][pt.cells])
        fps.append(fp)
    dev = torch.device("cuda", 0)
    R = mesh.dim + 3
    send = {(r, q): torch.as_tensor(s, device=dev) for r in range(nparts)
            for q, (s, _) in plans[r].items()}
    recv = {(r, q): torch.as_tensor(v, device=dev) for r in range(nparts)
            for q, (_, v) in plans[r].items()}
    buf = {k: torch.empty((v.numel(), R), dtype=torch.float64, device=dev)
           for k, v in send.items()}
    torch.cuda.synchronize()
    for _ in range(nsteps):
        for fp in fps:
            fp.step(dt, 1)
        for (r, q), idx in send.items():
            fps[r].pack_cells(idx, buf[(r, q)])
        for (r, q), idx in recv.items():
            fps[r].unpack_cells(idx, buf[(q, r)])
        ctx.synchronize()
    seen = np.zeros(mesh.n_cells, int)
    for pt, fp in zip(parts, fps):
        W, Q = fp.state()
        own = pt.cells[:pt.n_own]
        seen[own] += 1
        np.testing.assert_array_equal(W[:pt.n_own], Wg[own])
        np.testing.assert_array_equal(Q[:pt.n_own], Qg[own])
        # the ring cells hold their owners' W after the last exchange
        np.testing.assert_array_equal(W[pt.n_own:], Wg[pt.cells[pt.n_own:]])
    assert np.all(seen == 1)
    # the parts' totals (over their owned cells) add up to the whole mesh's
    tot = sum(fp.totals() for fp in fps)
    assert np.all(np.abs(tot - whole.totals()) <= 1e-12 * np.abs(Qg).sum(0))


def test_ranges_are_checked(cuda_ok):
    from shadowfax_b200._lib import SfxError
    from shadowfax_b200.hydro import FluxPass
    mesh, meta, _ = load_case("sod2d_exact")
    fp = FluxPass(_ctx(mesh, meta), mesh)
    n, F = mesh.n_cells, mesh.n_faces
    for bad in [(n + 1, F, n), (n, F + 1, n), (n - 5, F, n), (n, F, -1)]:
        with pytest.raises(SfxError):
            fp.set_ranges(*bad)
    fp.set_ranges(n, F, n)          # the whole mesh: the unrestricted pass
    fp2 = FluxPass(_ctx(mesh, meta, precision=1), mesh)
    twin = fp2.clone()
    with pytest.raises(SfxError):
        twin.set_ranges(n, F, n)    # not a split clone: it shares the owner's tables
    fp2.set_ranges(n, F, n)         # the split pass takes ranges
