"""sfx_flux_pass_noalloc: the flux pass for callers that cannot let the
library allocate device memory (they own every array; the gradient scratch
is a fixed device array inside the library).  Its output must equal the
allocating entry point's (sfx_flux_pass, plain FP64: bit for bit) on two
calls in a row, the second on a different mesh, so a stale scratch array
would show.  Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

from golden_util import load_case


def _device_mesh(mesh, torch):
    """the mesh in the field-major device layout, owned by the caller"""
    dev = "cuda:0"
    keep = []

    def d(a, dtype):
        t = torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)
        keep.append(t)
        return t.data_ptr()

    n = mesh.n_cells
    off, idx = mesh.cell_face_offset, mesh.cell_face_index
    owner = np.repeat(np.arange(n), np.diff(off))
    entry = idx.astype(np.uint32) | np.where(mesh.face_left[idx] != owner,
                                             np.uint32(1 << 31), np.uint32(0))
    from shadowfax_b200 import _lib as L
    dm = L.sfx_device_mesh(
        mesh.dim, n, mesh.n_faces,
        d(mesh.cell_pos.T, torch.float64), d(mesh.cell_centroid.T, torch.float64),
        d(mesh.cell_volume, torch.float64), d(mesh.cell_total_area, torch.float64),
        d(off, torch.int32), d(entry.view(np.int32), torch.int32),
        d(mesh.face_area, torch.float64), d(mesh.face_midpoint.T, torch.float64),
        d(mesh.face_left, torch.int32), d(mesh.face_right, torch.int32),
        d(mesh.face_kind, torch.int32), d(mesh.face_right_pos.T, torch.float64))
    return dm, keep


def _case(name, torch):
    from shadowfax_b200 import _lib as L
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    mesh, meta, _ = load_case(name)
    solver = RiemannSolverFactory.generate(meta["solver"], meta["gamma"])
    ctx = Context(mesh.dim, solver)
    fp = FluxPass(ctx, mesh)
    fp.set_primitive(meta["W0"])
    W, Q = fp.state()
    _, want, _, rc, _ = fp.flux_pass(meta["dt"])       # the allocating entry point
    assert rc == 0
    cfg = L.sfx_config(mesh.dim, solver.kind, solver.gamma, solver.tolerance, solver.cutoff,
                       L.PREC_FP64, 0)
    return mesh, meta, cfg, W, Q, want


@pytest.mark.gpu
def test_noalloc_pass_matches_allocating_pass_twice(cuda_ok):
    import torch
    from shadowfax_b200 import _lib as L
    lib = L.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for name in ("sod2d_hllc", "sedov3d_hllc"):       # two calls in a row
        mesh, meta, cfg, W, Q, want = _case(name, torch)
        dm, keep = _device_mesh(mesh, torch)
        S = mesh.dim + 2
        dW = torch.as_tensor(np.ascontiguousarray(W.T), device="cuda:0")
        dQ = torch.as_tensor(np.ascontiguousarray(Q.T), device="cuda:0")
        out = torch.full((S, mesh.n_faces), float("nan"), dtype=torch.float64, device="cuda:0")
        rc = lib.sfx_flux_pass_noalloc(C.byref(dm), C.byref(cfg), meta["dt"], dW.data_ptr(),
                                       dQ.data_ptr(), out.data_ptr(), C.c_void_p(stream))
        assert rc == L.SFX_OK
        got = out.cpu().numpy().T
        np.testing.assert_array_equal(got, want)


def test_noalloc_rejects_meshes_above_its_scratch_size():
    """size check happens before any CUDA call"""
    from shadowfax_b200 import _lib as L
    lib = L.lib()
    dm = L.sfx_device_mesh(3, 65536 + 1, 10, *([1] * 12))
    cfg = L.sfx_config(3, L.SOLVER_HLLC, 5 / 3, 1e-8, -5.0, L.PREC_FP64, 0)
    rc = lib.sfx_flux_pass_noalloc(C.byref(dm), C.byref(cfg), 1e-3, C.c_void_p(1),
                                   C.c_void_p(1), C.c_void_p(1), None)
    assert rc == 13  # SFX_ERR_TOO_LARGE
