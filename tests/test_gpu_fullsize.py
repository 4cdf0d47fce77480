"""The two large single-mesh workloads at their full sizes, against the
reference's own CPU flux pass.  tests/golden/fullsize.json holds SHA-256
fingerprints of the reference harness's results (made by
tests/golden/make_fullsize.py from the unmodified Shadowfax sources):

* Sedov 3D, 262,144 generators, HLLC, 50 CFL-0.4 steps: the plain FP64 pass
  equals the reference built with sfx_pow bit for bit (W and Q), and is
  within 1e-12 per field of the reference with glibc pow on every 997th cell;
  the FP32/FP64 split pass after the same 50 steps is within 1e-6 relative L1
  of the FP64 pass per conserved field, mass conserved to round-off;
* random field 3D, 2,097,152 generators, periodic, exact solver: the single
  pass's per-face dQ, gradients and branch codes equal the oracle's bit for
  bit, and one step equals the reference's bit for bit.

The meshes are rebuilt here by the face-list builder; their fingerprint is
checked first, so a different tessellation is told apart from a different
pass."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIX = json.loads((Path(__file__).resolve().parent / "golden" / "fullsize.json").read_text())


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _mesh_sha(m):
    h = hashlib.sha256()
    for name in m._ARRAYS:
        h.update(name.encode())
        h.update(np.ascontiguousarray(getattr(m, name)).tobytes())
    return h.hexdigest()


def _close_per_field(a, b, absmax, rtol=1e-12, atol_scale=1e-15):
    """per conserved field and cell: |a - b| <= rtol |b| + atol_scale * max|b|
    over the field (the absolute term only matters for values at the
    round-off level of their field)"""
    for k in range(b.shape[1]):
        lim = rtol * np.abs(b[:, k]) + atol_scale * absmax[k]
        err = np.abs(a[:, k] - b[:, k])
        assert np.all(err <= lim), (k, float(np.max(err / np.maximum(lim, 1e-300))))


def _check_case(pr, fix):
    assert pr.mesh.n_cells == fix["n_cells"] and pr.mesh.n_faces == fix["n_faces"]
    assert _mesh_sha(pr.mesh) == fix["mesh_sha256"], "the builder made another tessellation"
    assert _sha(pr.W0) == fix["W0_sha256"]
    assert pr.dt == fix["dt"]


def _fp64(pr):
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    ctx = Context(pr.mesh.dim, RiemannSolverFactory.generate(pr.solver, pr.gamma), 0)
    fp = FluxPass(ctx, pr.mesh)
    fp.set_primitive(pr.W0)
    return ctx, fp


@pytest.fixture(scope="module")
def sedov():
    from shadowfax_b200 import workloads as wl
    pr = wl.sedov3d()
    _check_case(pr, FIX["sedov3d"])
    return pr


def test_sedov3d_full_fp64_vs_reference(cuda_ok, sedov):
    fix = FIX["sedov3d"]
    pr = sedov
    ctx, fp = _fp64(pr)
    st = fp.step(pr.dt, fix["nsteps"])
    assert st.status == 0
    W, Q = fp.state()
    assert _sha(Q) == fix["ref_sfxpow_Q_sha256"]
    assert _sha(W) == fix["ref_sfxpow_W_sha256"]
    idx = np.arange(0, pr.mesh.n_cells, fix["ref_libm_sample_every"])
    _close_per_field(Q[idx], np.array(fix["ref_libm_Q_sample"]), fix["ref_libm_Q_absmax"])
    fp.close()
    ctx.close()


def test_sedov3d_full_split_vs_fp64_50_steps(cuda_ok, sedov):
    from shadowfax_b200.hydro import Context, FluxPass, RiemannSolverFactory
    pr = sedov
    nsteps = FIX["sedov3d"]["nsteps"]
    ctx, fp = _fp64(pr)
    fp.step(pr.dt, nsteps)
    Q64 = fp.state()[1]
    fp.close()
    ctx.close()
    ctx = Context(3, RiemannSolverFactory.generate(pr.solver, pr.gamma), 1)
    fp = FluxPass(ctx, pr.mesh)
    fp.set_primitive(pr.W0)
    Q0 = fp.state()[1]
    st = fp.step(pr.dt, nsteps)
    assert st.status == 0
    Q32 = fp.state()[1]
    den = np.abs(Q64).sum(0)
    den[1:4] = np.sqrt((Q64[:, 1:4] ** 2).sum(1)).sum()
    err = np.abs(Q32 - Q64).sum(0) / den
    assert np.all(err <= 1e-6), err
    assert abs(Q32[:, 0].sum() - Q0[:, 0].sum()) <= 1e-13 * Q0[:, 0].sum()
    fp.close()
    ctx.close()


def test_random3d_full_pass_vs_oracle_and_step_vs_reference(cuda_ok):
    from shadowfax_b200 import workloads as wl
    fix = FIX["random3d"]
    pr = wl.random_field3d()
    _check_case(pr, fix)
    ctx, fp = _fp64(pr)
    grad, dQ, br, rc, _ = fp.flux_pass(pr.dt)
    assert rc == 0
    assert _sha(br.astype(np.int32)) == fix["oracle_pass_branch_sha256"]
    assert _sha(dQ) == fix["oracle_pass_dQ_sha256"]
    assert _sha(grad) == fix["oracle_pass_grad_sha256"]
    st = fp.step(pr.dt, fix["nsteps"])
    assert st.status == 0
    W, Q = fp.state()
    assert _sha(Q) == fix["ref_sfxpow_Q_sha256"]
    assert _sha(W) == fix["ref_sfxpow_W_sha256"]
    idx = np.arange(0, pr.mesh.n_cells, fix["ref_libm_sample_every"])
    _close_per_field(Q[idx], np.array(fix["ref_libm_Q_sample"]), fix["ref_libm_Q_absmax"])
    fp.close()
    ctx.close()
