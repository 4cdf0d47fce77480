"""Generate tests/golden/fullsize.json: fingerprints of the reference's own
CPU flux pass on the two large single-mesh workloads at their full sizes, for
tests/test_gpu_fullsize.py (run where the reference harness binaries exist:
``python oracle/build.py`` first; several minutes of CPU time).

  sedov3d   262,144 generators (seed 2), reflective unit cube, HLLC, CFL-0.4
            dt, 50 steps: the reference harness with sfx_pow (bitwise target)
            -> SHA-256 of W and Q; with glibc pow -> every 997th cell's Q
            (the 1e-12 target)
  random3d  2,097,152 generators (seed 3), periodic unit cube, exact solver,
            one step: the same fingerprints, plus the oracle restatement's
            single pass (pinned bit for bit to the reference on the small
            golden meshes) -> SHA-256 of the per-face dQ, the gradients and
            the per-face branch codes

The arrays are fingerprinted, not stored (the random-field pass alone has
660 MB of per-face dQ); the mesh and the initial state are fingerprinted too,
so a test can tell a different tessellation from a different pass.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import Oracle, Params, run_reference  # noqa: E402
from shadowfax_b200 import workloads as wl  # noqa: E402

OUT = Path(__file__).resolve().parent / "fullsize.json"
SAMPLE_EVERY = 997


def sha(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()).hexdigest()


def mesh_sha(m) -> str:
    h = hashlib.sha256()
    for name in m._ARRAYS:
        a = np.ascontiguousarray(getattr(m, name))
        h.update(name.encode())
        h.update(a.tobytes())
    return h.hexdigest()


def case(name, pr, single_pass: bool):
    m = pr.mesh
    p = Params(solver=pr.solver, gamma=pr.gamma)
    out = {"n_cells": m.n_cells, "n_faces": m.n_faces, "solver": pr.solver, "dt": pr.dt,
           "nsteps": pr.nsteps, "mesh_sha256": mesh_sha(m), "W0_sha256": sha(pr.W0)}
    r = run_reference(m, p, pr.dt, pr.nsteps, pr.W0, pow_kind="sfxpow")
    assert r["status"] == 0 and r["steps"] == pr.nsteps, (name, r["status"])
    out["ref_sfxpow_W_sha256"] = sha(r["W"])
    out["ref_sfxpow_Q_sha256"] = sha(r["Q"])
    r = run_reference(m, Params(solver=pr.solver, gamma=pr.gamma, use_libm_pow=True), pr.dt,
                      pr.nsteps, pr.W0, pow_kind="libm")
    assert r["status"] == 0, (name, r["status"])
    idx = np.arange(0, m.n_cells, SAMPLE_EVERY)
    out["ref_libm_sample_every"] = SAMPLE_EVERY
    out["ref_libm_Q_sample"] = r["Q"][idx].tolist()
    out["ref_libm_Q_absmax"] = np.abs(r["Q"]).max(0).tolist()
    if single_pass:
        o = Oracle()
        Q0 = o.init_Q(m, p, pr.W0)
        g, dQ, code, rc, _ = o.flux_pass(m, p, pr.dt, pr.W0, Q0)
        assert rc == 0
        out["oracle_pass_dQ_sha256"] = sha(dQ)
        out["oracle_pass_grad_sha256"] = sha(g)
        out["oracle_pass_branch_sha256"] = sha(code.astype(np.int32))
    print(name, {k: v for k, v in out.items() if not k.startswith("ref_libm_Q")}, flush=True)
    return out


def main():
    res = {"sedov3d": case("sedov3d", wl.sedov3d(), False),
           "random3d": case("random3d", wl.random_field3d(), True)}
    OUT.write_text(json.dumps(res, indent=1) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
