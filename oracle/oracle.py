"""Python front end of the CPU checkers — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module, and only as the checker (never as the thing measured or
shipped).

* :class:`Oracle` wraps ``libsfxoracle.so``, the C restatement of the
  reference flux pass (sfx_oracle.c).
* :func:`run_reference` runs the reference's own CPU flux pass (the unmodified
  Shadowfax sources, oracle/_ref/refharness_*) on a mesh and returns its
  final state; :func:`riemann_reference` evaluates the reference Riemann
  solvers on state pairs; :func:`reference_tessellation` tessellates with the
  reference's own DelTess/VorTess (oracle/_ref/tessharness_*), exports the
  face list and can run the reference's step loop on that tessellation.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

SOLVERS = {"Exact": 0, "HLLC": 1, "EXAC": 0, 0: 0, 1: 1}


class sfxo_mesh(C.Structure):
    _fields_ = [("dim", C.c_int), ("ncell", C.c_int), ("nface", C.c_int),
                ("cell_pos", _dp), ("cell_centroid", _dp), ("cell_volume", _dp),
                ("cell_total_area", _dp), ("cell_face_offset", _ip),
                ("cell_face_index", _ip), ("face_area", _dp), ("face_midpoint", _dp),
                ("face_left", _ip), ("face_right", _ip), ("face_kind", _ip),
                ("face_right_pos", _dp), ("face_velocity", _dp)]


class sfxo_params(C.Structure):
    _fields_ = [("solver", C.c_int), ("gamma", C.c_double), ("tolerance", C.c_double),
                ("cutoff", C.c_double), ("use_libm_pow", C.c_int)]


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


@dataclass
class Params:
    solver: int = 0
    gamma: float = 5.0 / 3.0
    tolerance: float = 1e-8
    cutoff: float = -5.0
    use_libm_pow: bool = False

    def c(self) -> sfxo_params:
        return sfxo_params(SOLVERS[self.solver], self.gamma, self.tolerance, self.cutoff,
                           int(self.use_libm_pow))


class Oracle:
    """CPU restatement of the flux pass (bit-identical to the GPU FP64 pass
    when ``use_libm_pow`` is False)."""

    def __init__(self):
        so = HERE / "libsfxoracle.so"
        if not so.exists():
            from oracle.build import build_oracle
            build_oracle()
        L = C.CDLL(str(so))
        P = C.POINTER(sfxo_mesh), C.POINTER(sfxo_params)
        L.sfxo_init_Q.argtypes = [P[0], P[1], _dp, _dp]
        L.sfxo_gradients.argtypes = [P[0], _dp, _dp]
        L.sfxo_face_fluxes.argtypes = [P[0], P[1], C.c_double, _dp, _dp, _dp, _dp, _ip, _ip]
        L.sfxo_apply.argtypes = [P[0], P[1], _dp, _dp, _dp, _dp, _ip]
        L.sfxo_run.argtypes = [P[0], P[1], C.c_double, C.c_int, _dp, _dp, _dp, _dp, _ip,
                               C.POINTER(C.c_double)]
        L.sfxo_riemann.argtypes = [C.c_int, P[1], C.c_int, _dp, _dp, _dp, C.c_int, _dp, _dp,
                                   _ip]
        L.sfxo_move_velocities.argtypes = [P[0], P[1], C.c_double, C.c_int, _dp, _dp, _dp]
        _u64 = C.POINTER(C.c_uint64)
        L.sfxo_timestep_bins.argtypes = [P[0], P[1], _dp, _dp, _u64, _u64, C.c_uint64,
                                         C.c_double, C.c_double, C.c_uint64, C.c_uint64, _u64]
        L.sfxo_pow.argtypes = [C.c_double, C.c_double]
        L.sfxo_pow.restype = C.c_double
        L.sfxo_pow_fast.argtypes = [C.c_double, C.c_double]
        L.sfxo_pow_fast.restype = C.c_double
        self.L = L

    @staticmethod
    def _mesh(m) -> sfxo_mesh:
        m.normalized()
        s = sfxo_mesh()
        s.dim, s.ncell, s.nface = m.dim, m.n_cells, m.n_faces
        s.cell_pos, s.cell_centroid = _d(m.cell_pos), _d(m.cell_centroid)
        s.cell_volume, s.cell_total_area = _d(m.cell_volume), _d(m.cell_total_area)
        s.cell_face_offset, s.cell_face_index = _i(m.cell_face_offset), _i(m.cell_face_index)
        s.face_area, s.face_midpoint = _d(m.face_area), _d(m.face_midpoint)
        s.face_left, s.face_right, s.face_kind = _i(m.face_left), _i(m.face_right), _i(m.face_kind)
        s.face_right_pos = _d(m.face_right_pos)
        vel = m.face_velocity if m.face_velocity is not None else np.zeros_like(m.face_midpoint)
        s._vel = vel
        s.face_velocity = _d(vel)
        return s

    def init_Q(self, mesh, p: Params, W: np.ndarray) -> np.ndarray:
        W = np.ascontiguousarray(W, np.float64)
        Q = np.empty_like(W)
        rc = self.L.sfxo_init_Q(C.byref(self._mesh(mesh)), C.byref(p.c()), _d(W), _d(Q))
        if rc:
            raise RuntimeError(f"oracle init_Q status {rc}")
        return Q

    def flux_pass(self, mesh, p: Params, dt: float, W: np.ndarray, Q: np.ndarray):
        """gradients, per-face limited dQ of the left cell, branch codes"""
        S = mesh.dim + 2
        W = np.ascontiguousarray(W, np.float64)
        Q = np.ascontiguousarray(Q, np.float64)
        m = self._mesh(mesh)
        grad = np.empty((mesh.n_cells, mesh.dim, S))
        self.L.sfxo_gradients(C.byref(m), _d(W), _d(grad))
        dQ = np.empty((mesh.n_faces, S))
        code = np.empty(mesh.n_faces, np.int32)
        bad = C.c_int(-1)
        rc = self.L.sfxo_face_fluxes(C.byref(m), C.byref(p.c()), dt, _d(W), _d(Q), _d(grad),
                                     _d(dQ), _i(code), C.byref(bad))
        return grad, dQ, code, rc, bad.value

    def apply(self, mesh, p: Params, dQ_face: np.ndarray, W: np.ndarray, Q: np.ndarray):
        """scatter + update_Q + get_W; returns (W, Q, status, bad_cell)"""
        S = mesh.dim + 2
        W = np.array(W, np.float64, copy=True, order="C")
        Q = np.array(Q, np.float64, copy=True, order="C")
        dQ_face = np.ascontiguousarray(dQ_face, np.float64)
        dQc = np.empty((mesh.n_cells, S))
        bad = C.c_int(-1)
        rc = self.L.sfxo_apply(C.byref(self._mesh(mesh)), C.byref(p.c()), _d(dQ_face), _d(Q),
                               _d(W), _d(dQc), C.byref(bad))
        return W, Q, rc, bad.value

    def run(self, mesh, p: Params, dt: float, nsteps: int, W: np.ndarray,
            Q: np.ndarray | None = None):
        """nsteps of the full pass; returns (W, Q, status, steps_done, seconds)"""
        S = mesh.dim + 2
        W = np.array(W, np.float64, copy=True, order="C")
        Q = self.init_Q(mesh, p, W) if Q is None else np.array(Q, np.float64, copy=True, order="C")
        steps = C.c_int(0)
        secs = C.c_double(0)
        grad = np.empty((mesh.n_cells, mesh.dim, S))
        dQc = np.empty((mesh.n_cells, S))
        rc = self.L.sfxo_run(C.byref(self._mesh(mesh)), C.byref(p.c()), dt, nsteps, _d(W), _d(Q),
                             _d(grad), _d(dQc), C.byref(steps), C.byref(secs))
        return dict(W=W, Q=Q, status=rc, steps=steps.value, seconds=secs.value, grad=grad,
                    dQ=dQc)

    def run_moving(self, mesh, p: Params, dt: float, W: np.ndarray, periodic: bool):
        """one step with moving generators (the reference built without
        -DSTATIC): generator and face velocities, the step with the fluxes in
        the faces' frames, the drift; returns (W, Q, status, positions)"""
        W = np.array(W, np.float64, copy=True, order="C")
        vgen = np.empty((mesh.n_cells, mesh.dim))
        vface = np.empty((mesh.n_faces, mesh.dim))
        self.L.sfxo_move_velocities(C.byref(self._mesh(mesh)), C.byref(p.c()), dt,
                                    int(periodic), _d(W), _d(vgen), _d(vface))
        import dataclasses
        moved = dataclasses.replace(mesh, face_velocity=vface)
        r = self.run(moved, p, dt, 1, W)
        pos = mesh.cell_pos + dt * vgen
        return r["W"], r["Q"], r["status"], pos

    def timestep_bins(self, mesh, p: Params, W, vgen, start, end, t_next: int, t_total: float,
                      cfl: float, max_step: int, min_step: int):
        """TimeLine::calculate_timestep for the cells ending at t_next:
        returns (start, end, smallest new step, status)"""
        W = np.ascontiguousarray(W, np.float64)
        vgen = np.ascontiguousarray(vgen, np.float64)
        s = np.array(start, np.uint64, copy=True, order="C")
        e = np.array(end, np.uint64, copy=True, order="C")
        smin = C.c_uint64(0)
        u = C.POINTER(C.c_uint64)
        rc = self.L.sfxo_timestep_bins(C.byref(self._mesh(mesh)), C.byref(p.c()), _d(W),
                                       _d(vgen), s.ctypes.data_as(u), e.ctypes.data_as(u),
                                       int(t_next), t_total, cfl, int(max_step), int(min_step),
                                       C.byref(smin))
        return s, e, int(smin.value), rc

    def riemann(self, dim: int, p: Params, WL, WR, normal, reflective: bool = False):
        WL = np.ascontiguousarray(WL, np.float64)
        WR = np.ascontiguousarray(WR, np.float64)
        normal = np.ascontiguousarray(normal, np.float64)
        n = WL.shape[0]
        half = np.zeros_like(WL)
        flux = np.zeros_like(WL)
        code = np.zeros(n, np.int32)
        self.L.sfxo_riemann(dim, C.byref(p.c()), n, _d(WL), _d(WR), _d(normal), int(reflective),
                            _d(half), _d(flux), _i(code))
        return half, flux, code

    def pow(self, x: float, y: float) -> float:
        return self.L.sfxo_pow(x, y)

    def pow_fast(self, x: float, y: float) -> float:
        return self.L.sfxo_pow_fast(x, y)


# ---------------------------------------------------------------- reference

def ref_binary(dim: int, pow_kind: str = "libm", moving: bool = False) -> Path:
    return REF_DIR / f"refharness_{dim}d{'_moving' if moving else ''}_{pow_kind}"


def reference_available(dim: int = 2, pow_kind: str = "libm", moving: bool = False) -> bool:
    return ref_binary(dim, pow_kind, moving).exists()


def _write_mesh_input(f, mesh, p: Params, dt: float, nsteps: int, W0: np.ndarray,
                      moving: bool = False, local: dict | None = None):
    m = mesh.normalized()
    f.write(b"SFXMESH1")
    mode = 2 if local is not None else int(moving)
    np.array([m.dim, m.n_cells, m.n_faces, m.nnz, SOLVERS[p.solver], nsteps, mode,
              int(m.periodic)], np.int32).tofile(f)
    np.array([p.gamma, p.tolerance, p.cutoff, dt], np.float64).tofile(f)
    vel = m.face_velocity if m.face_velocity is not None else np.zeros_like(m.face_midpoint)
    for a in (m.cell_pos, m.cell_centroid, m.cell_volume, m.cell_total_area,
              m.cell_face_offset, m.cell_face_index, m.face_area, m.face_midpoint, m.face_left,
              m.face_right, m.face_kind, m.face_right_pos, vel,
              np.ascontiguousarray(W0, np.float64)):
        np.ascontiguousarray(a).tofile(f)
    if local is not None:
        np.ascontiguousarray(local["start"], np.uint64).tofile(f)
        np.ascontiguousarray(local["end"], np.uint64).tofile(f)
        np.array([local["t_now"], local["t_next"]], np.uint64).tofile(f)
        np.array([local["t_total"]], np.float64).tofile(f)
        np.ascontiguousarray(local["grad0"], np.float64).tofile(f)


def run_reference(mesh, p: Params, dt: float, nsteps: int, W0: np.ndarray,
                  pow_kind: str = "libm", timeout: float | None = None,
                  moving: bool = False, local: dict | None = None) -> dict:
    """Run the reference CPU pass (unmodified Shadowfax sources) for nsteps.
    moving=True: the build without -DSTATIC, one step with moving generators
    (VorCell::get_velocity, VorFace::set_v, the drift); the result then also
    holds the drifted generator positions ("pos").
    local={start, end, t_now, t_next, t_total, grad0}: one system step of
    local time steps on the 2^60-tick timeline (each particle's step bounds,
    the stored gradients of the inactive ones); the result also holds the
    velocities the active particles set ("vel", zero for the others)."""
    exe = ref_binary(mesh.dim, pow_kind, moving)
    if not exe.exists():
        raise FileNotFoundError(f"{exe} not built (oracle/build.py needs the reference tree)")
    S = mesh.dim + 2
    n = mesh.n_cells
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            _write_mesh_input(f, mesh, p, dt, nsteps, W0, moving, local)
        subprocess.run([str(exe), fin, fout, "step"], check=True, timeout=timeout)
        raw = open(fout, "rb").read()
    hdr = np.frombuffer(raw, np.int32, 4)
    secs = float(np.frombuffer(raw, np.float64, 1, 16)[0])
    step_secs = np.frombuffer(raw, np.float64, nsteps, 24).copy()
    body = np.frombuffer(raw, np.float64, offset=24 + 8 * nsteps)
    o = 0
    W = body[o:o + n * S].reshape(n, S).copy(); o += n * S
    Q = body[o:o + n * S].reshape(n, S).copy(); o += n * S
    grad = body[o:o + n * mesh.dim * S].reshape(n, mesh.dim, S).copy(); o += n * mesh.dim * S
    dQ = body[o:o + n * S].reshape(n, S).copy(); o += n * S
    out = dict(status=int(hdr[0]), steps=int(hdr[1]), seconds=secs, step_seconds=step_secs,
               W=W, Q=Q, grad=grad, dQ=dQ)
    if local is not None:
        out["vel"] = body[o:o + n * mesh.dim].reshape(n, mesh.dim).copy(); o += n * mesh.dim
    if moving:
        out["pos"] = body[o:o + n * mesh.dim].reshape(n, mesh.dim).copy()
    return out


def tess_binary(dim: int, pow_kind: str = "libm") -> Path:
    return REF_DIR / f"tessharness_{dim}d_{pow_kind}"


def reference_tessellation(pos: np.ndarray, periodic: bool, p: Params | None = None,
                           dt: float = 0., nsteps: int = 0, W0: np.ndarray | None = None,
                           pow_kind: str = "libm", tess_tolerance: float = 1e-9,
                           timeout: float | None = None) -> dict:
    """Tessellate generator positions in the unit box with the reference's own
    DelTess/VorTess (oracle/refharness/tessharness.cpp) and export its face
    list; cells come back in the reference's Hilbert order ("order": the
    input index of each cell).  With W0 (input order) the reference's step
    loop also runs nsteps on the objects VorTess built ("W", "Q", sorted
    order).  Returns {"mesh": Mesh, "order", "status", "steps", "W", "Q"}."""
    from shadowfax_b200.mesh import Mesh
    pos = np.ascontiguousarray(pos, np.float64)
    n, dim = pos.shape
    exe = tess_binary(dim, pow_kind)
    if not exe.exists():
        raise FileNotFoundError(f"{exe} not built (oracle/build.py needs the reference tree)")
    p = p or Params()
    S = dim + 2
    has_w = W0 is not None
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            np.array([dim, n, int(periodic), SOLVERS[p.solver], nsteps, int(has_w)],
                     np.int32).tofile(f)
            np.array([p.gamma, p.tolerance, p.cutoff, dt, tess_tolerance], np.float64).tofile(f)
            pos.tofile(f)
            if has_w:
                np.ascontiguousarray(W0, np.float64).tofile(f)
        subprocess.run([str(exe), fin, fout], check=True, timeout=timeout,
                       stdout=subprocess.DEVNULL)
        raw = open(fout, "rb").read()
    status, steps, nn, F, nnz = np.frombuffer(raw, np.int32, 5)
    o = 20

    def take(dtype, count, shape=None):
        nonlocal o
        a = np.frombuffer(raw, dtype, count, o).copy()
        o += a.nbytes
        return a.reshape(shape) if shape else a

    order = take(np.int32, n)
    mesh = Mesh(dim=dim, periodic=bool(periodic),
                cell_pos=take(np.float64, n * dim, (n, dim)),
                cell_centroid=take(np.float64, n * dim, (n, dim)),
                cell_volume=take(np.float64, n),
                cell_total_area=take(np.float64, n),
                cell_face_offset=take(np.int32, n + 1),
                cell_face_index=take(np.int32, int(nnz)),
                face_area=take(np.float64, int(F)),
                face_midpoint=take(np.float64, int(F) * dim, (int(F), dim)),
                face_left=take(np.int32, int(F)),
                face_right=take(np.int32, int(F)),
                face_kind=take(np.int32, int(F)),
                face_right_pos=take(np.float64, int(F) * dim, (int(F), dim)))
    out = dict(mesh=mesh, order=order, status=int(status), steps=int(steps))
    if has_w:
        out["W"] = take(np.float64, n * S, (n, S))
        out["Q"] = take(np.float64, n * S, (n, S))
    return out


def riemann_reference(dim: int, p: Params, WL, WR, normal, reflective: bool = False,
                      pow_kind: str = "libm") -> dict:
    """Reference solve() (exact) and solve_for_flux() on state pairs."""
    exe = ref_binary(dim, pow_kind)
    S = dim + 2
    WL = np.ascontiguousarray(WL, np.float64)
    n = WL.shape[0]
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(b"SFXMESH1")
            np.array([n, SOLVERS[p.solver], int(reflective), 0], np.int32).tofile(f)
            np.array([p.gamma, p.tolerance, p.cutoff, 0.], np.float64).tofile(f)
            WL.tofile(f)
            np.ascontiguousarray(WR, np.float64).tofile(f)
            np.ascontiguousarray(normal, np.float64).tofile(f)
        subprocess.run([str(exe), fin, fout, "riemann"], check=True)
        raw = open(fout, "rb").read()
    st = np.frombuffer(raw, np.int32, n).copy()
    body = np.frombuffer(raw, np.float64, offset=4 * n)
    return dict(status=st, half=body[:n * S].reshape(n, S).copy(),
                flux=body[n * S:2 * n * S].reshape(n, S).copy())
