"""Request server: continuous batching of static-mesh integrations (sfx_server_*).

    srv = Server(precision=PREC_SPLIT, memory_budget=150 << 30)
    mid = srv.add_mesh(mesh)                      # upload once to the device pool
    rid = srv.submit(mid, W0, "HLLC", dt, 100)    # queued, returns at once
    out = srv.poll(rid)                           # None while running
    srv.shutdown()

A native worker thread admits queued requests in arrival order under the
device-memory budget and the slot limit, keeps their states resident and, in
split precision, advances all requests of one (dimension, solver) class in
shared launches; requests that arrive meanwhile join at the next round.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .mesh import Mesh

SOLVER_CODES = {"Exact": L.SOLVER_EXACT, "HLLC": L.SOLVER_HLLC,
                L.SOLVER_EXACT: L.SOLVER_EXACT, L.SOLVER_HLLC: L.SOLVER_HLLC}


@dataclass
class Result:
    status: int
    steps_done: int
    mesh_id: int
    solver: int
    t_submit: float
    t_admit: float
    t_done: float
    face_steps: int
    W: np.ndarray | None = None
    Q: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class Server:
    def __init__(self, precision: int = L.PREC_SPLIT, gamma: float = 5.0 / 3.0,
                 tolerance: float = 1e-8, cutoff: float = -5.0, memory_budget: int = 150 << 30,
                 max_active: int = 4096, chunk_steps: int = 4, device: int = 0):
        cfg = L.sfx_server_config(device, precision, gamma, tolerance, cutoff, memory_budget,
                                  max_active, chunk_steps)
        h = C.c_void_p()
        L.check(L.lib().sfx_server_create(C.byref(cfg), C.byref(h)), "sfx_server_create")
        self.h = h
        self.meshes: list[Mesh] = []
        self._mesh_of: dict[int, int] = {}

    def set_tuning(self, dim: int, solver, lanes: int = 0, face_variant: int = 0) -> None:
        """split servers: kernel settings of one (dim, solver) class's launch
        group (lanes 0: the default), applied before its next round"""
        L.check(L.lib().sfx_server_set_tuning(self.h, dim, SOLVER_CODES[solver], lanes,
                                              face_variant), "sfx_server_set_tuning")

    def add_mesh(self, mesh: Mesh) -> int:
        mid = C.c_int32(-1)
        d = mesh.desc()
        L.check(L.lib().sfx_server_add_mesh(self.h, C.byref(d), C.byref(mid)),
                "sfx_server_add_mesh")
        self.meshes.append(mesh)
        return mid.value

    def submit(self, mesh_id: int, W0: np.ndarray, solver, dt: float, nsteps: int) -> int:
        W0 = np.ascontiguousarray(W0, np.float64)
        m = self.meshes[mesh_id]
        assert W0.shape == (m.n_cells, m.dim + 2), W0.shape
        rid = C.c_int64(0)
        L.check(L.lib().sfx_server_submit(self.h, mesh_id, L.dptr(W0), SOLVER_CODES[solver],
                                          float(dt), int(nsteps), C.byref(rid)),
                "sfx_server_submit")
        self._mesh_of[rid.value] = mesh_id
        return rid.value

    def poll(self, rid: int, want_state: bool = True) -> Result | None:
        """None while the request runs; then its Result (the server forgets it)"""
        info = L.sfx_request_info()
        info.status = -1
        W = Q = None
        m = self.meshes[self._mesh_of[rid]] if rid in self._mesh_of else None
        if want_state and m is not None:
            W = np.full((m.n_cells, m.dim + 2), np.nan)
            Q = np.full((m.n_cells, m.dim + 2), np.nan)
        rc = L.lib().sfx_server_poll(self.h, rid, L.dptr(W), L.dptr(Q), C.byref(info))
        if rc == L.SFX_ERR_NOT_READY:
            return None
        if info.status == -1:
            raise L.SfxError(rc, f"sfx_server_poll({rid})")
        self._mesh_of.pop(rid, None)
        return Result(info.status, info.steps_done, info.mesh_id, info.solver, info.t_submit,
                      info.t_admit, info.t_done, info.face_steps, W, Q)

    def drain(self, timeout: float = 0.0) -> bool:
        return L.lib().sfx_server_drain(self.h, timeout) == L.SFX_OK

    def stats(self) -> L.sfx_server_stats:
        st = L.sfx_server_stats()
        L.check(L.lib().sfx_server_stats_get(self.h, C.byref(st)), "sfx_server_stats_get")
        return st

    def shutdown(self):
        if self.h:
            L.lib().sfx_server_shutdown(self.h)
            self.h = None

    def __del__(self):
        try:
            self.shutdown()
        except Exception:
            pass
