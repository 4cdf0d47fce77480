"""Host-side mirror of Shadowfax's flux-pass interface over the C ABI.

* :class:`RiemannSolver` and :class:`RiemannSolverFactory` mirror the
  reference plugin selection (src/riemann/RiemannSolver.hpp:37-155,
  src/riemann/RiemannSolverFactory.hpp): ``tag()`` "EXAC"/"HLLC",
  ``get_gamma()``, tolerance and cutoff.  Unsupported solver names raise, as
  the factory's ``my_exit()`` does.
* :class:`FluxPass` is the device-side replacement of the gradient loop +
  ``VorTessManager::hydro`` + ``update_Q``/``get_W`` (src/Simulation.cpp:
  414-483, 791-836) for one uploaded mesh.

Errors map onto :class:`shadowfax_b200._lib.SfxError`, whose ``status`` is one
of the SFX_ERR_* codes (RiemannSolverException -> SFX_ERR_RIEMANN,
FluxCalculationException -> SFX_ERR_NAN_FLUX, UpdateQException ->
SFX_ERR_NEG_STATE).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .mesh import Mesh

DEFAULT_GAMMA = 5.0 / 3.0      # RIEMANNSOLVERFACTORY_DEFAULT_GAMMA
DEFAULT_TOLERANCE = 1e-8       # RIEMANNSOLVERFACTORY_DEFAULT_TOLERANCE
DEFAULT_CUTOFF = -5.0          # RIEMANNSOLVERFACTORY_DEFAULT_CUTOFF


class RiemannSolver:
    """Selection of the Riemann solver for the flux pass."""

    kind: int = -1
    _tag: str = ""

    def __init__(self, gamma: float = DEFAULT_GAMMA, tolerance: float = DEFAULT_TOLERANCE,
                 cutoff: float = DEFAULT_CUTOFF):
        self.gamma = float(gamma)
        self.tolerance = float(tolerance)
        self.cutoff = float(cutoff)

    def tag(self) -> str:
        return self._tag

    def get_gamma(self) -> float:
        return self.gamma

    def __repr__(self):
        return f"{type(self).__name__}(gamma={self.gamma!r})"


class ExactRiemannSolver(RiemannSolver):
    """src/riemann/ExactRiemannSolver.cpp"""
    kind = L.SOLVER_EXACT
    _tag = "EXAC"


class HLLCRiemannSolver(RiemannSolver):
    """src/riemann/HLLCRiemannSolver.cpp"""
    kind = L.SOLVER_HLLC
    _tag = "HLLC"


class RiemannSolverFactory:
    """Name / tag -> solver (src/riemann/RiemannSolverFactory.hpp)."""

    @staticmethod
    def generate(name: str, gamma: float = DEFAULT_GAMMA, tolerance: float = DEFAULT_TOLERANCE,
                 cutoff: float = DEFAULT_CUTOFF) -> RiemannSolver:
        if name == "Exact":
            return ExactRiemannSolver(gamma, tolerance, cutoff)
        if name == "HLLC":
            return HLLCRiemannSolver(gamma)
        if name in ("TRRS", "NoPressure", "Advection"):
            raise L.SfxError(L.SFX_ERR_UNSUPPORTED, f"Riemann solver {name!r}")
        raise ValueError(f"Unknown Riemann solver type: {name}!")

    @staticmethod
    def from_tag(tag: str, gamma: float = DEFAULT_GAMMA, tolerance: float = DEFAULT_TOLERANCE,
                 cutoff: float = DEFAULT_CUTOFF) -> RiemannSolver:
        if tag == "EXAC":
            return ExactRiemannSolver(gamma, tolerance, cutoff)
        if tag == "HLLC":
            return HLLCRiemannSolver(gamma)
        raise L.SfxError(L.SFX_ERR_UNSUPPORTED, f"Riemann solver tag {tag!r}")


class Context:
    """One device + solver configuration (sfx_ctx)."""

    def __init__(self, dim: int, solver: RiemannSolver, precision: int = L.PREC_FP64,
                 device: int = 0):
        self.dim = dim
        self.solver = solver
        self.precision = precision
        self.device = device
        cfg = L.sfx_config(dim, solver.kind, solver.gamma, solver.tolerance, solver.cutoff,
                           precision, device)
        h = C.c_void_p()
        L.check(L.lib().sfx_ctx_create(C.byref(cfg), C.byref(h)), "sfx_ctx_create")
        self.h = h

    def close(self):
        if self.h:
            L.lib().sfx_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None):
        L.check(L.lib().sfx_ctx_set_stream(self.h, C.c_void_p(stream_handle or 0)))

    def synchronize(self):
        L.check(L.lib().sfx_ctx_synchronize(self.h))

    def riemann(self, WL, WR, normal, reflective: bool = False):
        """RiemannSolver::solve (exact) and solve_for_flux on the GPU for n
        state pairs with the interface at rest; returns (half, flux, branch)."""
        WL = np.ascontiguousarray(WL, np.float64)
        WR = np.ascontiguousarray(WR, np.float64)
        normal = np.ascontiguousarray(normal, np.float64)
        n = WL.shape[0]
        half = np.zeros_like(WL)
        flux = np.zeros_like(WL)
        code = np.zeros(n, np.int32)
        L.check(L.lib().sfx_riemann_eval(self.h, n, L.dptr(WL), L.dptr(WR), L.dptr(normal),
                                         int(reflective), L.dptr(half), L.dptr(flux),
                                         L.iptr(code)), "sfx_riemann_eval")
        return half, flux, code


class FluxPass:
    """A mesh resident on the device with its hydro state."""

    def __init__(self, ctx: Context, mesh: Mesh):
        if mesh.dim != ctx.dim:
            raise ValueError("mesh dimension does not match the context")
        self.ctx = ctx
        self.mesh = mesh
        h = C.c_void_p()
        d = mesh.desc()
        L.check(L.lib().sfx_mesh_upload(ctx.h, C.byref(d), C.byref(h)), "sfx_mesh_upload")
        self.h = h
        self.S = mesh.dim + 2

    def clone(self, ctx: Context | None = None) -> "FluxPass":
        """a new state on this mesh's device geometry (sfx_mesh_clone): the
        clone owns only W, Q and per-step scratch; this FluxPass must outlive
        it"""
        ctx = ctx or self.ctx
        h = C.c_void_p()
        L.check(L.lib().sfx_mesh_clone(ctx.h, self.h, C.byref(h)), "sfx_mesh_clone")
        fp = FluxPass.__new__(FluxPass)
        fp.ctx, fp.mesh, fp.h, fp.S = ctx, self.mesh, h, self.S
        fp.base = self
        return fp

    def clone_bytes(self, precision: int) -> int:
        return int(L.lib().sfx_mesh_clone_bytes(self.h, precision))

    def close(self):
        if self.h:
            L.lib().sfx_mesh_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_primitive(self, W: np.ndarray):
        """W per cell; Q = get_Q(V, W) on the device (Simulation::initialize)."""
        W = np.ascontiguousarray(W, np.float64)
        assert W.shape == (self.mesh.n_cells, self.S)
        L.check(L.lib().sfx_state_upload_W(self.h, L.dptr(W)), "sfx_state_upload_W")

    def set_state(self, W: np.ndarray, Q: np.ndarray):
        W = np.ascontiguousarray(W, np.float64)
        Q = np.ascontiguousarray(Q, np.float64)
        L.check(L.lib().sfx_state_upload_WQ(self.h, L.dptr(W), L.dptr(Q)), "sfx_state_upload_WQ")

    def state(self) -> tuple[np.ndarray, np.ndarray]:
        W = np.empty((self.mesh.n_cells, self.S))
        Q = np.empty((self.mesh.n_cells, self.S))
        L.check(L.lib().sfx_state_download(self.h, L.dptr(W), L.dptr(Q)), "sfx_state_download")
        return W, Q

    def step(self, dt: float, nsteps: int = 1, stats: bool = True) -> L.sfx_stats | None:
        st = L.sfx_stats() if stats else None
        rc = L.lib().sfx_step(self.h, dt, nsteps, C.byref(st) if stats else None)
        if rc:
            idx = None
            if st is not None:
                idx = st.bad_face if st.bad_face >= 0 else st.bad_cell
            raise L.SfxError(rc, "sfx_step", idx)
        return st

    def set_lanes(self, lanes: int):
        L.check(L.lib().sfx_mesh_set_lanes(self.h, lanes), "sfx_mesh_set_lanes")

    # ---- local (hierarchical) time steps, plain FP64 ----
    def set_timesteps(self, start, end) -> None:
        """each cell's step [start, end) in ticks of the 2^60-tick timeline"""
        s = np.ascontiguousarray(start, np.uint64)
        e = np.ascontiguousarray(end, np.uint64)
        L.check(L.lib().sfx_mesh_set_timesteps(self.h, s.ctypes.data_as(L._u64p),
                                               e.ctypes.data_as(L._u64p)),
                "sfx_mesh_set_timesteps")

    def timesteps(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.mesh.n_cells
        s, e = np.empty(n, np.uint64), np.empty(n, np.uint64)
        L.check(L.lib().sfx_mesh_get_timesteps(self.h, s.ctypes.data_as(L._u64p),
                                               e.ctypes.data_as(L._u64p)),
                "sfx_mesh_get_timesteps")
        return s, e

    def set_gradients(self, grad) -> None:
        g = np.ascontiguousarray(grad, np.float64)
        L.check(L.lib().sfx_mesh_set_gradients(self.h, L.dptr(g)), "sfx_mesh_set_gradients")

    def gradients(self) -> np.ndarray:
        g = np.empty((self.mesh.n_cells, self.mesh.dim, self.S))
        L.check(L.lib().sfx_mesh_get_gradients(self.h, L.dptr(g)), "sfx_mesh_get_gradients")
        return g

    def step_window(self, t_total: float, t_now: int, t_next: int, periodic: bool):
        """one system step [t_now, t_next) of local time steps (sfx_step_window)"""
        st = L.sfx_stats()
        rc = L.lib().sfx_step_window(self.h, t_total, int(t_now), int(t_next), int(periodic),
                                     C.byref(st))
        if rc:
            raise L.SfxError(rc, "sfx_step_window",
                             st.bad_face if st.bad_face >= 0 else st.bad_cell)
        return st

    def timestep_bins(self, t_total: float, cfl: float, max_step: int, min_step: int,
                      t_next: int) -> int:
        """new steps for the cells ending at t_next; returns the next system step"""
        out = C.c_uint64(0)
        L.check(L.lib().sfx_timestep_bins(self.h, t_total, cfl, int(max_step), int(min_step),
                                          int(t_next), C.byref(out)), "sfx_timestep_bins")
        return int(out.value)

    def run_local(self, t_total: float, n_system_steps: int, cfl: float = 0.4,
                  max_step: int = 1 << 60, min_step: int = 0, periodic: bool = True,
                  t0: int = 0) -> int:
        """n_system_steps of local time stepping from tick t0 (0: every cell
        starts a step there), each followed by the new steps of the cells it
        ends (the reference's main loop for a static mesh); returns the tick
        reached.  One 8-byte read per system step for the next system step."""
        t = int(t0)
        dsys = self.timestep_bins(t_total, cfl, max_step, min_step, t)
        for _ in range(n_system_steps):
            t_next = t + dsys
            self.step_window(t_total, t, t_next, periodic)
            dsys = self.timestep_bins(t_total, cfl, max_step, min_step, t_next)
            t = t_next
        return t

    def step_moving(self, dt: float, periodic: bool) -> np.ndarray:
        """one step of a moving mesh (sfx_step_moving): generator velocities
        from the state, face velocities, the step in each face's frame, the
        drift; returns the drifted generator positions [n, dim] (the next
        tessellation's input)"""
        pos = np.empty((self.mesh.n_cells, self.mesh.dim))
        st = L.sfx_stats()
        rc = L.lib().sfx_step_moving(self.h, dt, int(periodic), L.dptr(pos), C.byref(st))
        if rc:
            raise L.SfxError(rc, "sfx_step_moving",
                             st.bad_face if st.bad_face >= 0 else st.bad_cell)
        return pos

    def set_face_variant(self, variant: int):
        """split pass: face-kernel variant (SFX_FACE_VARIANTS: 0 and 1 the
        64- and 80-register kernels; 2 and 3 the exact solver's gamma = 5/3
        forms, HLLC's stored dW/dt; include/sfxflux.h)"""
        L.check(L.lib().sfx_mesh_set_face_variant(self.h, variant), "sfx_mesh_set_face_variant")

    def tune_faces(self, dt: float, reps: int = 3) -> int:
        """split pass: time the face-kernel variants on this mesh and keep the
        fastest (advances the state by FACE_VARIANTS * (reps + 1) steps: call
        before loading the initial state); returns it"""
        best, best_ms = 0, 1e30
        for v in range(L.FACE_VARIANTS):
            self.set_face_variant(v)
            self.step_timed(dt, 1)
            ms, _ = self.step_timed(dt, reps)
            if ms[1] < best_ms:
                best, best_ms = v, ms[1]
        self.set_face_variant(best)
        return best

    def set_ranges(self, grad_cells: int, flux_faces: int, update_cells: int):
        """one part of a mesh split over several devices (plain FP64 or
        split): gradients of cells [0, grad_cells), fluxes of faces
        [0, flux_faces), update of cells [0, update_cells)
        (sfx_mesh_set_ranges)"""
        L.check(L.lib().sfx_mesh_set_ranges(self.h, grad_cells, flux_faces, update_cells),
                "sfx_mesh_set_ranges")

    def pack_cells(self, idx, out) -> None:
        """records [count, S + 1] (W, then the mass) of local cells idx into
        the device buffer out; idx an int32 and out a float64 device tensor"""
        L.check(L.lib().sfx_mesh_pack_cells(self.h, C.c_void_p(idx.data_ptr()), int(idx.numel()),
                                            C.c_void_p(out.data_ptr()), None),
                "sfx_mesh_pack_cells")

    def unpack_cells(self, idx, inp) -> None:
        """store records [count, S + 1] from the device buffer inp into the
        local cells idx"""
        L.check(L.lib().sfx_mesh_unpack_cells(self.h, C.c_void_p(idx.data_ptr()),
                                              int(idx.numel()), C.c_void_p(inp.data_ptr()), None),
                "sfx_mesh_unpack_cells")

    def tune(self, dt: float, reps: int = 3) -> int:
        """split pass: time the lanes-per-cell variants on this mesh's own
        gradient+update kernels and keep the fastest (advances the state by
        5 * (reps + 1) steps: call before loading the initial state)"""
        best, best_ms = 4, 1e30
        for lanes in (1, 2, 4, 8, 16):
            self.set_lanes(lanes)
            self.step_timed(dt, 1)
            ms, _ = self.step_timed(dt, reps)
            t = ms[0] + ms[2]
            if t < best_ms:
                best, best_ms = lanes, t
        self.set_lanes(best)
        return best

    def step_timed(self, dt: float, nsteps: int) -> tuple[np.ndarray, int]:
        """nsteps with per-kernel device times: (ms[gradients, faces, update],
        launches)"""
        ms = (C.c_float * 3)()
        nl = C.c_int32(0)
        L.check(L.lib().sfx_step_timed(self.h, dt, nsteps, ms, C.byref(nl)), "sfx_step_timed")
        return np.array(list(ms), dtype=np.float64), nl.value

    def flux_pass(self, dt: float):
        """gradients [n, dim, S], per-face dQ of the left cell [F, S], branch
        codes [F] of one pass without updating the state."""
        n, F, D, S = self.mesh.n_cells, self.mesh.n_faces, self.mesh.dim, self.S
        grad = np.empty((n, D, S))
        dQ = np.empty((F, S))
        br = np.empty(F, np.int32)
        st = L.sfx_stats()
        rc = L.lib().sfx_flux_pass(self.h, dt, L.dptr(grad), L.dptr(dQ), L.iptr(br), C.byref(st))
        return grad, dQ, br, rc, (st.bad_face if st.bad_face >= 0 else st.bad_cell)

    def totals(self) -> np.ndarray:
        out = np.zeros(5)
        L.check(L.lib().sfx_mesh_totals(self.h, L.dptr(out)), "sfx_mesh_totals")
        return out[: self.S]


class Group:
    """Many meshes of one split-precision context advanced together: one
    launch per phase for all members (sfx_group_*)."""

    def __init__(self, ctx: Context, members: list[FluxPass], dts):
        self.ctx = ctx
        self.members = list(members)
        n = len(self.members)
        arr = (C.c_void_p * n)(*[m.h.value for m in self.members])
        dt = np.ascontiguousarray(dts, np.float64)
        h = C.c_void_p()
        L.check(L.lib().sfx_group_create(ctx.h, n, arr, L.dptr(dt), C.byref(h)),
                "sfx_group_create")
        self.h = h

    def close(self):
        if self.h:
            L.lib().sfx_group_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_dt(self, dts):
        dt = np.ascontiguousarray(dts, np.float64)
        L.check(L.lib().sfx_group_set_dt(self.h, L.dptr(dt)), "sfx_group_set_dt")

    def tune(self, reps: int = 3) -> int:
        lanes = C.c_int32(0)
        L.check(L.lib().sfx_group_tune(self.h, reps, C.byref(lanes)), "sfx_group_tune")
        return lanes.value

    def set_lanes(self, lanes: int):
        L.check(L.lib().sfx_group_set_lanes(self.h, lanes), "sfx_group_set_lanes")

    def tune_faces(self, reps: int = 3) -> int:
        """time the face-kernel variants on this group's meshes (a gradient
        launch before each timed face launch; no state changes) and keep the
        fastest; returns it"""
        v = C.c_int32(0)
        L.check(L.lib().sfx_group_tune_faces(self.h, reps, C.byref(v)), "sfx_group_tune_faces")
        return v.value

    def set_face_variant(self, variant: int):
        L.check(L.lib().sfx_group_set_face_variant(self.h, variant),
                "sfx_group_set_face_variant")

    def set_steps(self, steps):
        """per-member remaining step counts on the device: a member at 0 is
        skipped, the others count down each step"""
        st = np.ascontiguousarray(steps, np.int32)
        L.check(L.lib().sfx_group_set_steps(self.h, L.iptr(st)), "sfx_group_set_steps")

    def get_steps(self) -> np.ndarray:
        st = np.zeros(len(self.members), np.int32)
        L.check(L.lib().sfx_group_get_steps(self.h, L.iptr(st)), "sfx_group_get_steps")
        return st

    def status(self) -> np.ndarray:
        st = np.zeros(len(self.members), np.int32)
        L.lib().sfx_group_status(self.h, L.iptr(st))
        return st

    def step_timed(self, nsteps: int) -> tuple[np.ndarray, int]:
        """nsteps without a graph; (ms[gradients, faces, update] summed over
        the steps, kernels launched)"""
        ms = (C.c_float * 3)()
        nl = C.c_int32(0)
        L.check(L.lib().sfx_group_step_timed(self.h, nsteps, ms, C.byref(nl)),
                "sfx_group_step_timed")
        return np.array(list(ms), dtype=np.float64), nl.value

    def step(self, nsteps: int = 1, graph: bool = True, status: bool = True):
        """nsteps for every member; returns the per-member status array"""
        st = np.zeros(len(self.members), np.int32) if status else None
        rc = L.lib().sfx_group_step(self.h, nsteps, int(graph), L.iptr(st) if status else None)
        if rc and not status:
            raise L.SfxError(rc, "sfx_group_step")
        if rc and st is not None and not np.any(st):
            raise L.SfxError(rc, "sfx_group_step")
        return st
