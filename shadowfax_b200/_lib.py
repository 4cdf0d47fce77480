"""ctypes binding of the sfxflux C ABI (include/sfxflux.h).

The library is the in-tree ``shadowfax_b200/libsfxflux.so``; it is built by
``shadowfax_b200.build`` (``__graft_entry__.build()``).  There is no Python or
CPU fallback for the flux pass: if the library is missing, loading fails
loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libsfxflux.so"

SFX_OK = 0
STATUS_NAMES = {
    0: "SFX_OK", 1: "SFX_ERR_INVALID", 2: "SFX_ERR_CUDA", 3: "SFX_ERR_RIEMANN",
    4: "SFX_ERR_NAN_FLUX", 5: "SFX_ERR_NEG_STATE", 6: "SFX_ERR_NOCONV",
    7: "SFX_ERR_BOUNDS", 8: "SFX_ERR_UNSUPPORTED", 9: "SFX_ERR_MESH",
    10: "SFX_ERR_NOMEM", 11: "SFX_ERR_NOT_READY", 12: "SFX_ERR_CLOSED",
    13: "SFX_ERR_TOO_LARGE", 14: "SFX_ERR_IO", 15: "SFX_ERR_TIMESTEP",
}
SFX_ERR_INVALID, SFX_ERR_CUDA, SFX_ERR_RIEMANN, SFX_ERR_NAN_FLUX = 1, 2, 3, 4
SFX_ERR_NEG_STATE, SFX_ERR_NOCONV, SFX_ERR_BOUNDS, SFX_ERR_UNSUPPORTED = 5, 6, 7, 8
SFX_ERR_MESH, SFX_ERR_NOMEM, SFX_ERR_NOT_READY, SFX_ERR_CLOSED = 9, 10, 11, 12
SFX_ERR_TOO_LARGE, SFX_ERR_IO, SFX_ERR_TIMESTEP = 13, 14, 15

SOLVER_EXACT, SOLVER_HLLC = 0, 1
PREC_FP64, PREC_SPLIT = 0, 1
FACE_VARIANTS = 5  # SFX_FACE_VARIANTS
FACE_REAL, FACE_PERIODIC, FACE_MIRROR = 0, 1, 2


class SfxError(RuntimeError):
    """A non-zero status returned by the library."""

    def __init__(self, status: int, what: str = "", index: int | None = None):
        self.status = status
        self.index = index
        name = STATUS_NAMES.get(status, str(status))
        msg = f"{what}: {name}" if what else name
        if index is not None and index >= 0:
            msg += f" (index {index})"
        super().__init__(msg)


class sfx_config(C.Structure):
    _fields_ = [("dim", C.c_int32), ("solver", C.c_int32), ("gamma", C.c_double),
                ("tolerance", C.c_double), ("cutoff", C.c_double),
                ("precision", C.c_int32), ("device", C.c_int32)]


_dp = C.POINTER(C.c_double)
_u64p = C.POINTER(C.c_uint64)
_ip = C.POINTER(C.c_int32)


class sfx_mesh_desc(C.Structure):
    _fields_ = [("dim", C.c_int32), ("n_cells", C.c_int32), ("n_faces", C.c_int32),
                ("cell_pos", _dp), ("cell_centroid", _dp), ("cell_volume", _dp),
                ("cell_total_area", _dp), ("cell_face_offset", _ip),
                ("cell_face_index", _ip), ("face_area", _dp), ("face_midpoint", _dp),
                ("face_left", _ip), ("face_right", _ip), ("face_kind", _ip),
                ("face_right_pos", _dp), ("face_velocity", _dp)]


class sfx_device_mesh(C.Structure):
    """device-pointer face list of sfx_flux_pass_noalloc (field-major)"""
    _fields_ = [("dim", C.c_int32), ("n_cells", C.c_int32), ("n_faces", C.c_int32),
                ("cell_pos", C.c_void_p), ("cell_centroid", C.c_void_p),
                ("cell_volume", C.c_void_p), ("cell_total_area", C.c_void_p),
                ("cell_face_offset", C.c_void_p), ("cell_face_entry", C.c_void_p),
                ("face_area", C.c_void_p), ("face_midpoint", C.c_void_p),
                ("face_left", C.c_void_p), ("face_right", C.c_void_p),
                ("face_kind", C.c_void_p), ("face_right_pos", C.c_void_p)]


class sfx_server_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32), ("gamma", C.c_double),
                ("tolerance", C.c_double), ("cutoff", C.c_double),
                ("memory_budget", C.c_int64), ("max_active", C.c_int32),
                ("chunk_steps", C.c_int32)]


class sfx_request_info(C.Structure):
    _fields_ = [("status", C.c_int32), ("steps_done", C.c_int32), ("mesh_id", C.c_int32),
                ("solver", C.c_int32), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("face_steps", C.c_int64)]


class sfx_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("failed", C.c_int64), ("active", C.c_int64), ("queued", C.c_int64),
                ("face_steps", C.c_int64), ("bytes_in_use", C.c_int64), ("rounds", C.c_int64),
                ("now", C.c_double), ("worker_s", C.c_double * 4)]


class sfx_stats(C.Structure):
    _fields_ = [("status", C.c_int32), ("bad_face", C.c_int32), ("bad_cell", C.c_int32),
                ("steps_done", C.c_int32), ("totals", C.c_double * 5)]


_lib = None

# name -> (restype, argtypes); every exported symbol of include/sfxflux.h
PROTOTYPES = {
    "sfx_version": (C.c_char_p, []),
    "sfx_launch_count": (C.c_int64, []),
    "sfx_ctx_create": (C.c_int, [C.POINTER(sfx_config), C.POINTER(C.c_void_p)]),
    "sfx_ctx_destroy": (C.c_int, [C.c_void_p]),
    "sfx_ctx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sfx_ctx_synchronize": (C.c_int, [C.c_void_p]),
    "sfx_mesh_upload": (C.c_int, [C.c_void_p, C.POINTER(sfx_mesh_desc), C.POINTER(C.c_void_p)]),
    "sfx_mesh_check": (C.c_int, [C.POINTER(sfx_mesh_desc), C.c_int32]),
    "sfx_mesh_free": (C.c_int, [C.c_void_p]),
    "sfx_mesh_device_bytes": (C.c_int64, [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_int32]),
    "sfx_state_upload_W": (C.c_int, [C.c_void_p, _dp]),
    "sfx_state_upload_WQ": (C.c_int, [C.c_void_p, _dp, _dp]),
    "sfx_state_download": (C.c_int, [C.c_void_p, _dp, _dp]),
    "sfx_step": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.POINTER(sfx_stats)]),
    "sfx_step_timed": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.POINTER(C.c_float),
                                 C.POINTER(C.c_int32)]),
    "sfx_flux_pass": (C.c_int, [C.c_void_p, C.c_double, _dp, _dp, _ip, C.POINTER(sfx_stats)]),
    "sfx_riemann_eval": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp, _dp, C.c_int32, _dp, _dp, _ip]),
    "sfx_mesh_totals": (C.c_int, [C.c_void_p, _dp]),
    "sfx_voronoi_build": (C.c_int, [C.c_int, C.c_int64, _dp, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "sfx_voronoi_counts": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int64)]),
    "sfx_voronoi_export": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _ip, _ip, _dp, _dp, _ip, _ip,
                                     _ip, _dp]),
    "sfx_voronoi_free": (None, [C.c_void_p]),
    "sfx_meshfile_write": (C.c_int, [C.c_char_p, C.POINTER(sfx_mesh_desc), C.c_int32]),
    "sfx_meshfile_info": (C.c_int, [C.c_char_p, _ip, _ip, C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int64), _ip]),
    "sfx_meshfile_read": (C.c_int, [C.c_char_p, _dp, _dp, _dp, _dp, _ip, _ip, _dp, _dp, _ip,
                                    _ip, _ip, _dp, _dp]),
    "sfx_mesh_set_lanes": (C.c_int, [C.c_void_p, C.c_int32]),
    "sfx_mesh_set_face_variant": (C.c_int, [C.c_void_p, C.c_int32]),
    "sfx_step_moving": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, _dp, C.c_void_p]),
    "sfx_mesh_set_timesteps": (C.c_int, [C.c_void_p, _u64p, _u64p]),
    "sfx_mesh_get_timesteps": (C.c_int, [C.c_void_p, _u64p, _u64p]),
    "sfx_mesh_set_gradients": (C.c_int, [C.c_void_p, _dp]),
    "sfx_mesh_get_gradients": (C.c_int, [C.c_void_p, _dp]),
    "sfx_step_window": (C.c_int, [C.c_void_p, C.c_double, C.c_uint64, C.c_uint64, C.c_int32,
                                  C.c_void_p]),
    "sfx_timestep_bins": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_uint64, C.c_uint64,
                                    C.c_uint64, C.POINTER(C.c_uint64)]),
    "sfx_mesh_set_ranges": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    "sfx_mesh_pack_cells": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                      C.c_void_p]),
    "sfx_mesh_unpack_cells": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                        C.c_void_p]),
    "sfx_mesh_clone": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "sfx_mesh_clone_bytes": (C.c_int64, [C.c_void_p, C.c_int32]),
    "sfx_group_set_steps": (C.c_int, [C.c_void_p, _ip]),
    "sfx_group_get_steps": (C.c_int, [C.c_void_p, _ip]),
    "sfx_group_status": (C.c_int, [C.c_void_p, _ip]),
    "sfx_group_step_timed": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_float),
                                       C.POINTER(C.c_int32)]),
    "sfx_server_create": (C.c_int, [C.POINTER(sfx_server_config), C.POINTER(C.c_void_p)]),
    "sfx_server_add_mesh": (C.c_int, [C.c_void_p, C.POINTER(sfx_mesh_desc), _ip]),
    "sfx_server_set_tuning": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                        C.c_int32]),
    "sfx_server_submit": (C.c_int, [C.c_void_p, C.c_int32, _dp, C.c_int32, C.c_double,
                                    C.c_int32, C.POINTER(C.c_int64)]),
    "sfx_server_poll": (C.c_int, [C.c_void_p, C.c_int64, _dp, _dp,
                                  C.POINTER(sfx_request_info)]),
    "sfx_server_drain": (C.c_int, [C.c_void_p, C.c_double]),
    "sfx_server_stats_get": (C.c_int, [C.c_void_p, C.POINTER(sfx_server_stats)]),
    "sfx_server_shutdown": (C.c_int, [C.c_void_p]),
    "sfx_group_create": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), _dp,
                                   C.POINTER(C.c_void_p)]),
    "sfx_group_set_dt": (C.c_int, [C.c_void_p, _dp]),
    "sfx_group_step": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, _ip]),
    "sfx_group_tune": (C.c_int, [C.c_void_p, C.c_int32, _ip]),
    "sfx_group_set_lanes": (C.c_int, [C.c_void_p, C.c_int32]),
    "sfx_group_tune_faces": (C.c_int, [C.c_void_p, C.c_int32, _ip]),
    "sfx_group_set_face_variant": (C.c_int, [C.c_void_p, C.c_int32]),
    "sfx_group_free": (C.c_int, [C.c_void_p]),
    "sfx_flux_pass_noalloc": (C.c_int, [C.POINTER(sfx_device_mesh), C.POINTER(sfx_config),
                                        C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
}


def lib() -> C.CDLL:
    """Load (once) and return the library; raise if it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m shadowfax_b200.build` "
                "(the flux pass has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, what: str = "", index: int | None = None) -> None:
    if status != SFX_OK:
        raise SfxError(status, what, index)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_ip)
