"""The C-ABI library builds in-tree, loads without a GPU and exports every
entry point include/sfxflux.h declares (no compute calls here)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    src = (ROOT / "include" / "sfxflux.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sfx_[A-Za-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from shadowfax_b200 import _lib
    lib = _lib.lib()
    syms = declared_symbols()
    assert len(syms) >= 19
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and the binding declares a prototype for each of them
    assert set(syms) <= set(_lib.PROTOTYPES), set(syms) - set(_lib.PROTOTYPES)


def test_version_string():
    from shadowfax_b200 import _lib
    assert b"sfxflux" in _lib.lib().sfx_version()


def test_ctx_rejects_unsupported_solver_without_touching_the_gpu():
    from shadowfax_b200 import _lib as L
    cfg = L.sfx_config(2, 7, 5 / 3, 1e-8, -5.0, 0, 0)
    h = ctypes.c_void_p()
    assert L.lib().sfx_ctx_create(ctypes.byref(cfg), ctypes.byref(h)) == L.SFX_ERR_UNSUPPORTED
    cfg = L.sfx_config(4, 0, 5 / 3, 1e-8, -5.0, 0, 0)
    assert L.lib().sfx_ctx_create(ctypes.byref(cfg), ctypes.byref(h)) == L.SFX_ERR_INVALID


def test_branch_code_layout_matches_oracle():
    """include/sfxflux.h and oracle/sfx_oracle.c use the same bit layout"""
    h = (ROOT / "include" / "sfxflux.h").read_text()
    o = (ROOT / "oracle" / "sfx_oracle.c").read_text()
    pairs = {"S_RSHOCK_STAR": "S_RSHOCK_STAR", "S_LFAN": "S_LFAN", "S_VAC": "S_VAC",
             "HLLC": "HLLC", "LIMIT_L": "LIMIT_L", "SKIPPED": "SKIPPED"}
    for a, b in pairs.items():
        va = re.search(rf"#define SFX_BRANCH_{a} (.+)", h).group(1).strip()
        vb = re.search(rf"#define SFXB_{b} (.+)", o).group(1).strip()
        assert eval(va) == eval(vb), (a, va, vb)


def test_server_rejects_bad_config():
    """argument checks run before any device work"""
    import ctypes as C
    from shadowfax_b200 import _lib as L
    for kw in ({"precision": 7}, {"max_active": 0}, {"memory_budget": 0}, {"chunk_steps": 0}):
        base = dict(device=0, precision=1, gamma=5 / 3, tolerance=1e-8, cutoff=-5.0,
                    memory_budget=1 << 30, max_active=16, chunk_steps=4)
        base.update(kw)
        cfg = L.sfx_server_config(**base)
        h = C.c_void_p()
        assert L.lib().sfx_server_create(C.byref(cfg), C.byref(h)) == L.SFX_ERR_INVALID
        assert not h.value
    assert L.lib().sfx_server_poll(None, 1, None, None, None) == L.SFX_ERR_INVALID
    assert L.lib().sfx_server_shutdown(None) == L.SFX_ERR_INVALID


def test_variant_counts_match_the_header():
    """the Python constants that drive the tuners match include/sfxflux.h"""
    from shadowfax_b200 import _lib as L
    h = (ROOT / "include" / "sfxflux.h").read_text()
    assert int(re.search(r"#define SFX_FACE_VARIANTS (\d+)", h).group(1)) == L.FACE_VARIANTS


def test_server_tuning_rejects_bad_arguments_without_a_server():
    from shadowfax_b200 import _lib as L
    assert L.lib().sfx_server_set_tuning(None, 2, 0, 0, 0) == L.SFX_ERR_INVALID


# entry points whose first argument is an object handle: a NULL handle is
# refused before any device call (sfx_mesh_clone_bytes answers -1)
NULL_HANDLE_ENTRY_POINTS = [
    "sfx_ctx_destroy", "sfx_ctx_set_stream", "sfx_ctx_synchronize", "sfx_mesh_upload",
    "sfx_mesh_free", "sfx_state_download", "sfx_step", "sfx_step_moving",
    "sfx_mesh_set_timesteps", "sfx_mesh_get_timesteps", "sfx_mesh_set_gradients",
    "sfx_mesh_get_gradients", "sfx_step_window", "sfx_timestep_bins", "sfx_step_timed",
    "sfx_flux_pass", "sfx_riemann_eval", "sfx_mesh_clone", "sfx_mesh_clone_bytes",
    "sfx_mesh_set_lanes", "sfx_mesh_set_face_variant", "sfx_mesh_set_ranges",
    "sfx_mesh_pack_cells", "sfx_mesh_unpack_cells", "sfx_mesh_totals",
    "sfx_group_create", "sfx_group_set_dt", "sfx_group_set_face_variant", "sfx_group_set_lanes",
    "sfx_group_step", "sfx_group_step_timed", "sfx_group_status", "sfx_group_tune",
    "sfx_group_tune_faces", "sfx_group_set_steps", "sfx_group_get_steps", "sfx_group_free",
    "sfx_server_add_mesh", "sfx_server_submit", "sfx_server_poll", "sfx_server_drain",
    "sfx_server_stats_get", "sfx_server_shutdown", "sfx_server_set_tuning",
]


def _plausible(argtype):
    """a value of the argument's type that is valid on its own"""
    if argtype in (ctypes.c_double, ctypes.c_float):
        return 1.0
    if argtype in (ctypes.c_int, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32,
                   ctypes.c_uint64):
        return 1
    return None  # pointers and handles


@pytest.mark.parametrize("name", NULL_HANDLE_ENTRY_POINTS)
def test_null_handles_are_refused_without_a_gpu(name):
    from shadowfax_b200 import _lib as L
    res, argtypes = L.PROTOTYPES[name]
    fn = getattr(L.lib(), name)
    rc = fn(*[_plausible(a) for a in argtypes])
    assert rc == (-1 if name == "sfx_mesh_clone_bytes" else L.SFX_ERR_INVALID), rc


def test_noalloc_pass_checks_its_arguments_before_any_device_call():
    """sfx_flux_pass_noalloc refuses a bad call before it asks the runtime for
    a device: these cases never reach the (here absent) GPU, and the host
    arrays standing in for device pointers are never read"""
    from shadowfax_b200 import _lib as L
    buf = ctypes.create_string_buffer(64)
    p = ctypes.cast(buf, ctypes.c_void_p)

    def mesh(**kw):
        d = dict(dim=2, n_cells=100, n_faces=300)
        d.update(kw)
        m = L.sfx_device_mesh(d["dim"], d["n_cells"], d["n_faces"], *([p] * 12))
        return m

    def call(m, cfg, dt=1e-4, W=p):
        return L.lib().sfx_flux_pass_noalloc(ctypes.byref(m), ctypes.byref(cfg), dt, W, p, p, None)

    limit = int(re.search(r"#define SFX_NOALLOC_MAX_CELLS (\d+)",
                          (ROOT / "include" / "sfxflux.h").read_text()).group(1))
    cfg = L.sfx_config(2, 0, 5 / 3, 1e-8, -5.0, 0, 0)
    assert call(mesh(n_cells=limit + 1), cfg) == L.SFX_ERR_TOO_LARGE
    assert call(mesh(dim=4), cfg) == L.SFX_ERR_INVALID
    assert call(mesh(), L.sfx_config(3, 0, 5 / 3, 1e-8, -5.0, 0, 0)) == L.SFX_ERR_INVALID
    assert call(mesh(), L.sfx_config(2, 7, 5 / 3, 1e-8, -5.0, 0, 0)) == L.SFX_ERR_UNSUPPORTED
    assert call(mesh(), L.sfx_config(2, 0, 1.0, 1e-8, -5.0, 0, 0)) == L.SFX_ERR_INVALID
    assert call(mesh(), cfg, dt=0.0) == L.SFX_ERR_INVALID
    assert call(mesh(), cfg, W=None) == L.SFX_ERR_INVALID
    assert call(mesh(n_cells=0), cfg) == L.SFX_ERR_INVALID


C_HOST = r"""
#include <stdio.h>
#include <string.h>
#include "sfxflux.h"

int main(void) {
    double pos[2] = {0.5, 0.5}, cen[2] = {0.5, 0.5}, vol = 1.0, tarea = 4.0;
    int32_t off[2] = {0, 0}, idx[1] = {0};
    sfx_mesh_desc d;
    memset(&d, 0, sizeof d);
    d.dim = 2;
    d.n_cells = 1;
    d.n_faces = 0;
    d.cell_pos = pos;
    d.cell_centroid = cen;
    d.cell_volume = &vol;
    d.cell_total_area = &tarea;
    d.cell_face_offset = off;
    d.cell_face_index = idx;
    int ok = sfx_mesh_check(&d, SFX_PREC_FP64);
    d.cell_face_offset = NULL;
    int bad = sfx_mesh_check(&d, SFX_PREC_FP64);
    printf("%s|%d|%d\n", sfx_version(), ok, bad);
    return !(ok == SFX_OK && bad == SFX_ERR_INVALID);
}
"""


def test_a_c_host_links_and_calls_the_library(tmp_path):
    """the boundary as a C or cgo host sees it: the header compiles as strict
    C99 and C++11, and a C program linked against the shared library calls
    it (host-only entry points: no GPU here)"""
    import shutil
    import subprocess
    from shadowfax_b200 import _lib as L
    if shutil.which("gcc") is None or shutil.which("g++") is None:
        pytest.skip("no C compiler")
    L.lib()   # the library is built
    inc, libdir = ROOT / "include", ROOT / "shadowfax_b200"
    src = tmp_path / "host.c"
    src.write_text(C_HOST)
    exe = tmp_path / "host"
    cmd = ["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", f"-I{inc}", str(src),
           f"-L{libdir}", "-lsfxflux", f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    cpp = tmp_path / "host.cpp"
    cpp.write_text('#include "sfxflux.h"\nint main() { return sizeof(sfx_mesh_desc) == 0; }\n')
    subprocess.run(["g++", "-std=c++11", "-Wall", "-Werror", "-pedantic", f"-I{inc}", "-c",
                    str(cpp), "-o", str(tmp_path / "host_cpp.o")], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    version, ok, bad = r.stdout.strip().split("|")
    assert version.startswith("sfxflux") and int(ok) == 0 and int(bad) == L.SFX_ERR_INVALID
