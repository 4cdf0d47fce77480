"""Build the in-tree sfxflux shared library for sm_100a.

``python -m shadowfax_b200.build`` (or ``build_library()``) compiles

* ``csrc/sfx_fp64.cu``   plain-FP64 kernels, ``-fmad=false`` (bit parity)
* ``csrc/sfx_split.cu``  FP32/FP64-split and batched kernels (FMA allowed, FP32
  division and square root approximate)
* ``csrc/sfx_api.cu``    C ABI (include/sfxflux.h)
* ``csrc/sfx_voronoi.cpp`` host face-list builder
* ``csrc/sfx_meshfile.cpp`` versioned binary mesh files

with ``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo`` into
``shadowfax_b200/libsfxflux.so``, and the host-only mesh-file generator
``shadowfax_b200/sfx_meshgen`` (``csrc/sfx_meshgen.cpp`` with the builder and
mesh-file sources, g++ only).  nvcc cross-compiles, so this runs on a
machine without a GPU.  A source newer than a target triggers its rebuild.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libsfxflux.so"
MESHGEN = PKG / "sfx_meshgen"
MESHGEN_SRC = ["sfx_meshgen.cpp", "sfx_voronoi.cpp", "sfx_meshfile.cpp"]
OBJ = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

COMMON = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I", str(PKG.parent / "include")]

# per-source extra flags
UNITS = {
    "sfx_fp64.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"],
    # FP32 division and square root by the hardware approximations (about
    # 2 ulp); FP64 operations stay IEEE
    "sfx_split.cu": ["-fmad=true", "-prec-div=false", "-prec-sqrt=false"],
    "sfx_api.cu": [],
    "sfx_noalloc.cu": [],
    "sfx_group.cu": [],
    "sfx_server.cu": [],
    "sfx_voronoi.cpp": [],
    "sfx_meshfile.cpp": [],
}


def _sources() -> list[Path]:
    return [CSRC / s for s in UNITS if (CSRC / s).exists()]


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list((PKG.parent / "include").glob("*.h"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _sources() + _headers() + [Path(__file__)])


def _compile(src: Path) -> Path:
    OBJ.mkdir(exist_ok=True)
    obj = OBJ / (src.name + ".o")
    cmd = [NVCC, *COMMON, *UNITS[src.name], "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-pthread",
               "-I", str(PKG.parent / "include"), "-c", str(src), "-o", str(obj)]
    subprocess.run(cmd, check=True)
    return obj


def build_meshgen(force: bool = False) -> Path:
    srcs = [CSRC / s for s in MESHGEN_SRC]
    deps = srcs + [PKG.parent / "include" / "sfxflux.h", Path(__file__)]
    if not force and MESHGEN.exists() and all(MESHGEN.stat().st_mtime >= d.stat().st_mtime
                                              for d in deps):
        return MESHGEN
    tmp = MESHGEN.with_suffix(".tmp")
    subprocess.run(["g++", "-std=c++17", "-O3", "-ffp-contract=off", "-pthread", "-I",
                    str(PKG.parent / "include"), *map(str, srcs), "-o", str(tmp)], check=True)
    os.replace(tmp, MESHGEN)
    return MESHGEN


def build_library(force: bool = False, verbose: bool = True) -> Path:
    build_meshgen(force)
    if not force and not needs_build():
        return LIB
    srcs = _sources()
    if verbose:
        print(f"[sfxflux] compiling {', '.join(s.name for s in srcs)} for sm_100a",
              file=sys.stderr)
    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(_compile, srcs))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
           "-Xcompiler", "-pthread"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv)
    print(LIB)
