"""Build the CPU checkers (TEST INFRASTRUCTURE ONLY).

* ``oracle/libsfxoracle.so`` - the C restatement of the flux pass
  (sfx_oracle.c), compiled with gcc from this directory.
* ``oracle/_ref/refharness_{2,3}d_{libm,sfxpow}`` - the reference Shadowfax
  flux-pass sources compiled UNMODIFIED from the reference tree
  (``$SFX_REFERENCE_SRC``; by default ``reference/src`` beside this
  repository's directory) together with
  oracle/refharness (single-rank MPI stand-in, version header, TimeLine
  constructor, driver).  Built only where the reference tree exists; the
  binaries then travel with the repository.  "libm" keeps glibc's pow,
  "sfxpow" routes pow() and cbrt() to sfx_pow and sfx_cbrt
  (refharness/pow_interpose.c).
* ``oracle/_ref/refharness_{2,3}d_moving_{libm,sfxpow}`` - the same sources
  built without -DSTATIC (moving generators: VorFace::set_v and the drift).
* ``oracle/_ref/tessharness_{2,3}d_{libm,sfxpow}`` - the reference's own
  tessellation (DelTess, VorTess, the exact predicates of ExArith with the
  fixed-width integer stand-in in refharness/shim/boost, the particle tree)
  and the same hot path, with oracle/refharness/tessharness.cpp: tessellate,
  export the face list, run the step loop on that tessellation.

Nothing here is linked into or called by the product library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_SRC = Path(os.environ.get("SFX_REFERENCE_SRC",
                              str(HERE.parent.parent / "reference" / "src")))
OUT = HERE / "_ref"
ORACLE_SO = HERE / "libsfxoracle.so"

# reference translation units of the hot path and the support code they link
REF_UNITS = [
    "riemann/RiemannSolver.cpp", "riemann/ExactRiemannSolver.cpp",
    "riemann/HLLCRiemannSolver.cpp", "VorFace.cpp", "VorCell.cpp", "VorGen.cpp",
    "utilities/GasParticle.cpp", "utilities/Particle.cpp", "utilities/Timer.cpp",
    "utilities/HelperFunctions.cpp", "utilities/Hilbert.cpp", "ColorMap.cpp", "MPIGlobal.cpp", "ProgramLog.cpp", "RestartFile.cpp",
]
# the reference's tessellation and what it links (the static build only)
TESS_UNITS = [
    "DelTess.cpp", "DelTess_mpi.cpp", "ExArith.cpp", "VorTess.cpp", "Simplex.cpp",
    "NgbSearch.cpp", "Line.cpp", "Plane.cpp", "RectangularBox.cpp", "utilities/Tree.cpp",
    "utilities/EwaldTable.cpp", "utilities/DMParticle.cpp", "utilities/StarParticle.cpp",
]
# the reference's release flags plus: no FMA contraction (matches x86-64 default
# code generation on every host), no builtin pow folding (so the sfxpow build
# can interpose pow), <array> pre-included (src/RestartFile.hpp uses std::array)
REF_FLAGS = ["-O2", "-ffp-contract=off", "-fno-builtin-pow", "-fno-builtin-cbrt", "-std=c++11",
             "-include", "array", "-w"]
# the two variants: static generators (the reference's -DSTATIC build) and
# moving ones
VARIANTS = {"": ["-DSTATIC"], "_moving": []}


def _newer(out: Path, deps: list[Path]) -> bool:
    return out.exists() and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps)


def build_oracle(force: bool = False) -> Path:
    deps = [HERE / "sfx_oracle.c", HERE / "sfx_oracle.h", HERE / "sfx_oracle_dim.h",
            HERE.parent / "shadowfax_b200" / "csrc" / "sfx_pow.h"]
    if not force and _newer(ORACLE_SO, deps):
        return ORACLE_SO
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-builtin", "-std=c99", "-shared",
                    "-fPIC", str(HERE / "sfx_oracle.c"), "-o", str(ORACLE_SO), "-lm"],
                   check=True)
    return ORACLE_SO


def ref_binary(dim: int, pow_kind: str, moving: bool = False) -> Path:
    return OUT / f"refharness_{dim}d{'_moving' if moving else ''}_{pow_kind}"


def tess_binary(dim: int, pow_kind: str) -> Path:
    return OUT / f"tessharness_{dim}d_{pow_kind}"


def build_reference(force: bool = False, jobs: int = 8) -> list[Path]:
    """Compile the reference harness binaries; returns [] if the reference
    tree is absent (the prebuilt binaries are used instead)."""
    if not (REF_SRC / "VorFace.cpp").exists():
        return []
    OUT.mkdir(exist_ok=True)
    obj = OUT / "obj"
    obj.mkdir(exist_ok=True)
    inc = ["-I", str(HERE / "refharness" / "shim"), "-I", str(HERE / "refharness"),
           "-I", str(REF_SRC), "-I", str(REF_SRC / "utilities")]
    harness = HERE / "refharness" / "harness.cpp"
    tessh = HERE / "refharness" / "tessharness.cpp"
    interpose = HERE / "refharness" / "pow_interpose.c"
    outs = [ref_binary(d, k, mv) for d in (2, 3) for k in ("libm", "sfxpow")
            for mv in (False, True)]
    outs += [tess_binary(d, k) for d in (2, 3) for k in ("libm", "sfxpow")]
    deps = [harness, tessh, interpose, HERE / "refharness" / "timeline_stub.hpp",
            HERE / "refharness" / "shim" / "mpi.h",
            HERE / "refharness" / "shim" / "boost" / "multiprecision" / "cpp_int.hpp",
            Path(__file__), HERE.parent / "shadowfax_b200" / "csrc" / "sfx_pow.h"]
    if not force and all(_newer(o, deps) for o in outs):
        return outs
    tasks = []
    for d in (2, 3):
        for var, vflags in VARIANTS.items():
            for u in REF_UNITS:
                o = obj / (u.replace("/", "_") + f".{d}d{var}.o")
                tasks.append(["g++", *REF_FLAGS, *vflags, f"-Dndim_={d}", *inc, "-c",
                              str(REF_SRC / u), "-o", str(o)])
            tasks.append(["g++", *REF_FLAGS, *vflags, f"-Dndim_={d}", *inc, "-c", str(harness),
                          "-o", str(obj / f"harness.{d}d{var}.o")])
        for u in TESS_UNITS:
            tasks.append(["g++", *REF_FLAGS, "-DSTATIC", f"-Dndim_={d}", *inc, "-c",
                          str(REF_SRC / u), "-o", str(obj / (u.replace("/", "_") + f".{d}d.o"))])
        tasks.append(["g++", *REF_FLAGS, "-DSTATIC", f"-Dndim_={d}", *inc, "-c", str(tessh),
                      "-o", str(obj / f"tessharness.{d}d.o")])
    tasks.append(["gcc", "-O2", "-ffp-contract=off", "-std=c99", "-c", str(interpose), "-o",
                  str(obj / "pow_interpose.o")])
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        for r in ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), tasks):
            if r.returncode:
                raise RuntimeError(f"reference build failed: {' '.join(r.args)}\n{r.stderr}")
    for d in (2, 3):
        for var in VARIANTS:
            objs = [str(obj / (u.replace("/", "_") + f".{d}d{var}.o")) for u in REF_UNITS]
            objs.append(str(obj / f"harness.{d}d{var}.o"))
            for k in ("libm", "sfxpow"):
                extra = [str(obj / "pow_interpose.o")] if k == "sfxpow" else []
                subprocess.run(["g++", "-o", str(ref_binary(d, k, var == "_moving")), *objs,
                                *extra, "-lm"], check=True)
        tobjs = [str(obj / (u.replace("/", "_") + f".{d}d.o")) for u in REF_UNITS + TESS_UNITS]
        tobjs.append(str(obj / f"tessharness.{d}d.o"))
        for k in ("libm", "sfxpow"):
            extra = [str(obj / "pow_interpose.o")] if k == "sfxpow" else []
            subprocess.run(["g++", "-o", str(tess_binary(d, k)), *tobjs, *extra, "-lm"],
                           check=True)
    return outs


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    for p in build_reference(force="--force" in sys.argv):
        print(p)
