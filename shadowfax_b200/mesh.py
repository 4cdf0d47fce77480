"""Face-list meshes: the VorTess/VorFace contract the flux pass consumes.

A :class:`Mesh` holds exactly what Shadowfax's host tessellation exports
once per tessellation (src/VorTess.cpp:153-396, src/VorFace.cpp:293-404,
src/VorCell.cpp:257-411): per cell the generator position, centroid, volume,
total face area and the cell's face list; per face the area, midpoint, left
(owner) cell, right neighbour, right kind (real cell / periodic image /
reflective mirror) and the right generator's position.

:func:`build_voronoi` produces such a mesh with the library's host builder
(``sfx_voronoi_*``) from generator positions in the unit square/cube.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib as L

# mesh file header and section entry (sfx_meshfile.cpp)
_MESHFILE_HEADER = struct.Struct("<8sIIIIqqqIIQQQ48x")
_MESHFILE_ENTRY = struct.Struct("<IIQQ")
MESHGEN = Path(__file__).resolve().parent / "sfx_meshgen"


@dataclass
class Mesh:
    dim: int
    periodic: bool
    cell_pos: np.ndarray          # [n, dim] float64
    cell_centroid: np.ndarray     # [n, dim]
    cell_volume: np.ndarray       # [n]
    cell_total_area: np.ndarray   # [n]
    cell_face_offset: np.ndarray  # [n+1] int32
    cell_face_index: np.ndarray   # [nnz] int32
    face_area: np.ndarray         # [F]
    face_midpoint: np.ndarray     # [F, dim]
    face_left: np.ndarray         # [F] int32
    face_right: np.ndarray        # [F] int32, -1 for mirrors
    face_kind: np.ndarray         # [F] int32 (0 real, 1 periodic, 2 mirror)
    face_right_pos: np.ndarray    # [F, dim]
    face_velocity: np.ndarray | None = None  # [F, dim] or None (static)
    _keep: list = field(default_factory=list, repr=False, compare=False)

    @property
    def n_cells(self) -> int:
        return int(self.cell_pos.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.face_area.shape[0])

    @property
    def n_active_faces(self) -> int:
        """faces with nonzero area (the unit of work of the flux pass)"""
        return int(np.count_nonzero(self.face_area))

    @property
    def nnz(self) -> int:
        return int(self.cell_face_index.shape[0])

    _ARRAYS = ("cell_pos", "cell_centroid", "cell_volume", "cell_total_area",
               "cell_face_offset", "cell_face_index", "face_area", "face_midpoint",
               "face_left", "face_right", "face_kind", "face_right_pos")

    def normalized(self) -> "Mesh":
        for name in self._ARRAYS:
            a = getattr(self, name)
            want = np.int32 if a.dtype.kind in "iu" else np.float64
            setattr(self, name, np.ascontiguousarray(a, dtype=want))
        if self.face_velocity is not None:
            self.face_velocity = np.ascontiguousarray(self.face_velocity, dtype=np.float64)
        return self

    def desc(self) -> L.sfx_mesh_desc:
        """C descriptor pointing at this mesh's host arrays."""
        self.normalized()
        d = L.sfx_mesh_desc()
        d.dim, d.n_cells, d.n_faces = self.dim, self.n_cells, self.n_faces
        d.cell_pos = L.dptr(self.cell_pos)
        d.cell_centroid = L.dptr(self.cell_centroid)
        d.cell_volume = L.dptr(self.cell_volume)
        d.cell_total_area = L.dptr(self.cell_total_area)
        d.cell_face_offset = L.iptr(self.cell_face_offset)
        d.cell_face_index = L.iptr(self.cell_face_index)
        d.face_area = L.dptr(self.face_area)
        d.face_midpoint = L.dptr(self.face_midpoint)
        d.face_left = L.iptr(self.face_left)
        d.face_right = L.iptr(self.face_right)
        d.face_kind = L.iptr(self.face_kind)
        d.face_right_pos = L.dptr(self.face_right_pos)
        d.face_velocity = L.dptr(self.face_velocity) if self.face_velocity is not None else None
        return d

    def save(self, path: str | Path) -> None:
        arrs = {n: getattr(self, n) for n in self._ARRAYS}
        arrs["meta"] = np.array([self.dim, int(self.periodic)], dtype=np.int64)
        np.savez_compressed(path, **arrs)

    @classmethod
    def load(cls, path: str | Path) -> "Mesh":
        z = np.load(path)
        dim, periodic = (int(x) for x in z["meta"])
        return cls(dim=dim, periodic=bool(periodic),
                   **{n: z[n] for n in cls._ARRAYS}).normalized()

    def check(self, precision: int = L.PREC_FP64) -> None:
        """the checks an upload to a context of this precision makes, on the
        host alone (sfx_mesh_check); raises SfxError with the status the
        upload would return"""
        d = self.desc()
        L.check(L.lib().sfx_mesh_check(C.byref(d), int(precision)), "sfx_mesh_check")

    def write_file(self, path: str | Path) -> None:
        """the library's versioned binary mesh file (sfx_meshfile_write)"""
        L.check(L.lib().sfx_meshfile_write(str(path).encode(), C.byref(self.desc()),
                                           int(self.periodic)), "sfx_meshfile_write")

    @classmethod
    def read_file(cls, path: str | Path) -> "Mesh":
        """a mesh from sfx_meshfile_write's file (sfx_meshfile_info/_read)"""
        p = str(path).encode()
        dim, per, vel = C.c_int32(), C.c_int32(), C.c_int32()
        n, nf, nnz = C.c_int64(), C.c_int64(), C.c_int64()
        L.check(L.lib().sfx_meshfile_info(p, C.byref(dim), C.byref(per), C.byref(n),
                                          C.byref(nf), C.byref(nnz), C.byref(vel)),
                "sfx_meshfile_info")
        d, n, nf, nnz = dim.value, n.value, nf.value, nnz.value
        m = cls(dim=d, periodic=bool(per.value),
                cell_pos=np.empty((n, d)), cell_centroid=np.empty((n, d)),
                cell_volume=np.empty(n), cell_total_area=np.empty(n),
                cell_face_offset=np.empty(n + 1, np.int32),
                cell_face_index=np.empty(nnz, np.int32),
                face_area=np.empty(nf), face_midpoint=np.empty((nf, d)),
                face_left=np.empty(nf, np.int32), face_right=np.empty(nf, np.int32),
                face_kind=np.empty(nf, np.int32), face_right_pos=np.empty((nf, d)),
                face_velocity=np.empty((nf, d)) if vel.value else None)
        L.check(L.lib().sfx_meshfile_read(
            p, L.dptr(m.cell_pos), L.dptr(m.cell_centroid), L.dptr(m.cell_volume),
            L.dptr(m.cell_total_area), L.iptr(m.cell_face_offset), L.iptr(m.cell_face_index),
            L.dptr(m.face_area), L.dptr(m.face_midpoint), L.iptr(m.face_left),
            L.iptr(m.face_right), L.iptr(m.face_kind), L.dptr(m.face_right_pos),
            L.dptr(m.face_velocity) if vel.value else None), "sfx_meshfile_read")
        return m

    @classmethod
    def read_file_numpy(cls, path: str | Path, verify_checksum: bool = False) -> "Mesh":
        """a mesh file read with numpy alone (no GPU library loaded), for
        CPU-only jobs: the same structural checks as sfx_meshfile_read
        (magic, major version, section table inside the file, cell face
        offsets covering the face list); the FNV-1a payload checksum only
        with verify_checksum (a byte-serial hash, slow in Python)"""
        raw = np.memmap(path, dtype=np.uint8, mode="r")
        head = _MESHFILE_HEADER.unpack_from(raw, 0)
        (magic, major, hbytes, dim, flags, n, nf, nnz, nsec, _minor, poff, pbytes,
         csum) = head
        if (magic != b"SFXMESH\0" or major == 0 or major > 1 or hbytes != 128
                or dim not in (2, 3) or min(n, nf, nnz) < 0 or nsec > 64
                or poff > raw.size or pbytes > raw.size - poff):
            raise ValueError(f"{path}: not a readable mesh file")
        if verify_checksum:
            h = 1469598103934665603
            for x in bytes(raw[poff:poff + pbytes]):
                h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
            if h != csum:
                raise ValueError(f"{path}: checksum mismatch")
        secs = {}
        for i in range(nsec):
            sid, eb, cnt, off = _MESHFILE_ENTRY.unpack_from(raw, 128 + i * _MESHFILE_ENTRY.size)
            if eb not in (4, 8) or off < poff or off + cnt * eb > poff + pbytes:
                raise ValueError(f"{path}: section {sid} outside the payload")
            secs[sid] = np.array(np.frombuffer(raw, "<f8" if eb == 8 else "<i4", cnt, off))
        want = {1: n * dim, 2: n * dim, 3: n, 4: n, 5: n + 1, 6: nnz, 7: nf, 8: nf * dim,
                9: nf, 10: nf, 11: nf, 12: nf * dim}
        if flags & 2:
            want[13] = nf * dim
        for sid, cnt in want.items():
            if sid not in secs or secs[sid].size != cnt:
                raise ValueError(f"{path}: section {sid} missing or of the wrong size")
        off = secs[5]
        if off[0] != 0 or off[-1] != nnz or np.any(np.diff(off) < 0):
            raise ValueError(f"{path}: cell face offsets do not cover the face list")
        return cls(dim=dim, periodic=bool(flags & 1),
                   cell_pos=secs[1].reshape(n, dim), cell_centroid=secs[2].reshape(n, dim),
                   cell_volume=secs[3], cell_total_area=secs[4], cell_face_offset=off,
                   cell_face_index=secs[6], face_area=secs[7],
                   face_midpoint=secs[8].reshape(nf, dim), face_left=secs[9],
                   face_right=secs[10], face_kind=secs[11],
                   face_right_pos=secs[12].reshape(nf, dim),
                   face_velocity=secs[13].reshape(nf, dim) if flags & 2 else None)

    def check_geometry(self, rtol: float = 1e-9) -> None:
        """Sanity checks of a tessellation of the unit box."""
        tot = float(self.cell_volume.sum())
        assert abs(tot - 1.0) < rtol * max(1, self.n_cells) ** 0.5 + 1e-12, tot
        assert np.all(self.cell_volume > 0)
        assert np.all(self.face_area >= 0)


def morton_order(pos: np.ndarray) -> np.ndarray:
    """Permutation sorting points in [0,1)^d along a Z-order curve (the
    reference orders particles along a Hilbert curve for locality,
    src/utilities/ParticleVector.cpp:222)."""
    dim = pos.shape[1]
    bits = 21 if dim == 3 else 31
    q = np.clip((pos * (1 << bits)).astype(np.uint64), 0, (1 << bits) - 1)
    key = np.zeros(pos.shape[0], dtype=np.uint64)
    for b in range(bits):
        for d in range(dim):
            key |= ((q[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * dim + d)
    return np.argsort(key, kind="stable")


def random_generators(n: int, dim: int, seed: int, sort: bool = True) -> np.ndarray:
    """n generator positions uniform in [0,1)^dim from numpy's PCG64 stream
    with the given seed, Z-ordered for memory locality."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = rng.random((n, dim))
    if sort:
        pos = pos[morton_order(pos)]
    return np.ascontiguousarray(pos)


def build_voronoi(pos: np.ndarray, periodic: bool = False, nthreads: int = 0) -> Mesh:
    """Tessellate generators in the unit box (reflective or periodic walls)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n, dim = pos.shape
    lib = L.lib()
    h = C.c_void_p()
    L.check(lib.sfx_voronoi_build(dim, n, L.dptr(pos), int(periodic), int(nthreads),
                                  C.byref(h)), "sfx_voronoi_build")
    try:
        nc, nf, nnz = C.c_int64(), C.c_int64(), C.c_int64()
        L.check(lib.sfx_voronoi_counts(h, C.byref(nc), C.byref(nf), C.byref(nnz)))
        nc, nf, nnz = nc.value, nf.value, nnz.value
        m = Mesh(dim=dim, periodic=periodic, cell_pos=pos,
                 cell_centroid=np.empty((nc, dim)), cell_volume=np.empty(nc),
                 cell_total_area=np.empty(nc),
                 cell_face_offset=np.empty(nc + 1, np.int32),
                 cell_face_index=np.empty(nnz, np.int32),
                 face_area=np.empty(nf), face_midpoint=np.empty((nf, dim)),
                 face_left=np.empty(nf, np.int32), face_right=np.empty(nf, np.int32),
                 face_kind=np.empty(nf, np.int32), face_right_pos=np.empty((nf, dim)))
        L.check(lib.sfx_voronoi_export(
            h, L.dptr(m.cell_centroid), L.dptr(m.cell_volume), L.dptr(m.cell_total_area),
            L.iptr(m.cell_face_offset), L.iptr(m.cell_face_index), L.dptr(m.face_area),
            L.dptr(m.face_midpoint), L.iptr(m.face_left), L.iptr(m.face_right),
            L.iptr(m.face_kind), L.dptr(m.face_right_pos)), "sfx_voronoi_export")
    finally:
        lib.sfx_voronoi_free(h)
    return m


def build_voronoi_file(pos: np.ndarray, periodic: bool, path: str | Path,
                       nthreads: int = 0) -> None:
    """Tessellate generators with the standalone sfx_meshgen program (the same
    builder as build_voronoi, run in a child process without the GPU
    library) and write the face list as a mesh file at `path`."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n, dim = pos.shape
    if not MESHGEN.exists():
        raise FileNotFoundError(f"{MESHGEN} not built (shadowfax_b200.build)")
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "pos.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<iq", dim, n))
            pos.tofile(f)
        subprocess.run([str(MESHGEN), fin, str(int(periodic)), str(path), str(nthreads)],
                       check=True)
