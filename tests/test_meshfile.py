"""The versioned binary mesh file (sfx_meshfile_*): round trips, the layout
read back by an independent parser written from the format's description,
forward compatibility (unknown sections and later minor versions are read)
and rejection of corrupt, truncated and other-major-version files, of header
sizes that do not fit the file and of cell face offsets that do not cover
the face list."""
import struct

import numpy as np
import pytest

from shadowfax_b200 import _lib as L
from shadowfax_b200.mesh import Mesh, build_voronoi, random_generators

ARRAYS = [("cell_pos", 1, 8), ("cell_centroid", 2, 8), ("cell_volume", 3, 8),
          ("cell_total_area", 4, 8), ("cell_face_offset", 5, 4), ("cell_face_index", 6, 4),
          ("face_area", 7, 8), ("face_midpoint", 8, 8), ("face_left", 9, 4),
          ("face_right", 10, 4), ("face_kind", 11, 4), ("face_right_pos", 12, 8),
          ("face_velocity", 13, 8)]
HEADER = struct.Struct("<8sIIIIqqqIIQQQ48x")
ENTRY = struct.Struct("<IIQQ")


def _fnv1a(b: bytes) -> int:
    h = 1469598103934665603
    for x in b:
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def _mesh(dim, periodic, n=1500, seed=3, velocity=False):
    m = build_voronoi(random_generators(n, dim, seed), periodic=periodic)
    if velocity:
        m.face_velocity = np.random.default_rng(seed).standard_normal(m.face_midpoint.shape)
    return m


def _same(a: Mesh, b: Mesh):
    assert a.dim == b.dim and a.periodic == b.periodic
    for name in Mesh._ARRAYS:
        x, y = getattr(a, name), getattr(b, name)
        assert x.dtype == y.dtype and np.array_equal(x.view(np.uint8), y.view(np.uint8)), name
    assert (a.face_velocity is None) == (b.face_velocity is None)
    if a.face_velocity is not None:
        assert np.array_equal(a.face_velocity, b.face_velocity)


@pytest.mark.parametrize("dim,periodic,velocity", [(2, False, False), (3, True, False),
                                                   (2, True, True)])
def test_round_trip(tmp_path, dim, periodic, velocity):
    m = _mesh(dim, periodic, velocity=velocity)
    f = tmp_path / "m.sfxmesh"
    m.write_file(f)
    _same(m, Mesh.read_file(f))


def _parse(raw: bytes):
    """the file by its description alone"""
    (magic, version, hbytes, dim, flags, n, nf, nnz, nsec, _, poff, pbytes,
     csum) = HEADER.unpack_from(raw, 0)
    assert magic == b"SFXMESH\0" and version == 1 and hbytes == 128
    assert _fnv1a(raw[poff:poff + pbytes]) == csum
    out = {}
    for i in range(nsec):
        sid, eb, cnt, off = ENTRY.unpack_from(raw, 128 + i * ENTRY.size)
        assert off % 64 == 0 and poff <= off and off + cnt * eb <= poff + pbytes
        out[sid] = np.frombuffer(raw, dtype="<f8" if eb == 8 else "<i4", count=cnt, offset=off)
    return dim, flags, n, nf, nnz, out


def test_layout_matches_its_description(tmp_path):
    m = _mesh(3, True, velocity=True)
    f = tmp_path / "m.sfxmesh"
    m.write_file(f)
    dim, flags, n, nf, nnz, secs = _parse(f.read_bytes())
    assert (dim, flags, n, nf, nnz) == (3, 3, m.n_cells, m.n_faces, m.nnz)
    for name, sid, _ in ARRAYS:
        assert np.array_equal(secs[sid], getattr(m, name).ravel()), name


def _write_py(path, m: Mesh, extra=None, version=1, minor=0):
    """an independent writer, with optional extra sections {id: bytes}"""
    arrs = [(sid, eb, getattr(m, name)) for name, sid, eb in ARRAYS
            if getattr(m, name) is not None]
    extra = extra or {}
    nsec = len(arrs) + len(extra)
    off = -(-(128 + ENTRY.size * nsec) // 64) * 64
    poff, table, body = off, [], bytearray()
    items = [(sid, eb, np.ascontiguousarray(a).tobytes(), a.size) for sid, eb, a in arrs]
    items += [(sid, 4, b, len(b) // 4) for sid, b in extra.items()]
    for sid, eb, b, cnt in items:
        off = -(-off // 64) * 64
        body += bytes(off - poff - len(body))
        table.append(ENTRY.pack(sid, eb, cnt, off))
        body += b
        off += len(b)
    flags = int(m.periodic) | (2 if m.face_velocity is not None else 0)
    head = HEADER.pack(b"SFXMESH\0", version, 128, m.dim, flags, m.n_cells, m.n_faces, m.nnz,
                       nsec, minor, poff, len(body), _fnv1a(bytes(body)))
    raw = head + b"".join(table)
    raw += bytes(poff - len(raw))
    path.write_bytes(raw + bytes(body))


def test_reader_skips_unknown_sections(tmp_path):
    m = _mesh(2, True)
    f = tmp_path / "m.sfxmesh"
    _write_py(f, m, extra={77: np.arange(10, dtype=np.int32).tobytes()})
    _same(m, Mesh.read_file(f))


def test_corrupt_truncated_and_other_versions_are_rejected(tmp_path):
    m = _mesh(2, False)
    f = tmp_path / "m.sfxmesh"
    m.write_file(f)
    raw = bytearray(f.read_bytes())
    cases = {}
    flip = bytearray(raw)
    flip[len(raw) - 100] ^= 0x10
    cases["flip"] = flip
    cases["truncated"] = raw[:len(raw) // 2]
    v2 = bytearray(raw)
    v2[8:12] = struct.pack("<I", 2)
    cases["version"] = v2
    magic = bytearray(raw)
    magic[0:1] = b"X"
    cases["magic"] = magic
    for name, b in cases.items():
        g = tmp_path / f"{name}.sfxmesh"
        g.write_bytes(bytes(b))
        with pytest.raises(L.SfxError, match="SFX_ERR_IO"):
            Mesh.read_file(g)
    with pytest.raises(L.SfxError, match="SFX_ERR_IO"):
        Mesh.read_file(tmp_path / "missing.sfxmesh")
    _write_py(tmp_path / "v2.sfxmesh", m, version=2)
    with pytest.raises(L.SfxError, match="SFX_ERR_IO"):
        Mesh.read_file(tmp_path / "v2.sfxmesh")


def test_serve_pool_reads_back_its_cached_meshes(tmp_path):
    from shadowfax_b200 import workloads as wl
    a = wl.serve_pool(only={0, 10}, cache_dir=tmp_path)
    files = sorted(p.name for p in tmp_path.iterdir())
    assert len(files) == 2 and all(p.endswith(".sfxmesh") for p in files)
    b = wl.serve_pool(only={0, 10}, cache_dir=tmp_path)
    for j in (0, 10):
        _same(a.meshes[j], b.meshes[j])
        for x, y in zip(a.states[j], b.states[j]):
            assert np.array_equal(x, y)


def test_later_minor_version_with_new_sections_is_read(tmp_path):
    m = _mesh(3, True)
    f = tmp_path / "m.sfxmesh"
    _write_py(f, m, extra={90: np.arange(6, dtype=np.int32).tobytes()}, minor=3)
    _same(m, Mesh.read_file(f))
    _write_py(f, m, version=0)
    with pytest.raises(L.SfxError, match="SFX_ERR_IO"):
        Mesh.read_file(f)


def test_header_sizes_beyond_the_file_are_rejected(tmp_path):
    """the header is not covered by the checksum: a payload size far beyond
    the file must be refused before anything is allocated for it"""
    m = _mesh(2, False)
    f = tmp_path / "m.sfxmesh"
    m.write_file(f)
    raw = bytearray(f.read_bytes())
    fields = list(HEADER.unpack_from(raw, 0))
    for k, v in ((11, 1 << 62), (11, len(raw)), (10, len(raw) + 64)):
        bad = list(fields)
        bad[k] = v
        g = tmp_path / f"bad{k}_{v}.sfxmesh"
        g.write_bytes(HEADER.pack(*bad) + bytes(raw[HEADER.size:]))
        with pytest.raises(L.SfxError, match="SFX_ERR_IO"):
            Mesh.read_file(g)


@pytest.mark.parametrize("how", ["past_end", "short", "decreasing", "nonzero_first"])
def test_cell_face_offsets_must_cover_the_face_list(tmp_path, how):
    """a well-formed file (valid checksum) whose cell face offsets do not run
    from 0 to n_cell_faces without decreasing is rejected (the upload would
    read past the face index array)"""
    m = _mesh(2, True, n=400)
    off = m.cell_face_offset.copy()
    if how == "past_end":
        off[-1] += 7
    elif how == "short":
        off[-1] -= 1
    elif how == "decreasing":
        off[5], off[6] = off[6], off[5]
    else:
        off[0] = 1
    m.cell_face_offset = off
    f = tmp_path / f"{how}.sfxmesh"
    _write_py(f, m)
    with pytest.raises(L.SfxError, match="SFX_ERR_IO"):
        Mesh.read_file(f)


@pytest.mark.parametrize("dim,periodic", [(2, True), (3, False)])
def test_standalone_builder_and_numpy_reader(tmp_path, dim, periodic):
    """sfx_meshgen (the builder as a program of its own, no GPU library)
    writes the same face list as build_voronoi, and the numpy reader reads
    back what sfx_meshfile_read reads, checksum included"""
    from shadowfax_b200.mesh import build_voronoi_file
    pos = random_generators(1200, dim, 11)
    f = tmp_path / "g.sfxmesh"
    build_voronoi_file(pos, periodic, f)
    ref = build_voronoi(pos, periodic=periodic)
    _same(ref, Mesh.read_file(f))
    _same(ref, Mesh.read_file_numpy(f, verify_checksum=True))


def test_numpy_reader_rejects_what_the_library_rejects(tmp_path):
    m = _mesh(2, True, n=300)
    off = m.cell_face_offset.copy()
    off[-1] += 3
    m.cell_face_offset = off
    f = tmp_path / "bad.sfxmesh"
    _write_py(f, m)
    with pytest.raises(ValueError):
        Mesh.read_file_numpy(f)
    m = _mesh(2, True, n=300)
    _write_py(f, m, version=2)
    with pytest.raises(ValueError):
        Mesh.read_file_numpy(f)
