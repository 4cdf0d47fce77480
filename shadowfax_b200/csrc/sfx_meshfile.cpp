/*
 * Versioned binary file of one tessellation's face list (the sfx_mesh_desc
 * contract: what Shadowfax's VorTess/VorFace/VorCell export once per
 * tessellation, src/VorTess.cpp:153-396), so that a pool of pre-tessellated
 * meshes is built once and read back by any caller of the C ABI.
 *
 * Layout, little-endian:
 *   header (128 bytes)   magic "SFXMESH\0", major version, header size, dim,
 *                        flags (bit 0 periodic, bit 1 face velocities),
 *                        n_cells, n_faces, n_cell_faces, section count,
 *                        minor version, payload offset and size, FNV-1a 64
 *                        checksum of the payload
 *   section table        per array: id, element size, element count, offset
 *   payload              the arrays, each at a 64-byte aligned offset, in
 *                        the descriptor's layout ([n][dim] row-major)
 * A reader skips sections whose id it does not know, so a later minor
 * version can add arrays and stay readable; a file with a higher major
 * version (a changed meaning of an existing array) is rejected.  Sizes in the
 * header are never trusted: the payload must lie inside the file, and the
 * cell face offsets must run from 0 to n_cell_faces without decreasing.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "sfxflux.h"

namespace {

constexpr char kMagic[8] = {'S', 'F', 'X', 'M', 'E', 'S', 'H', '\0'};
constexpr uint32_t kHeaderBytes = 128;
constexpr uint64_t kAlign = 64;

enum Section : uint32_t {
    kCellPos = 1,
    kCellCentroid,
    kCellVolume,
    kCellTotalArea,
    kCellFaceOffset,
    kCellFaceIndex,
    kFaceArea,
    kFaceMidpoint,
    kFaceLeft,
    kFaceRight,
    kFaceKind,
    kFaceRightPos,
    kFaceVelocity
};

struct Header {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    uint32_t dim;
    uint32_t flags;
    int64_t n_cells;
    int64_t n_faces;
    int64_t n_cell_faces;
    uint32_t n_sections;
    uint32_t minor_version; /* readers ignore it: later minors only add sections */
    uint64_t payload_offset;
    uint64_t payload_bytes;
    uint64_t checksum;
    uint8_t pad[128 - 80];
};
static_assert(sizeof(Header) == kHeaderBytes, "header layout");

struct Entry {
    uint32_t id;
    uint32_t elem_bytes;
    uint64_t count;
    uint64_t offset;
};
static_assert(sizeof(Entry) == 24, "section entry layout");

bool little_endian() {
    const uint16_t x = 1;
    uint8_t b;
    std::memcpy(&b, &x, 1);
    return b == 1;
}

uint64_t fnv1a(const uint8_t* p, size_t n, uint64_t h = 1469598103934665603ull) {
    for(size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

uint64_t align_up(uint64_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Array {
    uint32_t id;
    uint32_t elem_bytes;
    uint64_t count;
    const void* src;
};

/* the arrays of a mesh with these sizes, in file order */
std::vector<Array> layout(int dim, int64_t n, int64_t F, int64_t nnz, bool vel) {
    const uint64_t D = (uint64_t)dim;
    std::vector<Array> a = {
        {kCellPos, 8, n * D, nullptr},      {kCellCentroid, 8, n * D, nullptr},
        {kCellVolume, 8, (uint64_t)n, nullptr}, {kCellTotalArea, 8, (uint64_t)n, nullptr},
        {kCellFaceOffset, 4, (uint64_t)n + 1, nullptr},
        {kCellFaceIndex, 4, (uint64_t)nnz, nullptr},
        {kFaceArea, 8, (uint64_t)F, nullptr}, {kFaceMidpoint, 8, F * D, nullptr},
        {kFaceLeft, 4, (uint64_t)F, nullptr}, {kFaceRight, 4, (uint64_t)F, nullptr},
        {kFaceKind, 4, (uint64_t)F, nullptr}, {kFaceRightPos, 8, F * D, nullptr}};
    if(vel) a.push_back({kFaceVelocity, 8, F * D, nullptr});
    return a;
}

struct File {
    std::FILE* f = nullptr;
    ~File() {
        if(f) std::fclose(f);
    }
};

}  // namespace

extern "C" {

int sfx_meshfile_write(const char* path, const sfx_mesh_desc* m, int32_t periodic) {
    if(!path || !m || (m->dim != 2 && m->dim != 3) || m->n_cells < 0 || m->n_faces < 0 ||
       !m->cell_face_offset)
        return SFX_ERR_INVALID;
    if(!little_endian()) return SFX_ERR_UNSUPPORTED;
    const int64_t n = m->n_cells, F = m->n_faces;
    const int64_t nnz = m->cell_face_offset[n];
    if(nnz < 0) return SFX_ERR_INVALID;
    std::vector<Array> arrs = layout(m->dim, n, F, nnz, m->face_velocity != nullptr);
    const void* src[] = {m->cell_pos,         m->cell_centroid,   m->cell_volume,
                         m->cell_total_area,  m->cell_face_offset, m->cell_face_index,
                         m->face_area,        m->face_midpoint,   m->face_left,
                         m->face_right,       m->face_kind,       m->face_right_pos,
                         m->face_velocity};
    for(size_t i = 0; i < arrs.size(); ++i) {
        arrs[i].src = src[i];
        if(!arrs[i].src && arrs[i].count) return SFX_ERR_INVALID;
    }
    Header h;
    std::memset(&h, 0, sizeof h);
    std::memcpy(h.magic, kMagic, 8);
    h.version = SFX_MESHFILE_VERSION;
    h.minor_version = SFX_MESHFILE_MINOR_VERSION;
    h.header_bytes = kHeaderBytes;
    h.dim = (uint32_t)m->dim;
    h.flags = (periodic ? 1u : 0u) | (m->face_velocity ? 2u : 0u);
    h.n_cells = n;
    h.n_faces = F;
    h.n_cell_faces = nnz;
    h.n_sections = (uint32_t)arrs.size();
    std::vector<Entry> tab(arrs.size());
    uint64_t off = align_up(kHeaderBytes + sizeof(Entry) * tab.size());
    h.payload_offset = off;
    for(size_t i = 0; i < arrs.size(); ++i) {
        off = align_up(off);
        tab[i] = {arrs[i].id, arrs[i].elem_bytes, arrs[i].count, off};
        off += arrs[i].count * arrs[i].elem_bytes;
    }
    h.payload_bytes = off - h.payload_offset;
    /* the payload with its zero padding, checksummed as written */
    std::vector<uint8_t> payload;
    try {
        payload.assign(h.payload_bytes, 0);
    } catch(const std::bad_alloc&) {
        return SFX_ERR_NOMEM;
    }
    for(size_t i = 0; i < arrs.size(); ++i)
        if(tab[i].count)
            std::memcpy(payload.data() + (tab[i].offset - h.payload_offset), arrs[i].src,
                        tab[i].count * tab[i].elem_bytes);
    h.checksum = fnv1a(payload.data(), payload.size());
    File out;
    out.f = std::fopen(path, "wb");
    if(!out.f) return SFX_ERR_IO;
    std::vector<uint8_t> head(h.payload_offset, 0);
    std::memcpy(head.data(), &h, sizeof h);
    std::memcpy(head.data() + kHeaderBytes, tab.data(), sizeof(Entry) * tab.size());
    if(std::fwrite(head.data(), 1, head.size(), out.f) != head.size() ||
       std::fwrite(payload.data(), 1, payload.size(), out.f) != payload.size())
        return SFX_ERR_IO;
    if(std::fclose(out.f) != 0) {
        out.f = nullptr;
        return SFX_ERR_IO;
    }
    out.f = nullptr;
    return SFX_OK;
}

namespace {

/* header and section table of a file, checked for structure; the payload
 * read and checksummed when `payload` is not NULL */
int read_file(const char* path, Header& h, std::vector<Entry>& tab,
              std::vector<uint8_t>* payload) {
    if(!path) return SFX_ERR_INVALID;
    if(!little_endian()) return SFX_ERR_UNSUPPORTED;
    File in;
    in.f = std::fopen(path, "rb");
    if(!in.f) return SFX_ERR_IO;
    if(std::fseek(in.f, 0, SEEK_END) != 0) return SFX_ERR_IO;
    const long long file_bytes = std::ftell(in.f);
    if(file_bytes < 0 || std::fseek(in.f, 0, SEEK_SET) != 0) return SFX_ERR_IO;
    if(std::fread(&h, 1, sizeof h, in.f) != sizeof h) return SFX_ERR_IO;
    /* major version 0 never existed; a higher major is a format this reader
     * does not understand */
    if(std::memcmp(h.magic, kMagic, 8) != 0 || h.version == 0 ||
       h.version > SFX_MESHFILE_VERSION || h.header_bytes != kHeaderBytes ||
       (h.dim != 2 && h.dim != 3) || h.n_cells < 0 || h.n_faces < 0 || h.n_cell_faces < 0 ||
       h.n_cells > INT32_MAX - 1 || h.n_faces > INT32_MAX || h.n_cell_faces > INT32_MAX ||
       h.n_sections > 64)
        return SFX_ERR_IO;
    /* the payload lies inside the file (no allocation sized by a header
     * field alone) */
    const uint64_t fb = (uint64_t)file_bytes;
    if(h.payload_offset > fb || h.payload_bytes > fb - h.payload_offset) return SFX_ERR_IO;
    tab.resize(h.n_sections);
    if(h.n_sections &&
       std::fread(tab.data(), sizeof(Entry), h.n_sections, in.f) != h.n_sections)
        return SFX_ERR_IO;
    if(h.payload_offset < kHeaderBytes + sizeof(Entry) * (uint64_t)h.n_sections)
        return SFX_ERR_IO;
    for(const Entry& e : tab) {
        if(e.elem_bytes != 4 && e.elem_bytes != 8) return SFX_ERR_IO;
        if(e.count > (uint64_t)1 << 40 || e.offset < h.payload_offset ||
           e.offset - h.payload_offset > h.payload_bytes ||
           e.count * e.elem_bytes > h.payload_bytes - (e.offset - h.payload_offset))
            return SFX_ERR_IO;
    }
    if(!payload) return SFX_OK;
    if(std::fseek(in.f, (long)h.payload_offset, SEEK_SET) != 0) return SFX_ERR_IO;
    try {
        payload->assign(h.payload_bytes, 0);
    } catch(const std::bad_alloc&) {
        return SFX_ERR_NOMEM;
    }
    if(h.payload_bytes &&
       std::fread(payload->data(), 1, h.payload_bytes, in.f) != h.payload_bytes)
        return SFX_ERR_IO;
    if(fnv1a(payload->data(), payload->size()) != h.checksum) return SFX_ERR_IO;
    return SFX_OK;
}

}  // namespace

int sfx_meshfile_info(const char* path, int32_t* dim, int32_t* periodic, int64_t* n_cells,
                      int64_t* n_faces, int64_t* n_cell_faces, int32_t* has_velocity) {
    Header h;
    std::vector<Entry> tab;
    int rc;
    try {
        rc = read_file(path, h, tab, nullptr);
    } catch(const std::bad_alloc&) {
        return SFX_ERR_NOMEM;
    }
    if(rc) return rc;
    if(dim) *dim = (int32_t)h.dim;
    if(periodic) *periodic = (h.flags & 1u) ? 1 : 0;
    if(n_cells) *n_cells = h.n_cells;
    if(n_faces) *n_faces = h.n_faces;
    if(n_cell_faces) *n_cell_faces = h.n_cell_faces;
    if(has_velocity) *has_velocity = (h.flags & 2u) ? 1 : 0;
    return SFX_OK;
}

int sfx_meshfile_read(const char* path, double* cell_pos, double* cell_centroid,
                      double* cell_volume, double* cell_total_area, int32_t* cell_face_offset,
                      int32_t* cell_face_index, double* face_area, double* face_midpoint,
                      int32_t* face_left, int32_t* face_right, int32_t* face_kind,
                      double* face_right_pos, double* face_velocity) {
    Header h;
    std::vector<Entry> tab;
    std::vector<uint8_t> payload;
    int rc;
    try {
        rc = read_file(path, h, tab, &payload);
    } catch(const std::bad_alloc&) {
        return SFX_ERR_NOMEM;
    }
    if(rc) return rc;
    const bool vel = (h.flags & 2u) != 0;
    std::vector<Array> want = layout((int)h.dim, h.n_cells, h.n_faces, h.n_cell_faces, vel);
    void* dst[] = {cell_pos,        cell_centroid, cell_volume,   cell_total_area,
                   cell_face_offset, cell_face_index, face_area,  face_midpoint,
                   face_left,       face_right,    face_kind,     face_right_pos,
                   face_velocity};
    for(size_t i = 0; i < want.size(); ++i) {
        if(!dst[i]) {
            if(want[i].id == kFaceVelocity) continue; /* the caller does not want them */
            if(want[i].count) return SFX_ERR_INVALID;
            continue;
        }
        const Entry* e = nullptr;
        for(const Entry& t : tab)
            if(t.id == want[i].id) e = &t;
        if(!e || e->elem_bytes != want[i].elem_bytes || e->count != want[i].count)
            return SFX_ERR_IO;
        if(e->count)
            std::memcpy(dst[i], payload.data() + (e->offset - h.payload_offset),
                        e->count * e->elem_bytes);
    }
    /* the cell face lists must cover exactly the n_cell_faces entries the
     * caller sized cell_face_index for: sfx_mesh_upload reads up to
     * offset[n_cells] of them */
    const int32_t* off = cell_face_offset;
    if(off[0] != 0 || off[h.n_cells] != h.n_cell_faces) return SFX_ERR_IO;
    for(int64_t i = 0; i < h.n_cells; ++i)
        if(off[i + 1] < off[i]) return SFX_ERR_IO;
    if(!vel && face_velocity && h.n_faces)
        std::memset(face_velocity, 0, sizeof(double) * (size_t)h.n_faces * h.dim);
    return SFX_OK;
}

}  // extern "C"
