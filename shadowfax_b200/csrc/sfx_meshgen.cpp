/*
 * sfx_meshgen: command-line face-list builder.  Tessellates generator
 * positions with the library's host Voronoi builder (sfx_voronoi.cpp) and
 * writes the face list as a versioned mesh file (sfx_meshfile.cpp).
 *
 * A separate program (host code only, no CUDA runtime, no shared library)
 * so that a process that must not load the GPU library -- a CPU-only job
 * preparing meshes, or the reference CPU pass fed the very meshes the GPU
 * pass gets -- can still produce the face lists.
 *
 * Usage:  sfx_meshgen <positions.bin> <periodic 0|1> <out.sfxmesh> [threads]
 *   positions.bin: int32 dim, int64 n, then n*dim float64 positions in
 *   [0,1)^dim, row-major (exactly the array the Python builder takes).
 * Exit status 0 on success; otherwise the library status code (or 64 for a
 * usage or input error) with a message on stderr.
 */
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "sfxflux.h"

int main(int argc, char** argv) {
    if(argc < 4) {
        std::fprintf(stderr, "usage: %s <positions.bin> <periodic 0|1> <out.sfxmesh> [threads]\n",
                     argv[0]);
        return 64;
    }
    const int periodic = std::atoi(argv[2]) != 0;
    const int threads = argc > 4 ? std::atoi(argv[4]) : 0;
    std::FILE* f = std::fopen(argv[1], "rb");
    if(!f) {
        std::fprintf(stderr, "sfx_meshgen: cannot open %s\n", argv[1]);
        return 64;
    }
    int32_t dim = 0;
    int64_t n = 0;
    bool ok = std::fread(&dim, sizeof dim, 1, f) == 1 && std::fread(&n, sizeof n, 1, f) == 1 &&
              (dim == 2 || dim == 3) && n >= 2 && n <= 0x7ffffff0;
    std::vector<double> pos;
    if(ok) {
        pos.resize((size_t)n * dim);
        ok = std::fread(pos.data(), sizeof(double), pos.size(), f) == pos.size();
    }
    std::fclose(f);
    if(!ok) {
        std::fprintf(stderr, "sfx_meshgen: bad positions file %s\n", argv[1]);
        return 64;
    }
    sfx_voronoi* v = nullptr;
    int rc = sfx_voronoi_build(dim, n, pos.data(), periodic, threads, &v);
    if(rc != SFX_OK) {
        std::fprintf(stderr, "sfx_meshgen: sfx_voronoi_build failed (%d)\n", rc);
        return rc;
    }
    int64_t nc = 0, nf = 0, nnz = 0;
    sfx_voronoi_counts(v, &nc, &nf, &nnz);
    std::vector<double> cen((size_t)nc * dim), vol(nc), tarea(nc), farea(nf), mid((size_t)nf * dim),
            rpos((size_t)nf * dim);
    std::vector<int32_t> off(nc + 1), idx(nnz), left(nf), right(nf), kind(nf);
    rc = sfx_voronoi_export(v, cen.data(), vol.data(), tarea.data(), off.data(), idx.data(),
                            farea.data(), mid.data(), left.data(), right.data(), kind.data(),
                            rpos.data());
    sfx_voronoi_free(v);
    if(rc != SFX_OK) {
        std::fprintf(stderr, "sfx_meshgen: sfx_voronoi_export failed (%d)\n", rc);
        return rc;
    }
    sfx_mesh_desc d{};
    d.dim = dim;
    d.n_cells = (int32_t)nc;
    d.n_faces = (int32_t)nf;
    d.cell_pos = pos.data();
    d.cell_centroid = cen.data();
    d.cell_volume = vol.data();
    d.cell_total_area = tarea.data();
    d.cell_face_offset = off.data();
    d.cell_face_index = idx.data();
    d.face_area = farea.data();
    d.face_midpoint = mid.data();
    d.face_left = left.data();
    d.face_right = right.data();
    d.face_kind = kind.data();
    d.face_right_pos = rpos.data();
    d.face_velocity = nullptr;
    rc = sfx_meshfile_write(argv[3], &d, periodic);
    if(rc != SFX_OK) {
        std::fprintf(stderr, "sfx_meshgen: sfx_meshfile_write %s failed (%d)\n", argv[3], rc);
        return rc;
    }
    return 0;
}
