/*
 * C-ABI front end of the sfxflux library: contexts, mesh upload (VorTess
 * face-list contract -> device structure-of-arrays), state transfer, the
 * step driver and the parity entry points.  See include/sfxflux.h.
 */
#include <cuda_runtime.h>

#include <cstdio>
#include <atomic>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <unordered_map>
#include <vector>

#include "sfx_internal.h"

/* A context outlives its meshes: sfx_ctx_destroy on a context that still has
 * meshes only marks it, and the last sfx_mesh_free releases it.  Callers that
 * free in any order (garbage-collected bindings) stay safe. */
struct sfx_ctx {
    sfx_config cfg;
    sfx_solver_params sp;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int live_meshes = 0;
    bool closing = false;
};

struct sfx_mesh {
    sfx_ctx* ctx = nullptr;
    sfx_dmesh d;
    std::vector<void*> allocs;
    /* split pass: the mesh as a one-member launch group, so that a mesh
     * stepped alone runs the same kernels, and so the same arithmetic, as
     * in a group with other meshes */
    sfx_group_entry* self_tab = nullptr;
    int32_t* self_pre = nullptr;
    float self_dt = 0.f; /* time step held in self_tab (0: none yet) */
    bool clone = false;  /* geometry shared with the base mesh */
    unsigned long long* d_smin = nullptr; /* local time steps: smallest new step */
};

namespace {

int cuda_ok(cudaError_t e) {
    return e == cudaSuccess ? SFX_OK : SFX_ERR_CUDA;
}

#define SFX_TRY(x)                       \
    do {                                 \
        int _rc = (x);                   \
        if(_rc != SFX_OK) return _rc;    \
    } while(0)

template <typename T>
int dalloc(sfx_mesh* m, T** p, size_t count) {
    *p = nullptr;
    if(count == 0) count = 1;
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if(e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? SFX_ERR_NOMEM : SFX_ERR_CUDA;
    }
    m->allocs.push_back(q);
    *p = (T*)q;
    return SFX_OK;
}

template <typename T>
int h2d(T* dst, const T* src, size_t count, cudaStream_t s) {
    if(count == 0) return SFX_OK;
    return cuda_ok(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
}

/* [n][w] row-major host -> [w][n] field-major host buffer */
void transpose_in(const double* src, int64_t n, int w, std::vector<double>& out) {
    out.resize((size_t)n * w);
    for(int64_t i = 0; i < n; ++i)
        for(int k = 0; k < w; ++k) out[(size_t)k * n + i] = src[(size_t)i * w + k];
}

void transpose_out(const std::vector<double>& src, int64_t n, int w, double* out) {
    for(int64_t i = 0; i < n; ++i)
        for(int k = 0; k < w; ++k) out[(size_t)i * w + k] = src[(size_t)k * n + i];
}

int check_err(sfx_mesh* m, sfx_stats* st) {
    sfx_dev_error e;
    cudaStream_t s = m->ctx->stream;
    SFX_TRY(cuda_ok(cudaMemcpyAsync(&e, m->d.err, sizeof e, cudaMemcpyDeviceToHost, s)));
    SFX_TRY(cuda_ok(cudaStreamSynchronize(s)));
    int status = SFX_OK;
    if(st) {
        st->bad_face = -1;
        st->bad_cell = -1;
    }
    if(e.face_key != ~0ull) {
        status = (int)(e.face_key & 0xff);
        if(st) st->bad_face = (int32_t)(e.face_key >> 8);
    } else if(e.cell_key != ~0ull) {
        status = (int)(e.cell_key & 0xff);
        if(st) st->bad_cell = (int32_t)(e.cell_key >> 8);
    }
    if(st) st->status = status;
    return status;
}

/* one phase of a step: 0 gradients, 1 face fluxes, 2 update */
/* queued slow faces per mesh: room for every face, so the face kernel never
 * has to run Brent's method itself (and carries none of its code) */
int32_t slowq_capacity(int64_t n_faces) {
    return (int32_t)(n_faces > 0 ? n_faces : 1);
}

/* device table of a split mesh as a one-member launch group */
int setup_self(sfx_mesh* m, cudaStream_t s) {
    if(!m->self_tab) SFX_TRY(dalloc(m, &m->self_tab, 1));
    if(!m->self_pre) SFX_TRY(dalloc(m, &m->self_pre, 6));
    sfx_group_entry e;
    std::memset(&e, 0, sizeof e);
    e.m = m->d;
    m->self_dt = 0.f;
    SFX_TRY(cuda_ok(cudaMemsetAsync(m->self_pre, 0, 6 * sizeof(int32_t), s)));
    /* pageable source: staged before the call returns */
    return h2d(m->self_tab, &e, 1, s);
}

int run_phase(sfx_mesh* m, int phase, double dt, int write_branch, cudaStream_t s) {
    sfx_ctx* c = m->ctx;
    if(c->cfg.precision == SFX_PREC_SPLIT) {
        const float fdt = (float)dt;
        if(phase == 1 && fdt != m->self_dt) {
            m->self_dt = fdt;
            SFX_TRY(h2d(&m->self_tab->dt, &m->self_dt, 1, s));
        }
        sfx_group_dev g;
        std::memset(&g, 0, sizeof g);
        g.tab = m->self_tab;
        g.pre = m->self_pre;
        g.n_meshes = 1;
        g.dim = m->d.dim;
        g.lanes = m->d.lanes;
        g.face_variant = m->d.face_variant;
        g.moving = m->d.vel != nullptr ? 1 : 0; /* split meshes get face velocities
                                                   only from sfx_step_moving */
        sfx_split_blocks(m->d.dim, m->d.lanes, m->d.n_cells, m->d.n_faces, g.blocks);
        if(m->d.ranged) {
            /* one part of a mesh: the phases' own ranges */
            int32_t b[3];
            sfx_split_blocks(m->d.dim, m->d.lanes, sfx_grad_cells(m->d), sfx_flux_faces(m->d), b);
            g.blocks[0] = b[0];
            g.blocks[1] = b[1];
            sfx_split_blocks(m->d.dim, m->d.lanes, sfx_update_cells(m->d), 0, b);
            g.blocks[2] = b[0];
        }
        return sfx_split_group_phase(&g, phase, &c->sp, s);
    }
    switch(phase) {
    case 0:
        return sfx_fp64_gradients(&m->d, s);
    case 1:
        return sfx_fp64_faces(&m->d, &c->sp, dt, write_branch, s);
    default:
        return sfx_fp64_apply(&m->d, &c->sp, s);
    }
}

int reset_err_on(sfx_mesh* m, cudaStream_t s) {
    sfx_dev_error e;
    e.face_key = ~0ull;
    e.cell_key = ~0ull;
    /* pageable source: staged before the call returns */
    return cuda_ok(cudaMemcpyAsync(m->d.err, &e, sizeof e, cudaMemcpyHostToDevice, s));
}

int reset_err(sfx_mesh* m) {
    return reset_err_on(m, m->ctx->stream);
}

/* a state on base's geometry: one device block carved into the arrays,
 * set up on stream s (waited for when `wait`) */
int clone_impl(sfx_ctx* ctx, sfx_mesh* base, cudaStream_t s, bool wait, sfx_mesh** out) {
    if(!ctx || !base || !out) return SFX_ERR_INVALID;
    *out = nullptr;
    const sfx_dmesh& b = base->d;
    const bool split = ctx->cfg.precision == SFX_PREC_SPLIT;
    if(ctx->cfg.dim != b.dim || ctx->closing) return SFX_ERR_INVALID;
    if(split && !b.fg) return SFX_ERR_INVALID; /* base has no split geometry */
    if(cudaSetDevice(ctx->cfg.device) != cudaSuccess) return SFX_ERR_CUDA;
    sfx_mesh* m = new(std::nothrow) sfx_mesh;
    if(!m) return SFX_ERR_NOMEM;
    m->ctx = ctx;
    ctx->live_meshes++;
    m->d = b; /* geometry pointers shared with the base */
    m->clone = true;
    m->d.vgen = m->d.newpos = nullptr;
    m->d.tstart = m->d.tend = nullptr;
    m->d_smin = nullptr;
    sfx_dmesh& d = m->d;
    const int64_t n = d.n_cells, F = d.n_faces;
    const int S = d.S, dim = d.dim;
    d.W = d.Q = d.grad = d.dQf = d.gterm = nullptr;
    d.branch = nullptr;
    d.err = nullptr;
    d.totals_scratch = nullptr;
    d.cw = d.cg = d.cdw = nullptr;
    d.dqm = nullptr;
    d.dqv = nullptr;
    d.slowq = nullptr;
    d.slowq_n = nullptr;
    d.slowq_cap = 0;
    struct Slot {
        void** p;
        size_t bytes;
    };
    std::vector<Slot> slots;
    auto A = [&](auto** p, size_t c) { slots.push_back({(void**)p, c * sizeof(**p)}); };
    A(&d.W, n * S);
    A(&d.Q, n * S);
    A(&d.err, 1);
    A(&d.totals_scratch, (size_t)(S + 1) * 1024);
    if(split) {
        A(&d.cw, 2 * n);
        A(&d.cg, (size_t)sfx_split_grad_vec4(dim) * n);
        A(&d.cdw, (size_t)sfx_split_dwdt_vec4(dim) * n);
        A(&d.dqm, F);
        A(&d.dqv, (size_t)dim * F);
        d.slowq_cap = slowq_capacity(F);
        A(&d.slowq, (size_t)d.slowq_cap);
        A(&d.slowq_n, 1);
        A(&m->self_tab, 1);
        A(&m->self_pre, 6);
    } else {
        A(&d.grad, n * dim * S);
        if(d.gshare)
            A(&d.gterm, F * sfx_grad_term_stride(dim));
        else
            A(&d.dQf, F * S);
        A(&d.branch, F);
    }
    size_t total = 0;
    for(const Slot& sl : slots) total = ((total + 255) & ~(size_t)255) + sl.bytes;
    uint8_t* block = nullptr;
    int rc = dalloc(m, &block, total);
    if(!rc) {
        size_t off = 0;
        for(const Slot& sl : slots) {
            off = (off + 255) & ~(size_t)255;
            *sl.p = block + off;
            off += sl.bytes;
        }
        if(d.gterm) d.dQf = d.gterm;
    }
    if(!rc) rc = reset_err_on(m, s);
    if(!rc && split) rc = cuda_ok(cudaMemsetAsync(d.slowq_n, 0, sizeof(int32_t), s));
    if(!rc && split) rc = setup_self(m, s);
    if(!rc && wait) rc = cuda_ok(cudaStreamSynchronize(s));
    if(rc) {
        sfx_mesh_free(m);
        return rc;
    }
    *out = m;
    return SFX_OK;
}

}  // namespace

sfx_dmesh* sfx_mesh_dev(sfx_mesh* m) {
    return &m->d;
}
int sfx_mesh_last_status(sfx_mesh* m, int32_t* bad_index) {
    sfx_stats st;
    std::memset(&st, 0, sizeof st);
    const int rc = check_err(m, &st);
    if(bad_index) *bad_index = st.bad_face >= 0 ? st.bad_face : st.bad_cell;
    return rc;
}
sfx_ctx* sfx_mesh_ctx(sfx_mesh* m) {
    return m->ctx;
}
void* sfx_ctx_stream(sfx_ctx* c) {
    return (void*)c->stream;
}
const sfx_config* sfx_ctx_config(sfx_ctx* c) {
    return &c->cfg;
}
const sfx_solver_params* sfx_ctx_params(sfx_ctx* c) {
    return &c->sp;
}

namespace {
std::atomic<long long> g_launches{0};
thread_local bool t_capturing = false;
}  // namespace

void sfx_count_launches(int n) {
    if(!t_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}

void sfx_launch_capture(bool on) {
    t_capturing = on;
}

extern "C" {

int64_t sfx_launch_count(void) {
    return g_launches.load(std::memory_order_relaxed);
}

const char* sfx_version(void) {
    return "sfxflux 0.1 (sm_100a)";
}

int sfx_ctx_create(const sfx_config* cfg, sfx_ctx** out) {
    if(!cfg || !out) return SFX_ERR_INVALID;
    *out = nullptr;
    if(cfg->dim != 2 && cfg->dim != 3) return SFX_ERR_INVALID;
    if(cfg->solver != SFX_SOLVER_EXACT && cfg->solver != SFX_SOLVER_HLLC)
        return SFX_ERR_UNSUPPORTED;
    if(cfg->precision != SFX_PREC_FP64 && cfg->precision != SFX_PREC_SPLIT)
        return SFX_ERR_INVALID;
    if(!(cfg->gamma > 1.)) return SFX_ERR_INVALID;
    int ndev = 0;
    if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SFX_ERR_CUDA;
    }
    if(cfg->device < 0 || cfg->device >= ndev) return SFX_ERR_INVALID;
    SFX_TRY(cuda_ok(cudaSetDevice(cfg->device)));
    sfx_ctx* c = new(std::nothrow) sfx_ctx;
    if(!c) return SFX_ERR_NOMEM;
    c->cfg = *cfg;
    sfx_solver_params_init(&c->sp, cfg->solver, cfg->gamma, cfg->tolerance, cfg->cutoff);
    if(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return SFX_ERR_CUDA;
    }
    c->stream = c->own_stream;
    *out = c;
    return SFX_OK;
}

static void ctx_release(sfx_ctx* ctx) {
    cudaSetDevice(ctx->cfg.device);
    if(ctx->own_stream) {
        cudaStreamSynchronize(ctx->own_stream);
        cudaStreamDestroy(ctx->own_stream);
    }
    delete ctx;
}

int sfx_ctx_destroy(sfx_ctx* ctx) {
    if(!ctx || ctx->closing) return SFX_ERR_INVALID;
    ctx->closing = true;
    if(ctx->live_meshes > 0) return SFX_OK; /* released with the last mesh */
    ctx_release(ctx);
    return SFX_OK;
}

int sfx_ctx_set_stream(sfx_ctx* ctx, void* stream) {
    if(!ctx) return SFX_ERR_INVALID;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return SFX_OK;
}

int sfx_ctx_synchronize(sfx_ctx* ctx) {
    if(!ctx) return SFX_ERR_INVALID;
    return cuda_ok(cudaStreamSynchronize(ctx->stream));
}

int64_t sfx_mesh_device_bytes(int32_t dim, int32_t n_cells, int32_t n_faces,
                              int64_t nnz, int32_t precision) {
    const int64_t S = dim + 2, n = n_cells, F = n_faces;
    int64_t cells = n * (8 * (2 * dim + 2 + 2 * S + dim * S) + 4) + 4;
    int64_t faces = F * (8 * (1 + 3 * dim + S) + 4 * 4);
    int64_t bytes = cells + faces + nnz * 4 + 8 * 8 * 1024 + 4096;
    if(precision != SFX_PREC_SPLIT) /* the gradient terms, dQf inside them; the
                                       update's CSR copy (cells not in ascending
                                       face order) */
        bytes += F * 8 * (sfx_grad_term_stride(dim) - S) + nnz * 4;
    if(precision == SFX_PREC_SPLIT) {
        /* fg, fi, fsh, an, dqm, dqv, queue; cw, cg, cx, self table; nbe */
        bytes += F * (32 + 8 + 1 + 8 * dim + 8 + 8 * dim) + 4 * slowq_capacity(F) + 4;
        bytes += n * (32 + 16 * (sfx_split_grad_vec4((int)dim) + sfx_split_dwdt_vec4((int)dim)) +
                      16) + 256;
        bytes += nnz * 4;
    }
    return bytes;
}

namespace {

/* The host checks of a face list (sfx_mesh_check, and sfx_mesh_upload before
 * it allocates anything): every index a kernel will dereference, so device
 * code needs no bounds checks on mesh indices, and the one geometric
 * condition the split kernels rely on. */
int check_desc(const sfx_mesh_desc* desc, int precision) {
    const int dim = desc->dim;
    const int64_t n = desc->n_cells, F = desc->n_faces;
    if(n <= 0 || F < 0) return SFX_ERR_INVALID;
    if(!desc->cell_pos || !desc->cell_centroid || !desc->cell_volume ||
       !desc->cell_total_area || !desc->cell_face_offset || !desc->cell_face_index ||
       (F && (!desc->face_area || !desc->face_midpoint || !desc->face_left ||
              !desc->face_right || !desc->face_kind || !desc->face_right_pos)))
        return SFX_ERR_INVALID;
    const int32_t* off = desc->cell_face_offset;
    if(off[0] != 0) return SFX_ERR_BOUNDS;
    for(int64_t i = 0; i < n; ++i)
        if(off[i + 1] < off[i]) return SFX_ERR_BOUNDS;
    for(int64_t f = 0; f < F; ++f) {
        int L = desc->face_left[f], R = desc->face_right[f], k = desc->face_kind[f];
        if(L < 0 || L >= n) return SFX_ERR_BOUNDS;
        if(k == SFX_FACE_REAL || k == SFX_FACE_PERIODIC) {
            if(R < 0 || R >= n) return SFX_ERR_BOUNDS;
        } else if(k != SFX_FACE_MIRROR) {
            return SFX_ERR_BOUNDS;
        }
    }
    /* a cell lists the faces it owns and the real faces it is the right side of */
    for(int64_t i = 0; i < n; ++i)
        for(int64_t j = off[i]; j < off[i + 1]; ++j) {
            const int32_t f = desc->cell_face_index[j];
            if(f < 0 || f >= F) return SFX_ERR_BOUNDS;
            if(desc->face_left[f] != i &&
               !(desc->face_right[f] == i && desc->face_kind[f] == SFX_FACE_REAL))
                return SFX_ERR_BOUNDS;
        }
    if(precision == SFX_PREC_SPLIT) {
        /* the split kernels apply a periodic image's offset as one whole unit
         * box per axis (a code per axis: 0, +1 or -1); a mesh of another box
         * is refused rather than computed with the wrong offset */
        for(int64_t f = 0; f < F; ++f) {
            if(desc->face_kind[f] != SFX_FACE_PERIODIC) continue;
            for(int l = 0; l < dim; ++l) {
                const double a = std::fabs(desc->face_right_pos[f * dim + l] -
                                           desc->cell_pos[(int64_t)desc->face_right[f] * dim + l]);
                if(!(a <= 1e-9 || std::fabs(a - 1.) <= 1e-9)) return SFX_ERR_UNSUPPORTED;
            }
        }
    }
    return SFX_OK;
}

}  // namespace

int sfx_mesh_check(const sfx_mesh_desc* desc, int32_t precision) {
    if(!desc || (desc->dim != 2 && desc->dim != 3) ||
       (precision != SFX_PREC_FP64 && precision != SFX_PREC_SPLIT))
        return SFX_ERR_INVALID;
    return check_desc(desc, precision);
}

int sfx_mesh_upload(sfx_ctx* ctx, const sfx_mesh_desc* desc, sfx_mesh** out) {
    if(!ctx || !desc || !out) return SFX_ERR_INVALID;
    *out = nullptr;
    const int dim = desc->dim;
    if(dim != ctx->cfg.dim) return SFX_ERR_INVALID;
    SFX_TRY(check_desc(desc, ctx->cfg.precision));
    const int64_t n = desc->n_cells, F = desc->n_faces;
    const int32_t* off = desc->cell_face_offset;
    const int64_t nnz = off[n];
    std::vector<int32_t> idx(nnz);
    for(int64_t i = 0; i < n; ++i) {
        for(int64_t j = off[i]; j < off[i + 1]; ++j) {
            int32_t f = desc->cell_face_index[j];
            if(f < 0 || f >= F) return SFX_ERR_BOUNDS;
            if(desc->face_left[f] == i) {
                idx[j] = f;
            } else if(desc->face_right[f] == i && desc->face_kind[f] == SFX_FACE_REAL) {
                idx[j] = (int32_t)((uint32_t)f | 0x80000000u);
            } else {
                return SFX_ERR_BOUNDS;
            }
        }
    }
    /* The reference adds each face's dQ to its cells in its face loop, in
     * ascending face order (src/VorTessManager.cpp:198-212), while a cell's
     * gradient walks the cell's own face list (src/VorCell.cpp:464-530).  A
     * face list whose cells list their faces in ascending order (the
     * builder's) serves both; otherwise the plain-FP64 update gets a copy of
     * the CSR sorted per cell, so that its sums round as the reference's. */
    std::vector<int32_t> aidx;
    if(ctx->cfg.precision == SFX_PREC_FP64) {
        bool ascending = true;
        for(int64_t i = 0; i < n && ascending; ++i)
            for(int64_t j = off[i] + 1; j < off[i + 1]; ++j)
                if((idx[j] & 0x7fffffff) < (idx[j - 1] & 0x7fffffff)) {
                    ascending = false;
                    break;
                }
        if(!ascending) {
            aidx = idx;
            for(int64_t i = 0; i < n; ++i)
                std::sort(aidx.begin() + off[i], aidx.begin() + off[i + 1],
                          [](int32_t a, int32_t b) { return (a & 0x7fffffff) < (b & 0x7fffffff); });
        }
    }
    /* Split pass only: a face across a periodic boundary is listed twice, once
     * owned by each cell (the reference computes it twice and lets each copy
     * update only its owner, src/VorFace.cpp:913-955).  The split pass
     * applies one copy's flux to both cells: the other copy's owner takes its
     * negated flux (the CSR entry names the kept copy with the right-side
     * bit), so mass and energy leave one cell exactly as they enter the other.
     * Both copies are still solved; the dropped copy's flux reaches no cell
     * and only the per-face export reads it.  The copy kept is chosen by
     * geometry, not by face number: the one whose image shift has the smaller
     * code.  Any numbering of the same faces -- a part of the mesh
     * (shadowfax_b200/partition.py) renumbers them -- then applies the same
     * copy with the same rounding. */
    std::vector<uint8_t> skip;
    std::vector<int32_t> idx_split;
    if(ctx->cfg.precision == SFX_PREC_SPLIT) {
        skip.assign(F, 0);
        idx_split = idx;
        auto shcode = [&](int64_t f) {
            int code = 0;
            for(int l = 0; l < dim; ++l) {
                double s = desc->face_right_pos[f * dim + l] -
                           desc->cell_pos[(int64_t)desc->face_right[f] * dim + l];
                int c = s > 0.5 ? 1 : (s < -0.5 ? 2 : 0);
                code = code * 3 + c;
            }
            return code;
        };
        auto negcode = [&](int code) {
            int out = 0, mul = 1;
            for(int l = 0; l < dim; ++l) {
                int c = code % 3;
                code /= 3;
                out += (c == 1 ? 2 : (c == 2 ? 1 : 0)) * mul;
                mul *= 3;
            }
            return out;
        };
        auto key = [](int64_t L, int64_t R, int code) {
            return ((uint64_t)L * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)R << 20) ^ (uint64_t)code;
        };
        std::unordered_multimap<uint64_t, int64_t> per;
        for(int64_t f = 0; f < F; ++f)
            if(desc->face_kind[f] == SFX_FACE_PERIODIC)
                per.emplace(key(desc->face_left[f], desc->face_right[f], shcode(f)), f);
        std::vector<int32_t> twin(F, -1);
        for(int64_t g = 0; g < F; ++g) {
            if(desc->face_kind[g] != SFX_FACE_PERIODIC) continue;
            const int64_t L = desc->face_left[g], R = desc->face_right[g];
            const int want = negcode(shcode(g));
            auto rng = per.equal_range(key(R, L, want));
            for(auto it = rng.first; it != rng.second; ++it) {
                const int64_t f = it->second;
                if(desc->face_left[f] == R && desc->face_right[f] == L && shcode(f) == want &&
                   f < g && twin[f] < 0) {
                    twin[f] = (int32_t)g;
                    twin[g] = (int32_t)f;
                    if(want > shcode(g)) /* f has the larger code */
                        skip[f] = 1;
                    else
                        skip[g] = 1;
                    break;
                }
            }
        }
        for(int64_t i = 0; i < n; ++i)
            for(int64_t j = off[i]; j < off[i + 1]; ++j) {
                const int32_t g = desc->cell_face_index[j];
                if(skip[g]) idx_split[j] = (int32_t)((uint32_t)twin[g] | 0x80000000u);
            }
    }
    SFX_TRY(cuda_ok(cudaSetDevice(ctx->cfg.device)));
    if(ctx->closing) return SFX_ERR_INVALID;
    sfx_mesh* m = new(std::nothrow) sfx_mesh;
    if(!m) return SFX_ERR_NOMEM;
    m->ctx = ctx;
    ctx->live_meshes++;
    sfx_dmesh& d = m->d;
    std::memset(&d, 0, sizeof d);
    d.dim = dim;
    d.S = dim + 2;
    d.n_cells = (int32_t)n;
    d.n_faces = (int32_t)F;
    d.nnz = nnz;
    d.has_velocity = desc->face_velocity != nullptr;
    d.lanes = sfx_default_lanes(dim);
    /* the plain-FP64 gradients compute a face's terms once for both of its
     * cells when the right cell of every local face sits at the face's right
     * position, bit for bit */
    d.gshare = 1;
    for(int64_t f = 0; f < F && d.gshare; ++f)
        if(desc->face_kind[f] == SFX_FACE_REAL &&
           std::memcmp(desc->face_right_pos + f * dim,
                       desc->cell_pos + (int64_t)desc->face_right[f] * dim,
                       sizeof(double) * dim) != 0)
            d.gshare = 0;
    const int S = d.S;
    int rc = SFX_OK;
    auto A = [&](auto** p, size_t c) {
        if(rc == SFX_OK) rc = dalloc(m, p, c);
    };
    A(&d.pos, n * dim);
    A(&d.cen, n * dim);
    A(&d.vol, n);
    A(&d.tarea, n);
    A(&d.off, n + 1);
    A(&d.idx, nnz);
    if(!aidx.empty()) A(&d.aidx, nnz);
    A(&d.W, n * S);
    A(&d.Q, n * S);
    A(&d.grad, n * dim * S);
    A(&d.area, F);
    A(&d.mid, F * dim);
    A(&d.left, F);
    A(&d.right, F);
    A(&d.kind, F);
    A(&d.rpos, F * dim);
    if(d.has_velocity) A(&d.vel, F * dim);
    const bool split = ctx->cfg.precision == SFX_PREC_SPLIT;
    if(!split && d.gshare) {
        A(&d.gterm, F * sfx_grad_term_stride(dim));
        d.dQf = d.gterm;
    } else {
        A(&d.dQf, F * S);
    }
    A(&d.branch, F);
    A(&d.err, 1);
    A(&d.totals_scratch, (size_t)(S + 1) * 1024);
    if(split) {
        if(d.has_velocity) {
            sfx_mesh_free(m);
            return SFX_ERR_UNSUPPORTED; /* the split pass is for static meshes */
        }
        A(&d.fg, 2 * F);
        A(&d.fi, F);
        A(&d.fsh, F);
        A(&d.cw, 2 * n);
        A(&d.cg, (size_t)sfx_split_grad_vec4(dim) * n);
        A(&d.cdw, (size_t)sfx_split_dwdt_vec4(dim) * n);
        A(&d.cx, n);
        A(&d.nbe, nnz);
        A(&d.an, (size_t)dim * F);
        A(&d.dqm, F);
        A(&d.dqv, (size_t)dim * F);
        d.slowq_cap = slowq_capacity(F);
        A(&d.slowq, (size_t)d.slowq_cap);
        A(&d.slowq_n, 1);
    }
    if(rc != SFX_OK) {
        sfx_mesh_free(m);
        return rc;
    }
    cudaStream_t s = ctx->stream;
    std::vector<double> t1, t2, t3, t4, t5;
    transpose_in(desc->cell_pos, n, dim, t1);
    transpose_in(desc->cell_centroid, n, dim, t2);
    transpose_in(desc->face_midpoint, F, dim, t3);
    transpose_in(desc->face_right_pos, F, dim, t4);
    if(d.has_velocity) transpose_in(desc->face_velocity, F, dim, t5);
    rc = h2d(d.pos, t1.data(), t1.size(), s);
    if(!rc) rc = h2d(d.cen, t2.data(), t2.size(), s);
    if(!rc) rc = h2d(d.vol, desc->cell_volume, n, s);
    if(!rc) rc = h2d(d.tarea, desc->cell_total_area, n, s);
    if(!rc) rc = h2d(d.off, off, n + 1, s);
    if(!rc) rc = h2d(d.idx, split ? idx_split.data() : idx.data(), nnz, s);
    if(!rc && !aidx.empty()) rc = h2d(d.aidx, aidx.data(), nnz, s);
    if(aidx.empty()) d.aidx = d.idx;
    std::vector<int32_t> nbe;
    if(split) {
        /* the neighbour of each CSR entry, so the gradient kernel loads it
         * beside the face id instead of after it */
        nbe.resize(nnz);
        for(int64_t j = 0; j < nnz; ++j) {
            const uint32_t e = (uint32_t)idx_split[j];
            const int32_t f = (int32_t)(e & 0x7fffffffu);
            nbe[j] = (e >> 31) ? desc->face_left[f]
                               : (desc->face_kind[f] == SFX_FACE_MIRROR ? -1 : desc->face_right[f]);
        }
        if(!rc) rc = h2d(d.nbe, nbe.data(), nnz, s);
    }
    if(!rc) rc = h2d(d.area, desc->face_area, F, s);
    if(!rc) rc = h2d(d.mid, t3.data(), t3.size(), s);
    if(!rc) rc = h2d(d.left, desc->face_left, F, s);
    if(!rc) rc = h2d(d.right, desc->face_right, F, s);
    if(!rc) rc = h2d(d.kind, desc->face_kind, F, s);
    if(!rc) rc = h2d(d.rpos, t4.data(), t4.size(), s);
    if(!rc && d.has_velocity) rc = h2d(d.vel, t5.data(), t5.size(), s);
    if(!rc) rc = cuda_ok(cudaMemsetAsync(d.W, 0, sizeof(double) * n * S, s));
    if(!rc) rc = cuda_ok(cudaMemsetAsync(d.Q, 0, sizeof(double) * n * S, s));
    if(!rc) rc = reset_err(m);
    if(!rc && split) rc = cuda_ok(cudaMemsetAsync(d.slowq_n, 0, sizeof(int32_t), s));
    if(!rc && split) rc = sfx_split_prepare(&d, s);
    if(!rc && split) rc = setup_self(m, s);
    /* host staging buffers go out of scope: wait for the copies */
    if(!rc) rc = cuda_ok(cudaStreamSynchronize(s));
    if(rc != SFX_OK) {
        sfx_mesh_free(m);
        return rc;
    }
    *out = m;
    return SFX_OK;
}

int sfx_mesh_free(sfx_mesh* m) {
    if(!m) return SFX_ERR_INVALID;
    sfx_ctx* ctx = m->ctx;
    if(ctx) {
        cudaSetDevice(ctx->cfg.device);
        /* cudaFree waits for the device; a caller stream may already be gone */
        cudaStreamSynchronize(ctx->own_stream);
    }
    for(void* p : m->allocs) cudaFree(p);
    delete m;
    if(ctx && --ctx->live_meshes == 0 && ctx->closing) ctx_release(ctx);
    return SFX_OK;
}

int sfx_state_upload_W(sfx_mesh* m, const double* W) {
    if(!m || !W) return SFX_ERR_INVALID;
    const int64_t n = m->d.n_cells;
    cudaStream_t s = m->ctx->stream;
    std::vector<double> t;
    transpose_in(W, n, m->d.S, t);
    SFX_TRY(reset_err(m));
    SFX_TRY(h2d(m->d.W, t.data(), t.size(), s));
    SFX_TRY(sfx_fp64_init_Q(&m->d, &m->ctx->sp, s));
    if(m->ctx->cfg.precision == SFX_PREC_SPLIT) SFX_TRY(sfx_split_load_state(&m->d, s));
    return check_err(m, nullptr);
}

int sfx_state_upload_WQ(sfx_mesh* m, const double* W, const double* Q) {
    if(!m || !W || !Q) return SFX_ERR_INVALID;
    const int64_t n = m->d.n_cells;
    cudaStream_t s = m->ctx->stream;
    std::vector<double> t1, t2;
    transpose_in(W, n, m->d.S, t1);
    transpose_in(Q, n, m->d.S, t2);
    SFX_TRY(reset_err(m));
    SFX_TRY(h2d(m->d.W, t1.data(), t1.size(), s));
    SFX_TRY(h2d(m->d.Q, t2.data(), t2.size(), s));
    if(m->ctx->cfg.precision == SFX_PREC_SPLIT) SFX_TRY(sfx_split_load_state(&m->d, s));
    return cuda_ok(cudaStreamSynchronize(s));
}

int sfx_state_download(sfx_mesh* m, double* W, double* Q) {
    if(!m) return SFX_ERR_INVALID;
    const int64_t n = m->d.n_cells;
    const int S = m->d.S;
    cudaStream_t s = m->ctx->stream;
    std::vector<double> t1(W ? n * S : 0), t2(Q ? n * S : 0);
    if(W && m->ctx->cfg.precision == SFX_PREC_SPLIT) SFX_TRY(sfx_split_export_W(&m->d, s));
    if(W)
        SFX_TRY(cuda_ok(cudaMemcpyAsync(t1.data(), m->d.W, sizeof(double) * n * S,
                                        cudaMemcpyDeviceToHost, s)));
    if(Q)
        SFX_TRY(cuda_ok(cudaMemcpyAsync(t2.data(), m->d.Q, sizeof(double) * n * S,
                                        cudaMemcpyDeviceToHost, s)));
    SFX_TRY(cuda_ok(cudaStreamSynchronize(s)));
    if(W) transpose_out(t1, n, S, W);
    if(Q) transpose_out(t2, n, S, Q);
    return SFX_OK;
}

int sfx_step(sfx_mesh* m, double dt, int32_t nsteps, sfx_stats* st) {
    if(!m || nsteps < 0 || !(dt > 0.)) return SFX_ERR_INVALID;
    sfx_ctx* c = m->ctx;
    cudaStream_t s = c->stream;
    SFX_TRY(reset_err(m));
    for(int t = 0; t < nsteps; ++t)
        for(int ph = 0; ph < 3; ++ph) SFX_TRY(run_phase(m, ph, dt, 0, s));
    if(!st) return SFX_OK;
    std::memset(st, 0, sizeof *st);
    int rc = check_err(m, st);
    st->steps_done = rc == SFX_OK ? nsteps : -1;
    int rt = sfx_fp64_totals(&m->d, st->totals, s);
    return rc != SFX_OK ? rc : rt;
}

int sfx_step_moving(sfx_mesh* m, double dt, int32_t periodic, double* positions,
                    sfx_stats* st) {
    if(!m || !(dt > 0.)) return SFX_ERR_INVALID;
    sfx_ctx* c = m->ctx;
    if(m->clone || m->d.ranged) return SFX_ERR_UNSUPPORTED;
    const bool split = c->cfg.precision == SFX_PREC_SPLIT;
    cudaStream_t s = c->stream;
    sfx_dmesh& d = m->d;
    const int64_t n = d.n_cells, F = d.n_faces;
    const int D = d.dim;
    if(!d.vgen) SFX_TRY(dalloc(m, &d.vgen, (size_t)D * n));
    if(!d.newpos) SFX_TRY(dalloc(m, &d.newpos, (size_t)D * n));
    const bool fresh = d.vel == nullptr;
    if(fresh) SFX_TRY(dalloc(m, &d.vel, (size_t)D * (F > 0 ? F : 1)));
    d.has_velocity = 1;
    SFX_TRY(reset_err(m));
    /* the split pass keeps the state in FP32 cell records: the FP64 W the
     * velocity kernels read is exported from them first; the device copy of
     * the mesh (the one-member group table) learns the face velocities */
    if(split) SFX_TRY(sfx_split_export_W(&d, s));
    if(split && fresh) SFX_TRY(setup_self(m, s));
    SFX_TRY(sfx_fp64_move_velocities(&d, c->cfg.gamma, dt, periodic ? 1 : 0, 1, s));
    for(int ph = 0; ph < 3; ++ph) SFX_TRY(run_phase(m, ph, dt, 0, s));
    SFX_TRY(sfx_fp64_drift(&d, dt, s));
    if(positions) {
        std::vector<double> t((size_t)D * n);
        SFX_TRY(cuda_ok(cudaMemcpyAsync(t.data(), d.newpos, sizeof(double) * t.size(),
                                        cudaMemcpyDeviceToHost, s)));
        SFX_TRY(cuda_ok(cudaStreamSynchronize(s)));
        transpose_out(t, n, D, positions);
    }
    sfx_stats local;
    sfx_stats* out = st ? st : &local;
    std::memset(out, 0, sizeof *out);
    int rc = check_err(m, out);
    out->steps_done = rc == SFX_OK ? 1 : -1;
    int rt = sfx_fp64_totals(&m->d, out->totals, s);
    return rc != SFX_OK ? rc : rt;
}

/* local time steps: per-cell integer step bounds and generator velocities
 * (all zero at first) */
static int ensure_local(sfx_mesh* m) {
    sfx_dmesh& d = m->d;
    cudaStream_t s = m->ctx->stream;
    const size_t n = (size_t)d.n_cells;
    if(!d.tstart) {
        SFX_TRY(dalloc(m, &d.tstart, n));
        SFX_TRY(dalloc(m, &d.tend, n));
        SFX_TRY(cuda_ok(cudaMemsetAsync(d.tstart, 0, sizeof(uint64_t) * n, s)));
        SFX_TRY(cuda_ok(cudaMemsetAsync(d.tend, 0, sizeof(uint64_t) * n, s)));
    }
    if(!d.vgen) {
        SFX_TRY(dalloc(m, &d.vgen, (size_t)d.dim * n));
        SFX_TRY(cuda_ok(cudaMemsetAsync(d.vgen, 0, sizeof(double) * d.dim * n, s)));
    }
    if(!m->d_smin) SFX_TRY(dalloc(m, &m->d_smin, 1));
    return SFX_OK;
}

/* local time steps: plain FP64 meshes, and split meshes that are not
 * clones (a clone is a request instance of the server) */
static bool local_ok(const sfx_mesh* m) {
    if(m->d.ranged) return false;
    return m->ctx->cfg.precision == SFX_PREC_FP64 || !m->clone;
}

int sfx_mesh_set_timesteps(sfx_mesh* m, const uint64_t* start, const uint64_t* end) {
    if(!m || !start || !end) return SFX_ERR_INVALID;
    if(!local_ok(m)) return SFX_ERR_UNSUPPORTED;
    const int64_t n = m->d.n_cells;
    for(int64_t i = 0; i < n; ++i)
        if(end[i] < start[i] || end[i] > SFX_TIMELINE_TICKS) return SFX_ERR_INVALID;
    SFX_TRY(ensure_local(m));
    cudaStream_t s = m->ctx->stream;
    SFX_TRY(h2d(m->d.tstart, start, (size_t)n, s));
    SFX_TRY(h2d(m->d.tend, end, (size_t)n, s));
    return cuda_ok(cudaStreamSynchronize(s));
}

int sfx_mesh_get_timesteps(sfx_mesh* m, uint64_t* start, uint64_t* end) {
    if(!m || !start || !end) return SFX_ERR_INVALID;
    if(!local_ok(m)) return SFX_ERR_UNSUPPORTED;
    SFX_TRY(ensure_local(m));
    cudaStream_t s = m->ctx->stream;
    const size_t n = (size_t)m->d.n_cells;
    SFX_TRY(cuda_ok(cudaMemcpyAsync(start, m->d.tstart, sizeof(uint64_t) * n,
                                    cudaMemcpyDeviceToHost, s)));
    SFX_TRY(cuda_ok(cudaMemcpyAsync(end, m->d.tend, sizeof(uint64_t) * n,
                                    cudaMemcpyDeviceToHost, s)));
    return cuda_ok(cudaStreamSynchronize(s));
}

int sfx_mesh_set_gradients(sfx_mesh* m, const double* grad) {
    if(!m || !grad) return SFX_ERR_INVALID;
    if(m->ctx->cfg.precision != SFX_PREC_FP64 || !m->d.grad) return SFX_ERR_UNSUPPORTED;
    const int64_t n = m->d.n_cells;
    const int w = m->d.dim * m->d.S;
    std::vector<double> t;
    transpose_in(grad, n, w, t);
    cudaStream_t s = m->ctx->stream;
    SFX_TRY(h2d(m->d.grad, t.data(), t.size(), s));
    return cuda_ok(cudaStreamSynchronize(s));
}

int sfx_mesh_get_gradients(sfx_mesh* m, double* grad) {
    if(!m || !grad) return SFX_ERR_INVALID;
    if(m->ctx->cfg.precision != SFX_PREC_FP64 || !m->d.grad) return SFX_ERR_UNSUPPORTED;
    const int64_t n = m->d.n_cells;
    const int w = m->d.dim * m->d.S;
    std::vector<double> t((size_t)n * w);
    cudaStream_t s = m->ctx->stream;
    SFX_TRY(cuda_ok(cudaMemcpyAsync(t.data(), m->d.grad, sizeof(double) * t.size(),
                                    cudaMemcpyDeviceToHost, s)));
    SFX_TRY(cuda_ok(cudaStreamSynchronize(s)));
    transpose_out(t, n, w, grad);
    return SFX_OK;
}

int sfx_step_window(sfx_mesh* m, double t_total, uint64_t t_now, uint64_t t_next,
                    int32_t periodic, sfx_stats* st) {
    if(!m || !(t_total > 0.) || t_next <= t_now || t_next > SFX_TIMELINE_TICKS)
        return SFX_ERR_INVALID;
    if(!local_ok(m)) return SFX_ERR_UNSUPPORTED;
    SFX_TRY(ensure_local(m));
    sfx_ctx* c = m->ctx;
    cudaStream_t s = c->stream;
    sfx_dmesh& d = m->d;
    const bool split = c->cfg.precision == SFX_PREC_SPLIT;
    d.local = 1;
    d.t_now = t_now;
    d.t_next = t_next;
    d.t_total = t_total;
    int rc = reset_err(m);
    /* the cells starting a step set their generator velocity (the mesh
     * stays); a split mesh's FP32 states are exported to its FP64 W first */
    if(!rc && split) rc = sfx_split_export_W(&d, s);
    if(!rc) rc = sfx_fp64_move_velocities(&d, c->cfg.gamma, 0., periodic ? 1 : 0, 0, s);
    /* a split mesh's kernels read the window from its device table */
    if(!rc && split) rc = setup_self(m, s);
    for(int ph = 0; ph < 3 && !rc; ++ph) rc = run_phase(m, ph, 1., 0, s);
    d.local = 0;
    if(split) {
        const int r2 = setup_self(m, s);
        if(!rc) rc = r2;
    }
    if(rc) return rc;
    sfx_stats local;
    sfx_stats* out = st ? st : &local;
    std::memset(out, 0, sizeof *out);
    rc = check_err(m, out);
    out->steps_done = rc == SFX_OK ? 1 : -1;
    int rt = sfx_fp64_totals(&m->d, out->totals, s);
    return rc != SFX_OK ? rc : rt;
}

int sfx_timestep_bins(sfx_mesh* m, double t_total, double cfl, uint64_t max_step,
                      uint64_t min_step, uint64_t t_next, uint64_t* system_step) {
    if(!m || !(t_total > 0.) || !(cfl > 0.) || max_step == 0 || max_step > SFX_TIMELINE_TICKS ||
       min_step > max_step || !system_step)
        return SFX_ERR_INVALID;
    if(!local_ok(m)) return SFX_ERR_UNSUPPORTED;
    SFX_TRY(ensure_local(m));
    sfx_ctx* c = m->ctx;
    cudaStream_t s = c->stream;
    sfx_dmesh& d = m->d;
    d.t_next = t_next;
    d.t_total = t_total;
    SFX_TRY(reset_err(m));
    const unsigned long long smax = max_step;
    SFX_TRY(h2d(m->d_smin, &smax, 1, s));
    /* a split mesh: the CFL steps from its FP32 states, exported to FP64 */
    if(c->cfg.precision == SFX_PREC_SPLIT) SFX_TRY(sfx_split_export_W(&d, s));
    SFX_TRY(sfx_fp64_timestep_bins(&d, c->cfg.gamma, cfl, max_step, min_step, m->d_smin, s));
    unsigned long long out = 0;
    SFX_TRY(cuda_ok(cudaMemcpyAsync(&out, m->d_smin, sizeof out, cudaMemcpyDeviceToHost, s)));
    SFX_TRY(cuda_ok(cudaStreamSynchronize(s)));
    SFX_TRY(check_err(m, nullptr));
    *system_step = out;
    return SFX_OK;
}

int sfx_step_timed(sfx_mesh* m, double dt, int32_t nsteps, float* kernel_ms,
                   int32_t* launches) {
    if(!m || nsteps < 0 || !(dt > 0.) || !kernel_ms) return SFX_ERR_INVALID;
    sfx_ctx* c = m->ctx;
    cudaStream_t s = c->stream;
    cudaEvent_t ev[4];
    for(auto& e : ev)
        if(cudaEventCreate(&e) != cudaSuccess) return SFX_ERR_CUDA;
    double acc[3] = {0., 0., 0.};
    int rc = reset_err(m);
    const int64_t l0 = sfx_launch_count();
    for(int t = 0; t < nsteps && rc == SFX_OK; ++t) {
        cudaEventRecord(ev[0], s);
        rc = run_phase(m, 0, dt, 0, s);
        cudaEventRecord(ev[1], s);
        if(!rc) rc = run_phase(m, 1, dt, 0, s);
        cudaEventRecord(ev[2], s);
        if(!rc) rc = run_phase(m, 2, dt, 0, s);
        cudaEventRecord(ev[3], s);
        if(!rc) rc = cuda_ok(cudaEventSynchronize(ev[3]));
        for(int k = 0; k < 3 && !rc; ++k) {
            float ms = 0.f;
            rc = cuda_ok(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            acc[k] += ms;
        }
    }
    for(auto& e : ev) cudaEventDestroy(e);
    for(int k = 0; k < 3; ++k) kernel_ms[k] = (float)acc[k];
    if(launches) *launches = (int32_t)(sfx_launch_count() - l0);
    if(rc) return rc;
    return check_err(m, nullptr);
}

int sfx_flux_pass(sfx_mesh* m, double dt, double* grad, double* dQ_face,
                  int32_t* branch, sfx_stats* st) {
    if(!m || !(dt > 0.)) return SFX_ERR_INVALID;
    sfx_ctx* c = m->ctx;
    cudaStream_t s = c->stream;
    const int64_t n = m->d.n_cells, F = m->d.n_faces;
    const int S = m->d.S, D = m->d.dim;
    const bool split = c->cfg.precision == SFX_PREC_SPLIT;
    if(!m->d.dQf) return SFX_ERR_UNSUPPORTED; /* a split clone keeps no FP64 dQ */
    SFX_TRY(reset_err(m));
    SFX_TRY(run_phase(m, 0, dt, 1, s));
    SFX_TRY(run_phase(m, 1, dt, 1, s));
    if(split) SFX_TRY(sfx_split_export_dQ(&m->d, s));
    std::vector<double> tg(grad ? n * D * S : 0), tq(dQ_face ? F * S : 0);
    if(grad && split) {
        /* FP32 gradient records [n][G float4] -> [D*S][n] */
        const int G = sfx_split_grad_vec4(D);
        std::vector<float> tf((size_t)n * G * 4);
        SFX_TRY(cuda_ok(cudaMemcpyAsync(tf.data(), m->d.cg, sizeof(float) * tf.size(),
                                        cudaMemcpyDeviceToHost, s)));
        SFX_TRY(cuda_ok(cudaStreamSynchronize(s)));
        for(int64_t i = 0; i < n; ++i)
            for(int q = 0; q < D * S; ++q) tg[(size_t)q * n + i] = tf[(size_t)i * G * 4 + q];
    } else if(grad) {
        SFX_TRY(cuda_ok(cudaMemcpyAsync(tg.data(), m->d.grad, sizeof(double) * tg.size(),
                                        cudaMemcpyDeviceToHost, s)));
    }
    if(branch && split && F) SFX_TRY(cuda_ok(cudaMemsetAsync(m->d.branch, 0, 4 * F, s)));
    if(dQ_face)
        SFX_TRY(cuda_ok(cudaMemcpyAsync(tq.data(), m->d.dQf, sizeof(double) * tq.size(),
                                        cudaMemcpyDeviceToHost, s)));
    if(branch && F)
        SFX_TRY(cuda_ok(cudaMemcpyAsync(branch, m->d.branch, sizeof(int32_t) * F,
                                        cudaMemcpyDeviceToHost, s)));
    SFX_TRY(cuda_ok(cudaStreamSynchronize(s)));
    if(grad) transpose_out(tg, n, D * S, grad);
    if(dQ_face) transpose_out(tq, F, S, dQ_face);
    sfx_stats local;
    return check_err(m, st ? st : &local);
}

int sfx_riemann_eval(sfx_ctx* c, int32_t n, const double* WL, const double* WR,
                     const double* normal, int32_t reflective, double* half,
                     double* flux, int32_t* branch) {
    if(!c || n < 0 || (n && (!WL || !WR || !normal || !flux || !branch)))
        return SFX_ERR_INVALID;
    if(n == 0) return SFX_OK;
    const int D = c->cfg.dim, S = D + 2;
    cudaStream_t s = c->stream;
    double *dWL = nullptr, *dWR = nullptr, *dn = nullptr, *dh = nullptr, *df = nullptr;
    int32_t* dc = nullptr;
    int rc = SFX_OK;
    auto al = [&](auto** p, size_t bytes) {
        if(rc == SFX_OK && cudaMalloc((void**)p, bytes) != cudaSuccess) rc = SFX_ERR_CUDA;
    };
    al(&dWL, sizeof(double) * n * S);
    al(&dWR, sizeof(double) * n * S);
    al(&dn, sizeof(double) * n * D);
    al(&dh, sizeof(double) * n * S);
    al(&df, sizeof(double) * n * S);
    al(&dc, sizeof(int32_t) * n);
    if(!rc) rc = h2d(dWL, WL, (size_t)n * S, s);
    if(!rc) rc = h2d(dWR, WR, (size_t)n * S, s);
    if(!rc) rc = h2d(dn, normal, (size_t)n * D, s);
    if(!rc) rc = sfx_fp64_riemann(D, &c->sp, n, dWL, dWR, dn, reflective, dh, df, dc, s);
    if(!rc && half)
        rc = cuda_ok(cudaMemcpyAsync(half, dh, sizeof(double) * n * S, cudaMemcpyDeviceToHost, s));
    if(!rc)
        rc = cuda_ok(cudaMemcpyAsync(flux, df, sizeof(double) * n * S, cudaMemcpyDeviceToHost, s));
    if(!rc)
        rc = cuda_ok(cudaMemcpyAsync(branch, dc, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    if(!rc) rc = cuda_ok(cudaStreamSynchronize(s));
    cudaFree(dWL);
    cudaFree(dWR);
    cudaFree(dn);
    cudaFree(dh);
    cudaFree(df);
    cudaFree(dc);
    return rc;
}

int sfx_mesh_clone(sfx_ctx* ctx, sfx_mesh* base, sfx_mesh** out) {
    return clone_impl(ctx, base, ctx ? ctx->stream : nullptr, true, out);
}

int64_t sfx_mesh_clone_bytes(sfx_mesh* base, int32_t precision) {
    if(!base) return -1;
    const sfx_dmesh& b = base->d;
    const int64_t n = b.n_cells, F = b.n_faces, S = b.S, D = b.dim;
    int64_t bytes = n * S * 16 + (S + 1) * 1024 * 8 + 64;
    if(precision == SFX_PREC_SPLIT)
        bytes += n * 32 + n * 16 * (sfx_split_grad_vec4((int)D) + sfx_split_dwdt_vec4((int)D)) +
                 F * 8 + F * D * 8 +
                 4 * (int64_t)slowq_capacity(F) + 4 + (int64_t)sizeof(sfx_group_entry) + 24;
    else
        bytes += n * D * S * 8 + F * 4 +
                 F * 8 * (b.gshare ? sfx_grad_term_stride((int)D) : S) + 256;
    return bytes;
}

int sfx_mesh_set_lanes(sfx_mesh* m, int32_t lanes) {
    if(!m || (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16))
        return SFX_ERR_INVALID;
    m->d.lanes = lanes;
    return SFX_OK;
}

int sfx_mesh_set_face_variant(sfx_mesh* m, int32_t variant) {
    if(!m || variant < 0 || variant >= SFX_FACE_VARIANTS) return SFX_ERR_INVALID;
    m->d.face_variant = variant;
    return SFX_OK;
}

int sfx_mesh_set_ranges(sfx_mesh* m, int32_t grad_cells, int32_t flux_faces,
                        int32_t update_cells) {
    if(!m) return SFX_ERR_INVALID;
    const bool split = m->ctx->cfg.precision == SFX_PREC_SPLIT;
    if(split && m->clone) return SFX_ERR_UNSUPPORTED;
    sfx_dmesh& d = m->d;
    if(update_cells < 0 || update_cells > grad_cells || grad_cells > d.n_cells ||
       flux_faces < 0 || flux_faces > d.n_faces)
        return SFX_ERR_INVALID;
    d.ranged = 1;
    d.r_grad = grad_cells;
    d.r_flux = flux_faces;
    d.r_upd = update_cells;
    /* a split mesh's kernels read the ranges from its device table */
    if(split) return setup_self(m, m->ctx->stream);
    return SFX_OK;
}

int sfx_mesh_pack_cells(sfx_mesh* m, const int32_t* idx, int32_t count, double* out,
                        void* stream) {
    if(!m || count < 0 || (count > 0 && (!idx || !out))) return SFX_ERR_INVALID;
    if(m->ctx->cfg.precision == SFX_PREC_SPLIT)
        return sfx_split_pack_cells(&m->d, idx, count, out,
                                    stream ? stream : (void*)m->ctx->stream);
    return sfx_fp64_pack_cells(&m->d, idx, count, out,
                               stream ? stream : (void*)m->ctx->stream);
}

int sfx_mesh_unpack_cells(sfx_mesh* m, const int32_t* idx, int32_t count, const double* in,
                          void* stream) {
    if(!m || count < 0 || (count > 0 && (!idx || !in))) return SFX_ERR_INVALID;
    if(m->ctx->cfg.precision == SFX_PREC_SPLIT)
        return sfx_split_unpack_cells(&m->d, idx, count, in,
                                      stream ? stream : (void*)m->ctx->stream);
    return sfx_fp64_unpack_cells(&m->d, idx, count, in,
                                 stream ? stream : (void*)m->ctx->stream);
}

int sfx_mesh_totals(sfx_mesh* m, double* totals) {
    if(!m || !totals) return SFX_ERR_INVALID;
    return sfx_fp64_totals(&m->d, totals, m->ctx->stream);
}

}  // extern "C"

/* internal transfers for the request server (C++ linkage) */
int sfx_mesh_upload_W_fieldmajor(sfx_mesh* m, const double* W) {
    if(!m || !W) return SFX_ERR_INVALID;
    cudaStream_t s = m->ctx->stream;
    SFX_TRY(reset_err(m));
    SFX_TRY(h2d(m->d.W, W, (size_t)m->d.n_cells * m->d.S, s));
    SFX_TRY(sfx_fp64_init_Q(&m->d, &m->ctx->sp, s));
    if(m->ctx->cfg.precision == SFX_PREC_SPLIT) SFX_TRY(sfx_split_load_state(&m->d, s));
    return check_err(m, nullptr);
}

int sfx_mesh_download_fieldmajor_async(sfx_mesh* m, double* W, double* Q, void* stream) {
    if(!m || !W || !Q) return SFX_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = sizeof(double) * (size_t)m->d.n_cells * m->d.S;
    if(m->ctx->cfg.precision == SFX_PREC_SPLIT) SFX_TRY(sfx_split_export_W(&m->d, s));
    SFX_TRY(cuda_ok(cudaMemcpyAsync(W, m->d.W, bytes, cudaMemcpyDeviceToHost, s)));
    return cuda_ok(cudaMemcpyAsync(Q, m->d.Q, bytes, cudaMemcpyDeviceToHost, s));
}

int sfx_mesh_clone_async(sfx_ctx* ctx, sfx_mesh* base, void* stream, sfx_mesh** out) {
    return clone_impl(ctx, base, (cudaStream_t)stream, false, out);
}

int sfx_mesh_upload_W_fieldmajor_async(sfx_mesh* m, const double* W, void* stream) {
    if(!m || !W) return SFX_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    SFX_TRY(reset_err_on(m, s));
    SFX_TRY(h2d(m->d.W, W, (size_t)m->d.n_cells * m->d.S, s));
    SFX_TRY(sfx_fp64_init_Q(&m->d, &m->ctx->sp, s));
    if(m->ctx->cfg.precision == SFX_PREC_SPLIT) SFX_TRY(sfx_split_load_state(&m->d, s));
    return SFX_OK;
}
