/*
 * Request server: continuous batching of static-mesh integrations on one GPU.
 *
 * Shadowfax integrates one simulation per job; this server turns the flux
 * pass into a service.  Meshes are uploaded once into a device pool.  A
 * request (pool mesh, initial state, solver, dt, step count) is queued by
 * sfx_server_submit and admitted by the worker thread in arrival order while
 * the device-memory budget and the slot count allow: its state lives in an
 * instance on the pool mesh's geometry (sfx_mesh_clone) and stays resident
 * until it finishes.  Each scheduling round advances every admitted request
 * by up to `chunk_steps` steps:
 *   SFX_PREC_SPLIT  all requests of one (dimension, solver) class share one
 *                   launch group (one launch per phase for all of them, a
 *                   CUDA graph once the membership holds for a round);
 *                   per-request step counters live on the device, so a
 *                   request that finishes inside a round stops there while
 *                   the others go on;
 *   SFX_PREC_FP64   every request is stepped on its own (the per-request
 *                   baseline).
 * The classes run on their own streams and overlap on the device.  Requests
 * that arrive while a round runs join at the next round.
 *
 * The worker keeps the GPU busy between rounds: finished requests are copied
 * out on a separate stream into pinned buffers while the next round runs,
 * and their host-side transposes happen then too; instances of finished
 * requests are kept per (pool mesh, solver) and reused by later requests,
 * and launch groups keep their device tables, so a round in steady state
 * allocates and frees no device memory (cudaFree would wait for the whole
 * device).  Results wait in host memory until sfx_server_poll collects them.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "sfx_internal.h"

namespace {

/* pinned host staging for the asynchronous copies: one fixed block used as
 * a bump allocator and emptied once every copy it holds has completed
 * (cudaHostAlloc costs milliseconds per call, far more than the copies) */
struct Ring {
    uint8_t* base = nullptr;
    size_t cap = 0, used = 0;
    double* take(size_t n_doubles) {
        const size_t b = (n_doubles * sizeof(double) + 255) & ~(size_t)255;
        if(!base || used + b > cap) return nullptr;
        double* p = (double*)(base + used);
        used += b;
        return p;
    }
};
constexpr size_t kRingBytes = (size_t)256 << 20;

struct Request {
    int64_t id = 0;
    int32_t admit_status = SFX_OK;
    int32_t mesh_id = 0, solver = 0, nsteps = 0;
    double dt = 0.;
    std::vector<double> W0; /* field-major [S][n], transposed at submit */
    std::vector<double> W, Q;
    double t_submit = 0., t_admit = 0., t_done = 0.;
    int32_t status = SFX_OK, steps_done = 0;
    int64_t face_steps = 0;
    bool done = false;
    sfx_mesh* inst = nullptr;
    int64_t bytes = 0;
    int32_t remaining = 0;
    int32_t chunk = 0; /* steps launched this round (FP64 mode) */
    double* stage = nullptr; /* pinned staging of the copy in flight */
    bool stage_own = false;  /* staging allocated for this request alone */
};

struct PoolMesh {
    sfx_mesh* mesh = nullptr;
    int dim = 0, S = 0;
    int32_t n_cells = 0;
    int64_t active_faces = 0;
    int64_t clone_bytes = 0;
    std::vector<sfx_mesh*> cache[2]; /* idle instances per solver */
};

/* kernel settings of a class's launch group (sfx_server_set_tuning) */
struct Tuning {
    int32_t dim = 2;
    int32_t lanes = 0; /* 0: the library's default */
    int32_t face_variant = 0;
};

struct Class {
    sfx_ctx* ctx = nullptr;
    std::vector<Request*> members;
    sfx_group* group = nullptr;
    bool dirty = false;
    int reused = 0; /* rounds the current membership has run */
    std::atomic<int> tune_gen{0}; /* bumped by sfx_server_set_tuning */
    int applied_gen = 0;          /* worker thread: the tuning the group has */
    int applied_lanes = 0;        /* worker thread: lanes the group runs, 0: its default */
    Tuning tune;                  /* under sfx_server::mu */
};

}  // namespace

struct sfx_server {
    sfx_server_config cfg;
    sfx_ctx* pool_ctx[2] = {nullptr, nullptr};
    Class cls[2][2]; /* [dim - 2][solver] */
    std::vector<std::unique_ptr<PoolMesh>> pool;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<int64_t, Request*> reqs;
    int64_t next_id = 1;
    int64_t n_submitted = 0, n_admitted = 0, n_completed = 0, n_failed = 0;
    int64_t face_steps = 0, rounds = 0;
    int64_t bytes_in_use = 0; /* instances of admitted requests */
    int64_t bytes_cached = 0; /* idle instances kept for reuse */
    int active = 0;
    bool stop = false;
    double worker_s[4] = {0., 0., 0., 0.}; /* admit, launch, finish, collect */
    std::thread worker;
    std::chrono::steady_clock::time_point t0;
    /* worker thread only */
    cudaStream_t copy_stream = nullptr; /* results out */
    cudaStream_t up_stream = nullptr;   /* admitted states in */
    Ring up, down; /* staging of admitted states and of results */
    std::vector<Request*> leaving;  /* results being copied out */
    std::vector<Request*> arriving; /* admitted, states being copied in */
};

namespace {

double now_s(const sfx_server* s) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

sfx_config make_cfg(const sfx_server* s, int dim, int solver) {
    sfx_config c;
    std::memset(&c, 0, sizeof c);
    c.dim = dim;
    c.solver = solver;
    c.gamma = s->cfg.gamma;
    c.tolerance = s->cfg.tolerance;
    c.cutoff = s->cfg.cutoff;
    c.precision = s->cfg.precision;
    c.device = s->cfg.device;
    return c;
}

/* staging for n doubles: from the ring, or (larger than the ring) a block of
 * its own */
double* stage_take(Ring& ring, size_t n, bool* own) {
    *own = false;
    if(double* p = ring.take(n)) return p;
    if(ring.used > 0) return nullptr;
    double* p = nullptr;
    if(cudaHostAlloc((void**)&p, n * sizeof(double), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    *own = true;
    return p;
}

void stage_release(Request* r) {
    if(r->stage_own && r->stage) cudaFreeHost(r->stage);
    r->stage = nullptr;
    r->stage_own = false;
}

void finish_leaving(sfx_server* s);

/* bookkeeping of a request that has left the device (worker thread) */
void mark_done(sfx_server* s, Request* r, int status) {
    PoolMesh* pm;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        pm = s->pool[r->mesh_id].get();
    }
    r->steps_done = r->nsteps - r->remaining;
    r->face_steps = (int64_t)r->steps_done * pm->active_faces;
    r->status = status;
    r->t_done = now_s(s);
    std::lock_guard<std::mutex> lk(s->mu);
    s->active -= 1;
    r->done = true;
    if(status == SFX_OK) {
        s->n_completed += 1;
        s->face_steps += r->face_steps;
    } else {
        s->n_failed += 1;
    }
    s->cv_done.notify_all();
}

/* the instance goes back to its pool mesh's cache */
void release_instance(sfx_server* s, Request* r) {
    if(!r->inst) return;
    PoolMesh* pm;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        pm = s->pool[r->mesh_id].get();
        s->bytes_in_use -= r->bytes;
        s->bytes_cached += r->bytes;
    }
    pm->cache[r->solver].push_back(r->inst);
    r->inst = nullptr;
}

/* a request leaves the device: its final state is copied out on the copy
 * stream (the class stream has finished with it); finish_leaving completes
 * it after the next round has been launched */
void leave(sfx_server* s, Request* r, int status) {
    r->status = status;
    if(r->inst) {
        const size_t n = (size_t)sfx_mesh_dev(r->inst)->n_cells * sfx_mesh_dev(r->inst)->S;
        r->stage = stage_take(s->down, 2 * n, &r->stage_own);
        if(!r->stage) {
            /* the ring is full: complete the results already in it first */
            finish_leaving(s);
            r->stage = stage_take(s->down, 2 * n, &r->stage_own);
        }
        if(r->stage) {
            const int rc = sfx_mesh_download_fieldmajor_async(r->inst, r->stage, r->stage + n,
                                                              s->copy_stream);
            if(rc && r->status == SFX_OK) r->status = rc;
        } else if(r->status == SFX_OK) {
            r->status = SFX_ERR_NOMEM;
        }
    }
    s->leaving.push_back(r);
}

void finish_leaving(sfx_server* s) {
    if(s->leaving.empty()) return;
    const bool copy_ok = cudaStreamSynchronize(s->copy_stream) == cudaSuccess;
    for(Request* r : s->leaving) {
        int status = r->status;
        if(r->inst && r->stage) {
            if(!copy_ok && status == SFX_OK) status = SFX_ERR_CUDA;
            const sfx_dmesh* d = sfx_mesh_dev(r->inst);
            const int64_t n = d->n_cells;
            const int S = d->S;
            r->W.resize((size_t)n * S);
            r->Q.resize((size_t)n * S);
            const double* w = r->stage;
            const double* q = r->stage + (size_t)n * S;
            for(int64_t i = 0; i < n; ++i)
                for(int k = 0; k < S; ++k) {
                    r->W[(size_t)i * S + k] = w[(size_t)k * n + i];
                    r->Q[(size_t)i * S + k] = q[(size_t)k * n + i];
                }
        }
        stage_release(r);
        release_instance(s, r);
        mark_done(s, r, status);
    }
    s->leaving.clear();
    s->down.used = 0;
}

/* free cached instances until `need` more bytes fit the budget (waits for
 * the device; only when the budget is tight) */
bool make_room(sfx_server* s, int64_t need) {
    for(auto& pm : s->pool)
        for(auto& cache : pm->cache)
            while(!cache.empty()) {
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    if(s->bytes_in_use + s->bytes_cached + need <= s->cfg.memory_budget)
                        return true;
                    s->bytes_cached -= pm->clone_bytes;
                }
                sfx_mesh_free(cache.back());
                cache.pop_back();
            }
    std::lock_guard<std::mutex> lk(s->mu);
    return s->bytes_in_use + s->bytes_cached + need <= s->cfg.memory_budget;
}

/* admit queued requests in arrival order while budget and slots allow: take
 * an instance (cached, or a new clone) and start copying the state in on the
 * upload stream; join_arrivals adds them to their classes once it has run.
 * Called while a round runs, so the host work overlaps the GPU. */
void admit(sfx_server* s) {
    for(;;) {
        Request* r;
        PoolMesh* pm;
        bool reuse;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if(s->stop || s->queue.empty() || s->active >= s->cfg.max_active) return;
            r = s->queue.front();
            pm = s->pool[r->mesh_id].get();
            reuse = !pm->cache[r->solver].empty();
        }
        if(!reuse) {
            bool fits = make_room(s, pm->clone_bytes);
            std::lock_guard<std::mutex> lk(s->mu);
            /* one request is always admitted when nothing runs */
            if(!fits && s->active > 0) return;
        }
        /* staging for the state; a full ring waits for the next round */
        r->stage = stage_take(s->up, r->W0.size(), &r->stage_own);
        if(!r->stage && s->up.used > 0) return;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->queue.pop_front();
            s->bytes_in_use += pm->clone_bytes;
            if(reuse) s->bytes_cached -= pm->clone_bytes;
            s->active += 1;
            s->n_admitted += 1;
        }
        r->bytes = pm->clone_bytes;
        r->remaining = r->nsteps;
        r->t_admit = now_s(s);
        Class& c = s->cls[pm->dim - 2][r->solver];
        int rc = SFX_OK;
        if(reuse) {
            r->inst = pm->cache[r->solver].back();
            pm->cache[r->solver].pop_back();
        } else {
            rc = sfx_mesh_clone_async(c.ctx, pm->mesh, s->up_stream, &r->inst);
            if(rc) {
                r->inst = nullptr;
                std::lock_guard<std::mutex> lk(s->mu);
                s->bytes_in_use -= r->bytes;
            }
        }
        if(!rc) {
            if(r->stage) {
                std::memcpy(r->stage, r->W0.data(), r->W0.size() * sizeof(double));
                rc = sfx_mesh_upload_W_fieldmajor_async(r->inst, r->stage, s->up_stream);
            } else {
                rc = SFX_ERR_NOMEM;
            }
        }
        std::vector<double>().swap(r->W0);
        r->admit_status = rc;
        s->arriving.push_back(r);
    }
}

/* admitted requests whose states have arrived join their classes */
void join_arrivals(sfx_server* s) {
    if(s->arriving.empty()) return;
    const bool up_ok = cudaStreamSynchronize(s->up_stream) == cudaSuccess;
    for(Request* r : s->arriving) {
        stage_release(r);
        int rc = r->admit_status;
        if(!rc && !up_ok) rc = SFX_ERR_CUDA;
        if(!rc) {
            int32_t bad = -1;
            rc = sfx_mesh_last_status(r->inst, &bad);
        }
        if(rc || r->nsteps == 0) {
            leave(s, r, rc);
            continue;
        }
        PoolMesh* pm;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            pm = s->pool[r->mesh_id].get();
        }
        Class& c = s->cls[pm->dim - 2][r->solver];
        c.members.push_back(r);
        c.dirty = true;
    }
    s->arriving.clear();
    s->up.used = 0;
}

int rebuild_group(sfx_server* s, Class& c);

int apply_tuning(sfx_server* s, Class& c) {
    const int gen = c.tune_gen.load();
    if(!c.group || gen == c.applied_gen) return SFX_OK;
    Tuning t;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        t = c.tune;
    }
    int rc = SFX_OK;
    if(t.lanes != c.applied_lanes) {
        /* 0 takes a group tuned before back to the library's default */
        rc = sfx_group_set_lanes(c.group, t.lanes ? t.lanes : sfx_default_lanes(t.dim));
        if(!rc) c.applied_lanes = t.lanes;
    }
    if(!rc) rc = sfx_group_set_face_variant(c.group, t.face_variant);
    c.applied_gen = gen;
    c.reused = 0; /* the captured graph holds the old kernels */
    return rc;
}

int rebuild_group(sfx_server* s, Class& c) {
    c.dirty = false;
    c.reused = 0;
    std::vector<sfx_mesh*> ms;
    std::vector<double> dts;
    std::vector<int32_t> steps;
    for(Request* r : c.members) {
        ms.push_back(r->inst);
        dts.push_back(r->dt);
        steps.push_back(r->remaining);
    }
    const int32_t n = (int32_t)ms.size();
    if(c.group) {
        const int rc = sfx_group_set_members(c.group, n, ms.data(), dts.data(), steps.data());
        return rc ? rc : apply_tuning(s, c);
    }
    int rc = sfx_group_create(c.ctx, n, ms.data(), dts.data(), &c.group);
    if(!rc) rc = sfx_group_set_steps(c.group, steps.data());
    c.applied_gen = 0;
    c.applied_lanes = 0; /* a new group runs the default lanes */
    if(!rc && c.tune_gen.load() != 0) {
        c.applied_gen = -1; /* a new group: apply whatever tuning there is */
        rc = apply_tuning(s, c);
    }
    return rc;
}

void fail_class(sfx_server* s, Class& c, int rc) {
    for(Request* r : c.members) leave(s, r, rc);
    c.members.clear();
    c.dirty = true;
}

void launch_split(sfx_server* s) {
    const int chunk = std::max(1, s->cfg.chunk_steps);
    for(auto& row : s->cls)
        for(Class& c : row) {
            if(c.members.empty()) continue;
            if(c.dirty || !c.group) {
                const int rc = rebuild_group(s, c);
                if(rc) {
                    fail_class(s, c, rc);
                    continue;
                }
            } else if(c.tune_gen.load() != c.applied_gen) {
                const int rc = apply_tuning(s, c);
                if(rc) {
                    fail_class(s, c, rc);
                    continue;
                }
            } else {
                c.reused += 1;
            }
            /* a membership that has held for a round is replayed as a graph */
            const int rc = sfx_group_step(c.group, chunk, c.reused > 0, nullptr);
            if(rc) fail_class(s, c, rc);
        }
}

void collect_split(sfx_server* s) {
    for(auto& row : s->cls)
        for(Class& c : row) {
            if(c.members.empty() || !c.group) continue;
            const size_t nm = c.members.size();
            std::vector<int32_t> left(nm), st(nm);
            int rc = sfx_group_get_steps(c.group, left.data());
            if(!rc) {
                const int rs = sfx_group_status(c.group, st.data());
                /* a member's failure comes back in st; other codes are the
                 * group's own */
                bool any = false;
                for(int32_t v : st) any = any || v != SFX_OK;
                if(rs && !any) rc = rs;
            }
            std::vector<Request*> keep;
            for(size_t i = 0; i < nm; ++i) {
                Request* r = c.members[i];
                if(rc) {
                    leave(s, r, rc);
                    continue;
                }
                r->remaining = left[i];
                if(st[i] != SFX_OK)
                    leave(s, r, st[i]);
                else if(left[i] == 0)
                    leave(s, r, SFX_OK);
                else
                    keep.push_back(r);
            }
            if(keep.size() != nm) c.dirty = true;
            c.members.swap(keep);
        }
}

void launch_fp64(sfx_server* s) {
    const int chunk = std::max(1, s->cfg.chunk_steps);
    for(auto& row : s->cls)
        for(Class& c : row)
            for(Request* r : c.members) {
                r->chunk = std::min(chunk, r->remaining);
                if(sfx_step(r->inst, r->dt, r->chunk, nullptr) != SFX_OK) r->chunk = -1;
            }
}

void collect_fp64(sfx_server* s) {
    for(auto& row : s->cls)
        for(Class& c : row) {
            if(c.members.empty()) continue;
            sfx_ctx_synchronize(c.ctx);
            std::vector<Request*> keep;
            for(Request* r : c.members) {
                int32_t bad = -1;
                const int st = r->chunk < 0 ? SFX_ERR_CUDA : sfx_mesh_last_status(r->inst, &bad);
                if(r->chunk > 0) r->remaining -= r->chunk;
                if(st != SFX_OK)
                    leave(s, r, st);
                else if(r->remaining == 0)
                    leave(s, r, SFX_OK);
                else
                    keep.push_back(r);
            }
            c.members.swap(keep);
        }
}

void worker_main(sfx_server* s) {
    cudaSetDevice(s->cfg.device);
    const bool split = s->cfg.precision == SFX_PREC_SPLIT;
    double tw[4] = {0., 0., 0., 0.};
    auto lap = [&](double& t0, int k) {
        const double t1 = now_s(s);
        tw[k] += t1 - t0;
        t0 = t1;
    };
    for(;;) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if(s->stop) break;
            for(int k = 0; k < 4; ++k) s->worker_s[k] = tw[k];
        }
        double t = now_s(s);
        bool any = false;
        for(auto& row : s->cls)
            for(Class& c : row) any = any || !c.members.empty();
        /* launch the round first; admissions and finished results are
         * handled while it runs */
        if(any) {
            if(split)
                launch_split(s);
            else
                launch_fp64(s);
        }
        lap(t, 1);
        admit(s);
        lap(t, 0);
        finish_leaving(s);
        lap(t, 2);
        if(any) {
            if(split)
                collect_split(s);
            else
                collect_fp64(s);
        }
        lap(t, 3);
        join_arrivals(s);
        lap(t, 0);
        if(any) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->rounds += 1;
            continue;
        }
        bool more = !s->leaving.empty();
        for(auto& row : s->cls)
            for(Class& c : row) more = more || !c.members.empty();
        if(more) continue;
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_work.wait_for(lk, std::chrono::milliseconds(20),
                            [&] { return s->stop || !s->queue.empty(); });
    }
    finish_leaving(s);
    join_arrivals(s);
    finish_leaving(s);
}

}  // namespace

extern "C" int sfx_server_create(const sfx_server_config* cfg, sfx_server** out) {
    if(!cfg || !out) return SFX_ERR_INVALID;
    *out = nullptr;
    if(cfg->precision != SFX_PREC_SPLIT && cfg->precision != SFX_PREC_FP64) return SFX_ERR_INVALID;
    if(cfg->max_active <= 0 || cfg->memory_budget <= 0 || cfg->chunk_steps <= 0)
        return SFX_ERR_INVALID;
    sfx_server* s = new(std::nothrow) sfx_server;
    if(!s) return SFX_ERR_NOMEM;
    s->cfg = *cfg;
    s->t0 = std::chrono::steady_clock::now();
    int rc = cudaSetDevice(cfg->device) == cudaSuccess ? SFX_OK : SFX_ERR_CUDA;
    if(!rc && cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = SFX_ERR_CUDA;
    if(!rc && cudaStreamCreateWithFlags(&s->up_stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = SFX_ERR_CUDA;
    for(Ring* g : {&s->up, &s->down}) {
        if(rc) break;
        if(cudaHostAlloc((void**)&g->base, kRingBytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            g->base = nullptr;
            rc = SFX_ERR_NOMEM;
        } else {
            g->cap = kRingBytes;
        }
    }
    for(int d = 0; d < 2 && !rc; ++d) {
        sfx_config pc = make_cfg(s, d + 2, SFX_SOLVER_HLLC);
        rc = sfx_ctx_create(&pc, &s->pool_ctx[d]);
        for(int k = 0; k < 2 && !rc; ++k) {
            sfx_config cc = make_cfg(s, d + 2, k);
            rc = sfx_ctx_create(&cc, &s->cls[d][k].ctx);
        }
    }
    if(rc) {
        sfx_server_shutdown(s);
        return rc;
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return SFX_OK;
}

extern "C" int sfx_server_set_tuning(sfx_server* s, int32_t dim, int32_t solver, int32_t lanes,
                                     int32_t face_variant) {
    if(!s || (dim != 2 && dim != 3) ||
       (solver != SFX_SOLVER_EXACT && solver != SFX_SOLVER_HLLC) ||
       (lanes != 0 && lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16) ||
       face_variant < 0 || face_variant >= SFX_FACE_VARIANTS)
        return SFX_ERR_INVALID;
    if(s->cfg.precision != SFX_PREC_SPLIT) return SFX_ERR_UNSUPPORTED;
    Class& c = s->cls[dim - 2][solver];
    {
        std::lock_guard<std::mutex> lk(s->mu);
        c.tune.dim = dim;
        c.tune.lanes = lanes;
        c.tune.face_variant = face_variant;
    }
    c.tune_gen.fetch_add(1); /* the worker applies it before the class's next round */
    return SFX_OK;
}

extern "C" int sfx_server_add_mesh(sfx_server* s, const sfx_mesh_desc* desc, int32_t* mesh_id) {
    if(!s || !desc || !mesh_id) return SFX_ERR_INVALID;
    if(desc->dim != 2 && desc->dim != 3) return SFX_ERR_INVALID;
    std::unique_ptr<PoolMesh> pm(new(std::nothrow) PoolMesh);
    if(!pm) return SFX_ERR_NOMEM;
    int rc = sfx_mesh_upload(s->pool_ctx[desc->dim - 2], desc, &pm->mesh);
    if(rc) return rc;
    pm->dim = desc->dim;
    pm->S = desc->dim + 2;
    pm->n_cells = desc->n_cells;
    for(int32_t f = 0; f < desc->n_faces; ++f) pm->active_faces += desc->face_area[f] != 0.;
    pm->clone_bytes = sfx_mesh_clone_bytes(pm->mesh, s->cfg.precision);
    std::lock_guard<std::mutex> lk(s->mu);
    *mesh_id = (int32_t)s->pool.size();
    s->pool.push_back(std::move(pm));
    return SFX_OK;
}

extern "C" int sfx_server_submit(sfx_server* s, int32_t mesh_id, const double* W0,
                                 int32_t solver, double dt, int32_t nsteps,
                                 int64_t* request_id) {
    if(!s || !W0 || !request_id || nsteps < 0 || !(dt > 0.)) return SFX_ERR_INVALID;
    if(solver != SFX_SOLVER_EXACT && solver != SFX_SOLVER_HLLC) return SFX_ERR_UNSUPPORTED;
    Request* r = new(std::nothrow) Request;
    if(!r) return SFX_ERR_NOMEM;
    int64_t n;
    int S;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if(s->stop) {
            delete r;
            return SFX_ERR_CLOSED;
        }
        if(mesh_id < 0 || mesh_id >= (int32_t)s->pool.size()) {
            delete r;
            return SFX_ERR_INVALID;
        }
        n = s->pool[mesh_id]->n_cells;
        S = s->pool[mesh_id]->S;
    }
    /* the device layout, transposed here on the caller's thread */
    r->W0.resize((size_t)n * S);
    for(int64_t i = 0; i < n; ++i)
        for(int k = 0; k < S; ++k) r->W0[(size_t)k * n + i] = W0[(size_t)i * S + k];
    r->mesh_id = mesh_id;
    r->solver = solver;
    r->dt = dt;
    r->nsteps = nsteps;
    r->t_submit = now_s(s);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        s->queue.push_back(r);
        s->n_submitted += 1;
        *request_id = r->id;
    }
    s->cv_work.notify_one();
    return SFX_OK;
}

extern "C" int sfx_server_poll(sfx_server* s, int64_t id, double* W, double* Q,
                               sfx_request_info* info) {
    if(!s) return SFX_ERR_INVALID;
    Request* r;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if(it == s->reqs.end()) return SFX_ERR_INVALID;
        r = it->second;
        if(!r->done) return SFX_ERR_NOT_READY;
        s->reqs.erase(it);
    }
    if(W && !r->W.empty()) std::memcpy(W, r->W.data(), r->W.size() * sizeof(double));
    if(Q && !r->Q.empty()) std::memcpy(Q, r->Q.data(), r->Q.size() * sizeof(double));
    if(info) {
        info->status = r->status;
        info->steps_done = r->steps_done;
        info->mesh_id = r->mesh_id;
        info->solver = r->solver;
        info->t_submit = r->t_submit;
        info->t_admit = r->t_admit;
        info->t_done = r->t_done;
        info->face_steps = r->face_steps;
    }
    const int st = r->status;
    delete r;
    return st;
}

extern "C" int sfx_server_drain(sfx_server* s, double timeout_s) {
    if(!s) return SFX_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto idle = [&] { return s->queue.empty() && s->active == 0; };
    if(timeout_s <= 0.) {
        s->cv_done.wait(lk, idle);
        return SFX_OK;
    }
    return s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), idle)
                   ? SFX_OK
                   : SFX_ERR_NOT_READY;
}

extern "C" int sfx_server_stats_get(sfx_server* s, sfx_server_stats* st) {
    if(!s || !st) return SFX_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    st->submitted = s->n_submitted;
    st->admitted = s->n_admitted;
    st->completed = s->n_completed;
    st->failed = s->n_failed;
    st->active = s->active;
    st->queued = (int64_t)s->queue.size();
    st->face_steps = s->face_steps;
    st->bytes_in_use = s->bytes_in_use;
    st->rounds = s->rounds;
    st->now = now_s(s);
    for(int k = 0; k < 4; ++k) st->worker_s[k] = s->worker_s[k];
    return SFX_OK;
}

extern "C" int sfx_server_shutdown(sfx_server* s) {
    if(!s) return SFX_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if(s->worker.joinable()) s->worker.join();
    for(auto& row : s->cls)
        for(Class& c : row) {
            if(c.group) sfx_group_free(c.group);
            c.group = nullptr;
            for(Request* r : c.members)
                if(r->inst) {
                    sfx_mesh_free(r->inst);
                    r->inst = nullptr;
                }
            c.members.clear();
        }
    for(auto& kv : s->reqs) {
        if(kv.second->inst) sfx_mesh_free(kv.second->inst);
        stage_release(kv.second);
        delete kv.second;
    }
    s->reqs.clear();
    for(auto& pm : s->pool) {
        for(auto& cache : pm->cache)
            for(sfx_mesh* m : cache) sfx_mesh_free(m);
        if(pm->mesh) sfx_mesh_free(pm->mesh);
    }
    s->pool.clear();
    for(Ring* g : {&s->up, &s->down})
        if(g->base) cudaFreeHost(g->base);
    for(auto& row : s->cls)
        for(Class& c : row)
            if(c.ctx) sfx_ctx_destroy(c.ctx);
    for(sfx_ctx* c : s->pool_ctx)
        if(c) sfx_ctx_destroy(c);
    if(s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if(s->up_stream) cudaStreamDestroy(s->up_stream);
    delete s;
    return SFX_OK;
}
