/*
 * Launch groups: many independent meshes advanced with one launch per phase.
 *
 * The group keeps, in device memory, a table with each member mesh's device
 * view and time step, and per phase the prefix sum of thread blocks over the
 * members.  A step is three launches (gradients, faces, update) for all
 * members together, optionally captured in a CUDA graph, so small meshes share
 * the GPU instead of each paying its own launch latency and leaving most SMs
 * idle.  The per-mesh error records stay separate: a failing member stops
 * only itself, and its status is reported per mesh.
 */
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <vector>

#include "sfx_internal.h"

struct sfx_group {
    sfx_ctx* ctx = nullptr;
    std::vector<sfx_mesh*> meshes;
    std::vector<sfx_group_entry> host_tab;
    sfx_group_dev dev{};
    sfx_dev_error* d_err_out = nullptr;
    int32_t* d_steps = nullptr; /* per-member step counters (after set_steps) */
    cudaGraphExec_t graph = nullptr;
    int graph_steps = -1;
    int cap = 0; /* members the device buffers hold */
};

namespace {

int cuda_ok(cudaError_t e) {
    if(e == cudaSuccess) return SFX_OK;
    cudaGetLastError();
    return SFX_ERR_CUDA;
}

void drop_graph(sfx_group* g) {
    if(g->graph) cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
    g->graph_steps = -1;
}

/* block prefix sums for the current lanes-per-cell and upload of the table */
int upload_layout(sfx_group* g) {
    const int nm = (int)g->meshes.size();
    std::vector<int32_t> pre(3 * (nm + 1), 0);
    for(int mi = 0; mi < nm; ++mi) {
        const sfx_dmesh& d = g->host_tab[mi].m;
        int32_t b[3];
        sfx_split_blocks(d.dim, g->dev.lanes, d.n_cells, d.n_faces, b);
        for(int p = 0; p < 3; ++p) {
            const long long next = (long long)pre[p * (nm + 1) + mi] + b[p];
            if(next > 0x7fffffffLL) return SFX_ERR_TOO_LARGE;
            pre[p * (nm + 1) + mi + 1] = (int32_t)next;
        }
    }
    for(int p = 0; p < 3; ++p) g->dev.blocks[p] = pre[p * (nm + 1) + nm];
    cudaStream_t s = (cudaStream_t)sfx_ctx_stream(g->ctx);
    int rc = cuda_ok(cudaMemcpyAsync(g->dev.pre, pre.data(), sizeof(int32_t) * pre.size(),
                                     cudaMemcpyHostToDevice, s));
    if(!rc)
        rc = cuda_ok(cudaMemcpyAsync(g->dev.tab, g->host_tab.data(),
                                     sizeof(sfx_group_entry) * nm, cudaMemcpyHostToDevice, s));
    if(!rc) rc = cuda_ok(cudaStreamSynchronize(s));
    drop_graph(g);
    return rc;
}

int run_steps(sfx_group* g, int nsteps, cudaStream_t s) {
    const sfx_solver_params* sp = sfx_ctx_params(g->ctx);
    for(int t = 0; t < nsteps; ++t) {
        for(int ph = 0; ph < 3; ++ph) {
            int rc = sfx_split_group_phase(&g->dev, ph, sp, s);
            if(rc) return rc;
        }
        if(g->d_steps) {
            int rc = sfx_split_group_tick(&g->dev, s);
            if(rc) return rc;
        }
    }
    return SFX_OK;
}

/* device buffers for at least n members (contents are not kept) */
int reserve(sfx_group* g, int n) {
    if(n <= g->cap) return SFX_OK;
    const int cap = n > 2 * g->cap ? n : 2 * g->cap;
    if(g->dev.tab) cudaFree(g->dev.tab);
    if(g->dev.pre) cudaFree(g->dev.pre);
    if(g->d_err_out) cudaFree(g->d_err_out);
    if(g->d_steps) cudaFree(g->d_steps);
    g->dev.tab = nullptr;
    g->dev.pre = nullptr;
    g->d_err_out = nullptr;
    g->d_steps = nullptr;
    g->cap = 0;
    int rc = cuda_ok(cudaMalloc((void**)&g->dev.tab, sizeof(sfx_group_entry) * cap));
    if(!rc) rc = cuda_ok(cudaMalloc((void**)&g->dev.pre, sizeof(int32_t) * 3 * (cap + 1)));
    if(!rc) rc = cuda_ok(cudaMalloc((void**)&g->d_err_out, sizeof(sfx_dev_error) * cap));
    if(!rc) g->cap = cap;
    return rc;
}

bool same_config(const sfx_config* a, const sfx_config* b) {
    return a->dim == b->dim && a->solver == b->solver && a->precision == b->precision &&
           a->gamma == b->gamma && a->tolerance == b->tolerance && a->cutoff == b->cutoff &&
           a->device == b->device;
}

}  // namespace

extern "C" int sfx_group_create(sfx_ctx* ctx, int32_t n, sfx_mesh* const* meshes,
                                const double* dt, sfx_group** out) {
    if(!ctx || !meshes || !dt || !out || n <= 0) return SFX_ERR_INVALID;
    *out = nullptr;
    const sfx_config* cfg = sfx_ctx_config(ctx);
    if(cfg->precision != SFX_PREC_SPLIT) return SFX_ERR_UNSUPPORTED;
    for(int i = 0; i < n; ++i) {
        if(!meshes[i] || !(dt[i] > 0.)) return SFX_ERR_INVALID;
        if(!same_config(sfx_ctx_config(sfx_mesh_ctx(meshes[i])), cfg)) return SFX_ERR_INVALID;
    }
    sfx_group* g = new(std::nothrow) sfx_group;
    if(!g) return SFX_ERR_NOMEM;
    g->ctx = ctx;
    g->meshes.assign(meshes, meshes + n);
    g->host_tab.resize(n);
    for(int i = 0; i < n; ++i) {
        std::memset(&g->host_tab[i], 0, sizeof(sfx_group_entry));
        g->host_tab[i].m = *sfx_mesh_dev(meshes[i]);
        g->host_tab[i].dt = (float)dt[i];
    }
    g->dev.n_meshes = n;
    g->dev.dim = cfg->dim;
    g->dev.lanes = sfx_default_lanes(cfg->dim);
    int rc = cuda_ok(cudaSetDevice(cfg->device));
    if(!rc) rc = reserve(g, n);
    if(!rc) rc = upload_layout(g);
    if(rc) {
        sfx_group_free(g);
        return rc;
    }
    *out = g;
    return SFX_OK;
}

extern "C" int sfx_group_set_dt(sfx_group* g, const double* dt) {
    if(!g || !dt) return SFX_ERR_INVALID;
    for(size_t i = 0; i < g->meshes.size(); ++i) {
        if(!(dt[i] > 0.)) return SFX_ERR_INVALID;
        g->host_tab[i].dt = (float)dt[i];
    }
    return upload_layout(g);
}

extern "C" int sfx_group_set_face_variant(sfx_group* g, int32_t variant) {
    if(!g || variant < 0 || variant >= SFX_FACE_VARIANTS) return SFX_ERR_INVALID;
    g->dev.face_variant = variant;
    drop_graph(g); /* a captured step holds the old kernel */
    return SFX_OK;
}

extern "C" int sfx_group_set_lanes(sfx_group* g, int32_t lanes) {
    if(!g || (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16))
        return SFX_ERR_INVALID;
    g->dev.lanes = lanes;
    return upload_layout(g);
}

extern "C" int sfx_group_step(sfx_group* g, int32_t nsteps, int32_t use_graph,
                              int32_t* mesh_status) {
    if(!g || nsteps < 0) return SFX_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)sfx_ctx_stream(g->ctx);
    int rc = sfx_split_group_reset(&g->dev, s);
    if(rc) return rc;
    if(use_graph && nsteps > 0) {
        if(!g->graph || g->graph_steps != nsteps) {
            drop_graph(g);
            cudaGraph_t graph = nullptr;
            rc = cuda_ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            if(rc) return rc;
            sfx_launch_capture(true);
            const int rr = run_steps(g, nsteps, s);
            sfx_launch_capture(false);
            rc = cuda_ok(cudaStreamEndCapture(s, &graph));
            if(!rc && rr) rc = rr;
            if(!rc) rc = cuda_ok(cudaGraphInstantiate(&g->graph, graph, 0));
            if(graph) cudaGraphDestroy(graph);
            if(rc) {
                drop_graph(g);
                return rc;
            }
            g->graph_steps = nsteps;
        }
        rc = cuda_ok(cudaGraphLaunch(g->graph, s));
        if(!rc) {
            int per_step = g->d_steps ? 1 : 0;
            for(int p = 0; p < 3; ++p) per_step += g->dev.blocks[p] > 0;
            /* the queued faces (both solvers: the exact solver's refused
             * faces, HLLC's non-finite FP32 fluxes) */
            if(g->dev.blocks[1] > 0) per_step += 1;
            sfx_count_launches(per_step * nsteps);
        }
    } else {
        rc = run_steps(g, nsteps, s);
    }
    if(rc) return rc;
    if(!mesh_status) return SFX_OK;
    const int nm = g->dev.n_meshes;
    std::vector<sfx_dev_error> e(nm);
    rc = sfx_split_group_collect(&g->dev, g->d_err_out, s);
    if(!rc)
        rc = cuda_ok(cudaMemcpyAsync(e.data(), g->d_err_out, sizeof(sfx_dev_error) * nm,
                                     cudaMemcpyDeviceToHost, s));
    if(!rc) rc = cuda_ok(cudaStreamSynchronize(s));
    if(rc) return rc;
    int first = SFX_OK;
    for(int i = 0; i < nm; ++i) {
        int st = SFX_OK;
        if(e[i].face_key != ~0ull)
            st = (int)(e[i].face_key & 0xff);
        else if(e[i].cell_key != ~0ull)
            st = (int)(e[i].cell_key & 0xff);
        mesh_status[i] = st;
        if(st && !first) first = st;
    }
    return first;
}

extern "C" int sfx_group_step_timed(sfx_group* g, int32_t nsteps, float* phase_ms,
                                    int32_t* launches) {
    if(!g || nsteps < 0 || !phase_ms) return SFX_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)sfx_ctx_stream(g->ctx);
    const sfx_solver_params* sp = sfx_ctx_params(g->ctx);
    cudaEvent_t ev[4];
    int made = 0;
    int rc = SFX_OK;
    for(; made < 4 && !rc; ++made)
        if(cudaEventCreate(&ev[made]) != cudaSuccess) rc = SFX_ERR_CUDA;
    if(rc) made -= 1;
    double acc[3] = {0., 0., 0.};
    int nl = 0;
    if(!rc) rc = sfx_split_group_reset(&g->dev, s);
    for(int t = 0; t < nsteps && !rc; ++t) {
        for(int ph = 0; ph < 3 && !rc; ++ph) {
            cudaEventRecord(ev[ph], s);
            rc = sfx_split_group_phase(&g->dev, ph, sp, s);
            nl += 1;
        }
        cudaEventRecord(ev[3], s);
        if(!rc && g->d_steps) {
            rc = sfx_split_group_tick(&g->dev, s);
            nl += 1;
        }
        if(!rc) rc = cuda_ok(cudaEventSynchronize(ev[3]));
        for(int k = 0; k < 3 && !rc; ++k) {
            float ms = 0.f;
            rc = cuda_ok(cudaEventElapsedTime(&ms, ev[k], k < 2 ? ev[k + 1] : ev[3]));
            acc[k] += ms;
        }
    }
    if(!rc) rc = cuda_ok(cudaStreamSynchronize(s));
    for(int k = 0; k < made; ++k) cudaEventDestroy(ev[k]);
    for(int k = 0; k < 3; ++k) phase_ms[k] = (float)acc[k];
    if(launches) *launches = nl;
    return rc;
}

extern "C" int sfx_group_status(sfx_group* g, int32_t* mesh_status) {
    if(!g || !mesh_status) return SFX_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)sfx_ctx_stream(g->ctx);
    const int nm = g->dev.n_meshes;
    std::vector<sfx_dev_error> e(nm);
    int rc = sfx_split_group_collect(&g->dev, g->d_err_out, s);
    if(!rc)
        rc = cuda_ok(cudaMemcpyAsync(e.data(), g->d_err_out, sizeof(sfx_dev_error) * nm,
                                     cudaMemcpyDeviceToHost, s));
    if(!rc) rc = cuda_ok(cudaStreamSynchronize(s));
    if(rc) return rc;
    int first = SFX_OK;
    for(int i = 0; i < nm; ++i) {
        int st = SFX_OK;
        if(e[i].face_key != ~0ull)
            st = (int)(e[i].face_key & 0xff);
        else if(e[i].cell_key != ~0ull)
            st = (int)(e[i].cell_key & 0xff);
        mesh_status[i] = st;
        if(st && !first) first = st;
    }
    return first;
}

extern "C" int sfx_group_tune(sfx_group* g, int32_t reps, int32_t* lanes_out) {
    if(!g || reps <= 0) return SFX_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)sfx_ctx_stream(g->ctx);
    const sfx_solver_params* sp = sfx_ctx_params(g->ctx);
    cudaEvent_t e0, e1;
    if(cudaEventCreate(&e0) != cudaSuccess) return SFX_ERR_CUDA;
    if(cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return SFX_ERR_CUDA;
    }
    const int cand[5] = {1, 2, 4, 8, 16};
    int best = g->dev.lanes;
    float best_ms = 1e30f;
    int rc = SFX_OK;
    for(int c = 0; c < 5 && !rc; ++c) {
        rc = sfx_group_set_lanes(g, cand[c]);
        if(rc) break;
        /* timed on the gradient kernel, which only reads the states (the
         * update kernel shares the setting); one untimed launch, then reps */
        for(int r = 0; r <= reps && !rc; ++r) {
            if(r == 1) cudaEventRecord(e0, s);
            rc = sfx_split_group_phase(&g->dev, 0, sp, s);
        }
        cudaEventRecord(e1, s);
        if(!rc) rc = cuda_ok(cudaEventSynchronize(e1));
        float ms = 0.f;
        if(!rc) rc = cuda_ok(cudaEventElapsedTime(&ms, e0, e1));
        if(!rc && ms < best_ms) {
            best_ms = ms;
            best = cand[c];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int r2 = sfx_group_set_lanes(g, best);
    if(lanes_out) *lanes_out = best;
    return rc ? rc : r2;
}

extern "C" int sfx_group_tune_faces(sfx_group* g, int32_t reps, int32_t* variant_out) {
    if(!g || reps <= 0) return SFX_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)sfx_ctx_stream(g->ctx);
    const sfx_solver_params* sp = sfx_ctx_params(g->ctx);
    cudaEvent_t e0, e1;
    if(cudaEventCreate(&e0) != cudaSuccess) return SFX_ERR_CUDA;
    if(cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return SFX_ERR_CUDA;
    }
    int best = g->dev.face_variant;
    float best_ms = 1e30f;
    int rc = SFX_OK;
    bool timed[SFX_FACE_VARIANTS] = {};
    for(int v = 0; v < SFX_FACE_VARIANTS && !rc; ++v) {
        /* a variant that runs an already timed kernel is not timed again */
        const int k = sfx_split_face_variant_kernel(sp, v);
        if(timed[k]) continue;
        timed[k] = true;
        g->dev.face_variant = v;
        float total = 0.f;
        /* every face launch follows a gradient launch, which also empties
         * the queued-face lists; one untimed pair, then reps timed */
        for(int r = 0; r <= reps && !rc; ++r) {
            rc = sfx_split_group_phase(&g->dev, 0, sp, s);
            if(!rc) rc = cuda_ok(cudaEventRecord(e0, s));
            if(!rc) rc = sfx_split_group_phase(&g->dev, 1, sp, s);
            if(!rc) rc = cuda_ok(cudaEventRecord(e1, s));
            if(!rc) rc = cuda_ok(cudaEventSynchronize(e1));
            float ms = 0.f;
            if(!rc) rc = cuda_ok(cudaEventElapsedTime(&ms, e0, e1));
            if(r > 0) total += ms;
        }
        if(!rc && total < best_ms) {
            best_ms = total;
            best = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g->dev.face_variant = best;
    drop_graph(g);
    if(variant_out) *variant_out = best;
    return rc;
}

extern "C" int sfx_group_set_steps(sfx_group* g, const int32_t* steps) {
    if(!g || !steps) return SFX_ERR_INVALID;
    const int nm = g->dev.n_meshes;
    for(int i = 0; i < nm; ++i)
        if(steps[i] < 0) return SFX_ERR_INVALID;
    if(!g->d_steps) {
        int rc = cuda_ok(cudaMalloc((void**)&g->d_steps, sizeof(int32_t) * g->cap));
        if(rc) return rc;
    }
    for(int i = 0; i < nm; ++i) g->host_tab[i].steps_left = g->d_steps + i;
    cudaStream_t s = (cudaStream_t)sfx_ctx_stream(g->ctx);
    int rc = cuda_ok(cudaMemcpyAsync(g->d_steps, steps, sizeof(int32_t) * nm,
                                     cudaMemcpyHostToDevice, s));
    if(rc) return rc;
    return upload_layout(g); /* the table now points at the counters */
}

extern "C" int sfx_group_get_steps(sfx_group* g, int32_t* steps) {
    if(!g || !steps) return SFX_ERR_INVALID;
    if(!g->d_steps) return SFX_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)sfx_ctx_stream(g->ctx);
    int rc = cuda_ok(cudaMemcpyAsync(steps, g->d_steps, sizeof(int32_t) * g->dev.n_meshes,
                                     cudaMemcpyDeviceToHost, s));
    if(rc) return rc;
    return cuda_ok(cudaStreamSynchronize(s));
}

int sfx_group_set_members(sfx_group* g, int32_t n, sfx_mesh* const* meshes, const double* dt,
                          const int32_t* steps) {
    if(!g || n <= 0 || !meshes || !dt) return SFX_ERR_INVALID;
    const sfx_config* cfg = sfx_ctx_config(g->ctx);
    for(int i = 0; i < n; ++i) {
        if(!meshes[i] || !(dt[i] > 0.)) return SFX_ERR_INVALID;
        if(!same_config(sfx_ctx_config(sfx_mesh_ctx(meshes[i])), cfg)) return SFX_ERR_INVALID;
    }
    drop_graph(g);
    const bool had_steps = g->d_steps != nullptr;
    int rc = reserve(g, n);
    if(rc) return rc;
    g->meshes.assign(meshes, meshes + n);
    g->host_tab.assign(n, sfx_group_entry{});
    for(int i = 0; i < n; ++i) {
        std::memset(&g->host_tab[i], 0, sizeof(sfx_group_entry));
        g->host_tab[i].m = *sfx_mesh_dev(meshes[i]);
        g->host_tab[i].dt = (float)dt[i];
    }
    g->dev.n_meshes = n;
    if(steps || had_steps) {
        std::vector<int32_t> zero;
        if(!steps) zero.assign(n, 0);
        return sfx_group_set_steps(g, steps ? steps : zero.data());
    }
    return upload_layout(g);
}

extern "C" int sfx_group_free(sfx_group* g) {
    if(!g) return SFX_ERR_INVALID;
    drop_graph(g);
    if(g->d_steps) cudaFree(g->d_steps);
    if(g->dev.tab) cudaFree(g->dev.tab);
    if(g->dev.pre) cudaFree(g->dev.pre);
    if(g->d_err_out) cudaFree(g->d_err_out);
    delete g;
    return SFX_OK;
}
