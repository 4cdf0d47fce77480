/*
 * sfx_flux_pass_noalloc: one plain-FP64 flux pass (gradients + per-face dQ)
 * that allocates no device memory.
 *
 * Who needs it: applications that manage all device memory themselves (their
 * own pools, memory reserved up front) or that must not allocate while work
 * is in flight cannot let the library cudaMalloc a mesh.  They pass their own
 * device arrays in; the only scratch this pass needs, the per-cell gradients,
 * lives in the fixed array below.
 *
 * The array is a file-scope __device__ variable, so every GPU that loads the
 * library holds it (SFX_NOALLOC_MAX_CELLS x 15 doubles = 7.5 MiB) until the
 * process exits.  In host code its name is only a host-side stand-in, not a
 * device address: the address is looked up once per device context with
 * cudaGetSymbolAddress (on the first call made on that device, which should
 * therefore come before any stream capture) and passed to the kernels.  The
 * lookup is repeated when the device's context changes (after a
 * cudaDeviceReset the module is loaded again and the old address is gone);
 * the first call after such a reset should again come before any capture.
 * Every call reuses the array and overwrites all the gradients it reads, so
 * nothing but the error record has to be cleared; calls that overlap on the
 * GPU race on the array.
 */
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "sfx_internal.h"

namespace {

constexpr int kMaxDevices = 64;

/* gradients: [dim * S][n_cells] doubles, at most 3 * 5 per cell */
static __device__ __align__(256) double g_noalloc_grad[SFX_NOALLOC_MAX_CELLS * 15];
static __device__ __align__(256) sfx_dev_error g_noalloc_err;

std::mutex g_setup_mutex;
void* g_grad_addr[kMaxDevices];
void* g_err_addr[kMaxDevices];
unsigned long long g_ctx_id[kMaxDevices]; /* context the addresses belong to */

typedef CUresult (*ctx_current_fn)(CUcontext*);
typedef CUresult (*ctx_id_fn)(CUcontext, unsigned long long*);
ctx_current_fn g_ctx_current = nullptr;
ctx_id_fn g_ctx_get_id = nullptr;
std::once_flag g_ctx_fn_once;

/* the unique id of the calling thread's current context, 0 when there is
 * none or the driver cannot report it (then every call looks the addresses
 * up again) */
unsigned long long current_context_id() {
    std::call_once(g_ctx_fn_once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) ==
                   cudaSuccess &&
           q == cudaDriverEntryPointSuccess)
            g_ctx_current = (ctx_current_fn)f;
        f = nullptr;
        if(cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
           q == cudaDriverEntryPointSuccess)
            g_ctx_get_id = (ctx_id_fn)f;
        cudaGetLastError();
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if(!g_ctx_current || !g_ctx_get_id || g_ctx_current(&c) != CUDA_SUCCESS || !c ||
       g_ctx_get_id(c, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

/* per device, with that device current: device addresses of the arrays in
 * the current context */
int scratch_addresses(int dev, double** grad, sfx_dev_error** err) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long id = current_context_id();
    if(!g_grad_addr[dev] || id == 0 || id != g_ctx_id[dev]) {
        void* g = nullptr;
        void* e = nullptr;
        if(cudaGetSymbolAddress(&g, g_noalloc_grad) != cudaSuccess ||
           cudaGetSymbolAddress(&e, g_noalloc_err) != cudaSuccess) {
            cudaGetLastError();
            return SFX_ERR_CUDA;
        }
        g_err_addr[dev] = e;
        g_grad_addr[dev] = g;
        /* the lookup made the device's context current if it was not */
        g_ctx_id[dev] = current_context_id();
    }
    *grad = (double*)g_grad_addr[dev];
    *err = (sfx_dev_error*)g_err_addr[dev];
    return SFX_OK;
}

}  // namespace

extern "C" int sfx_flux_pass_noalloc(const sfx_device_mesh* dm, const sfx_config* cfg,
                                     double dt, const double* W, const double* Q,
                                     double* dQ_face, void* cuda_stream) {
    if(!dm || !cfg || !W || !Q || !dQ_face || !(dt > 0.)) return SFX_ERR_INVALID;
    if(dm->dim != 2 && dm->dim != 3) return SFX_ERR_INVALID;
    if(cfg->dim != dm->dim || !(cfg->gamma > 1.)) return SFX_ERR_INVALID;
    if(cfg->solver != SFX_SOLVER_EXACT && cfg->solver != SFX_SOLVER_HLLC)
        return SFX_ERR_UNSUPPORTED;
    if(dm->n_cells <= 0 || dm->n_faces < 0) return SFX_ERR_INVALID;
    if(dm->n_cells > SFX_NOALLOC_MAX_CELLS) return SFX_ERR_TOO_LARGE;
    if(!dm->cell_pos || !dm->cell_centroid || !dm->cell_volume || !dm->cell_total_area ||
       !dm->cell_face_offset || !dm->cell_face_entry ||
       (dm->n_faces && (!dm->face_area || !dm->face_midpoint || !dm->face_left ||
                        !dm->face_right || !dm->face_kind || !dm->face_right_pos)))
        return SFX_ERR_INVALID;
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return SFX_ERR_CUDA;
    }
    double* grad = nullptr;
    sfx_dev_error* err = nullptr;
    int rc = scratch_addresses(dev, &grad, &err);
    if(rc != SFX_OK) return rc;

    sfx_dmesh d;
    std::memset(&d, 0, sizeof d);
    d.dim = dm->dim;
    d.S = dm->dim + 2;
    d.n_cells = dm->n_cells;
    d.n_faces = dm->n_faces;
    d.pos = const_cast<double*>(dm->cell_pos);
    d.cen = const_cast<double*>(dm->cell_centroid);
    d.vol = const_cast<double*>(dm->cell_volume);
    d.tarea = const_cast<double*>(dm->cell_total_area);
    d.off = const_cast<int32_t*>(dm->cell_face_offset);
    d.idx = const_cast<int32_t*>(dm->cell_face_entry);
    d.W = const_cast<double*>(W);
    d.Q = const_cast<double*>(Q);
    d.grad = grad;
    d.area = const_cast<double*>(dm->face_area);
    d.mid = const_cast<double*>(dm->face_midpoint);
    d.left = const_cast<int32_t*>(dm->face_left);
    d.right = const_cast<int32_t*>(dm->face_right);
    d.kind = const_cast<int32_t*>(dm->face_kind);
    d.rpos = const_cast<double*>(dm->face_right_pos);
    d.vel = nullptr;
    d.dQf = dQ_face;
    d.err = err;

    sfx_solver_params sp;
    sfx_solver_params_init(&sp, cfg->solver, cfg->gamma, cfg->tolerance, cfg->cutoff);
    cudaStream_t s = (cudaStream_t)cuda_stream;
    /* the error record keeps the previous call's contents: clear it */
    if(cudaMemsetAsync(err, 0xff, sizeof(sfx_dev_error), s) != cudaSuccess) {
        cudaGetLastError();
        return SFX_ERR_CUDA;
    }
    rc = sfx_fp64_gradients(&d, s);
    if(rc == SFX_OK) rc = sfx_fp64_faces(&d, &sp, dt, 0, s);
    if(rc != SFX_OK) return rc;
    sfx_dev_error e;
    if(cudaMemcpyAsync(&e, err, sizeof e, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
       cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return SFX_ERR_CUDA;
    }
    if(e.face_key != ~0ull) return (int)(e.face_key & 0xff);
    if(e.cell_key != ~0ull) return (int)(e.cell_key & 0xff);
    return SFX_OK;
}
