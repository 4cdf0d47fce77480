/*
 * Internal declarations of the sfxflux library (not part of the C ABI).
 */
#ifndef SFX_INTERNAL_H
#define SFX_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "../../include/sfxflux.h"

/* hard cap on Newton and Brent iterations of the exact solver (the reference
 * has none; a face that reaches it reports SFX_ERR_NOCONV) */
#define SFX_MAX_ITER 1000

/* device error record.  Each key packs (index << 8) | status, and the
 * kernels take the minimum, so the record names the lowest failing face or
 * cell -- the one at which the reference's loops would have thrown. */
struct sfx_dev_error {
    unsigned long long face_key; /* ~0ull when no face failed */
    unsigned long long cell_key; /* ~0ull when no cell failed */
};

/* device-resident mesh in structure-of-arrays layout.  Field-major arrays:
 * W[k * n_cells + i] etc.  All pointers are device pointers. */
struct sfx_dmesh {
    int32_t dim, S;
    int32_t n_cells, n_faces;
    int64_t nnz;
    int32_t has_velocity;
    int32_t lanes; /* split pass: lanes per cell of the gradient/update kernels */
    int32_t face_variant; /* split pass: register cap of the face kernel (sfx_split.cu) */
    /* cells */
    double* pos;    /* [dim][n]  */
    double* cen;    /* [dim][n]  */
    double* vol;    /* [n]       */
    double* tarea;  /* [n]       */
    int32_t* off;   /* [n+1]     */
    int32_t* idx;   /* [nnz] face id | (1u << 31 if the cell is the right) */
    int32_t* aidx;  /* [nnz] the same entries in ascending face order per cell, the
                       order the plain-FP64 update sums them in; == idx when every
                       cell lists its faces that way */
    double* W;      /* [S][n]    */
    double* Q;      /* [S][n]    */
    double* grad;   /* [dim*S][n]: grad[(l*S + k)*n + i] = dW_k/dx_l       */
    /* faces */
    double* area;   /* [F]       */
    double* mid;    /* [dim][F]  */
    int32_t* left;  /* [F]       */
    int32_t* right; /* [F]       */
    int32_t* kind;  /* [F]       */
    double* rpos;   /* [dim][F]  */
    double* vel;    /* [dim][F] or NULL */
    double* dQf;    /* [S][F] scratch: limited dQ received by the left cell */
    /* plain-FP64 pass: the first gradient loop's terms as seen from each
     * face's left cell, [F][sfx_grad_term_stride(dim)] (the right cell of a
     * local face takes their negation).  NULL: one kernel computes the
     * gradients without it.  The array is dead between the gradient and the
     * face kernels, so dQf lives inside it. */
    double* gterm;
    int32_t gshare; /* every local face's right position equals its right cell's */
    /* one part of a mesh split over several devices (plain FP64): gradients
     * of cells [0, r_grad), fluxes of faces [0, r_flux), update of cells
     * [0, r_upd) (the owned cells, numbered first); ranged == 0: all */
    int32_t ranged, r_grad, r_flux, r_upd;
    int32_t* branch; /* [F] scratch or NULL */
    sfx_dev_error* err;
    double* totals_scratch; /* [S * 1024] */
    /* ---- FP32/FP64-split arrays (precision SFX_PREC_SPLIT only) ----
     * fg [2F] float4: {A, c0, c1, c2}, {r0, r1, r2, |r|} (2D: {A, c0, c1, r0},
     *     {r1, |r|, 0, 0}) with c = midpoint - (x_L + x_R)/2 and
     *     r = x_L - x_R (right generator at its image/mirror position),
     *     computed in FP64 and rounded once;
     * fi [F] int2: {L, R}; R = -1 mirror, R | 1<<30 periodic image;
     * fsh [F]: periodic image shift, 2 bits per axis (0, +1, -1 box);
     * cw [2n] float4 cell record {rho, v.., p | Q.m, total area ..};
     * cg [G*n] float4 gradients (G = 4 in 3D, 2 in 2D: 64 / 32 bytes, so a
     *     record never straddles more 32-byte sectors than it fills);
     * cdw [H*n] float4 dW/dt (the Euler Jacobian at the cell state times its
     *     gradients: the MUSCL-Hancock prediction every face of the cell
     *     shares), read by the exact solver's face kernels (H = 2 in 3D, 1 in 2D);
     * cx [n] float4 {x - centroid, volume};
     * an [dim][F] FP64 area vector A n (n from x_L to x_R), for the pressure
     *     force, so that the forces on a cell cancel to FP64 round-off in a
     *     uniform region;
     * dqm [F] float2 {mass, energy} and dqv [dim][F] FP64 momentum: the
     *     limited dQ received by the left cell. */
    float4* fg;
    int2* fi;
    uint8_t* fsh;
    float4* cw;
    float4* cg;
    float4* cdw;
    float4* cx;
    int32_t* nbe; /* [nnz] neighbour cell of each CSR entry (-1 mirror) */
    /* moving generators (plain FP64, sfx_step_moving; allocated on first
     * use): generator velocities [dim][n], drifted positions [dim][n] */
    double* vgen;
    double* newpos;
    /* local (hierarchical) time steps, plain FP64 (sfx_step_window): the
     * start and end of every cell's step on the integer timeline of 2^60
     * ticks spanning t_total; with `local` set a cell is active when its
     * start is t_now (gradients, fluxes of its faces) and gets get_W when its
     * end is t_next */
    uint64_t* tstart;
    uint64_t* tend;
    int32_t local;
    uint64_t t_now, t_next;
    double t_total;
    double* an;
    float2* dqm;
    double* dqv;
    /* exact solver, split pass: faces whose p* iteration falls back to
     * Brent's method are queued here by the face kernel (face ids; room for
     * every face; slowq_n counts them) and solved by a follow-up launch in
     * which every lane works on a queued face, instead of one lane of a warp
     * iterating while the other 31 wait.  The gradient kernel resets the
     * count each step. */
    int32_t* slowq;
    int32_t* slowq_n;
    int32_t slowq_cap;
};

#if defined(__CUDACC__)
#define SFX_RANGE_HD __host__ __device__ inline
#else
#define SFX_RANGE_HD inline
#endif
SFX_RANGE_HD int sfx_grad_cells(const sfx_dmesh& m) { return m.ranged ? m.r_grad : m.n_cells; }
SFX_RANGE_HD int sfx_flux_faces(const sfx_dmesh& m) { return m.ranged ? m.r_flux : m.n_faces; }
SFX_RANGE_HD int sfx_update_cells(const sfx_dmesh& m) { return m.ranged ? m.r_upd : m.n_cells; }

/* the integer timeline of local time steps: 2^60 ticks from time 0 to
 * t_total (TimeLine, src/TimeLine.hpp:145-178) */
#define SFX_TIMELINE_TICKS (1ull << 60)
/* TimeLine::get_realtime (the timeline starts at 0) */
SFX_RANGE_HD double sfx_realtime(double t_total, uint64_t ticks) {
    const double t = (double)ticks / (double)SFX_TIMELINE_TICKS;
    return t_total * t + 0.;
}
/* TimeLine::get_realtime_interval */
SFX_RANGE_HD double sfx_realtime_interval(double t_total, uint64_t ticks) {
    const double dt = (double)ticks / (double)SFX_TIMELINE_TICKS;
    return t_total * dt;
}

/* one mesh of a launch group (device table entry); steps_left, when not
 * NULL, is the member's remaining step count: the kernels skip a member at 0
 * and a tick after each step counts it down */
struct sfx_group_entry {
    sfx_dmesh m;
    float dt;
    int32_t pad;
    int32_t* steps_left;
};

/* device view of a launch group: table of meshes and, per phase, the prefix
 * sum of blocks over the meshes (3 arrays of n_meshes + 1) */
struct sfx_group_dev {
    sfx_group_entry* tab;
    int32_t* pre;
    int32_t n_meshes;
    int32_t dim;
    int32_t lanes; /* lanes per cell of the gradient and update kernels */
    int32_t face_variant; /* SFX_FACE_VARIANTS (include/sfxflux.h) */
    int32_t moving;       /* a moving mesh stepped alone: face kernels with the boost */
    int32_t blocks[3];
};

struct sfx_solver_params {
    int32_t kind;
    double gamma, tol, cutoff;
    double gp1d2g, gm1d2g, gm1dgp1, tdgp1, tdgm1, gm1d2, tgdgm1, ginv;
};

void sfx_solver_params_init(sfx_solver_params* p, int kind, double gamma,
                            double tol, double cutoff);

/* FP64 kernels (sfx_fp64.cu) */
inline int64_t sfx_grad_term_stride(int dim) { return dim == 3 ? 16 : 8; }
int sfx_fp64_gradients(const sfx_dmesh* m, void* stream);
int sfx_fp64_faces(const sfx_dmesh* m, const sfx_solver_params* sp, double dt,
                   int write_branch, void* stream);
int sfx_fp64_apply(const sfx_dmesh* m, const sfx_solver_params* sp,
                   void* stream);
int sfx_fp64_init_Q(const sfx_dmesh* m, const sfx_solver_params* sp,
                    void* stream);
int sfx_fp64_totals(const sfx_dmesh* m, double* host_out, void* stream);
/* halo records [count][S + 1] (W, then the mass Q[0]) of the listed cells */
int sfx_fp64_pack_cells(const sfx_dmesh* m, const int32_t* idx, int count, double* out,
                        void* stream);
int sfx_fp64_unpack_cells(const sfx_dmesh* m, const int32_t* idx, int count, const double* in,
                          void* stream);
/* moving generators: generator velocities (VorCell::get_velocity with the
 * reflective-box check) into m->vgen, then (faces != 0) face velocities
 * (VorFace::set_v) into m->vel; with m->local only the cells starting a step
 * at t_now, each with its own step in the box check */
int sfx_fp64_move_velocities(const sfx_dmesh* m, double gamma, double dt, int periodic,
                             int faces, void* stream);
/* m->newpos = m->pos + dt m->vgen (Particle::drift) */
int sfx_fp64_drift(const sfx_dmesh* m, double dt, void* stream);
/* TimeLine::calculate_timestep for the cells whose step ends at t_next: the
 * CFL step h / (|v - v_gen| + c), its power-of-two subdivision of the
 * timeline, synchronised with the end, clamped to [min_step, max_step];
 * start <- end, end <- end + step; *d_smin (device) receives the smallest */
int sfx_fp64_timestep_bins(const sfx_dmesh* m, double gamma, double cfl, uint64_t max_step,
                           uint64_t min_step, unsigned long long* d_smin, void* stream);
int sfx_fp64_riemann(int dim, const sfx_solver_params* sp, int n,
                     const double* dWL, const double* dWR, const double* dn,
                     int reflective, double* dhalf, double* dflux,
                     int32_t* dcode, void* stream);

/* FP32/FP64-split kernels (sfx_split.cu) */
int sfx_split_prepare(const sfx_dmesh* m, void* stream);
int sfx_split_load_state(const sfx_dmesh* m, void* stream);
/* W (FP64 SoA) from the FP32 cell records, for downloads */
int sfx_split_export_W(const sfx_dmesh* m, void* stream);
/* per-face dQ (FP32) widened into dQf (FP64 SoA), for parity checks */
int sfx_split_export_dQ(const sfx_dmesh* m, void* stream);
/* kernel launch counter behind sfx_launch_count (sfx_api.cu).  Launches made
 * while the calling thread captures a CUDA graph are not counted (the
 * graph's kernels are counted when it is launched). */
void sfx_count_launches(int n);
void sfx_launch_capture(bool on);
/* accessors of the C-ABI handles (sfx_api.cu) */
sfx_dmesh* sfx_mesh_dev(sfx_mesh* m);
/* status of the mesh's error record (waits for its stream) */
int sfx_mesh_last_status(sfx_mesh* m, int32_t* bad_index);
sfx_ctx* sfx_mesh_ctx(sfx_mesh* m);
void* sfx_ctx_stream(sfx_ctx* c);
const sfx_config* sfx_ctx_config(sfx_ctx* c);
const sfx_solver_params* sfx_ctx_params(sfx_ctx* c);

/* replace a launch group's members (same context), reusing its device
 * buffers when they are large enough; steps (may be NULL) as in
 * sfx_group_set_steps (sfx_group.cu) */
int sfx_group_set_members(sfx_group* g, int32_t n, sfx_mesh* const* meshes, const double* dt,
                          const int32_t* steps);
/* state transfers in the device's field-major layout [S][n] (sfx_api.cu):
 * upload W, derive Q (waits and returns the status, as sfx_state_upload_W);
 * the download enqueues the copies on `stream` and returns at once */
int sfx_mesh_upload_W_fieldmajor(sfx_mesh* m, const double* W);
int sfx_mesh_download_fieldmajor_async(sfx_mesh* m, double* W, double* Q, void* stream);
/* the same without waiting, all device work on `stream` (W must stay valid
 * until the stream has run it); errors of the upload land in the mesh's
 * error record (sfx_mesh_last_status after the stream has finished) */
int sfx_mesh_upload_W_fieldmajor_async(sfx_mesh* m, const double* W, void* stream);
/* sfx_mesh_clone with its device setup on `stream`, not waited for */
int sfx_mesh_clone_async(sfx_ctx* ctx, sfx_mesh* base, void* stream, sfx_mesh** out);

/* lanes per cell of the split gradient and update kernels before any
 * tuning, the same for a mesh alone and in a group: one in 2D (about six
 * faces per cell), four in 3D (about sixteen); measured fastest on 300,000-cell
 * meshes */
/* float4s of the split pass's per-cell gradient record (cg) and of its
 * per-cell dW/dt record (cdw) */
inline int sfx_split_grad_vec4(int dim) {
    const int S = dim + 2;
    return (dim * S + 3) / 4;
}
inline int sfx_split_dwdt_vec4(int dim) {
    return (dim + 2 + 3) / 4;
}

inline int sfx_default_lanes(int dim) {
    return dim == 2 ? 1 : 4;
}

/* grouped launches (sfx_split.cu) */
int sfx_split_blocks(int dim, int lanes, int n_cells, int n_faces, int32_t* out);
/* a part's ring exchange in the split pass (the plain-FP64 record layout:
 * W, then the mass, per listed cell) */
int sfx_split_pack_cells(const sfx_dmesh* m, const int32_t* idx, int count, double* out,
                         void* stream);
int sfx_split_unpack_cells(const sfx_dmesh* m, const int32_t* idx, int count, const double* in,
                           void* stream);
/* the face-kernel variant that variant `variant` runs for this solver (the
 * variants that do not apply to it run another one's kernel) */
int sfx_split_face_variant_kernel(const sfx_solver_params* sp, int variant);
int sfx_split_group_phase(const sfx_group_dev* g, int phase, const sfx_solver_params* sp,
                          void* stream);
int sfx_split_group_reset(const sfx_group_dev* g, void* stream);
int sfx_split_group_tick(const sfx_group_dev* g, void* stream);
int sfx_split_group_collect(const sfx_group_dev* g, sfx_dev_error* d_out, void* stream);

#endif
