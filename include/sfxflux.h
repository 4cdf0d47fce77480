/*
 * sfxflux — B200-native finite-volume flux pass over a static Voronoi mesh.
 *
 * C ABI (extern "C", plain pointers and sizes, no exceptions).  Every entry
 * point returns an int status (SFX_OK == 0).  It replaces, in Shadowfax's
 * own C++ host code:
 *
 *   - the gradient loop   for i: VorTessManager::estimate_gradients(i, g);
 *                                gas(i)->set_gradients(g)
 *                         (src/Simulation.cpp:414-420,
 *                          src/VorTessManager.cpp:290-296,
 *                          src/VorCell.cpp:464-530)
 *   - the face loop       VorTessManager::hydro -> VorFace::calculate_flux
 *                         (src/VorTessManager.cpp:198-212,
 *                          src/VorFace.cpp:670-1024)
 *   - update_Q / get_W    (src/Simulation.cpp:473-483 and 791-836,
 *                          src/utilities/GasParticle.cpp:617-624)
 *
 * keeping the RiemannSolver plugin selection (tag "EXAC" / "HLLC", gamma,
 * tolerance, cutoff: src/riemann/RiemannSolverFactory.hpp) and the
 * VorTess/VorFace face-list contract (src/VorTess.cpp:153-396).
 *
 * Array conventions on the host side: per-cell and per-face vectors are
 * row-major [n][dim]; states are [n][S] with S = dim + 2 and the component
 * order of StateVector (rho, vx, vy[, vz], p for primitive variables;
 * m, px, py[, pz], e for conserved ones), src/StateVector.hpp:52-116.
 */
#ifndef SFXFLUX_H
#define SFXFLUX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference's exceptions map onto these) ---- */
#define SFX_OK 0
#define SFX_ERR_INVALID 1     /* bad argument or mesh layout               */
#define SFX_ERR_CUDA 2        /* CUDA runtime failure                      */
#define SFX_ERR_RIEMANN 3     /* RiemannSolverException (RiemannSolver.hpp:202) */
#define SFX_ERR_NAN_FLUX 4    /* FluxCalculationException (VorFace.cpp:1022)    */
#define SFX_ERR_NEG_STATE 5   /* UpdateQException (GasParticle.cpp:619-621) and
                                 ConservedVariablesException in get_Q          */
#define SFX_ERR_NOCONV 6      /* exact solver hit its iteration cap       */
#define SFX_ERR_BOUNDS 7      /* face/cell index outside the mesh          */
#define SFX_ERR_UNSUPPORTED 8 /* solver tag other than EXAC/HLLC, etc.     */
#define SFX_ERR_MESH 9        /* tessellation failed                       */
#define SFX_ERR_NOMEM 10      /* device memory budget exceeded             */
#define SFX_ERR_NOT_READY 11  /* server: result not available yet          */
#define SFX_ERR_CLOSED 12     /* server: shut down                         */
#define SFX_ERR_IO 14         /* mesh file missing, truncated, corrupt or of
                                 another version                            */
#define SFX_ERR_TIMESTEP 15   /* a local time step of zero ticks ("Timestep 0!",
                                 TimeLine.cpp:287-290)                      */

/* ---- solver kinds and precision modes ---- */
#define SFX_SOLVER_EXACT 0 /* ExactRiemannSolver, tag "EXAC" */
#define SFX_SOLVER_HLLC 1  /* HLLCRiemannSolver, tag "HLLC"  */

#define SFX_PREC_FP64 0  /* plain FP64, bit-identical to the CPU oracle      */
#define SFX_PREC_SPLIT 1 /* FP32 reconstruction/prediction/HLLC and p*
                            Newton iteration, FP64 final p* step, sampling
                            and accumulation of Q                          */

/* ---- face kinds (the right generator of a VorFace) ---- */
#define SFX_FACE_REAL 0     /* right is a local cell                        */
#define SFX_FACE_PERIODIC 1 /* right is a periodic image (id 1, has particle)*/
#define SFX_FACE_MIRROR 2   /* right is a reflective mirror (no particle)    */

/* ---- exact-solver branch codes (per face, debug output) ----
 * bits 0-2   vacuum case: 0 none, 1 both sides vacuum, 2 right vacuum,
 *            3 left vacuum, 4 vacuum generation
 *            (ExactRiemannSolver.cpp:304-446)
 * bits 3-4   pressure iteration: 1 Newton only (f(0) < cutoff),
 *            2 Newton (converged), 3 Newton then Brent
 *            (ExactRiemannSolver.cpp:142-176)
 * bits 5-8   sampled region at x/t = 0 (see SFX_BRANCH_S_*)
 * bits 9-15  Newton steps (saturating at 127)
 * bits 16-22 Brent steps (saturating at 127)
 * bit  23    Brent error exit (f(a) f(b) >= 0, ExactRiemannSolver.cpp:480-486)
 * bit  24    set for HLLC faces; bits 5-8 then hold SFX_BRANCH_HLLC_*
 * bit  25/26 over-flux limiter applied on the left / right side
 *            (VorFace.cpp:837-866)
 * bit  27    face skipped (zero area)                                       */
#define SFX_BRANCH_VAC_MASK 0x7
#define SFX_BRANCH_S_SHIFT 5
#define SFX_BRANCH_S_MASK (0xf << 5)
#define SFX_BRANCH_S_RSHOCK_STAR (1 << 5)
#define SFX_BRANCH_S_RUP_SHOCK (2 << 5)
#define SFX_BRANCH_S_RFAN (3 << 5)
#define SFX_BRANCH_S_RRARE_STAR (4 << 5)
#define SFX_BRANCH_S_RUP (5 << 5)
#define SFX_BRANCH_S_LSHOCK_STAR (6 << 5)
#define SFX_BRANCH_S_LUP_SHOCK (7 << 5)
#define SFX_BRANCH_S_LFAN (8 << 5)
#define SFX_BRANCH_S_LRARE_STAR (9 << 5)
#define SFX_BRANCH_S_LUP (10 << 5)
#define SFX_BRANCH_S_VAC (11 << 5)
#define SFX_BRANCH_HLLC (1 << 24)
#define SFX_BRANCH_HLLC_L (1 << 5)
#define SFX_BRANCH_HLLC_LSTAR (2 << 5)
#define SFX_BRANCH_HLLC_R (3 << 5)
#define SFX_BRANCH_HLLC_RSTAR (4 << 5)
#define SFX_BRANCH_LIMIT_L (1 << 25)
#define SFX_BRANCH_LIMIT_R (1 << 26)
#define SFX_BRANCH_SKIPPED (1 << 27)

/* ---- configuration: what the RiemannSolver factory carries ---- */
typedef struct sfx_config {
    int32_t dim;       /* 2 or 3                                        */
    int32_t solver;    /* SFX_SOLVER_EXACT or SFX_SOLVER_HLLC           */
    double gamma;      /* adiabatic index (factory default 5/3)          */
    double tolerance;  /* exact solver p* tolerance (default 1e-8)       */
    double cutoff;     /* Newton-only threshold on f(0) (default -5)     */
    int32_t precision; /* SFX_PREC_FP64 or SFX_PREC_SPLIT                */
    int32_t device;    /* CUDA device ordinal                            */
} sfx_config;

/* ---- the face list exported once per tessellation (host arrays) ----
 * Faces follow the VorTess order (each face owned by the first cell that
 * meets it).  For face f: face_left[f] is the owner cell; face_right[f] is
 * the neighbour cell (or, for a periodic image, the cell it is an image of;
 * -1 for a reflective mirror); face_right_pos is the right generator's
 * position (image/mirror position), used for the normal and the gradient
 * geometry.  The per-cell face list (CSR) is the VorCell::_faces order;
 * it lists every face whose left is the cell or whose right is the cell
 * with kind SFX_FACE_REAL.  face_velocity may be NULL for a static mesh.  */
typedef struct sfx_mesh_desc {
    int32_t dim;
    int32_t n_cells;
    int32_t n_faces;
    const double* cell_pos;         /* [n_cells][dim] generator positions  */
    const double* cell_centroid;    /* [n_cells][dim]                      */
    const double* cell_volume;      /* [n_cells]                           */
    const double* cell_total_area;  /* [n_cells]                           */
    const int32_t* cell_face_offset; /* [n_cells + 1]                      */
    const int32_t* cell_face_index;  /* [cell_face_offset[n_cells]]        */
    const double* face_area;        /* [n_faces]                           */
    const double* face_midpoint;    /* [n_faces][dim]                      */
    const int32_t* face_left;       /* [n_faces]                           */
    const int32_t* face_right;      /* [n_faces]                           */
    const int32_t* face_kind;       /* [n_faces] SFX_FACE_*                */
    const double* face_right_pos;   /* [n_faces][dim]                      */
    const double* face_velocity;    /* [n_faces][dim] or NULL (static)     */
} sfx_mesh_desc;

/* ---- per-call statistics ---- */
typedef struct sfx_stats {
    int32_t status;      /* first error of the call, SFX_OK otherwise    */
    int32_t bad_face;    /* face index of a face error, else -1          */
    int32_t bad_cell;    /* cell index of a cell error, else -1          */
    int32_t steps_done;  /* completed steps                              */
    double totals[5];    /* sum over cells of Q (m, p[dim], e) after the
                            call, deterministic FP64 reduction           */
} sfx_stats;

typedef struct sfx_ctx sfx_ctx;
typedef struct sfx_mesh sfx_mesh;

/* ---- context: one per device and solver configuration ----
 * Replaces RiemannSolverFactory::generate (RiemannSolverFactory.hpp:60-81);
 * any other solver kind returns SFX_ERR_UNSUPPORTED. */
int sfx_ctx_create(const sfx_config* cfg, sfx_ctx** out);
int sfx_ctx_destroy(sfx_ctx* ctx);
/* run all work of this context on a caller stream (cudaStream_t); NULL =
 * the context's own stream */
int sfx_ctx_set_stream(sfx_ctx* ctx, void* cuda_stream);
/* block until the context's stream is idle */
int sfx_ctx_synchronize(sfx_ctx* ctx);

/* ---- mesh: upload the face list once per tessellation ----
 * (VorTess::construct output, src/VorTess.cpp:153-396).  The caller keeps
 * ownership of the host arrays and may free them after return.  A split
 * context takes periodic meshes of the unit box only (a periodic image
 * offset of 0 or +-1 on every axis, to 1e-9): SFX_ERR_UNSUPPORTED for
 * others; the plain-FP64 pass takes any box. */
int sfx_mesh_upload(sfx_ctx* ctx, const sfx_mesh_desc* desc, sfx_mesh** out);
/* the checks sfx_mesh_upload makes of a face list before it allocates, on the
 * host alone (no context, no device): SFX_OK or the status the upload to a
 * context of this precision would return -- SFX_ERR_INVALID for missing
 * arrays or sizes, SFX_ERR_BOUNDS for an index out of range or a cell listing
 * a face it is not on, SFX_ERR_UNSUPPORTED for a periodic mesh outside the
 * unit box in SFX_PREC_SPLIT.  For checking an exporter's output where no
 * GPU is. */
int sfx_mesh_check(const sfx_mesh_desc* desc, int32_t precision);
int sfx_mesh_free(sfx_mesh* mesh);
/* bytes of device memory a mesh of this size needs (admission control) */
int64_t sfx_mesh_device_bytes(int32_t dim, int32_t n_cells, int32_t n_faces,
                              int64_t n_cell_faces, int32_t precision);

/* ---- states ----
 * sfx_state_upload_W: primitive variables [n_cells][S]; conserved ones are
 * derived as in Simulation::initialize (Q = solver->get_Q(V, W),
 * src/Simulation.cpp:1231-1251).  sfx_state_upload_WQ sets both.       */
int sfx_state_upload_W(sfx_mesh* mesh, const double* W);
int sfx_state_upload_WQ(sfx_mesh* mesh, const double* W, const double* Q);
int sfx_state_download(sfx_mesh* mesh, double* W, double* Q);

/* ---- the pass ----
 * sfx_step: nsteps of gradients -> face fluxes -> update_Q -> get_W with a
 * global time step dt (every cell active).  Stops at the first error and
 * reports it in stats (may be NULL).  Asynchronous unless stats != NULL. */
int sfx_step(sfx_mesh* mesh, double dt, int32_t nsteps, sfx_stats* stats);
/* One step of a moving mesh (plain FP64 meshes that own their geometry):
 * the generator velocities of VorCell::get_velocity from the current state
 * (src/VorCell.cpp:966-1008), without the fluid velocity for a generator
 * that would leave the reflective unit box within dt (periodic = 0;
 * src/Simulation.cpp:366-398), the face velocities of VorFace::set_v
 * (src/VorFace.cpp:586-660), the step with every face's flux computed in
 * its moving frame, and the drift x + dt v (src/Simulation.cpp:473-481).
 * The tessellation is then stale: `positions` ([n_cells][dim] host, may be
 * NULL) receives the drifted generators, from which the caller builds the
 * next face list, as the reference re-tessellates after every drift.
 * Split-precision meshes take the boost into the face frame in FP32 and the
 * reference's de-boost of each solver's flux; the velocities and the drift
 * stay FP64.  SFX_ERR_UNSUPPORTED for clones and parts. */
int sfx_step_moving(sfx_mesh* mesh, double dt, int32_t periodic, double* positions,
                    sfx_stats* stats);

/* ---- local (hierarchical) time steps, plain FP64 and split ----
 * Every cell advances on its own step of the integer timeline: 2^60 ticks
 * from time 0 to t_total (TimeLine, src/TimeLine.hpp:145-178).  A cell is
 * active at tick t_now when its step starts there.
 * sfx_mesh_set_timesteps / _get_timesteps: each cell's step [start, end)
 * in ticks (all 0 until set; end <= 2^60).
 * sfx_mesh_set_gradients / _get_gradients: the stored gradients
 * [n_cells][dim][S] (an inactive cell keeps its last ones).
 * sfx_step_window: one system step [t_now, t_next): the cells starting at
 * t_now set their generator velocity (VorCell::get_velocity with the
 * reflective-box check over their own step; the mesh does not move) and
 * their gradients; every face with an active cell gets its flux over the
 * shorter of its cells' steps, the over-flux limiter scaled by that over the
 * longer one (VorFace.cpp:672-697, 837-866); every cell takes its faces'
 * dQ into Q (src/Simulation.cpp:473-483); the cells whose step ends at
 * t_next get W (src/Simulation.cpp:791-836).  Step bounds are not changed.
 * sfx_timestep_bins: TimeLine::calculate_timestep (src/TimeLine.cpp:233-317)
 * for the cells whose step ends at t_next: CFL step cfl h / (|v - v_gen| +
 * c), as a power-of-two subdivision of the timeline synchronised with the
 * cell's end and clamped to [min_step, max_step] ticks; the cell's next step
 * starts at its end; *system_step receives the smallest new step (the next
 * system step).  Start a run with t_next = 0 (every cell's end is 0).
 * Split-precision meshes (not clones) run the same window with their
 * kernels (per-face step and timefac in FP32 beside the FP64 accumulation;
 * the CFL steps from their FP32 states); sfx_mesh_set/get_gradients are
 * plain FP64 only.  SFX_ERR_UNSUPPORTED for parts and split clones. */
int sfx_mesh_set_timesteps(sfx_mesh* mesh, const uint64_t* start, const uint64_t* end);
int sfx_mesh_get_timesteps(sfx_mesh* mesh, uint64_t* start, uint64_t* end);
int sfx_mesh_set_gradients(sfx_mesh* mesh, const double* grad);
int sfx_mesh_get_gradients(sfx_mesh* mesh, double* grad);
int sfx_step_window(sfx_mesh* mesh, double t_total, uint64_t t_now, uint64_t t_next,
                    int32_t periodic, sfx_stats* stats);
int sfx_timestep_bins(sfx_mesh* mesh, double t_total, double cfl, uint64_t max_step,
                      uint64_t min_step, uint64_t t_next, uint64_t* system_step);

/* sfx_step with CUDA events around every phase: kernel_ms[0..2] receive
 * the summed device time (ms) of the gradient, face and update kernels over
 * the nsteps, *launches the number of kernels launched.  For profiling. */
int sfx_step_timed(sfx_mesh* mesh, double dt, int32_t nsteps, float* kernel_ms,
                   int32_t* launches);

/* one pass for parity checks: gradients and per-face limited dQ (the amount
 * the left cell receives; a real right cell receives its negation) without
 * updating the state.  Outputs are host arrays, each may be NULL:
 * grad [n_cells][dim][S], dQ_face [n_faces][S], branch [n_faces]. */
int sfx_flux_pass(sfx_mesh* mesh, double dt, double* grad, double* dQ_face,
                  int32_t* branch, sfx_stats* stats);

/* Riemann solver on n independent state pairs (host arrays), interface at
 * rest: RiemannSolver::solve (exact only) and solve_for_flux
 * (ExactRiemannSolver.cpp:108-290, 858-880; HLLCRiemannSolver.cpp:258-403).
 * half/flux/branch are [n][S], [n][S], [n]; half may be NULL. */
int sfx_riemann_eval(sfx_ctx* ctx, int32_t n, const double* WL, const double* WR,
                     const double* normal, int32_t reflective, double* half,
                     double* flux, int32_t* branch);

/* conserved totals sum_i Q_i (m, p[dim], e), deterministic FP64 */
int sfx_mesh_totals(sfx_mesh* mesh, double* totals);

/* A new mesh handle on `ctx` that shares `base`'s device geometry and owns
 * only a state (W, Q and the per-step scratch of ctx's precision): several
 * integrations of one tessellation without copying it again.  `base` must
 * outlive the clone and have been uploaded with the split arrays if ctx is
 * SFX_PREC_SPLIT.  sfx_flux_pass is not available on split clones. */
int sfx_mesh_clone(sfx_ctx* ctx, sfx_mesh* base, sfx_mesh** out);
/* device bytes a clone of `base` at `precision` allocates */
int64_t sfx_mesh_clone_bytes(sfx_mesh* base, int32_t precision);

/* split pass: lanes of a warp that share one cell in the gradient and update
 * kernels (1, 2, 4, 8 or 16; default 1 in 2D, 4 in 3D).  Changes the summation
 * tree of the per-cell sums, not the algorithm. */
int sfx_mesh_set_lanes(sfx_mesh* mesh, int32_t lanes);
/* split pass: face-kernel variant: 0 (64 registers, four 256-thread blocks
 * per SM; the default), 1 (80 registers, three blocks), 2 (HLLC: the
 * half-step prediction's dW/dt read from the per-cell record instead of
 * formed per face; exact solver with gamma = 5/3: the p* step's powers as a
 * fifth root by Newton's method and the sampling's powers as integer powers;
 * other gamma: as 0), 3 (exact solver with gamma = 5/3: 2 with 80
 * registers; other gamma: as 1; HLLC: 48 registers, five blocks), 4 (the
 * left cells of each 256-face block staged in shared memory by bulk copies:
 * exact solver as 2 at gamma = 5/3, as 0 otherwise; HLLC as 3).  Variants 0
 * and 1, 3 for HLLC and 4 change the schedule only, not the results of the
 * variant they stage for; 2, and 3 for the exact solver, change round-off
 * within the split pass's tolerance. */
#define SFX_FACE_VARIANTS 5
int sfx_mesh_set_face_variant(sfx_mesh* mesh, int32_t variant);

/* ---- one mesh over several devices (plain FP64 and split) ----
 * Replaces the reference's MPI halo updates for the flux pass
 * (DelTess::update_Ws / update_gradients / update_dQs, src/DelTess_mpi.cpp:1614,
 * 1781, 2024): each device holds its owned cells, numbered first, then the
 * cells one face away (their gradients are computed here too) and the cells
 * two faces away (state only), with every face of the first two groups, the
 * faces touching an owned cell first.  sfx_mesh_set_ranges makes the pass
 * compute gradients of cells [0, grad_cells), fluxes of faces
 * [0, flux_faces) and update cells [0, update_cells) only; the owned cells
 * then receive exactly the values a pass over the whole mesh gives them.
 * Between steps the other cells' W and mass Q[0] come from their owners:
 * sfx_mesh_pack_cells writes records [count][S + 1] (W, then Q[0]) of the
 * listed local cells to a device buffer, sfx_mesh_unpack_cells stores such
 * records into the listed cells.  idx, out and in are device pointers;
 * stream NULL is the context's stream.  The lists are made once per
 * partition and are not checked on every call: an index outside the mesh
 * is skipped (never dereferenced).  A split-precision mesh packs its FP32
 * states (exact in the doubles) and its FP64 mass, and its owned cells also
 * receive exactly the values of a split pass over the whole mesh when the
 * part also holds the other copy of every periodic face of its first two
 * groups, those of owned cells inside [0, flux_faces): the split pass applies
 * one copy of a periodic pair to both cells, the copy whose image shift has
 * the smaller code; SFX_ERR_UNSUPPORTED for a split clone. */
int sfx_mesh_set_ranges(sfx_mesh* mesh, int32_t grad_cells, int32_t flux_faces,
                        int32_t update_cells);
int sfx_mesh_pack_cells(sfx_mesh* mesh, const int32_t* idx, int32_t count, double* out,
                        void* stream);
int sfx_mesh_unpack_cells(sfx_mesh* mesh, const int32_t* idx, int32_t count, const double* in,
                          void* stream);

/* ---- launch groups: many meshes per launch (SFX_PREC_SPLIT) ----
 * A group runs one step of every member mesh with one launch per phase
 * (gradients, faces, update): block b of a launch works on the mesh whose
 * block range contains b.  Each mesh keeps its own time step, state and error
 * record (a failing mesh stops only itself).  The member meshes must belong
 * to `ctx` and stay alive while the group exists; their states are set and
 * read with the per-mesh sfx_state_* calls.  With use_graph != 0 the nsteps
 * steps are captured once in a CUDA graph and replayed on later calls with
 * the same nsteps.  mesh_status (may be NULL) receives one status per mesh. */
typedef struct sfx_group sfx_group;
int sfx_group_create(sfx_ctx* ctx, int32_t n_meshes, sfx_mesh* const* meshes,
                     const double* dt, sfx_group** out);
int sfx_group_set_dt(sfx_group* group, const double* dt);
int sfx_group_step(sfx_group* group, int32_t nsteps, int32_t use_graph,
                   int32_t* mesh_status);
/* time each lanes-per-cell variant (1, 2, 4, 8, 16) of the gradient kernel on
 * this group (reads the states, changes none) and keep the fastest for the
 * gradient and update kernels; *lanes receives it */
int sfx_group_tune(sfx_group* group, int32_t reps, int32_t* lanes);
int sfx_group_set_lanes(sfx_group* group, int32_t lanes);
/* time each face-kernel variant (SFX_FACE_VARIANTS) on this group, every
 * timed face launch after a gradient launch (the states are read, none
 * changes), and keep the fastest; *variant receives it */
int sfx_group_tune_faces(sfx_group* group, int32_t reps, int32_t* variant);
int sfx_group_set_face_variant(sfx_group* group, int32_t variant);
/* per-member remaining step counts, kept on the device: a member at 0 is
 * skipped by the launches and each step counts the others down, so members
 * with different step counts share launches without host round trips */
int sfx_group_set_steps(sfx_group* group, const int32_t* steps);
int sfx_group_get_steps(sfx_group* group, int32_t* steps);
/* nsteps without a graph, with CUDA events around each phase's launch:
 * phase_ms[3] receives the summed device time of the gradient, face and
 * update launches, *launches (may be NULL) the number of kernels launched */
int sfx_group_step_timed(sfx_group* group, int32_t nsteps, float* phase_ms,
                         int32_t* launches);
/* per-member status of the last sfx_group_step (waits for the group) */
int sfx_group_status(sfx_group* group, int32_t* mesh_status);
int sfx_group_free(sfx_group* group);

/* ---- host Voronoi face-list builder (inputs for the pass) ---- */
typedef struct sfx_voronoi sfx_voronoi;
int sfx_voronoi_build(int dim, int64_t n, const double* pos, int periodic,
                      int nthreads, sfx_voronoi** out);
int sfx_voronoi_counts(const sfx_voronoi* v, int64_t* n_cells,
                       int64_t* n_faces, int64_t* n_cell_faces);
int sfx_voronoi_export(const sfx_voronoi* v, double* cell_centroid,
                       double* cell_volume, double* cell_total_area,
                       int32_t* cell_face_offset, int32_t* cell_face_index,
                       double* face_area, double* face_midpoint,
                       int32_t* face_left, int32_t* face_right,
                       int32_t* face_kind, double* face_right_pos);
void sfx_voronoi_free(sfx_voronoi* v);

/* ---- versioned binary mesh file (no counterpart in the reference, which
 * re-tessellates at every start; the pre-tessellated pool of the request
 * service is built once and read back through these) ----
 * sfx_meshfile_write stores a face list in the sfx_mesh_desc layout with its
 * periodicity (face velocities when not NULL); sfx_meshfile_info returns its
 * sizes (any output may be NULL); sfx_meshfile_read fills caller arrays of
 * those sizes (face_velocity may be NULL; zeros when the file has none).
 * Every read checks the magic, the major version (a higher major is
 * rejected; a later minor version only adds sections, which this reader
 * skips), the section table against the file size, a checksum of the
 * payload and the cell face offsets (0 first, never decreasing, n_cell_faces
 * last): SFX_ERR_IO otherwise, SFX_ERR_NOMEM when the payload cannot be
 * held in host memory. */
#define SFX_MESHFILE_VERSION 1
#define SFX_MESHFILE_MINOR_VERSION 0
int sfx_meshfile_write(const char* path, const sfx_mesh_desc* mesh, int32_t periodic);
int sfx_meshfile_info(const char* path, int32_t* dim, int32_t* periodic, int64_t* n_cells,
                      int64_t* n_faces, int64_t* n_cell_faces, int32_t* has_velocity);
int sfx_meshfile_read(const char* path, double* cell_pos, double* cell_centroid,
                      double* cell_volume, double* cell_total_area, int32_t* cell_face_offset,
                      int32_t* cell_face_index, double* face_area, double* face_midpoint,
                      int32_t* face_left, int32_t* face_right, int32_t* face_kind,
                      double* face_right_pos, double* face_velocity);

/* ---- request server: continuous batching of static-mesh integrations ----
 * No counterpart in the reference (Shadowfax runs one simulation per job).
 * Meshes are added once to a device-resident pool; a request names a pool
 * mesh, an initial state, a solver, a time step and a step count.  A worker
 * thread admits queued requests in arrival order while the device-memory
 * budget and the slot count allow, keeps admitted states resident, and
 * advances all admitted requests of one (dimension, solver) class together:
 * SFX_PREC_SPLIT co-batches them into one launch group per class and chunk
 * of steps (per-request step counters on the device), SFX_PREC_FP64 steps
 * each request alone (the per-request baseline).  Requests arriving while
 * others run join at the next chunk.  Results wait in host memory until
 * sfx_server_poll collects them. */
typedef struct sfx_server sfx_server;

typedef struct sfx_server_config {
    int32_t device;
    int32_t precision;      /* SFX_PREC_SPLIT (co-batched) or SFX_PREC_FP64     */
    double gamma;
    double tolerance;
    double cutoff;
    int64_t memory_budget;  /* device bytes for admitted request states       */
    int32_t max_active;     /* admitted requests at most                      */
    int32_t chunk_steps;    /* steps per scheduling round (4 measured best)    */
} sfx_server_config;

typedef struct sfx_request_info {
    int32_t status;         /* SFX_OK or the request's error                  */
    int32_t steps_done;
    int32_t mesh_id;
    int32_t solver;
    double t_submit;        /* seconds on the server's clock                  */
    double t_admit;
    double t_done;
    int64_t face_steps;     /* nonzero-area faces x steps done                */
} sfx_request_info;

typedef struct sfx_server_stats {
    int64_t submitted, admitted, completed, failed, active, queued;
    int64_t face_steps;     /* over completed requests                        */
    int64_t bytes_in_use;   /* device bytes of admitted request states        */
    int64_t rounds;         /* scheduling rounds run                          */
    double now;             /* server clock, seconds                          */
    double worker_s[4];     /* worker thread time in admission, launches,
                               completing results, and waiting for rounds    */
} sfx_server_stats;

int sfx_server_create(const sfx_server_config* cfg, sfx_server** out);
/* split servers: the kernel settings of the launch group of one (dim, solver)
 * class (lanes per cell, 0: the default; face variant, SFX_FACE_VARIANTS),
 * e.g. what sfx_group_tune / sfx_group_tune_faces kept on meshes like the
 * pool's; applied before the class's next round.  SFX_ERR_UNSUPPORTED for
 * FP64. */
int sfx_server_set_tuning(sfx_server* srv, int32_t dim, int32_t solver, int32_t lanes,
                          int32_t face_variant);
/* add a mesh to the device pool (upload once); *mesh_id identifies it */
int sfx_server_add_mesh(sfx_server* srv, const sfx_mesh_desc* desc, int32_t* mesh_id);
/* queue a request; W0 [n_cells][S] is copied; returns at once */
int sfx_server_submit(sfx_server* srv, int32_t mesh_id, const double* W0, int32_t solver,
                      double dt, int32_t nsteps, int64_t* request_id);
/* SFX_ERR_NOT_READY while the request runs; then copies W and Q (either may
 * be NULL to discard), fills info (may be NULL), forgets the request and
 * returns its status */
int sfx_server_poll(sfx_server* srv, int64_t request_id, double* W, double* Q,
                    sfx_request_info* info);
/* wait until nothing is queued or running (timeout_s <= 0: no limit);
 * SFX_ERR_NOT_READY on timeout */
int sfx_server_drain(sfx_server* srv, double timeout_s);
int sfx_server_stats_get(sfx_server* srv, sfx_server_stats* stats);
/* stop the worker, free every request and the pool */
int sfx_server_shutdown(sfx_server* srv);

/* ---- one FP64 flux pass that allocates nothing ----
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory through the library: applications that hand out all device memory
 * from their own pools or reserve it up front, or that must not allocate
 * while requests are in flight.  The caller owns every input and output
 * array (device pointers, field-major layout below); the gradient scratch is
 * a fixed file-scope device array of SFX_NOALLOC_MAX_CELLS cells (7.5 MiB on
 * every GPU that loads the library, held until the process exits), so
 * meshes with more cells are rejected with SFX_ERR_TOO_LARGE.
 *
 * Same arithmetic as sfx_flux_pass in SFX_PREC_FP64: gradients, then the
 * limited dQ each face gives its left cell.  Runs on the current device and
 * on `cuda_stream` (NULL = legacy default stream), and waits for it before
 * returning the status.  The first call on a device looks up the scratch
 * array's device address; make that first call before any stream capture.
 * The lookup is repeated when the device's context has changed (after a
 * cudaDeviceReset), so make the first call after a reset before any capture
 * too.
 * All calls share the scratch array: calls that overlap on the GPU (other
 * threads, other streams) race and must be serialised by the caller.
 * Mesh indices are not range-checked on the device: they must be valid. */
#define SFX_ERR_TOO_LARGE 13
#define SFX_NOALLOC_MAX_CELLS 65536

typedef struct sfx_device_mesh {
    int32_t dim;
    int32_t n_cells;
    int32_t n_faces;
    const double* cell_pos;          /* [dim][n_cells]                      */
    const double* cell_centroid;     /* [dim][n_cells]                      */
    const double* cell_volume;       /* [n_cells]                           */
    const double* cell_total_area;   /* [n_cells]                           */
    const int32_t* cell_face_offset; /* [n_cells + 1]                       */
    const int32_t* cell_face_entry;  /* face id, bit 31 set when the cell is
                                        the face's (real) right cell         */
    const double* face_area;         /* [n_faces]                           */
    const double* face_midpoint;     /* [dim][n_faces]                      */
    const int32_t* face_left;        /* [n_faces]                           */
    const int32_t* face_right;       /* [n_faces]                           */
    const int32_t* face_kind;        /* [n_faces] SFX_FACE_*                */
    const double* face_right_pos;    /* [dim][n_faces]                      */
} sfx_device_mesh;

/* W, Q: [S][n_cells] device (S = dim + 2); dQ_face: [S][n_faces] device out */
int sfx_flux_pass_noalloc(const sfx_device_mesh* mesh, const sfx_config* cfg, double dt,
                          const double* W, const double* Q, double* dQ_face,
                          void* cuda_stream);

/* library version string */
const char* sfx_version(void);
/* kernels this library has launched since it was loaded (all contexts;
 * a replayed CUDA graph counts each kernel it runs) */
int64_t sfx_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
