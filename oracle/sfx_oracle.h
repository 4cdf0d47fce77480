/*
 * sfx_oracle — CPU restatement of the Shadowfax per-step finite-volume flux
 * pass (TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py, never by the product library).
 *
 * Plain C99, double precision, one thread.  Every routine follows the
 * reference's expression order so that, with the same pow(), it reproduces
 * the reference bit for bit; the reference file:line is cited at each routine.
 * Parity is pinned by oracle/refharness (the unmodified reference sources run
 * on the same mesh) and by the reference's Riemann golden vectors
 * (test/testRiemannSolver.cpp:217-248).
 */
#ifndef SFX_ORACLE_H
#define SFX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Face-list mesh, host arrays (cell-major, [n][dim] for vectors). */
typedef struct sfxo_mesh {
    int dim;
    int ncell;
    int nface;
    const double* cell_pos;        /* [ncell][dim] generator positions    */
    const double* cell_centroid;   /* [ncell][dim]                        */
    const double* cell_volume;     /* [ncell]                             */
    const double* cell_total_area; /* [ncell]                             */
    const int* cell_face_offset;   /* [ncell+1] CSR into cell_face_index  */
    const int* cell_face_index;    /* faces of each cell, cell's order    */
    const double* face_area;       /* [nface]                             */
    const double* face_midpoint;   /* [nface][dim]                        */
    const int* face_left;          /* [nface] owning (left) cell          */
    const int* face_right;         /* [nface] right cell, or -1 (mirror)  */
    const int* face_kind;          /* 0 real, 1 periodic image, 2 mirror  */
    const double* face_right_pos;  /* [nface][dim] right generator pos    */
    const double* face_velocity;   /* [nface][dim]                        */
} sfxo_mesh;

typedef struct sfxo_params {
    int solver;     /* 0 exact, 1 HLLC */
    double gamma;
    double tolerance;
    double cutoff;
    int use_libm_pow; /* 0: sfx_pow (bit-identical to the GPU), 1: libm pow */
} sfxo_params;

/* status codes (mirror include/sfxflux.h) */
#define SFXO_OK 0
#define SFXO_ERR_RIEMANN 3  /* RiemannSolverException (negative/NaN state) */
#define SFXO_ERR_NAN_FLUX 4 /* FluxCalculationException                   */
#define SFXO_ERR_NEG_STATE 5 /* UpdateQException / ConservedVariables    */
#define SFXO_ERR_NOCONV 6   /* iteration cap reached                      */

int sfxo_init_Q(const sfxo_mesh* m, const sfxo_params* p, const double* W,
                double* Q);
int sfxo_gradients(const sfxo_mesh* m, const double* W, double* grad);
int sfxo_face_fluxes(const sfxo_mesh* m, const sfxo_params* p, double dt,
                     const double* W, const double* Q, const double* grad,
                     double* dQL, int* code, int* bad_face);
int sfxo_apply(const sfxo_mesh* m, const sfxo_params* p, const double* dQL,
               double* Q, double* W, double* dQcell, int* bad_cell);
int sfxo_run(const sfxo_mesh* m, const sfxo_params* p, double dt, int nsteps,
             double* W, double* Q, double* grad_last, double* dQ_last,
             int* steps_done, double* seconds);
/* local time steps: new steps of the cells ending at t_next
 * (TimeLine::calculate_timestep); returns 0 or 15 (a zero step) */
int sfxo_timestep_bins(const sfxo_mesh* m, const sfxo_params* p, const double* W,
                       const double* vgen, uint64_t* start, uint64_t* end, uint64_t t_next,
                       double t_total, double cfl, uint64_t max_step, uint64_t min_step,
                       uint64_t* smin);
/* moving generators: generator velocities [ncell][dim] (VorCell::get_velocity
 * with the reflective-box check) and face velocities [nface][dim]
 * (VorFace::set_v) from the state W */
int sfxo_move_velocities(const sfxo_mesh* m, const sfxo_params* p, double dt, int periodic,
                         const double* W, double* vgen, double* vface);
int sfxo_riemann(int dim, const sfxo_params* p, int n, const double* WL,
                 const double* WR, const double* normal, int reflective,
                 double* half, double* flux, int* code);
double sfxo_pow(double x, double y);
double sfxo_pow_fast(double x, double y);

#ifdef __cplusplus
}
#endif
#endif
