/*
 * CPU oracle for the Shadowfax flux pass — TEST INFRASTRUCTURE ONLY.
 *
 * Imported by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py as the checker; the product library never links or calls it.
 * See sfx_oracle.h for the interface and sfx_oracle_dim.h for the per-
 * dimension restatement (each routine cites the reference file:line).
 *
 * Build: gcc -O2 -ffp-contract=off -fno-builtin -std=c99 -shared -fPIC
 * (oracle/build.py).  -ffp-contract=off keeps every a*b+c as two
 * roundings, as the reference's own x86-64 build does.
 */
#define _POSIX_C_SOURCE 200809L
#include "sfx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../shadowfax_b200/csrc/sfx_pow.h"

/* iteration cap for the exact solver's Newton and Brent loops (the reference
 * has none; a capped face reports SFXO_ERR_NOCONV) */
#define SFXO_MAX_ITER 1000

/* branch codes: same bit layout as SFX_BRANCH_* in include/sfxflux.h */
#define SFXB_VAC_MASK 0x7
#define SFXB_VAC_BOTH 0x1
#define SFXB_VAC_RIGHT 0x2
#define SFXB_VAC_LEFT 0x3
#define SFXB_VAC_SPEED 0x4
#define SFXB_VAC_GEN SFXB_VAC_SPEED
#define SFXB_IT_NEWTON_ONLY (1 << 3)
#define SFXB_IT_NEWTON (2 << 3)
#define SFXB_IT_BRENT (3 << 3)
#define SFXB_S_RSHOCK_STAR (1 << 5)
#define SFXB_S_RUP_SHOCK (2 << 5)
#define SFXB_S_RFAN (3 << 5)
#define SFXB_S_RRARE_STAR (4 << 5)
#define SFXB_S_RUP (5 << 5)
#define SFXB_S_LSHOCK_STAR (6 << 5)
#define SFXB_S_LUP_SHOCK (7 << 5)
#define SFXB_S_LFAN (8 << 5)
#define SFXB_S_LRARE_STAR (9 << 5)
#define SFXB_S_LUP (10 << 5)
#define SFXB_S_VAC (11 << 5)
#define SFXB_NEWTON_SHIFT 9
#define SFXB_BRENT_SHIFT 16
#define SFXB_BRENT_ERREXIT (1 << 23)
#define SFXB_HLLC (1 << 24)
#define SFXB_HLLC_L (1 << 5)
#define SFXB_HLLC_LSTAR (2 << 5)
#define SFXB_HLLC_R (3 << 5)
#define SFXB_HLLC_RSTAR (4 << 5)
#define SFXB_LIMIT_L (1 << 25)
#define SFXB_LIMIT_R (1 << 26)
#define SFXB_SKIPPED (1 << 27)

static int g_use_libm_pow = 0;

double sfxo_pow(double x, double y) {
    return g_use_libm_pow ? pow(x, y) : sfx_pow(x, y);
}

/* the library's plain-double pow of the split pass (checked against exact
 * arithmetic by the tests) */
double sfxo_pow_fast(double x, double y) {
    return sfx_pow_fast(x, y);
}

#define opow sfxo_pow
/* the value of M_PI in the reference's <cmath> (not defined under -std=c99) */
#define SFXO_PI 3.14159265358979323846

#define D 2
#define FN(x) x##_2d
#include "sfx_oracle_dim.h"
#undef FN
#undef D

#define D 3
#define FN(x) x##_3d
#include "sfx_oracle_dim.h"
#undef FN
#undef D

static void set_pow(const sfxo_params* p) {
    g_use_libm_pow = p->use_libm_pow;
}

int sfxo_init_Q(const sfxo_mesh* m, const sfxo_params* p, const double* W,
                double* Q) {
    set_pow(p);
    return m->dim == 3 ? init_Q_3d(m, p, W, Q) : init_Q_2d(m, p, W, Q);
}

int sfxo_gradients(const sfxo_mesh* m, const double* W, double* grad) {
    return m->dim == 3 ? gradients_3d(m, W, grad) : gradients_2d(m, W, grad);
}

int sfxo_face_fluxes(const sfxo_mesh* m, const sfxo_params* p, double dt,
                     const double* W, const double* Q, const double* grad,
                     double* dQL, int* code, int* bad_face) {
    set_pow(p);
    return m->dim == 3 ? face_fluxes_3d(m, p, dt, W, Q, grad, dQL, code, bad_face)
                       : face_fluxes_2d(m, p, dt, W, Q, grad, dQL, code, bad_face);
}

int sfxo_apply(const sfxo_mesh* m, const sfxo_params* p, const double* dQL,
               double* Q, double* W, double* dQcell, int* bad_cell) {
    return m->dim == 3 ? apply_3d(m, p, dQL, Q, W, dQcell, bad_cell)
                       : apply_2d(m, p, dQL, Q, W, dQcell, bad_cell);
}

int sfxo_run(const sfxo_mesh* m, const sfxo_params* p, double dt, int nsteps,
             double* W, double* Q, double* grad_last, double* dQ_last,
             int* steps_done, double* seconds) {
    const int S = m->dim + 2;
    size_t ng = (size_t)m->ncell * m->dim * S;
    double* grad = grad_last ? grad_last : (double*)malloc(ng * sizeof(double));
    double* dQL = (double*)malloc((size_t)m->nface * S * sizeof(double));
    double* dQc = dQ_last ? dQ_last : (double*)malloc((size_t)m->ncell * S * sizeof(double));
    int rc = SFXO_OK;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    *steps_done = 0;
    for(int step = 0; step < nsteps; ++step) {
        sfxo_gradients(m, W, grad);
        rc = sfxo_face_fluxes(m, p, dt, W, Q, grad, dQL, NULL, NULL);
        if(rc) break;
        rc = sfxo_apply(m, p, dQL, Q, W, dQc, NULL);
        if(rc) break;
        ++*steps_done;
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if(seconds) *seconds = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
    if(!grad_last) free(grad);
    if(!dQ_last) free(dQc);
    free(dQL);
    return rc;
}

int sfxo_move_velocities(const sfxo_mesh* m, const sfxo_params* p, double dt, int periodic,
                         const double* W, double* vgen, double* vface) {
    if(m->dim == 3)
        move_velocities_3d(m, p, dt, periodic, W, vgen, vface);
    else
        move_velocities_2d(m, p, dt, periodic, W, vgen, vface);
    return SFXO_OK;
}

int sfxo_timestep_bins(const sfxo_mesh* m, const sfxo_params* p, const double* W,
                       const double* vgen, uint64_t* start, uint64_t* end, uint64_t t_next,
                       double t_total, double cfl, uint64_t max_step, uint64_t min_step,
                       uint64_t* smin) {
    return m->dim == 3 ? timestep_bins_3d(m, p, W, vgen, start, end, t_next, t_total, cfl,
                                          max_step, min_step, smin)
                       : timestep_bins_2d(m, p, W, vgen, start, end, t_next, t_total, cfl,
                                          max_step, min_step, smin);
}

int sfxo_riemann(int dim, const sfxo_params* p, int n, const double* WL,
                 const double* WR, const double* normal, int reflective,
                 double* half, double* flux, int* code) {
    set_pow(p);
    return dim == 3 ? riemann_3d(p, n, WL, WR, normal, reflective, half, flux, code)
                    : riemann_2d(p, n, WL, WR, normal, reflective, half, flux, code);
}
