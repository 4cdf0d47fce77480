/*
 * Plain-FP64 flux pass for sm_100a: gradients, per-face fluxes, update_Q and
 * get_W, bit-identical to Shadowfax's CPU pass.
 *
 * This translation unit is compiled with -fmad=false (no a*b+c contraction)
 * and IEEE division / square root, and keeps the reference's expression
 * order, so each value is rounded exactly as the reference rounds it.  pow()
 * is sfx_pow (sfx_pow.h), shared with the CPU oracle, because glibc's and
 * CUDA's pow differ in the last bit.
 *
 * Kernels (one step = three or four launches):
 *   k_gradients  one thread per cell: VorCell::estimate_gradient
 *                (src/VorCell.cpp:464-530); or k_grad_terms (one thread
 *                per face) + k_grad_sum (one per cell and variable), the
 *                same values with each face's terms computed once
 *   k_faces      one thread per face: VorFace::calculate_flux
 *                (src/VorFace.cpp:670-1024) with the Exact or HLLC solver;
 *                writes the limited dQ of the left cell once per face
 *   k_apply      one thread per cell: the face contributions in ascending
 *                face order (the order of VorTessManager::hydro's loop,
 *                src/VorTessManager.cpp:205-209), Q -= dQ
 *                (GasParticle::update_Q, GasParticle.cpp:617-624), get_W.
 * No floating-point atomics: every cell sums its own faces in a fixed order,
 * so reruns are bitwise identical.
 */
#include <cuda_runtime.h>

#include "sfx_internal.h"
#include "sfx_limiter.h"
#include "sfx_pow.h"

namespace {

constexpr unsigned kRightBit = 0x80000000u;

__device__ __forceinline__ void report_face(sfx_dev_error* e, int f, int st) {
    unsigned long long key = ((unsigned long long)(unsigned)f << 8) | (unsigned)st;
    atomicMin(&e->face_key, key);
}

__device__ __forceinline__ void report_cell(sfx_dev_error* e, int i, int st) {
    unsigned long long key = ((unsigned long long)(unsigned)i << 8) | (unsigned)st;
    atomicMin(&e->cell_key, key);
}

__device__ __forceinline__ bool failed(const sfx_dev_error* e) {
    return (*(volatile const unsigned long long*)&e->face_key != ~0ull) ||
           (*(volatile const unsigned long long*)&e->cell_key != ~0ull);
}

/* ---------------- time derivative (Exact :892-934 / HLLC :415-450) ------- */
template <int D>
__device__ __forceinline__ void time_derivative(double gamma, const double* W,
                                                const double (*g)[D + 2],
                                                double* dW);

template <>
__device__ __forceinline__ void time_derivative<3>(double gamma, const double* W,
                                                   const double (*g)[5],
                                                   double* dW) {
    dW[0] = -W[0] * (g[0][1] + g[1][2] + g[2][3]) - W[1] * g[0][0] -
            W[2] * g[1][0] - W[3] * g[2][0];
    dW[1] = -W[1] * g[0][1] - W[2] * g[1][1] - W[3] * g[2][1] - g[0][4] / W[0];
    dW[2] = -W[1] * g[0][2] - W[2] * g[1][2] - W[3] * g[2][2] - g[1][4] / W[0];
    dW[3] = -W[1] * g[0][3] - W[2] * g[1][3] - W[3] * g[2][3] - g[2][4] / W[0];
    dW[4] = -gamma * W[4] * (g[0][1] + g[1][2] + g[2][3]) - W[1] * g[0][4] -
            W[2] * g[1][4] - W[3] * g[2][4];
}

template <>
__device__ __forceinline__ void time_derivative<2>(double gamma, const double* W,
                                                   const double (*g)[4],
                                                   double* dW) {
    dW[0] = -W[1] * g[0][0] - W[2] * g[1][0] - W[0] * (g[0][1] + g[1][2]);
    dW[1] = -W[1] * g[0][1] - W[2] * g[1][1] - g[0][3] / W[0];
    /* the reference uses d(vy)/dy in both terms (ExactRiemannSolver.cpp:920) */
    dW[2] = -W[1] * g[1][2] - W[2] * g[1][2] - g[1][3] / W[0];
    dW[3] = -gamma * W[3] * (g[0][1] + g[1][2]) - W[1] * g[0][3] - W[2] * g[1][3];
}

template <int D>
__device__ __forceinline__ double dot(const double* a, const double* b) {
    double s = a[0] * b[0] + a[1] * b[1];
    if(D == 3) s = s + a[2] * b[2];
    return s;
}

template <int D>
__device__ __forceinline__ double norm(const double* a) {
    return sqrt(dot<D>(a, a));
}

/* VorFace.hpp:174-196 */
template <int D>
__device__ __forceinline__ void reconstruct(double* W, const double (*g)[D + 2],
                                            const double* d) {
#pragma unroll
    for(int k = 0; k < D + 2; ++k) {
        double s = g[0][k] * d[0] + g[1][k] * d[1];
        if(D == 3) s = s + g[2][k] * d[2];
        W[k] = W[k] + s;
    }
}

/* VorFace.hpp:92-137 */
template <int D>
__device__ __forceinline__ double limit1(double phimid0, double phiL, double phiR,
                                         double dnrm, double r) {
    const double psi1 = 0.5, psi2 = 0.25;
    double delta1 = psi1 * fabs(phiL - phiR);
    double delta2 = psi2 * fabs(phiL - phiR);
    double phimin = fmin(phiL, phiR);
    double phimax = fmax(phiL, phiR);
    double phibar = phiL + dnrm / r * (phiR - phiL);
    if(phiL == phiR) return phiL;
    /* only the bound the result uses (phi- when phiL < phiR, else phi+), with
     * the sign-preserving fallback where the shifted extreme changes sign:
     * the reference's values, without the other bound's divisions */
    const bool up = phiL < phiR;
    const double ext = up ? phimin : phimax;
    double bound = up ? ext - delta1 : ext + delta1;
    if(!(bound * ext > 0.)) bound = ext / (1. + delta1 / fabs(ext));
    if(up) return fmax(bound, fmin(phibar + delta2, phimid0));
    return fmin(bound, fmax(phibar - delta2, phimid0));
}

/* mirror a state across a reflective face: transform, flip the normal
 * velocity, invtransform (VorFace.cpp:417-542, VorCell.cpp:479-485) */
template <int D>
__device__ __forceinline__ void mirror_state(double* W, const double* left,
                                             const double* right);

template <>
__device__ __forceinline__ void mirror_state<3>(double* W, const double* left,
                                                const double* right) {
    double n0 = right[0] - left[0], n1 = right[1] - left[1], n2 = right[2] - left[2];
    double n3 = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    n0 /= n3;
    n1 /= n3;
    n2 /= n3;
    double o0, o1, o3, p0, p1, p2;
    if(n0 != 0. || n1 != 0.) {
        o0 = -n1;
        o1 = n0;
        o3 = sqrt(o0 * o0 + o1 * o1);
        o0 /= o3;
        o1 /= o3;
        p0 = -n2 * o1;
        p1 = n2 * o0;
        p2 = o3;
    } else {
        o0 = 0.;
        o1 = 1.;
        p0 = -1.;
        p1 = 0.;
        p2 = 0.;
    }
    double v0 = W[1], v1 = W[2], v2 = W[3];
    double t1 = v0 * n0 + v1 * n1 + v2 * n2;
    double t2 = v0 * o0 + v1 * o1;
    double t3 = v0 * p0 + v1 * p1 + v2 * p2;
    t1 = -t1;
    W[1] = t1 * n0 + t2 * o0 + t3 * p0;
    W[2] = t1 * n1 + t2 * o1 + t3 * p1;
    W[3] = t1 * n2 + t3 * p2;
}

template <>
__device__ __forceinline__ void mirror_state<2>(double* W, const double* left,
                                                const double* right) {
    double d0 = left[0] - right[0], d1 = left[1] - right[1];
    double d2 = sqrt(d0 * d0 + d1 * d1);
    double cost = -d0 / d2;
    double sint = -d1 / d2;
    double W1 = W[1] * cost + W[2] * sint;
    double W2 = -W[1] * sint + W[2] * cost;
    W1 = -W1;
    W[1] = W1 * cost - W2 * sint;
    W[2] = W1 * sint + W2 * cost;
}

/* ------------------------------ gradients ------------------------------ */
template <int D>
__global__ void __launch_bounds__(128) k_gradients(sfx_dmesh m) {
    constexpr int S = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= sfx_grad_cells(m) || failed(m.err)) return;
    /* local time steps: an inactive cell keeps its gradients (src/Simulation.cpp:414-420) */
    if(m.local && m.tstart[i] != m.t_now) return;
    const int n = m.n_cells, F = m.n_faces;
    double W[S], xi[D], Wmax[S], Wmin[S], delta[D][S];
#pragma unroll
    for(int k = 0; k < S; ++k) {
        W[k] = m.W[(size_t)k * n + i];
        Wmax[k] = W[k];
        Wmin[k] = W[k];
#pragma unroll
        for(int l = 0; l < D; ++l) delta[l][k] = 0.;
    }
#pragma unroll
    for(int l = 0; l < D; ++l) xi[l] = m.pos[(size_t)l * n + i];
    const int beg = m.off[i], end = m.off[i + 1];
    for(int j = end - 1; j >= beg; --j) {
        const unsigned e = (unsigned)m.idx[j];
        const int f = (int)(e & ~kRightBit);
        const double A = m.area[f];
        if(A == 0.) continue;
        double mid[D], xj[D], Wj[S];
#pragma unroll
        for(int l = 0; l < D; ++l) mid[l] = m.mid[(size_t)l * F + f];
        if(!(e & kRightBit)) {
#pragma unroll
            for(int l = 0; l < D; ++l) xj[l] = m.rpos[(size_t)l * F + f];
            if(m.kind[f] == SFX_FACE_MIRROR) {
#pragma unroll
                for(int k = 0; k < S; ++k) Wj[k] = W[k];
                mirror_state<D>(Wj, xi, xj);
            } else {
                const int r = m.right[f];
#pragma unroll
                for(int k = 0; k < S; ++k) Wj[k] = m.W[(size_t)k * n + r];
            }
        } else {
            const int jl = m.left[f];
#pragma unroll
            for(int l = 0; l < D; ++l) xj[l] = m.pos[(size_t)l * n + jl];
#pragma unroll
            for(int k = 0; k < S; ++k) Wj[k] = m.W[(size_t)k * n + jl];
        }
        double c[D], rij[D];
#pragma unroll
        for(int l = 0; l < D; ++l) {
            c[l] = mid[l] - 0.5 * (xi[l] + xj[l]);
            rij[l] = xi[l] - xj[l];
        }
        const double rnorm = norm<D>(rij);
#pragma unroll
        for(int l = 0; l < D; ++l) {
#pragma unroll
            for(int k = 0; k < S; ++k) {
                delta[l][k] = delta[l][k] +
                              A * ((Wj[k] - W[k]) * c[l] / rnorm -
                                   0.5 * (W[k] + Wj[k]) * rij[l] / rnorm);
            }
        }
#pragma unroll
        for(int k = 0; k < S; ++k) {
            Wmax[k] = (Wmax[k] < Wj[k]) ? Wj[k] : Wmax[k];
            Wmin[k] = (Wj[k] < Wmin[k]) ? Wj[k] : Wmin[k];
        }
    }
    const double V = m.vol[i];
#pragma unroll
    for(int l = 0; l < D; ++l)
#pragma unroll
        for(int k = 0; k < S; ++k) delta[l][k] = delta[l][k] / V;
    double cen[D], alpha[S];
#pragma unroll
    for(int l = 0; l < D; ++l) cen[l] = m.cen[(size_t)l * n + i];
#pragma unroll
    for(int k = 0; k < S; ++k) alpha[k] = 1.;
    for(int j = end - 1; j >= beg; --j) {
        const int f = (int)((unsigned)m.idx[j] & ~kRightBit);
        if(m.area[f] == 0.) continue;
        double d[D];
#pragma unroll
        for(int l = 0; l < D; ++l) d[l] = m.mid[(size_t)l * F + f] - cen[l];
#pragma unroll
        for(int k = 0; k < S; ++k) {
            double dp = delta[0][k] * d[0] + delta[1][k] * d[1];
            if(D == 3) dp = dp + delta[2][k] * d[2];
            double q1 = Wmax[k] - W[k];
            double q2 = Wmin[k] - W[k];
            if(dp != 0.) {
                q1 = q1 / dp;
                q2 = q2 / dp;
            } else {
                q1 = 1.;
                q2 = 1.;
            }
            const double mx = (q1 < q2) ? q2 : q1;
            alpha[k] = (mx < alpha[k]) ? mx : alpha[k];
        }
    }
#pragma unroll
    for(int l = 0; l < D; ++l)
#pragma unroll
        for(int k = 0; k < S; ++k)
            m.grad[((size_t)l * S + k) * n + i] = delta[l][k] * alpha[k];
}

constexpr int kGradBlock = 128;

/* The same gradients in two kernels, when every local face's right position
 * is its right cell's position (gshare).  The first loop's term of a face,
 *   t = A ((W_j - W_i) c / |r| - (W_i + W_j) / 2 r / |r|),
 * is then exactly negated between the face's two cells: c is the same for
 * both (the midpoint sum commutes), r and W_j - W_i change sign, and IEEE
 * rounding is symmetric under negation, so the right cell's term equals -t
 * bit for bit, except that a zero term may carry the other sign, which no
 * sum starting at +0 can tell apart.  k_grad_terms evaluates t once per face
 * (its 2 D S divisions, the bulk of the gradients' cost, are no longer done
 * twice); k_grad_sum adds the terms in each cell's face order exactly as the
 * one-kernel loop does, and runs the limiter. */
template <int D>
__global__ void __launch_bounds__(128) k_grad_terms(sfx_dmesh m) {
    constexpr int S = D + 2, TS = D == 3 ? 16 : 8;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if(f >= m.n_faces || failed(m.err)) return;
    const double A = m.area[f];
    if(A == 0.) return; /* skipped by both cells */
    const int n = m.n_cells, F = m.n_faces;
    const int i = m.left[f];
    double W[S], Wj[S], xi[D], xj[D], c[D], rij[D];
#pragma unroll
    for(int k = 0; k < S; ++k) W[k] = m.W[(size_t)k * n + i];
#pragma unroll
    for(int l = 0; l < D; ++l) {
        xi[l] = m.pos[(size_t)l * n + i];
        xj[l] = m.rpos[(size_t)l * F + f];
    }
    if(m.kind[f] == SFX_FACE_MIRROR) {
#pragma unroll
        for(int k = 0; k < S; ++k) Wj[k] = W[k];
        mirror_state<D>(Wj, xi, xj);
    } else {
        const int r = m.right[f];
#pragma unroll
        for(int k = 0; k < S; ++k) Wj[k] = m.W[(size_t)k * n + r];
    }
#pragma unroll
    for(int l = 0; l < D; ++l) {
        c[l] = m.mid[(size_t)l * F + f] - 0.5 * (xi[l] + xj[l]);
        rij[l] = xi[l] - xj[l];
    }
    const double rnorm = norm<D>(rij);
    double t[TS];
#pragma unroll
    for(int l = 0; l < D; ++l)
#pragma unroll
        for(int k = 0; k < S; ++k)
            t[l * S + k] =
                A * ((Wj[k] - W[k]) * c[l] / rnorm - 0.5 * (W[k] + Wj[k]) * rij[l] / rnorm);
#pragma unroll
    for(int q = D * S; q < TS; ++q) t[q] = 0.;
    double2* out = reinterpret_cast<double2*>(m.gterm + (size_t)f * TS);
#pragma unroll
    for(int q = 0; q < TS / 2; ++q) out[q] = make_double2(t[2 * q], t[2 * q + 1]);
}

/* one thread per (cell, primitive variable): the first loop adds the
 * faces' terms (subtracts them where the cell is the face's right one) in
 * the cell's face order, the second is the limiter; the variables are
 * independent in both loops, so each thread rounds exactly as the
 * one-kernel loop does */
template <int D>
__global__ void __launch_bounds__(kGradBlock, 8) k_grad_sum(sfx_dmesh m) {
    constexpr int S = D + 2, TS = D == 3 ? 16 : 8;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t / S), k = (int)(t % S);
    if(i >= sfx_grad_cells(m) || failed(m.err)) return;
    if(m.local && m.tstart[i] != m.t_now) return;
    const int n = m.n_cells, F = m.n_faces;
    const double W = m.W[(size_t)k * n + i];
    double delta[D];
    double Wmax = W, Wmin = W;
#pragma unroll
    for(int l = 0; l < D; ++l) delta[l] = 0.;
    const int beg = m.off[i], end = m.off[i + 1];
    for(int j = end - 1; j >= beg; --j) {
        const unsigned e = (unsigned)m.idx[j];
        const int f = (int)(e & ~kRightBit);
        const bool rside = (e & kRightBit) != 0;
        /* the face's loads all issued before the area test (the record of a
         * face of zero area holds stale values, never used) */
        const double A = m.area[f];
        const int kd = m.kind[f];
        const int nb = rside ? m.left[f] : m.right[f];
        const double* tf = m.gterm + (size_t)f * TS + k;
        double tv[D];
#pragma unroll
        for(int l = 0; l < D; ++l) tv[l] = tf[l * S];
        if(A == 0.) continue;
        double Wj;
        if(!rside && kd == SFX_FACE_MIRROR) {
            double Wm[S], xi[D], xj[D];
#pragma unroll
            for(int q = 0; q < S; ++q) Wm[q] = m.W[(size_t)q * n + i];
#pragma unroll
            for(int l = 0; l < D; ++l) {
                xi[l] = m.pos[(size_t)l * n + i];
                xj[l] = m.rpos[(size_t)l * F + f];
            }
            mirror_state<D>(Wm, xi, xj);
            Wj = Wm[0];
#pragma unroll
            for(int q = 1; q < S; ++q)
                if(q == k) Wj = Wm[q];
        } else {
            Wj = m.W[(size_t)k * n + nb];
        }
        if(!rside) {
#pragma unroll
            for(int l = 0; l < D; ++l) delta[l] = delta[l] + tv[l];
        } else {
#pragma unroll
            for(int l = 0; l < D; ++l) delta[l] = delta[l] - tv[l];
        }
        Wmax = (Wmax < Wj) ? Wj : Wmax;
        Wmin = (Wj < Wmin) ? Wj : Wmin;
    }
    const double V = m.vol[i];
    double cen[D];
#pragma unroll
    for(int l = 0; l < D; ++l) {
        delta[l] = delta[l] / V;
        cen[l] = m.cen[(size_t)l * n + i];
    }
    const double a = Wmax - W, b = Wmin - W;
    double alpha = 1.;
    for(int j = end - 1; j >= beg; --j) {
        const int f = (int)((unsigned)m.idx[j] & ~kRightBit);
        const double A = m.area[f];
        double d[D];
#pragma unroll
        for(int l = 0; l < D; ++l) d[l] = m.mid[(size_t)l * F + f] - cen[l];
        if(A == 0.) continue;
        double dp = delta[0] * d[0] + delta[1] * d[1];
        if(D == 3) dp = dp + delta[2] * d[2];
        const double mx = sfx_limiter_ratio(a, b, dp);
        alpha = (mx < alpha) ? mx : alpha;
    }
#pragma unroll
    for(int l = 0; l < D; ++l) m.grad[((size_t)l * S + k) * n + i] = delta[l] * alpha;
}

/* --------------------------- exact solver --------------------------- */
struct ExactOut {
    int status;
    int code;
};

template <int D>
__device__ __forceinline__ double sound(const sfx_solver_params& s, const double* W) {
    return W[0] != 0. ? sqrt(s.gamma * W[D + 1] / W[0]) : 0.;
}

template <int D>
__device__ __forceinline__ double fb(const sfx_solver_params& s, double p,
                                     const double* Wb, double a) {
    if(p > Wb[D + 1]) {
        double A = s.tdgp1 / Wb[0];
        double B = s.gm1dgp1 * Wb[D + 1];
        return (p - Wb[D + 1]) * sqrt(A / (p + B));
    }
    return s.tdgm1 * a * (sfx_pow(p / Wb[D + 1], s.gm1d2g) - 1.);
}

template <int D>
__device__ __forceinline__ double gbf(const sfx_solver_params& s, double p,
                                      const double* Wb) {
    double A = s.tdgp1 / Wb[0];
    double B = s.gm1dgp1 * Wb[D + 1];
    return sqrt(A / (p + B));
}

template <int D>
__device__ __forceinline__ double fprimeb(const sfx_solver_params& s, double p,
                                          const double* Wb, double a) {
    if(p > Wb[D + 1]) {
        double A = s.tdgp1 / Wb[0];
        double B = s.gm1dgp1 * Wb[D + 1];
        return (1. - 0.5 * (p - Wb[D + 1]) / (B + p)) * sqrt(A / (p + B));
    }
    return 1. / (Wb[0] * a) * sfx_pow(p / Wb[D + 1], -s.gp1d2g);
}

template <int D>
__device__ __forceinline__ double ff(const sfx_solver_params& s, double p,
                                     const double* WL, const double* WR,
                                     double vL, double vR, double aL, double aR) {
    return fb<D>(s, p, WL, aL) + fb<D>(s, p, WR, aR) + (vR - vL);
}

/* The last f(p) of the iteration, per side, with its power
 * sfx_pow(p / p_K, (g-1)/(2g)) on a rarefaction side.  The reference
 * evaluates f_K(p) again for the wave velocity and that power again for the
 * sampling at the same p (ExactRiemannSolver.cpp:207-265): the kept values
 * are the same operations on the same operands, so reusing them changes no
 * bit and saves the double-double powers. */
struct FLast {
    double p, fL, fR, zL, zR;
    bool ok;
};

template <int D>
__device__ __forceinline__ double fbz(const sfx_solver_params& s, double p, const double* Wb,
                                      double a, double* z) {
    if(p > Wb[D + 1]) {
        double A = s.tdgp1 / Wb[0];
        double B = s.gm1dgp1 * Wb[D + 1];
        *z = 0.;
        return (p - Wb[D + 1]) * sqrt(A / (p + B));
    }
    *z = sfx_pow(p / Wb[D + 1], s.gm1d2g);
    return s.tdgm1 * a * (*z - 1.);
}

template <int D>
__device__ __forceinline__ double ffl(const sfx_solver_params& s, double p, const double* WL,
                                      const double* WR, double vL, double vR, double aL,
                                      double aR, FLast& c) {
    c.p = p;
    c.fL = fbz<D>(s, p, WL, aL, &c.zL);
    c.fR = fbz<D>(s, p, WR, aR, &c.zR);
    c.ok = true;
    return c.fL + c.fR + (vR - vL);
}

template <int D>
__device__ __forceinline__ double fprime(const sfx_solver_params& s, double p,
                                         const double* WL, const double* WR,
                                         double aL, double aR) {
    return fprimeb<D>(s, p, WL, aL) + fprimeb<D>(s, p, WR, aR);
}

/* ExactRiemannSolver.cpp:644-673 */
template <int D>
__device__ double guess_p(const sfx_solver_params& s, const double* WL,
                          const double* WR, double vL, double vR, double aL,
                          double aR) {
    const double pL = WL[D + 1], pR = WR[D + 1];
    double pguess;
    const double pmin = (pR < pL) ? pR : pL;
    const double pmax = (pL < pR) ? pR : pL;
    const double qmax = pmax / pmin;
    double ppv = 0.5 * (pL + pR) - 0.125 * (vR - vL) * (WL[0] + WR[0]) * (aL + aR);
    double fl = s.tol * 0.5 * (pL + pR);
    ppv = (fl < ppv) ? ppv : fl;
    if(qmax <= 2. && pmin <= ppv && ppv <= pmax) {
        pguess = ppv;
    } else if(ppv < pmin) {
        pguess = sfx_pow((aL + aR - s.gm1d2 * (vR - vL)) /
                                 (aL / sfx_pow(pL, s.gm1d2g) + aR / sfx_pow(pR, s.gm1d2g)),
                         s.tgdgm1);
    } else {
        const double gL = gbf<D>(s, ppv, WL), gR = gbf<D>(s, ppv, WR);
        pguess = (gL * pL + gR * pR - vR + vL) / (gL + gR);
    }
    fl = s.tol * 0.5 * (pL + pR);
    return (fl < pguess) ? pguess : fl;
}

/* ExactRiemannSolver.cpp:462-546, capped at SFX_MAX_ITER steps */
template <int D>
__device__ double brent(const sfx_solver_params& s, double lowerLimit,
                        double upperLimit, double errorTol, const double* WL,
                        const double* WR, double vL, double vR, double aL,
                        double aR, int* iters, int* errexit, int* noconv) {
    double a = lowerLimit, b = upperLimit, c = 0., d = 1e230;
    double fa = ff<D>(s, a, WL, WR, vL, vR, aL, aR);
    double fbv = ff<D>(s, b, WL, WR, vL, vR, aL, aR);
    double fc = 0., sv = 0., fs = 0.;
    *iters = 0;
    *errexit = 0;
    if(fa * fbv >= 0) {
        *errexit = 1;
        return (fa < fbv) ? a : b;
    }
    if(fabs(fa) < fabs(fbv)) {
        double t = a;
        a = b;
        b = t;
        t = fa;
        fa = fbv;
        fbv = t;
    }
    c = a;
    fc = fa;
    bool mflag = true;
    while(!(fbv == 0) && (fabs(a - b) > errorTol * (a + b) * 0.5)) {
        if(*iters >= SFX_MAX_ITER) {
            *noconv = 1;
            break;
        }
        ++*iters;
        if((fa != fc) && (fbv != fc))
            sv = a * fbv * fc / (fa - fbv) / (fa - fc) +
                 b * fa * fc / (fbv - fa) / (fbv - fc) +
                 c * fa * fbv / (fc - fa) / (fc - fbv);
        else
            sv = b - fbv * (b - a) / (fbv - fa);
        const double tmp2 = (3. * a + b) / 4.;
        if(!(((sv > tmp2) && (sv < b)) || ((sv < tmp2) && (sv > b))) ||
           (mflag && (fabs(sv - b) >= (fabs(b - c) / 2.))) ||
           (!mflag && (fabs(sv - b) >= (fabs(c - d) / 2.))) ||
           (mflag && (fabs(b - c) < errorTol * (b + c) * 0.5)) ||
           (!mflag && (fabs(c - d) < errorTol * (c + d) * 0.5))) {
            sv = (a + b) / 2.;
            mflag = true;
        } else {
            mflag = false;
        }
        fs = ff<D>(s, sv, WL, WR, vL, vR, aL, aR);
        d = c;
        c = b;
        fc = fbv;
        if(fa * fs < 0.) {
            b = sv;
            fbv = fs;
        } else {
            a = sv;
            fa = fs;
        }
        if(fabs(fa) < fabs(fbv)) {
            double t = a;
            a = b;
            b = t;
            t = fa;
            fa = fbv;
            fbv = t;
        }
    }
    return b;
}

template <int D>
__device__ __forceinline__ bool bad_state(const double* sol) {
    bool bad = (sol[0] < 0.) || (sol[0] != sol[0]);
#pragma unroll
    for(int k = 0; k < D; ++k) bad |= (sol[1 + k] != sol[1 + k]);
    bad |= (sol[D + 1] < 0.) || (sol[D + 1] != sol[D + 1]);
    return bad;
}

/* rarefaction fan state next to vacuum or at the interface; shared shape of
 * ExactRiemannSolver.cpp:318-330 / 350-362 and HLLCRiemannSolver.cpp:59-71 */
template <int D>
__device__ __forceinline__ void fan_left(double g, const double* WL, double vL,
                                         double aL, double* sol, double* vhalf) {
    sol[0] = WL[0] * sfx_pow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * vL, 2. / (g - 1.));
    *vhalf = 2. / (g + 1.) * (aL + 0.5 * (g - 1.) * vL) - vL;
    sol[D + 1] = WL[D + 1] *
                 sfx_pow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * vL, 2. * g / (g - 1.));
}

template <int D>
__device__ __forceinline__ void fan_right(double g, const double* WR, double vR,
                                          double aR, double* sol, double* vhalf) {
    sol[0] = WR[0] * sfx_pow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * vR, 2. / (g - 1.));
    *vhalf = 2. / (g + 1.) * (-aR + 0.5 * (g - 1.) * vR) - vR;
    sol[D + 1] = WR[D + 1] *
                 sfx_pow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * vR, 2. * g / (g - 1.));
}

/* vacuum sampling shared by ExactRiemannSolver::solve_vacuum
 * (ExactRiemannSolver.cpp:304-446) and HLLCRiemannSolver::vacuum_flux's
 * first half (HLLCRiemannSolver.cpp:44-156); the conditions are written in
 * the two sources with the operands swapped but are the same predicates */
template <int D>
__device__ void vacuum_sample(double g, const double* WL, const double* WR,
                              double vL, double vR, double aL, double aR,
                              const double* n, double* sol, int* code) {
    constexpr int S = D + 2;
    double vhalf = 0.;
    if(WR[0] == 0.) {
#pragma unroll
        for(int k = 0; k < S; ++k) sol[k] = WL[k];
        if(vL < aL) {
            double SL = vL + 2. * aL / (g - 1.);
            if(SL > 0.) {
                fan_left<D>(g, WL, vL, aL, sol, &vhalf);
                *code = 2 | SFX_BRANCH_S_LFAN;
            } else {
#pragma unroll
                for(int k = 0; k < S; ++k) sol[k] = 0.;
                *code = 2 | SFX_BRANCH_S_VAC;
            }
        } else {
            *code = 2 | SFX_BRANCH_S_LUP;
        }
    } else if(WL[0] == 0.) {
#pragma unroll
        for(int k = 0; k < S; ++k) sol[k] = WR[k];
        if(-aR < vR) {
            double SR = vR - 2. * aR / (g - 1.);
            if(SR >= 0.) {
#pragma unroll
                for(int k = 0; k < S; ++k) sol[k] = 0.;
                *code = 3 | SFX_BRANCH_S_VAC;
            } else {
                fan_right<D>(g, WR, vR, aR, sol, &vhalf);
                *code = 3 | SFX_BRANCH_S_RFAN;
            }
        } else {
            *code = 3 | SFX_BRANCH_S_RUP;
        }
    } else {
        double SR = vR - 2. * aR / (g - 1.);
        double SL = vL + 2. * aL / (g - 1.);
        if(SR > 0. && SL < 0.) {
#pragma unroll
            for(int k = 0; k < S; ++k) sol[k] = 0.;
            *code = 4 | SFX_BRANCH_S_VAC;
        } else if(SL >= 0.) {
#pragma unroll
            for(int k = 0; k < S; ++k) sol[k] = WL[k];
            if(aL > vL) {
                fan_left<D>(g, WL, vL, aL, sol, &vhalf);
                *code = 4 | SFX_BRANCH_S_LFAN;
            } else {
                *code = 4 | SFX_BRANCH_S_LUP;
            }
        } else {
#pragma unroll
            for(int k = 0; k < S; ++k) sol[k] = WR[k];
            if(-aR < vR) {
                fan_right<D>(g, WR, vR, aR, sol, &vhalf);
                *code = 4 | SFX_BRANCH_S_RFAN;
            } else {
                *code = 4 | SFX_BRANCH_S_RUP;
            }
        }
    }
#pragma unroll
    for(int k = 0; k < D; ++k) sol[1 + k] = sol[1 + k] + vhalf * n[k];
}

/* ExactRiemannSolver::solve (ExactRiemannSolver.cpp:108-290).  WR becomes WL
 * for a reflective face, as in the reference. */
template <int D>
__device__ ExactOut exact_solve(const sfx_solver_params& s, double* WL, double* WR,
                                const double* n, bool reflective, double* sol) {
    constexpr int S = D + 2;
    ExactOut out{SFX_OK, 0};
    double vL = WL[1] * n[0] + WL[2] * n[1];
    double vR = WR[1] * n[0] + WR[2] * n[1];
    if(D == 3) {
        vL = vL + WL[3] * n[2];
        vR = vR + WR[3] * n[2];
    }
    if(reflective) {
#pragma unroll
        for(int k = 0; k < S; ++k) WR[k] = WL[k];
        vR = -vL;
    }
    const double aL = sound<D>(s, WL), aR = sound<D>(s, WR);
    const double g = s.gamma;
    if(WL[0] == 0. || WR[0] == 0.) {
        if(WR[0] == 0. && WL[0] == 0.) {
#pragma unroll
            for(int k = 0; k < S; ++k) sol[k] = 0.;
            out.code = 1;
            return out;
        }
        vacuum_sample<D>(g, WL, WR, vL, vR, aL, aR, n, sol, &out.code);
        if(bad_state<D>(sol)) out.status = SFX_ERR_RIEMANN;
        return out;
    }
    if(2. * aL / (g - 1.) + 2. * aR / (g - 1.) <= vR - vL) {
        vacuum_sample<D>(g, WL, WR, vL, vR, aL, aR, n, sol, &out.code);
        if(bad_state<D>(sol)) out.status = SFX_ERR_RIEMANN;
        return out;
    }
    const double tol = s.tol;
    double p = 0.;
    double pguess = guess_p<D>(s, WL, WR, vL, vR, aL, aR);
    /* f(0): on both sides the rarefaction branch with sfx_pow(0, e) = +0
     * (e > 0), i.e. (2/(g-1) a_K) * (0 - 1) exactly */
    const double fp = WL[D + 1] > 0. && WR[D + 1] > 0.
                              ? s.tdgm1 * aL * (0. - 1.) + s.tdgm1 * aR * (0. - 1.) + (vR - vL)
                              : ff<D>(s, p, WL, WR, vL, vR, aL, aR);
    FLast last;
    last.ok = false;
    double fpguess = ffl<D>(s, pguess, WL, WR, vL, vR, aL, aR, last);
    int newton = 0, brent_it = 0, errexit = 0, noconv = 0, mode;
    if(fp < s.cutoff) {
        mode = 1 << 3;
        while(fabs(p - pguess) > tol * 0.5 * (p + pguess)) {
            if(newton >= SFX_MAX_ITER) {
                noconv = 1;
                break;
            }
            ++newton;
            p = pguess;
            pguess = pguess - fpguess / fprime<D>(s, pguess, WL, WR, aL, aR);
            if(pguess < 0.) pguess = 0.;
            fpguess = ffl<D>(s, pguess, WL, WR, vL, vR, aL, aR, last);
        }
        p = pguess;
    } else {
        mode = 2 << 3;
        if(fp * fpguess >= 0.) {
            while(fabs(p - pguess) > tol * 0.5 * (p + pguess) && fpguess < 0.) {
                if(newton >= SFX_MAX_ITER) {
                    noconv = 1;
                    break;
                }
                ++newton;
                p = pguess;
                pguess = pguess - fpguess / fprime<D>(s, pguess, WL, WR, aL, aR);
                fpguess = ffl<D>(s, pguess, WL, WR, vL, vR, aL, aR, last);
            }
        }
        if(!noconv && fabs(p - pguess) > tol * 0.5 * (p + pguess) && fpguess > 0.) {
            mode = 3 << 3;
            p = brent<D>(s, 0., pguess, tol, WL, WR, vL, vR, aL, aR, &brent_it,
                         &errexit, &noconv);
        } else {
            p = pguess;
        }
    }
    const bool at_p = last.ok && last.p == p;
    const double u = 0.5 * (vL + vR) + 0.5 * ((at_p ? last.fR : fb<D>(s, p, WR, aR)) -
                                             (at_p ? last.fL : fb<D>(s, p, WL, aL)));
    double vhalf;
    int region;
    if(u < 0) {
#pragma unroll
        for(int k = 0; k < S; ++k) sol[k] = WR[k];
        const double pdpR = p / WR[D + 1];
        if(p > WR[D + 1]) {
            const double SR = vR + aR * sqrt(s.gp1d2g * pdpR + s.gm1d2g);
            if(SR > 0) {
                sol[0] = WR[0] * (pdpR + s.gm1dgp1) / (s.gm1dgp1 * pdpR + 1.);
                sol[D + 1] = p;
                vhalf = u - vR;
                region = SFX_BRANCH_S_RSHOCK_STAR;
            } else {
                vhalf = 0.;
                region = SFX_BRANCH_S_RUP_SHOCK;
            }
        } else {
            const double SHR = vR + aR;
            if(SHR > 0) {
                const double STR = u + aR * (at_p ? last.zR : sfx_pow(pdpR, s.gm1d2g));
                if(STR <= 0) {
                    sol[0] = WR[0] * sfx_pow(s.tdgp1 - s.gm1dgp1 / aR * vR, s.tdgm1);
                    vhalf = s.tdgp1 * (-aR + s.gm1d2 * vR) - vR;
                    sol[D + 1] = WR[D + 1] * sfx_pow(s.tdgp1 - s.gm1dgp1 / aR * vR, s.tgdgm1);
                    region = SFX_BRANCH_S_RFAN;
                } else {
                    sol[0] = WR[0] * sfx_pow(pdpR, s.ginv);
                    sol[D + 1] = p;
                    vhalf = u - vR;
                    region = SFX_BRANCH_S_RRARE_STAR;
                }
            } else {
                vhalf = 0.;
                region = SFX_BRANCH_S_RUP;
            }
        }
    } else {
#pragma unroll
        for(int k = 0; k < S; ++k) sol[k] = WL[k];
        const double pdpL = p / WL[D + 1];
        if(p > WL[D + 1]) {
            const double SL = vL - aL * sqrt(s.gp1d2g * pdpL + s.gm1d2g);
            if(SL < 0) {
                sol[0] = WL[0] * (pdpL + s.gm1dgp1) / (s.gm1dgp1 * pdpL + 1.);
                sol[D + 1] = p;
                vhalf = u - vL;
                region = SFX_BRANCH_S_LSHOCK_STAR;
            } else {
                vhalf = 0.;
                region = SFX_BRANCH_S_LUP_SHOCK;
            }
        } else {
            const double SHL = vL - aL;
            if(SHL < 0) {
                const double STL = u - aL * (at_p ? last.zL : sfx_pow(pdpL, s.gm1d2g));
                if(STL > 0) {
                    sol[0] = WL[0] * sfx_pow(s.tdgp1 + s.gm1dgp1 / aL * vL, s.tdgm1);
                    vhalf = s.tdgp1 * (aL + s.gm1d2 * vL) - vL;
                    sol[D + 1] = WL[D + 1] * sfx_pow(s.tdgp1 + s.gm1dgp1 / aL * vL, s.tgdgm1);
                    region = SFX_BRANCH_S_LFAN;
                } else {
                    sol[0] = WL[0] * sfx_pow(pdpL, s.ginv);
                    vhalf = u - vL;
                    sol[D + 1] = p;
                    region = SFX_BRANCH_S_LRARE_STAR;
                }
            } else {
                vhalf = 0.;
                region = SFX_BRANCH_S_LUP;
            }
        }
    }
#pragma unroll
    for(int k = 0; k < D; ++k) sol[1 + k] = sol[1 + k] + vhalf * n[k];
    out.code = mode | region | (min(newton, 127) << 9) | (min(brent_it, 127) << 16) |
               (errexit ? (1 << 23) : 0);
    if(noconv)
        out.status = SFX_ERR_NOCONV;
    else if(bad_state<D>(sol))
        out.status = SFX_ERR_RIEMANN;
    return out;
}

/* ExactRiemannSolver::get_flux (:815-836) contracted with the normal
 * (solve_for_flux :858-880) */
template <int D>
__device__ __forceinline__ void exact_flux_from_half(double gamma, const double* Wh,
                                                     const double* v, const double* n,
                                                     double* flux) {
    constexpr int S = D + 2;
    double F[D][S];
#pragma unroll
    for(int idx = 0; idx < D; ++idx) {
#pragma unroll
        for(int k = 0; k < S; ++k) F[idx][k] = 0.;
        if(Wh[0] == 0.) continue;
        const double un = Wh[1 + idx] - v[idx];
        F[idx][0] = Wh[0] * un;
        F[idx][1] = Wh[0] * un * Wh[1];
        F[idx][2] = Wh[0] * un * Wh[2];
        if(D == 3) F[idx][3] = Wh[0] * un * Wh[3];
        double v2 = Wh[1] * Wh[1] + Wh[2] * Wh[2];
        if(D == 3) v2 = v2 + Wh[3] * Wh[3];
        const double e = 0.5 * Wh[0] * v2 + Wh[D + 1] / (gamma - 1.);
        F[idx][1 + idx] = F[idx][1 + idx] + Wh[D + 1];
        F[idx][D + 1] = un * e + Wh[D + 1] * Wh[1 + idx];
    }
#pragma unroll
    for(int k = 0; k < S; ++k) {
        double s = F[0][k] * n[0] + F[1][k] * n[1];
        if(D == 3) s = s + F[2][k] * n[2];
        flux[k] = s;
    }
}

/* ----------------------------- HLLC solver ----------------------------- */
template <int D>
__device__ __forceinline__ void hllc_deboost(const double* v, double* flux) {
    flux[1] = flux[1] + v[0] * flux[0];
    flux[2] = flux[2] + v[1] * flux[0];
    if(D == 3) {
        flux[3] = flux[3] + v[2] * flux[0];
        const double nrm2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        flux[4] = flux[4] + (v[0] * flux[1] + v[1] * flux[2] + v[2] * flux[3] +
                             0.5 * nrm2 * flux[0]);
    } else {
        const double nrm2 = v[0] * v[0] + v[1] * v[1];
        flux[D + 1] = flux[D + 1] + (v[0] * flux[1] + v[1] * flux[2] + 0.5 * nrm2 * flux[0]);
    }
}

/* HLLCRiemannSolver::solve_for_flux (HLLCRiemannSolver.cpp:258-403) */
template <int D>
__device__ int hllc_flux(const sfx_solver_params& s, double* WL, double* WR,
                         const double* n, const double* v, bool reflective,
                         double* flux) {
    constexpr int S = D + 2;
    const double g = s.gamma;
    int code = SFX_BRANCH_HLLC;
#pragma unroll
    for(int k = 0; k < S; ++k) flux[k] = 0.;
    if(WL[0] == 0. && (reflective || WR[0] == 0.)) return code | 1;
    double uL = WL[1] * n[0] + WL[2] * n[1];
    double uR = WR[1] * n[0] + WR[2] * n[1];
    if(D == 3) {
        uL = uL + WL[3] * n[2];
        uR = uR + WR[3] * n[2];
    }
    if(reflective) {
#pragma unroll
        for(int k = 0; k < S; ++k) WR[k] = WL[k];
        uR = -uL;
    }
    const double aL = sqrt(g * WL[D + 1] / WL[0]);
    const double aR = sqrt(g * WR[D + 1] / WR[0]);
    if(WL[0] == 0. || WR[0] == 0. || 2. * aL / (g - 1.) + 2. * aR / (g - 1.) <= uR - uL) {
        double sol[S];
        int vc = 0;
        vacuum_sample<D>(g, WL, WR, uL, uR, aL, aR, n, sol, &vc);
        code |= vc;
        if(sol[0] == 0.) return code;
        double vsol = sol[1] * n[0] + sol[2] * n[1];
        double v2 = sol[1] * sol[1] + sol[2] * sol[2];
        if(D == 3) {
            vsol = vsol + sol[3] * n[2];
            v2 = v2 + sol[3] * sol[3];
        }
        flux[0] = sol[0] * vsol;
        flux[1] = sol[0] * sol[1] * vsol + sol[D + 1] * n[0];
        flux[2] = sol[0] * sol[2] * vsol + sol[D + 1] * n[1];
        if(D == 3) flux[3] = sol[0] * sol[3] * vsol + sol[D + 1] * n[2];
        const double e = sol[D + 1] / (g - 1.) / sol[0] + 0.5 * v2;
        flux[D + 1] = sol[0] * e * vsol + sol[D + 1] * vsol;
        hllc_deboost<D>(v, flux);
        return code;
    }
    const double rhobar = 0.5 * (WL[0] + WR[0]);
    const double abar = 0.5 * (aL + aR);
    const double pPVRS = 0.5 * (WL[D + 1] + WR[D + 1]) - 0.5 * (uR - uL) * rhobar * abar;
    const double pstar = (0. < pPVRS) ? pPVRS : 0.;
    double qL = 1., qR = 1.;
    if(pstar > WL[D + 1]) qL = sqrt(1. + 0.5 * (g + 1.) / g * (pstar / WL[D + 1] - 1.));
    if(pstar > WR[D + 1]) qR = sqrt(1. + 0.5 * (g + 1.) / g * (pstar / WR[D + 1] - 1.));
    const double SL = uL - aL * qL;
    const double SR = uR + aR * qR;
    const double Sstar = (WR[D + 1] - WL[D + 1] + WL[0] * uL * (SL - uL) -
                          WR[0] * uR * (SR - uR)) /
                         (WL[0] * (SL - uL) - WR[0] * (SR - uR));
    const bool left = Sstar >= 0.;
    const double* Wk = left ? WL : WR;
    const double uk = left ? uL : uR;
    const double Sk = left ? SL : SR;
    flux[0] = Wk[0] * uk;
    flux[1] = Wk[0] * Wk[1] * uk + Wk[D + 1] * n[0];
    flux[2] = Wk[0] * Wk[2] * uk + Wk[D + 1] * n[1];
    double v2 = Wk[1] * Wk[1] + Wk[2] * Wk[2];
    if(D == 3) {
        flux[3] = Wk[0] * Wk[3] * uk + Wk[D + 1] * n[2];
        v2 = v2 + Wk[3] * Wk[3];
    }
    const double ek = Wk[D + 1] / (g - 1.) / Wk[0] + 0.5 * v2;
    flux[D + 1] = Wk[0] * ek * uk + Wk[D + 1] * uk;
    const bool star = left ? (SL < 0.) : (SR > 0.);
    if(star) {
        double U[S];
        U[0] = 1.;
        U[1] = Wk[1] + (Sstar - uk) * n[0];
        U[2] = Wk[2] + (Sstar - uk) * n[1];
        if(D == 3) U[3] = Wk[3] + (Sstar - uk) * n[2];
        U[D + 1] = ek + (Sstar - uk) * (Sstar + Wk[D + 1] / (Wk[0] * (Sk - uk)));
        const double fac = Wk[0] * (Sk - uk) / (Sk - Sstar);
#pragma unroll
        for(int k = 0; k < S; ++k) U[k] = U[k] * fac;
        flux[0] = flux[0] + Sk * (U[0] - Wk[0]);
        flux[1] = flux[1] + Sk * (U[1] - Wk[0] * Wk[1]);
        flux[2] = flux[2] + Sk * (U[2] - Wk[0] * Wk[2]);
        if(D == 3) flux[3] = flux[3] + Sk * (U[3] - Wk[0] * Wk[3]);
        flux[D + 1] = flux[D + 1] + Sk * (U[D + 1] - Wk[0] * ek);
    }
    code |= left ? (star ? SFX_BRANCH_HLLC_LSTAR : SFX_BRANCH_HLLC_L)
                 : (star ? SFX_BRANCH_HLLC_RSTAR : SFX_BRANCH_HLLC_R);
    hllc_deboost<D>(v, flux);
    return code;
}

/* -------------------------------- faces -------------------------------- */

/* MUSCL-Hancock prediction + reconstruction + pairwise limiter + positivity
 * fallbacks for one side (VorFace.cpp:715-759 right, 762-804 left) */
template <int D>
__device__ __forceinline__ void predict_side(double gamma, double dt, double* Wt,
                                             const double* Wself, const double* Wother,
                                             const double (*g)[D + 2], const double* d,
                                             bool do_limit, double r) {
    constexpr int S = D + 2;
    double dW0[S], dW[S];
    time_derivative<D>(gamma, Wt, g, dW0);
#pragma unroll
    for(int k = 0; k < S; ++k) dW[k] = 0.5 * dt * dW0[k];
    reconstruct<D>(Wt, g, d);
    if(do_limit) {
        double dn = sqrt(dot<D>(d, d));
#pragma unroll
        for(int k = 0; k < S; ++k) Wt[k] = limit1<D>(Wt[k], Wself[k], Wother[k], dn, r);
    }
    if(Wt[0] < 0. || Wt[D + 1] < 0.) {
#pragma unroll
        for(int k = 0; k < S; ++k) Wt[k] = Wself[k];
    }
#pragma unroll
    for(int k = 0; k < S; ++k) Wt[k] = Wt[k] + dW[k];
    if(Wt[0] < 0. || Wt[D + 1] < 0.) {
#pragma unroll
        for(int k = 0; k < S; ++k) Wt[k] = Wt[k] - dW[k];
    }
}

template <int D, int SOLVER>
__global__ void __launch_bounds__(128) k_faces(sfx_dmesh m, sfx_solver_params sp,
                                               double dt, int write_branch) {
    constexpr int S = D + 2;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if(f >= sfx_flux_faces(m) || failed(m.err)) return;
    const int n = m.n_cells, F = m.n_faces;
    const double A = m.area[f];
    if(A == 0.) {
#pragma unroll
        for(int k = 0; k < S; ++k) m.dQf[(size_t)k * F + f] = 0.;
        if(write_branch) m.branch[f] = SFX_BRANCH_SKIPPED;
        return;
    }
    const int iL = m.left[f];
    const int kind = m.kind[f];
    const bool has_right = kind != SFX_FACE_MIRROR;
    const int iR = has_right ? m.right[f] : 0;
    /* local time steps (VorFace.cpp:672-697): a face is computed when its
     * left cell is active, or (with a right cell) either cell is; its time
     * step is the shorter of the two cells' steps */
    double dtmax = dt;
    if(m.local) {
        const bool aL = m.tstart[iL] == m.t_now;
        const bool aR = has_right && m.tstart[iR] == m.t_now;
        if(!aL && !aR) {
#pragma unroll
            for(int k = 0; k < S; ++k) m.dQf[(size_t)k * F + f] = 0.;
            if(write_branch) m.branch[f] = SFX_BRANCH_SKIPPED;
            return;
        }
        dt = sfx_realtime(m.t_total, m.tend[iL] - m.tstart[iL]);
        dtmax = dt;
        if(has_right) {
            const double dtR = sfx_realtime(m.t_total, m.tend[iR] - m.tstart[iR]);
            dt = fmin(dt, dtR);
            dtmax = fmax(dtmax, dtR);
        }
    }
    double v[D], mid[D], xL[D], xRi[D], cenL[D];
#pragma unroll
    for(int l = 0; l < D; ++l) {
        v[l] = m.vel ? m.vel[(size_t)l * F + f] : 0.;
        mid[l] = m.mid[(size_t)l * F + f];
        xL[l] = m.pos[(size_t)l * n + iL];
        xRi[l] = m.rpos[(size_t)l * F + f];
        cenL[l] = m.cen[(size_t)l * n + iL];
    }
    double WL[S], WR[S], WRrec[S], Wt[S];
#pragma unroll
    for(int k = 0; k < S; ++k) {
        WL[k] = m.W[(size_t)k * n + iL];
        WR[k] = has_right ? m.W[(size_t)k * n + iR] : 0.;
        WRrec[k] = 0.;
    }
#pragma unroll
    for(int l = 0; l < D; ++l) {
        WL[1 + l] = WL[1 + l] - v[l];
        WR[1 + l] = WR[1 + l] - v[l];
    }
    double r = 0.;
    if(has_right) {
        double cenR[D], xR[D], d[D], g[D][S];
#pragma unroll
        for(int l = 0; l < D; ++l) {
            cenR[l] = m.cen[(size_t)l * n + iR];
            xR[l] = m.pos[(size_t)l * n + iR];
            d[l] = mid[l] - cenR[l] + (xR[l] - xRi[l]);
        }
#pragma unroll
        for(int l = 0; l < D; ++l)
#pragma unroll
            for(int k = 0; k < S; ++k) g[l][k] = m.grad[((size_t)l * S + k) * n + iR];
        double cd[D];
#pragma unroll
        for(int l = 0; l < D; ++l) cd[l] = cenL[l] - cenR[l];
        r = norm<D>(cd);
#pragma unroll
        for(int k = 0; k < S; ++k) Wt[k] = WR[k];
        predict_side<D>(sp.gamma, dt, Wt, WR, WL, g, d, true, r);
#pragma unroll
        for(int k = 0; k < S; ++k) WRrec[k] = Wt[k];
    }
    {
        double d[D], g[D][S];
#pragma unroll
        for(int l = 0; l < D; ++l) d[l] = mid[l] - cenL[l] + (xL[l] - xL[l]);
#pragma unroll
        for(int l = 0; l < D; ++l)
#pragma unroll
            for(int k = 0; k < S; ++k) g[l][k] = m.grad[((size_t)l * S + k) * n + iL];
#pragma unroll
        for(int k = 0; k < S; ++k) Wt[k] = WL[k];
        predict_side<D>(sp.gamma, dt, Wt, WL, WR, g, d, has_right, r);
    }
    if(WL[0] != 0.) {
#pragma unroll
        for(int k = 0; k < S; ++k) WL[k] = Wt[k];
    }
    if(WR[0] != 0.) {
#pragma unroll
        for(int k = 0; k < S; ++k) WR[k] = WRrec[k];
    }
    /* VorFace::get_normal (VorFace.cpp:553-571) */
    double nrm[D];
    {
        double dd[D];
#pragma unroll
        for(int l = 0; l < D; ++l) dd[l] = xL[l] - xRi[l];
        const double dn = norm<D>(dd);
#pragma unroll
        for(int l = 0; l < D; ++l) nrm[l] = -dd[l] / dn;
    }
    double flux[S];
    int status = SFX_OK, code;
    if(SOLVER == SFX_SOLVER_EXACT) {
        double half[S];
        ExactOut eo = exact_solve<D>(sp, WL, WR, nrm, !has_right, half);
        status = eo.status;
        code = eo.code;
#pragma unroll
        for(int l = 0; l < D; ++l) half[1 + l] = half[1 + l] + v[l];
        exact_flux_from_half<D>(sp.gamma, half, v, nrm, flux);
    } else {
        code = hllc_flux<D>(sp, WL, WR, nrm, v, !has_right, flux);
    }
    double dQL[S], dQR[S];
#pragma unroll
    for(int k = 0; k < S; ++k) {
        dQL[k] = dt * A * flux[k];
        dQR[k] = -dt * A * flux[k];
    }
    /* over-flux limiter (VorFace.cpp:837-866): timefac = dt / (the longer
     * of the two cells' steps); dt / dt with one global step */
    double timefac = 1.;
    if(has_right) timefac = dt / dtmax;
    double areafac = A / m.tarea[iL];
    areafac = areafac * timefac;
    const double QLm = m.Q[iL];
    if(dQL[0] > areafac * QLm) {
        const double corfac = fabs(areafac * QLm / dQL[0]);
#pragma unroll
        for(int k = 0; k < S; ++k) dQL[k] = dQL[k] * corfac;
#pragma unroll
        for(int k = 0; k < S; ++k) dQR[k] = -1. * dQL[k];
        code |= SFX_BRANCH_LIMIT_L;
    }
    if(has_right) {
        double areafacR = A / m.tarea[iR];
        areafacR = areafacR * timefac;
        const double QRm = m.Q[iR];
        if(dQR[0] > areafacR * QRm) {
            const double corfac = fabs(areafacR * QRm / dQR[0]);
#pragma unroll
            for(int k = 0; k < S; ++k) dQR[k] = dQR[k] * corfac;
#pragma unroll
            for(int k = 0; k < S; ++k) dQL[k] = -1. * dQR[k];
            code |= SFX_BRANCH_LIMIT_R;
        }
    }
#pragma unroll
    for(int k = 0; k < S; ++k) m.dQf[(size_t)k * F + f] = dQL[k];
    if(write_branch) m.branch[f] = code;
    if(status == SFX_OK && flux[0] != flux[0]) status = SFX_ERR_NAN_FLUX;
    if(status != SFX_OK) report_face(m.err, f, status);
}

/* ------------------------------ update ------------------------------ */

/* get_W (ExactRiemannSolver.cpp:716-766 == HLLCRiemannSolver.cpp:495-535 on
 * the hydro fields); may rewrite Q[D+1] (pressure floor) */
template <int D>
__device__ __forceinline__ void get_W(double gamma, double V, double* Q, double* W) {
    constexpr int S = D + 2;
#pragma unroll
    for(int k = 0; k < S; ++k) W[k] = 0.;
    if(Q[0] == 0.) return;
    W[0] = Q[0] / V;
    W[1] = Q[1] / Q[0];
    W[2] = Q[2] / Q[0];
    double p2 = Q[1] * Q[1] + Q[2] * Q[2];
    if(D == 3) {
        W[3] = Q[3] / Q[0];
        p2 = p2 + Q[3] * Q[3];
    }
    W[D + 1] = (gamma - 1.) * (Q[D + 1] - 0.5 * p2 / Q[0]) / V;
    if(W[D + 1] < 1.e-30) {
        W[D + 1] = 1.e-30;
        Q[D + 1] = 0.5 * p2 / Q[0] + W[D + 1] * V / (gamma - 1.);
    }
    if(W[0] < 1.e-30) {
#pragma unroll
        for(int k = 0; k < S; ++k) W[k] = 0.;
    }
}

template <int D>
__global__ void __launch_bounds__(128) k_apply(sfx_dmesh m, double gamma) {
    constexpr int S = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= sfx_update_cells(m) || failed(m.err)) return;
    const int n = m.n_cells, F = m.n_faces;
    double dQ[S];
#pragma unroll
    for(int k = 0; k < S; ++k) dQ[k] = 0.;
    const int beg = m.off[i], end = m.off[i + 1];
    /* the cell's faces in ascending face order (aidx), the order in which
     * the reference's face loop adds them */
    for(int j = beg; j < end; ++j) {
        const unsigned e = (unsigned)m.aidx[j];
        const int f = (int)(e & ~kRightBit);
        if(m.area[f] == 0.) continue;
        if(e & kRightBit) {
#pragma unroll
            for(int k = 0; k < S; ++k) dQ[k] = dQ[k] + -1. * m.dQf[(size_t)k * F + f];
        } else {
#pragma unroll
            for(int k = 0; k < S; ++k) dQ[k] = dQ[k] + m.dQf[(size_t)k * F + f];
        }
    }
    double Q[S], W[S];
#pragma unroll
    for(int k = 0; k < S; ++k) Q[k] = m.Q[(size_t)k * n + i] - dQ[k];
    if(Q[0] < 0. || Q[D + 1] < 0.) {
        report_cell(m.err, i, SFX_ERR_NEG_STATE);
        return;
    }
    if(m.local && m.tend[i] != m.t_next) {
        /* local time steps: a cell in the middle of its step takes the flux
         * of its active neighbours into Q; its W waits for the end of its
         * step (src/Simulation.cpp:791-836) */
#pragma unroll
        for(int k = 0; k < S; ++k) m.Q[(size_t)k * n + i] = Q[k];
        return;
    }
    get_W<D>(gamma, m.vol[i], Q, W);
#pragma unroll
    for(int k = 0; k < S; ++k) {
        m.Q[(size_t)k * n + i] = Q[k];
        m.W[(size_t)k * n + i] = W[k];
    }
}

/* Q = get_Q(V, W): ExactRiemannSolver.cpp:776-804 / HLLCRiemannSolver.cpp:471-483 */
template <int D>
__global__ void k_init_Q(sfx_dmesh m, double gamma, int kind) {
    constexpr int S = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m.n_cells) return;
    const int n = m.n_cells;
    double W[S], Q[S];
#pragma unroll
    for(int k = 0; k < S; ++k) W[k] = m.W[(size_t)k * n + i];
    const double V = m.vol[i];
    Q[0] = W[0] * V;
    Q[1] = Q[0] * W[1];
    Q[2] = Q[0] * W[2];
    double v2 = W[1] * W[1] + W[2] * W[2];
    if(D == 3) {
        Q[3] = Q[0] * W[3];
        v2 = v2 + W[3] * W[3];
    }
    if(kind == SFX_SOLVER_EXACT) {
        Q[D + 1] = (0.5 * W[0] * v2 + W[D + 1] / (gamma - 1.)) * V;
        if(Q[0] < 0. || Q[D + 1] < 0.) report_cell(m.err, i, SFX_ERR_NEG_STATE);
    } else {
        Q[D + 1] = V * W[D + 1] / (gamma - 1.) + 0.5 * Q[0] * v2;
    }
#pragma unroll
    for(int k = 0; k < S; ++k) m.Q[(size_t)k * n + i] = Q[k];
}

/* deterministic totals: fixed 1024 blocks over fixed ranges, fixed tree */
constexpr int kTotBlocks = 1024;
constexpr int kTotThreads = 256;

/* sums of the fields over cells [0, count) of Q [S][n] */
__global__ void k_totals_partial(const double* Q, int n, int count, int S, double* part) {
    __shared__ double sh[kTotThreads];
    const int per = (count + kTotBlocks - 1) / kTotBlocks;
    const int b0 = blockIdx.x * per;
    const int b1 = min(count, b0 + per);
    for(int k = 0; k < S; ++k) {
        double acc = 0.;
        for(int i = b0 + threadIdx.x; i < b1; i += kTotThreads) acc = acc + Q[(size_t)k * n + i];
        sh[threadIdx.x] = acc;
        __syncthreads();
        for(int w = kTotThreads / 2; w > 0; w >>= 1) {
            if(threadIdx.x < w) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + w];
            __syncthreads();
        }
        if(threadIdx.x == 0) part[k * kTotBlocks + blockIdx.x] = sh[0];
        __syncthreads();
    }
}

__global__ void k_totals_final(double* part, int S) {
    __shared__ double sh[kTotBlocks];
    for(int k = 0; k < S; ++k) {
        for(int t = threadIdx.x; t < kTotBlocks; t += blockDim.x) sh[t] = part[k * kTotBlocks + t];
        __syncthreads();
        for(int w = kTotBlocks / 2; w > 0; w >>= 1) {
            for(int t = threadIdx.x; t < w; t += blockDim.x) sh[t] = sh[t] + sh[t + w];
            __syncthreads();
        }
        if(threadIdx.x == 0) part[S * kTotBlocks + k] = sh[0];
        __syncthreads();
    }
}

template <int D, int SOLVER>
__global__ void k_riemann(sfx_solver_params sp, int n, const double* WLa,
                          const double* WRa, const double* na, int reflective,
                          double* half, double* flux, int32_t* code) {
    constexpr int S = D + 2;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= n) return;
    double L[S], R[S], nn[D], v[D], fl[S];
#pragma unroll
    for(int l = 0; l < D; ++l) {
        nn[l] = na[(size_t)t * D + l];
        v[l] = 0.;
    }
    int c, st = SFX_OK;
    if(SOLVER == SFX_SOLVER_EXACT) {
#pragma unroll
        for(int k = 0; k < S; ++k) {
            L[k] = WLa[(size_t)t * S + k];
            R[k] = WRa[(size_t)t * S + k];
        }
        double h[S];
        ExactOut eo = exact_solve<D>(sp, L, R, nn, reflective != 0, h);
        if(half) {
#pragma unroll
            for(int k = 0; k < S; ++k) half[(size_t)t * S + k] = h[k];
        }
        st = eo.status;
        c = eo.code;
#pragma unroll
        for(int l = 0; l < D; ++l) h[1 + l] = h[1 + l] + v[l];
        exact_flux_from_half<D>(sp.gamma, h, v, nn, fl);
    } else {
#pragma unroll
        for(int k = 0; k < S; ++k) {
            L[k] = WLa[(size_t)t * S + k];
            R[k] = WRa[(size_t)t * S + k];
        }
        c = hllc_flux<D>(sp, L, R, nn, v, reflective != 0, fl);
    }
#pragma unroll
    for(int k = 0; k < S; ++k) flux[(size_t)t * S + k] = fl[k];
    code[t] = st ? -st : c;
}

/* halo records of a split mesh: [count][S + 1], the cell's W then its mass
 * Q[0] (the only Q field the face kernel reads of a cell it does not
 * update); an index outside the mesh is skipped, never dereferenced */
__global__ void k_pack_cells(sfx_dmesh m, const int32_t* idx, int count, double* out) {
    const int S = m.S, R = S + 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= (long long)count * R) return;
    const int j = (int)(t / R), q = (int)(t % R);
    const int c = idx[j];
    if(c < 0 || c >= m.n_cells) return;
    out[t] = q < S ? m.W[(size_t)q * m.n_cells + c] : m.Q[c];
}

__global__ void k_unpack_cells(sfx_dmesh m, const int32_t* idx, int count, const double* in) {
    const int S = m.S, R = S + 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= (long long)count * R) return;
    const int j = (int)(t / R), q = (int)(t % R);
    const int c = idx[j];
    if(c < 0 || c >= m.n_cells) return;
    if(q < S)
        m.W[(size_t)q * m.n_cells + c] = in[t];
    else
        m.Q[c] = in[t];
}

inline int grid_for(long long n, int block) {
    return (int)((n + block - 1) / block);
}

inline int cuda_status(cudaError_t e) {
    return e == cudaSuccess ? SFX_OK : SFX_ERR_CUDA;
}

/* --------------------------- moving generators ---------------------------
 * One step of a moving mesh (a build of the reference without -DSTATIC):
 * every generator gets the velocity of VorCell::get_velocity
 * (src/VorCell.cpp:966-1008: the fluid velocity plus a term that steers the
 * generator towards its cell's centroid, at the sound speed when the offset
 * exceeds 1/4 of the cell radius, ramped in between; suppressed linearly
 * below density 1e-10), without the fluid velocity when a reflective unit
 * box would be left within dt (src/Simulation.cpp:366-398, RectangularBox::
 * inside); every face the velocity of VorFace::set_v
 * (src/VorFace.cpp:586-660: the mean of its generators' velocities plus the
 * part that keeps the face between them; a 3D mirror face does not move, a
 * 2D mirror generator moves as the mirror image of its cell's generator);
 * after the update the generators drift, x + dt v (Particle::drift,
 * src/utilities/Particle.cpp:281-283).  Same IEEE operations in the same
 * order as the reference, cube roots by sfx_cbrt. */
constexpr double kPi = 3.14159265358979323846;

template <int D>
__global__ void __launch_bounds__(128) k_gen_velocity(sfx_dmesh m, double gamma, double dt,
                                                      int periodic) {
    constexpr int S = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m.n_cells) return;
    /* local time steps: only the cells starting a step set their velocity
     * (the first kick of src/Simulation.cpp:366-398) */
    if(m.local && m.tstart[i] != m.t_now) return;
    const int n = m.n_cells;
    double W[S];
#pragma unroll
    for(int k = 0; k < S; ++k) W[k] = m.W[(size_t)k * n + i];
    double vel[D];
#pragma unroll
    for(int l = 0; l < D; ++l) vel[l] = 0.;
    if(W[0] != 0.) {
        double d[D];
#pragma unroll
        for(int l = 0; l < D; ++l) d[l] = m.cen[(size_t)l * n + i] - m.pos[(size_t)l * n + i];
        double Ri = m.vol[i];
        /* GasParticle::get_soundspeed: the solver's sqrt(gamma p / rho) */
        const double csnd = sqrt(gamma * W[D + 1] / W[0]);
        if(D == 3)
            Ri = sfx_cbrt(3. * Ri / 4. / kPi);
        else
            Ri = sqrt(Ri / kPi);
        const double dn = norm<D>(d);
        const double check = 4. * dn / Ri;
        if(check > 0.9) {
            double fac;
            if(check < 1.1)
                fac = csnd / dn * (dn - 0.9 * 0.25 * Ri) / (0.2 * 0.25 * Ri);
            else
                fac = csnd / dn;
#pragma unroll
            for(int l = 0; l < D; ++l) vel[l] = fac * d[l];
        }
    }
    double v[D];
#pragma unroll
    for(int l = 0; l < D; ++l) v[l] = W[1 + l] + vel[l];
    if(W[0] < 1.e-10) {
        const double fac = W[0] * 1.e10;
#pragma unroll
        for(int l = 0; l < D; ++l) v[l] = fac * v[l];
    }
    if(!periodic) {
        /* with local time steps, the cell's own step
         * (get_realtime_interval(end - start)) */
        const double dti = m.local ? sfx_realtime_interval(m.t_total, m.tend[i] - m.tstart[i]) : dt;
        bool inside = true;
#pragma unroll
        for(int l = 0; l < D; ++l) {
            const double nx = m.pos[(size_t)l * n + i] + dti * v[l];
            if(fabs(0.5 - nx) > 0.5) inside = false;
        }
        if(!inside) {
#pragma unroll
            for(int l = 0; l < D; ++l) v[l] -= W[1 + l];
        }
    }
#pragma unroll
    for(int l = 0; l < D; ++l) m.vgen[(size_t)l * n + i] = v[l];
}

template <int D>
__global__ void __launch_bounds__(128) k_face_velocity(sfx_dmesh m) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if(f >= m.n_faces) return;
    const int n = m.n_cells, F = m.n_faces;
    const int iL = m.left[f];
    const int kind = m.kind[f];
    double xl[D], xr[D], mid[D], vl[D], vr[D];
#pragma unroll
    for(int l = 0; l < D; ++l) {
        xl[l] = m.pos[(size_t)l * n + iL];
        xr[l] = m.rpos[(size_t)l * F + f];
        mid[l] = m.mid[(size_t)l * F + f];
        vl[l] = m.vgen[(size_t)l * n + iL];
    }
    if(kind != SFX_FACE_MIRROR) {
        const int iR = m.right[f];
#pragma unroll
        for(int l = 0; l < D; ++l) vr[l] = m.vgen[(size_t)l * n + iR];
    } else if(D == 3) {
#pragma unroll
        for(int l = 0; l < D; ++l) m.vel[(size_t)l * F + f] = 0.;
        return;
    } else {
        double Wd[4] = {0., vl[0], vl[1], 0.};
        mirror_state<2>(Wd, xl, xr);
        vr[0] = Wd[1];
        vr[1] = Wd[2];
    }
    double rRL[D];
#pragma unroll
    for(int l = 0; l < D; ++l) rRL[l] = xr[l] - xl[l];
    double r2 = rRL[0] * rRL[0] + rRL[1] * rRL[1];
    if(D == 3) r2 = r2 + rRL[2] * rRL[2];
    double fac = (vl[0] - vr[0]) * (mid[0] - 0.5 * (xl[0] + xr[0]));
#pragma unroll
    for(int l = 1; l < D; ++l) fac += (vl[l] - vr[l]) * (mid[l] - 0.5 * (xl[l] + xr[l]));
    fac /= r2;
#pragma unroll
    for(int l = 0; l < D; ++l) m.vel[(size_t)l * F + f] = 0.5 * (vl[l] + vr[l]) + fac * rRL[l];
}

template <int D>
__global__ void __launch_bounds__(128) k_drift(sfx_dmesh m, double dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m.n_cells) return;
    const int n = m.n_cells;
#pragma unroll
    for(int l = 0; l < D; ++l)
        m.newpos[(size_t)l * n + i] = m.pos[(size_t)l * n + i] + dt * m.vgen[(size_t)l * n + i];
}

/* ---------------------------- local time steps ----------------------------
 * TimeLine::calculate_timestep (src/TimeLine.cpp:233-317, the gas particles
 * of a run without gravity or a global step) for the cells whose step ends
 * at t_next: h = VorCell::get_h (src/VorCell.cpp:948-956), the CFL step
 * h / (|v - v_gen| + c) with the generator velocity set at the start of the
 * step, S = cfl x that; the step is max_step when max_step is shorter than
 * S, otherwise the largest power-of-two fraction of the timeline not longer
 * than S, halved until the timeline's end is a whole number of steps from
 * the cell's end (synchronisation), then clamped to [min_step, max_step].
 * The cell's next step is [end, end + step).  A zero step (the reference's
 * "Timestep 0!" exit) is SFX_ERR_TIMESTEP. */
template <int D>
__global__ void __launch_bounds__(128) k_timestep_bins(sfx_dmesh m, double gamma, double cfl,
                                                       unsigned long long max_step,
                                                       unsigned long long min_step,
                                                       unsigned long long* smin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m.n_cells) return;
    const uint64_t end = m.tend[i];
    if(end != m.t_next) return;
    const int n = m.n_cells;
    const double V = m.vol[i];
    const double h = D == 3 ? sfx_cbrt(V * 3. / 4. / kPi) : sqrt(V / kPi);
    const double rho = m.W[i], p = m.W[(size_t)(D + 1) * n + i];
    double v[D];
#pragma unroll
    for(int l = 0; l < D; ++l)
        v[l] = m.W[(size_t)(1 + l) * n + i] - (m.vgen ? m.vgen[(size_t)l * n + i] : 0.);
    double v2 = v[0] * v[0] + v[1] * v[1];
    if(D == 3) v2 = v2 + v[2] * v[2];
    const double vi = sqrt(v2);
    const double ci = rho != 0. ? sqrt(gamma * p / rho) : 0.;
    const double S = cfl * (h / (vi + ci));
    const uint64_t Smax = max_step;
    uint64_t S2;
    if(sfx_realtime_interval(m.t_total, Smax) < S) {
        S2 = Smax;
    } else {
        S2 = SFX_TIMELINE_TICKS;
        while(S2 && sfx_realtime_interval(m.t_total, S2) > S) S2 >>= 1;
        if(!S2) {
            report_cell(m.err, i, SFX_ERR_TIMESTEP);
            return;
        }
        while((SFX_TIMELINE_TICKS - end) % S2) S2 >>= 1;
        S2 = S2 > min_step ? S2 : min_step;
        S2 = S2 < Smax ? S2 : Smax;
    }
    m.tstart[i] = end;
    m.tend[i] = end + S2;
    atomicMin(smin, (unsigned long long)S2);
}

}  // namespace

int sfx_fp64_timestep_bins(const sfx_dmesh* m, double gamma, double cfl, uint64_t max_step,
                           uint64_t min_step, unsigned long long* d_smin, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int gc = (m->n_cells + 127) / 128;
    if(m->dim == 3)
        k_timestep_bins<3><<<gc, 128, 0, s>>>(*m, gamma, cfl, max_step, min_step, d_smin);
    else
        k_timestep_bins<2><<<gc, 128, 0, s>>>(*m, gamma, cfl, max_step, min_step, d_smin);
    sfx_count_launches(1);
    return cudaGetLastError() == cudaSuccess ? SFX_OK : SFX_ERR_CUDA;
}

namespace {
}  // namespace

int sfx_fp64_move_velocities(const sfx_dmesh* m, double gamma, double dt, int periodic,
                             int faces, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int gc = (m->n_cells + 127) / 128, gf = faces ? (m->n_faces + 127) / 128 : 0;
    if(m->dim == 3) {
        k_gen_velocity<3><<<gc, 128, 0, s>>>(*m, gamma, dt, periodic);
        if(gf) k_face_velocity<3><<<gf, 128, 0, s>>>(*m);
    } else {
        k_gen_velocity<2><<<gc, 128, 0, s>>>(*m, gamma, dt, periodic);
        if(gf) k_face_velocity<2><<<gf, 128, 0, s>>>(*m);
    }
    sfx_count_launches(gf ? 2 : 1);
    return cudaGetLastError() == cudaSuccess ? SFX_OK : SFX_ERR_CUDA;
}

int sfx_fp64_drift(const sfx_dmesh* m, double dt, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int gc = (m->n_cells + 127) / 128;
    if(m->dim == 3)
        k_drift<3><<<gc, 128, 0, s>>>(*m, dt);
    else
        k_drift<2><<<gc, 128, 0, s>>>(*m, dt);
    sfx_count_launches(1);
    return cudaGetLastError() == cudaSuccess ? SFX_OK : SFX_ERR_CUDA;
}

namespace {
}  // namespace

void sfx_solver_params_init(sfx_solver_params* p, int kind, double g, double tol,
                            double cutoff) {
    p->kind = kind;
    p->gamma = g;
    p->tol = tol;
    p->cutoff = cutoff;
    /* ExactRiemannSolver.cpp:48-64 */
    p->gp1d2g = 0.5 * (g + 1.) / g;
    p->gm1d2g = 0.5 * (g - 1.) / g;
    p->gm1dgp1 = (g - 1.) / (g + 1.);
    p->tdgp1 = 2. / (g + 1.);
    p->tdgm1 = 2. / (g - 1.);
    p->gm1d2 = 0.5 * (g - 1.);
    p->tgdgm1 = 2. * g / (g - 1.);
    p->ginv = 1. / g;
}

int sfx_fp64_gradients(const sfx_dmesh* m, void* stream) {
    const int nc = sfx_grad_cells(*m);
    if(nc == 0) return SFX_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int B = 128;
    if(m->gterm && m->gshare) {
        const long long cs = (long long)nc * m->S;
        if(m->dim == 3) {
            if(m->n_faces) k_grad_terms<3><<<grid_for(m->n_faces, B), B, 0, s>>>(*m);
            k_grad_sum<3><<<grid_for(cs, kGradBlock), kGradBlock, 0, s>>>(*m);
        } else {
            if(m->n_faces) k_grad_terms<2><<<grid_for(m->n_faces, B), B, 0, s>>>(*m);
            k_grad_sum<2><<<grid_for(cs, kGradBlock), kGradBlock, 0, s>>>(*m);
        }
        sfx_count_launches(m->n_faces ? 2 : 1);
        return cuda_status(cudaGetLastError());
    }
    if(m->dim == 3)
        k_gradients<3><<<grid_for(nc, B), B, 0, s>>>(*m);
    else
        k_gradients<2><<<grid_for(nc, B), B, 0, s>>>(*m);
    sfx_count_launches(1);
    return cuda_status(cudaGetLastError());
}

int sfx_fp64_faces(const sfx_dmesh* m, const sfx_solver_params* sp, double dt,
                   int write_branch, void* stream) {
    const int nf = sfx_flux_faces(*m);
    if(nf == 0) return SFX_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int B = 128;
    const int G = grid_for(nf, B);
    if(m->dim == 3) {
        if(sp->kind == SFX_SOLVER_EXACT)
            k_faces<3, SFX_SOLVER_EXACT><<<G, B, 0, s>>>(*m, *sp, dt, write_branch);
        else
            k_faces<3, SFX_SOLVER_HLLC><<<G, B, 0, s>>>(*m, *sp, dt, write_branch);
    } else {
        if(sp->kind == SFX_SOLVER_EXACT)
            k_faces<2, SFX_SOLVER_EXACT><<<G, B, 0, s>>>(*m, *sp, dt, write_branch);
        else
            k_faces<2, SFX_SOLVER_HLLC><<<G, B, 0, s>>>(*m, *sp, dt, write_branch);
    }
    sfx_count_launches(1);
    return cuda_status(cudaGetLastError());
}

int sfx_fp64_apply(const sfx_dmesh* m, const sfx_solver_params* sp, void* stream) {
    const int nc = sfx_update_cells(*m);
    if(nc == 0) return SFX_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int B = 128;
    if(m->dim == 3)
        k_apply<3><<<grid_for(nc, B), B, 0, s>>>(*m, sp->gamma);
    else
        k_apply<2><<<grid_for(nc, B), B, 0, s>>>(*m, sp->gamma);
    sfx_count_launches(1);
    return cuda_status(cudaGetLastError());
}

int sfx_fp64_init_Q(const sfx_dmesh* m, const sfx_solver_params* sp, void* stream) {
    if(m->n_cells == 0) return SFX_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int B = 128;
    if(m->dim == 3)
        k_init_Q<3><<<grid_for(m->n_cells, B), B, 0, s>>>(*m, sp->gamma, sp->kind);
    else
        k_init_Q<2><<<grid_for(m->n_cells, B), B, 0, s>>>(*m, sp->gamma, sp->kind);
    sfx_count_launches(1);
    return cuda_status(cudaGetLastError());
}

int sfx_fp64_totals(const sfx_dmesh* m, double* host_out, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    k_totals_partial<<<kTotBlocks, kTotThreads, 0, s>>>(m->Q, m->n_cells, sfx_update_cells(*m),
                                                         m->S, m->totals_scratch);
    k_totals_final<<<1, 256, 0, s>>>(m->totals_scratch, m->S);
    sfx_count_launches(2);
    cudaError_t e = cudaMemcpyAsync(host_out, m->totals_scratch + (size_t)m->S * kTotBlocks,
                                    sizeof(double) * m->S, cudaMemcpyDeviceToHost, s);
    if(e != cudaSuccess) return SFX_ERR_CUDA;
    return cuda_status(cudaStreamSynchronize(s));
}

int sfx_fp64_riemann(int dim, const sfx_solver_params* sp, int n, const double* dWL,
                     const double* dWR, const double* dn, int reflective, double* dhalf,
                     double* dflux, int32_t* dcode, void* stream) {
    if(n == 0) return SFX_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int B = 128, G = grid_for(n, B);
    if(dim == 3) {
        if(sp->kind == SFX_SOLVER_EXACT)
            k_riemann<3, SFX_SOLVER_EXACT><<<G, B, 0, s>>>(*sp, n, dWL, dWR, dn, reflective,
                                                          dhalf, dflux, dcode);
        else
            k_riemann<3, SFX_SOLVER_HLLC><<<G, B, 0, s>>>(*sp, n, dWL, dWR, dn, reflective,
                                                         dhalf, dflux, dcode);
    } else {
        if(sp->kind == SFX_SOLVER_EXACT)
            k_riemann<2, SFX_SOLVER_EXACT><<<G, B, 0, s>>>(*sp, n, dWL, dWR, dn, reflective,
                                                          dhalf, dflux, dcode);
        else
            k_riemann<2, SFX_SOLVER_HLLC><<<G, B, 0, s>>>(*sp, n, dWL, dWR, dn, reflective,
                                                         dhalf, dflux, dcode);
    }
    sfx_count_launches(1);
    return cuda_status(cudaGetLastError());
}

int sfx_fp64_pack_cells(const sfx_dmesh* m, const int32_t* idx, int count, double* out,
                        void* stream) {
    if(count <= 0) return SFX_OK;
    const long long t = (long long)count * (m->S + 1);
    k_pack_cells<<<grid_for(t, 256), 256, 0, (cudaStream_t)stream>>>(*m, idx, count, out);
    sfx_count_launches(1);
    return cuda_status(cudaGetLastError());
}

int sfx_fp64_unpack_cells(const sfx_dmesh* m, const int32_t* idx, int count, const double* in,
                          void* stream) {
    if(count <= 0) return SFX_OK;
    const long long t = (long long)count * (m->S + 1);
    k_unpack_cells<<<grid_for(t, 256), 256, 0, (cudaStream_t)stream>>>(*m, idx, count, in);
    sfx_count_launches(1);
    return cuda_status(cudaGetLastError());
}
