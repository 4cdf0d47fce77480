/*
 * FP32/FP64-split flux pass for sm_100a.
 *
 * Same algorithm as the plain-FP64 pass (VorCell::estimate_gradient,
 * VorFace::calculate_flux, update_Q/get_W; src/VorCell.cpp:464-530,
 * src/VorFace.cpp:670-1024, src/Simulation.cpp:473-483, 791-836), with the
 * precision chosen per step:
 *   FP32  gradients, slope limiters, reconstruction, MUSCL-Hancock prediction,
 *         HLLC fluxes, per-face dQ
 *   FP64  the exact solver's pressure iteration and wave sampling (pressure
 *         ratio powers lose digits near vacuum and strong shocks), the
 *         per-cell accumulation of dQ and Q -= dQ, get_W, the conservation
 *         totals.
 * Geometry is precomputed once per mesh in FP64 and rounded once to FP32 as
 * differences (c = midpoint - (x_L + x_R)/2, r = x_L - x_R, x - centroid), so
 * no FP32 subtraction of nearby absolute positions happens per step.
 *
 * Memory layout (one 32-byte cell record, 64-byte gradient record, 32-byte
 * face geometry record, 8-byte face index record) keeps every gather a pair
 * of 16-byte vector loads.  No floating-point atomics: each cell sums its own
 * faces in ascending face order in FP64, so reruns are bitwise identical and
 * the face flux leaving one cell enters the other exactly.
 */
#include <cuda_runtime.h>

#include "sfx_internal.h"

/* sfx_pow for the arguments outside sfx_pow_fast's domain, out of line so
 * that its code is not inlined into the exact solver */
__host__ __device__ __noinline__ double sfx_pow_rare(double x, double y);
#define SFX_POW_FAST_RARE sfx_pow_rare
#include "sfx_pow.h"
__host__ __device__ __noinline__ double sfx_pow_rare(double x, double y) {
    return sfx_pow(x, y);
}

namespace {

constexpr unsigned kRightBit = 0x80000000u;
constexpr int kPeriodicBit = 1 << 30;
constexpr int kIndexMask = (1 << 30) - 1;
/* faces per lane whose midpoint - centroid the gradient kernel keeps in
 * shared memory between its two passes */
constexpr int kGradSlots = 6;
/* exact solver: "this face needs Brent's method", queued instead of solved */
constexpr int kDefer = 0x7f;
/* how the exact solver treats a face whose p* needs a bracketing search:
 * search in this lane, or queue the face (kDefer) for a follow-up launch */
constexpr int kSolveInline = 0, kSolveDefer = 1;
/* blocks of the group's queued-face launch (two waves of 128-thread blocks
 * on 148 SMs; the launch strides over each member's queue) */
constexpr int kSlowGroupBlocks = 296;

__device__ __forceinline__ void report_face(sfx_dev_error* e, int f, int st) {
    atomicMin(&e->face_key, ((unsigned long long)(unsigned)f << 8) | (unsigned)st);
}
__device__ __forceinline__ void report_cell(sfx_dev_error* e, int i, int st) {
    atomicMin(&e->cell_key, ((unsigned long long)(unsigned)i << 8) | (unsigned)st);
}
__device__ __forceinline__ bool failed(const sfx_dev_error* e) {
    return (*(volatile const unsigned long long*)&e->face_key != ~0ull) ||
           (*(volatile const unsigned long long*)&e->cell_key != ~0ull);
}

template <int D>
struct Cell {
    static constexpr int S = D + 2;
    float W[S];
    float Qm, tarea;
};

/* GL: global memory through the read-only path; otherwise plain loads (a
 * copy in shared memory) */
template <bool GL>
__device__ __forceinline__ float4 ld4(const float4* p) {
    if constexpr(GL)
        return __ldg(p);
    else
        return *p;
}

template <int D, bool GL = true>
__device__ __forceinline__ Cell<D> load_cell(const float4* __restrict__ cw, int i) {
    const float4 a = ld4<GL>(cw + 2 * i);
    const float4 b = ld4<GL>(cw + 2 * i + 1);
    Cell<D> c;
    c.W[0] = a.x;
    c.W[1] = a.y;
    c.W[2] = a.z;
    c.W[3] = a.w;
    if(D == 3) {
        c.W[D + 1] = b.x;
        c.Qm = b.y;
        c.tarea = b.z;
    } else {
        c.Qm = b.x;
        c.tarea = b.y;
    }
    return c;
}

template <int D>
__device__ __forceinline__ void store_cell(float4* cw, int i, const float* W, float Qm,
                                           float tarea) {
    if(D == 3) {
        cw[2 * i] = make_float4(W[0], W[1], W[2], W[3]);
        cw[2 * i + 1] = make_float4(W[4], Qm, tarea, 0.f);
    } else {
        cw[2 * i] = make_float4(W[0], W[1], W[2], W[3]);
        cw[2 * i + 1] = make_float4(Qm, tarea, 0.f, 0.f);
    }
}

/* per-cell gradient record: g[l][k] at flat l*S+k, padded to float4s
 * (GradVec4<D>::value of them); dW/dt in a record of its own
 * (DwdtVec4<D>::value float4s) */
template <int D>
struct GradVec4 {
    static constexpr int value = (D * (D + 2) + 3) / 4;
};
template <int D>
struct DwdtVec4 {
    static constexpr int value = (D + 2 + 3) / 4;
};

template <int D>
__device__ __forceinline__ void sdwdt(float gamma, const float* W, const float (*g)[D + 2],
                                      float* dW);

/* a cell's gradients and dW/dt: with STORED dW/dt from its record (the
 * exact solver's kernels, bound by instruction issue), otherwise formed here
 * (the HLLC face kernel, closer to the memory bound) */
template <int D, bool STORED, bool GL = true>
__device__ __forceinline__ void load_grad(const float4* __restrict__ cg,
                                          const float4* __restrict__ cdw, int i, float gamma,
                                          const float* W, float (*g)[D + 2], float* dWdt,
                                          bool boosted = false) {
    constexpr int S = D + 2, G = GradVec4<D>::value, H = DwdtVec4<D>::value;
    float t[4 * G];
#pragma unroll
    for(int q = 0; q < G; ++q) {
        const float4 v = ld4<GL>(cg + (size_t)G * i + q);
        t[4 * q] = v.x;
        t[4 * q + 1] = v.y;
        t[4 * q + 2] = v.z;
        t[4 * q + 3] = v.w;
    }
#pragma unroll
    for(int l = 0; l < D; ++l)
#pragma unroll
        for(int k = 0; k < S; ++k) g[l][k] = t[l * S + k];
    if(STORED && !boosted) {
        float u[4 * H];
#pragma unroll
        for(int q = 0; q < H; ++q) {
            const float4 v = ld4<GL>(cdw + (size_t)H * i + q);
            u[4 * q] = v.x;
            u[4 * q + 1] = v.y;
            u[4 * q + 2] = v.z;
            u[4 * q + 3] = v.w;
        }
#pragma unroll
        for(int k = 0; k < S; ++k) dWdt[k] = u[k];
    } else {
        sdwdt<D>(gamma, W, g, dWdt);
    }
}

template <int D>
__device__ __forceinline__ void geom(const float4* __restrict__ fg, int f, float& A, float* c,
                                     float* r, float& rn) {
    const float4 g0 = __ldg(fg + 2 * (size_t)f);
    const float4 g1 = __ldg(fg + 2 * (size_t)f + 1);
    A = g0.x;
    c[0] = g0.y;
    c[1] = g0.z;
    if(D == 3) {
        c[2] = g0.w;
        r[0] = g1.x;
        r[1] = g1.y;
        r[2] = g1.z;
        rn = g1.w;
    } else {
        r[0] = g0.w;
        r[1] = g1.x;
        rn = g1.y;
    }
}

/* ------------------------------- prepare ------------------------------- */
template <int D>
__global__ void k_prep_faces(sfx_dmesh m) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if(f >= m.n_faces) return;
    const int n = m.n_cells, F = m.n_faces;
    const int L = m.left[f];
    double c[D], r[D], xl[D], xr[D];
    for(int l = 0; l < D; ++l) {
        xl[l] = m.pos[(size_t)l * n + L];
        xr[l] = m.rpos[(size_t)l * F + f];
        c[l] = m.mid[(size_t)l * F + f] - 0.5 * (xl[l] + xr[l]);
        r[l] = xl[l] - xr[l];
    }
    double rn2 = 0.;
    for(int l = 0; l < D; ++l) rn2 += r[l] * r[l];
    const double rn64 = sqrt(rn2);
    for(int l = 0; l < D; ++l) m.an[(size_t)l * F + f] = m.area[f] * (-r[l] / rn64);
    const float A = (float)m.area[f];
    const float rn = (float)rn64;
    if(D == 3) {
        m.fg[2 * f] = make_float4(A, (float)c[0], (float)c[1], (float)c[2]);
        m.fg[2 * f + 1] = make_float4((float)r[0], (float)r[1], (float)r[2], rn);
    } else {
        m.fg[2 * f] = make_float4(A, (float)c[0], (float)c[1], (float)r[0]);
        m.fg[2 * f + 1] = make_float4((float)r[1], rn, 0.f, 0.f);
    }
    const int kind = m.kind[f];
    int R = -1;
    uint8_t sh = 0;
    if(kind == SFX_FACE_REAL) {
        R = m.right[f];
    } else if(kind == SFX_FACE_PERIODIC) {
        R = m.right[f] | kPeriodicBit;
        for(int l = 0; l < D; ++l) {
            const double s = xr[l] - m.pos[(size_t)l * n + m.right[f]];
            const int code = s > 0.5 ? 1 : (s < -0.5 ? 2 : 0);
            sh |= (uint8_t)(code << (2 * l));
        }
    }
    m.fi[f] = make_int2(L, R);
    m.fsh[f] = sh;
}

template <int D>
__global__ void k_prep_cells(sfx_dmesh m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m.n_cells) return;
    const int n = m.n_cells;
    float v[3] = {0.f, 0.f, 0.f};
    for(int l = 0; l < D; ++l)
        v[l] = (float)(m.pos[(size_t)l * n + i] - m.cen[(size_t)l * n + i]);
    m.cx[i] = make_float4(v[0], v[1], v[2], (float)m.vol[i]);
}

/* W (FP64 SoA) and Q (FP64 SoA) -> FP32 cell records */
template <int D>
__global__ void k_load_state(sfx_dmesh m) {
    constexpr int S = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m.n_cells) return;
    const int n = m.n_cells;
    float W[S];
    for(int k = 0; k < S; ++k) W[k] = (float)m.W[(size_t)k * n + i];
    store_cell<D>(m.cw, i, W, (float)m.Q[i], (float)m.tarea[i]);
}

template <int D>
__global__ void k_export_W(sfx_dmesh m) {
    constexpr int S = D + 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m.n_cells) return;
    const int n = m.n_cells;
    const Cell<D> c = load_cell<D>(m.cw, i);
    for(int k = 0; k < S; ++k) m.W[(size_t)k * n + i] = c.W[k];
}

/* a part's ring exchange (split pass): per listed cell its FP32 state W (S
 * values) and its FP64 mass Q[0], as S + 1 doubles, the record layout of the
 * plain-FP64 pass; W goes through double and back exactly */
template <int D>
__global__ void k_pack_cells_split(sfx_dmesh m, const int32_t* idx, int count, double* out) {
    constexpr int S = D + 2, R = S + 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= (long long)count * R) return;
    const int j = (int)(t / R), q = (int)(t % R);
    const int c = idx[j];
    if(c < 0 || c >= m.n_cells) return;
    if(q < S) {
        const Cell<D> cell = load_cell<D>(m.cw, c);
        out[t] = cell.W[q];
    } else {
        out[t] = m.Q[c];
    }
}

/* one thread per listed cell: the received W and mass into the cell's FP32
 * record (total area kept) and its FP64 mass */
template <int D>
__global__ void k_unpack_cells_split(sfx_dmesh m, const int32_t* idx, int count,
                                     const double* in) {
    constexpr int S = D + 2, R = S + 1;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if(j >= count) return;
    const int c = idx[j];
    if(c < 0 || c >= m.n_cells) return;
    float W[S];
    for(int k = 0; k < S; ++k) W[k] = (float)in[(size_t)j * R + k];
    const double mass = in[(size_t)j * R + S];
    const Cell<D> cell = load_cell<D>(m.cw, c);
    store_cell<D>(m.cw, c, W, (float)mass, cell.tarea);
    m.Q[c] = mass;
}

template <int D>
__global__ void k_export_dQ(sfx_dmesh m) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if(f >= m.n_faces) return;
    const int F = m.n_faces;
    const float2 me = m.dqm[f];
    m.dQf[f] = me.x;
    for(int l = 0; l < D; ++l) m.dQf[(size_t)(1 + l) * F + f] = m.dqv[(size_t)l * F + f];
    m.dQf[(size_t)(D + 1) * F + f] = me.y;
}

/* face flux split as: mass m, momentum m v + P n, energy E (the momentum's
 * pressure part P n is assembled in FP64 with the FP64 area vector) */
template <int D>
struct SFlux {
    float m, mv[D], P, E;
};

/* ------------------------------ gradients ------------------------------ */
/* Lanes per cell: a group of LPC lanes of one warp shares a cell, each lane
 * takes every LPC-th of the cell's faces, and the group combines its partial
 * sums / maxima / minima with shuffles.  All loads of a group are independent,
 * so a warp keeps 32 face gathers in flight instead of one. */
template <int D>
struct Lanes {
    static constexpr int value = D == 3 ? 16 : 8;
};

template <int LPC>
__device__ __forceinline__ float seg_sum(float v) {
#pragma unroll
    for(int o = LPC / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, LPC);
    return v;
}
template <int LPC>
__device__ __forceinline__ float seg_max(float v) {
#pragma unroll
    for(int o = LPC / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o, LPC));
    return v;
}
template <int LPC>
__device__ __forceinline__ float seg_min(float v) {
#pragma unroll
    for(int o = LPC / 2; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o, LPC));
    return v;
}
template <int LPC>
__device__ __forceinline__ double seg_sum(double v) {
#pragma unroll
    for(int o = LPC / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, LPC);
    return v;
}

template <int D, int LPC>
__device__ __forceinline__ void sgrad_body(const sfx_dmesh& m, const float gamma, const int t) {
    constexpr int S = D + 2, G = GradVec4<D>::value;
    const int i = t / LPC, lane = t % LPC;
    if(t == 0) *m.slowq_n = 0; /* a new step: empty the queued-face list */
    /* whole warps stay alive for the shuffles; lanes past the end idle, and so
     * do the lanes of a cell that is not active (local time steps: it keeps
     * its gradients, src/Simulation.cpp:414-420) */
    const bool live = i < sfx_grad_cells(m) && !failed(m.err) &&
                      !(m.local && i < m.n_cells && m.tstart[i] != m.t_now);
    const int ic = live ? i : 0;
    const Cell<D> own = load_cell<D>(m.cw, ic);
    const float4 xv = __ldg(m.cx + ic);
    const float xmc[3] = {xv.x, xv.y, xv.z};
    float W[S], Wmax[S], Wmin[S], delta[D][S];
#pragma unroll
    for(int k = 0; k < S; ++k) {
        W[k] = own.W[k];
        Wmax[k] = W[k];
        Wmin[k] = W[k];
#pragma unroll
        for(int l = 0; l < D; ++l) delta[l][k] = 0.f;
    }
    const int beg = live ? __ldg(m.off + ic) : 0;
    const int end = live ? __ldg(m.off + ic + 1) : 0;
    /* the limiter pass below needs each face's midpoint - centroid again:
     * the first kGradSlots faces of each lane keep it in shared memory (NaN:
     * a face of zero area), the rest are loaded again */
    __shared__ float sd[kGradSlots * D][256];
    int k0 = 0;
    /* software pipelined: the next entry's face id and neighbour are loaded
     * before this entry's gathers, and both gathers (face geometry, the
     * neighbour's record) are issued before either is used */
    unsigned e_next = 0u;
    int nb_next = -1;
    if(beg + lane < end) {
        e_next = (unsigned)__ldg(m.idx + beg + lane);
        nb_next = __ldg(m.nbe + beg + lane);
    }
    for(int j = beg + lane; j < end; j += LPC, ++k0) {
        const unsigned e = e_next;
        const int nb = nb_next;
        if(j + LPC < end) {
            e_next = (unsigned)__ldg(m.idx + j + LPC);
            nb_next = __ldg(m.nbe + j + LPC);
        }
        const int f = (int)(e & ~kRightBit);
        const bool right = e & kRightBit;
        float A, c[D], r[D], rn;
        geom<D>(m.fg, f, A, c, r, rn);
        const Cell<D> cn = load_cell<D>(m.cw, nb < 0 ? ic : nb);
        if(A == 0.f) {
            if(k0 < kGradSlots) sd[k0 * D][threadIdx.x] = __int_as_float(0x7fc00000);
            continue;
        }
        if(right) {
#pragma unroll
            for(int l = 0; l < D; ++l) r[l] = -r[l];
        }
        if(k0 < kGradSlots) {
            /* midpoint - centroid = c + (x - centroid) - r_cell / 2 */
#pragma unroll
            for(int l = 0; l < D; ++l) sd[k0 * D + l][threadIdx.x] = c[l] + xmc[l] - 0.5f * r[l];
        }
        float Wj[S];
        if(nb < 0) {
            /* reflective mirror: flip the velocity component along the face
             * normal (VorFace::transform / invtransform, VorFace.cpp:417-542) */
            float vn = 0.f;
#pragma unroll
            for(int l = 0; l < D; ++l) vn += W[1 + l] * r[l];
            vn = 2.f * vn / (rn * rn);
#pragma unroll
            for(int k = 0; k < S; ++k) Wj[k] = W[k];
#pragma unroll
            for(int l = 0; l < D; ++l) Wj[1 + l] = W[1 + l] - vn * r[l];
        } else {
#pragma unroll
            for(int k = 0; k < S; ++k) Wj[k] = cn.W[k];
        }
        const float s = A / rn;
#pragma unroll
        for(int k = 0; k < S; ++k) {
            const float dW = Wj[k] - W[k];
            const float sW = 0.5f * (W[k] + Wj[k]);
#pragma unroll
            for(int l = 0; l < D; ++l) delta[l][k] += s * (dW * c[l] - sW * r[l]);
            Wmax[k] = fmaxf(Wmax[k], Wj[k]);
            Wmin[k] = fminf(Wmin[k], Wj[k]);
        }
    }
    const float iv = 1.f / xv.w;
#pragma unroll
    for(int k = 0; k < S; ++k) {
#pragma unroll
        for(int l = 0; l < D; ++l) delta[l][k] = seg_sum<LPC>(delta[l][k]) * iv;
        Wmax[k] = seg_max<LPC>(Wmax[k]);
        Wmin[k] = seg_min<LPC>(Wmin[k]);
    }
    float alpha[S];
#pragma unroll
    for(int k = 0; k < S; ++k) alpha[k] = 1.f;
    int k1 = 0;
    for(int j = beg + lane; j < end; j += LPC, ++k1) {
        float d[D];
        if(k1 < kGradSlots) {
            d[0] = sd[k1 * D][threadIdx.x];
            if(d[0] != d[0]) continue;
#pragma unroll
            for(int l = 1; l < D; ++l) d[l] = sd[k1 * D + l][threadIdx.x];
        } else {
            const unsigned e = (unsigned)__ldg(m.idx + j);
            const int f = (int)(e & ~kRightBit);
            const bool right = e & kRightBit;
            float A, c[D], r[D], rn;
            geom<D>(m.fg, f, A, c, r, rn);
            if(A == 0.f) continue;
#pragma unroll
            for(int l = 0; l < D; ++l) d[l] = c[l] + xmc[l] + (right ? 0.5f : -0.5f) * r[l];
        }
#pragma unroll
        for(int k = 0; k < S; ++k) {
            float dp = 0.f;
#pragma unroll
            for(int l = 0; l < D; ++l) dp += delta[l][k] * d[l];
            /* max((Wmax - W) / dp, (Wmin - W) / dp): the sign of dp picks
             * the operand (Wmax - W >= 0 >= Wmin - W) */
            float mx = 1.f;
            if(dp != 0.f) mx = (dp > 0.f ? Wmax[k] - W[k] : Wmin[k] - W[k]) * (1.f / dp);
            alpha[k] = fminf(alpha[k], mx);
        }
    }
#pragma unroll
    for(int k = 0; k < S; ++k) alpha[k] = seg_min<LPC>(alpha[k]);
    if(!live) return;
    /* lane q % LPC writes float4 q of the gradient record, lane (G + q) % LPC
     * float4 q of the dW/dt record (dW/dt at the cell state: every face of
     * the cell predicts its half step with it) */
    constexpr int H = DwdtVec4<D>::value;
    float out[4 * G], dw[4 * H];
    float lg[D][S];
#pragma unroll
    for(int l = 0; l < D; ++l)
#pragma unroll
        for(int k = 0; k < S; ++k) {
            lg[l][k] = delta[l][k] * alpha[k];
            out[l * S + k] = lg[l][k];
        }
#pragma unroll
    for(int q = D * S; q < 4 * G; ++q) out[q] = 0.f;
    sdwdt<D>(gamma, W, lg, dw);
#pragma unroll
    for(int q = S; q < 4 * H; ++q) dw[q] = 0.f;
#pragma unroll
    for(int q = 0; q < H; ++q)
        if(lane == (G + q) % LPC)
            m.cdw[(size_t)H * i + q] = make_float4(dw[4 * q], dw[4 * q + 1], dw[4 * q + 2],
                                                   dw[4 * q + 3]);
#pragma unroll
    for(int q = 0; q < G; ++q)
        if(lane == q % LPC)
            m.cg[(size_t)G * i + q] = make_float4(out[4 * q], out[4 * q + 1], out[4 * q + 2],
                                                  out[4 * q + 3]);
}

/* ----------------------------- face physics ----------------------------- */
template <int D>
__device__ __forceinline__ void sdwdt(float gamma, const float* W, const float (*g)[D + 2],
                                      float* dW) {
    const float ir = 1.f / W[0];
    if(D == 3) {
        const float div = g[0][1] + g[1][2] + g[2][3];
        dW[0] = -W[0] * div - W[1] * g[0][0] - W[2] * g[1][0] - W[3] * g[2][0];
        dW[1] = -W[1] * g[0][1] - W[2] * g[1][1] - W[3] * g[2][1] - g[0][4] * ir;
        dW[2] = -W[1] * g[0][2] - W[2] * g[1][2] - W[3] * g[2][2] - g[1][4] * ir;
        dW[3] = -W[1] * g[0][3] - W[2] * g[1][3] - W[3] * g[2][3] - g[2][4] * ir;
        dW[4] = -gamma * W[4] * div - W[1] * g[0][4] - W[2] * g[1][4] - W[3] * g[2][4];
    } else {
        dW[0] = -W[1] * g[0][0] - W[2] * g[1][0] - W[0] * (g[0][1] + g[1][2]);
        dW[1] = -W[1] * g[0][1] - W[2] * g[1][1] - g[0][3] * ir;
        /* the reference's 2D row uses d(vy)/dy twice (ExactRiemannSolver.cpp:920) */
        dW[2] = -W[1] * g[1][2] - W[2] * g[1][2] - g[1][3] * ir;
        dW[3] = -gamma * W[3] * (g[0][1] + g[1][2]) - W[1] * g[0][3] - W[2] * g[1][3];
    }
}

/* VorFace.hpp:92-137 in FP32 */
/* The two branches share one select and the sign-preserving fallback (two
 * divisions) runs only where the shifted extreme changes sign: written as
 * ternaries, both fallbacks were evaluated on every call (10% of the HLLC
 * face kernel's time).  The same arithmetic as the branchy form, NaN inputs
 * included. */
__device__ __forceinline__ float slimit(float phimid0, float phiL, float phiR, float dr) {
    const float delta1 = 0.5f * fabsf(phiL - phiR);
    const float delta2 = 0.25f * fabsf(phiL - phiR);
    const float phibar = phiL + dr * (phiR - phiL);
    const bool up = phiL < phiR;
    /* phi- (up) or phi+ (down) */
    const float ext = up ? fminf(phiL, phiR) : fmaxf(phiL, phiR);
    float lim = up ? ext - delta1 : ext + delta1;
    if(__builtin_expect(!(lim * ext > 0.f), 0)) lim = ext / (1.f + delta1 / fabsf(ext));
    const float r = up ? fmaxf(lim, fminf(phibar + delta2, phimid0))
                       : fminf(lim, fmaxf(phibar - delta2, phimid0));
    return phiL == phiR ? phiL : r;
}

template <int D>
__device__ __forceinline__ void spredict(float hdt, float* Wt, const float* Wself,
                                         const float* Wother, const float (*g)[D + 2],
                                         const float* dWdt, const float* d, bool do_limit,
                                         float r) {
    constexpr int S = D + 2;
    float dW[S];
#pragma unroll
    for(int k = 0; k < S; ++k) dW[k] = dWdt[k];
#pragma unroll
    for(int k = 0; k < S; ++k) {
        float s = 0.f;
#pragma unroll
        for(int l = 0; l < D; ++l) s += g[l][k] * d[l];
        Wt[k] += s;
    }
    if(do_limit) {
        float dn = 0.f;
#pragma unroll
        for(int l = 0; l < D; ++l) dn += d[l] * d[l];
        const float dr = sqrtf(dn) / r;
#pragma unroll
        for(int k = 0; k < S; ++k) Wt[k] = slimit(Wt[k], Wself[k], Wother[k], dr);
    }
    if(Wt[0] < 0.f || Wt[D + 1] < 0.f) {
#pragma unroll
        for(int k = 0; k < S; ++k) Wt[k] = Wself[k];
    }
    bool neg = false;
#pragma unroll
    for(int k = 0; k < S; ++k) dW[k] *= hdt;
    float t0 = Wt[0] + dW[0], tp = Wt[D + 1] + dW[D + 1];
    neg = t0 < 0.f || tp < 0.f;
    if(!neg) {
#pragma unroll
        for(int k = 0; k < S; ++k) Wt[k] += dW[k];
    }
}

/* HLLC (HLLCRiemannSolver.cpp:258-403) in precision T; the vacuum branch
 * (HLLCRiemannSolver.cpp:44-209) samples the exact vacuum solution.
 *
 * The wave speeds S_K = u_K -+ a_K q_K are formed as
 * a_K q_K = sqrt(gamma / rho_K (p_K + (gamma+1)/(2 gamma) (pstar - p_K)))
 * (the same quantity as the reference's a_K sqrt(1 + (gamma+1)/(2 gamma)
 * (pstar / p_K - 1)), without the ratio pstar / p_K): a predicted face
 * pressure far below the cell pressures (down to FP32 subnormals near the
 * 1e-30 floor) would overflow that ratio in FP32, and 0 * inf in S_star then
 * gives NaN.  The FP64 pass keeps the reference's form. */
template <typename T>
struct RT;
template <>
struct RT<float> {
    static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float pow_(float x, float y) { return powf(x, y); }
    static __device__ __forceinline__ float max_(float x, float y) { return fmaxf(x, y); }
};
template <>
struct RT<double> {
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double pow_(double x, double y) { return pow(x, y); }
    static __device__ __forceinline__ double max_(double x, double y) { return fmax(x, y); }
};

template <int D, typename T>
struct TFlux {
    T m, mv[D], P, E;
};

template <int D, typename T>
__device__ __forceinline__ void thllc(T g, const T* WL, const T* WRin, const T* n,
                                      bool reflective, TFlux<D, T>& F) {
    using R = RT<T>;
    constexpr int S = D + 2;
    const T zero = T(0), one = T(1), two = T(2), half = T(0.5);
    F.m = zero;
    F.P = zero;
    F.E = zero;
#pragma unroll
    for(int l = 0; l < D; ++l) F.mv[l] = zero;
    if(WL[0] == zero && (reflective || WRin[0] == zero)) return;
    /* the reflective right state is the left state with its normal velocity
     * reversed (only u_R enters below).  States are selected by value, element
     * by element: a select between two arrays' addresses would keep both
     * arrays in local memory */
    T WR[S];
#pragma unroll
    for(int k = 0; k < S; ++k) WR[k] = reflective ? WL[k] : WRin[k];
    T uL = zero, uR = zero;
#pragma unroll
    for(int l = 0; l < D; ++l) uL += WL[1 + l] * n[l];
    if(reflective) {
        uR = -uL;
    } else {
#pragma unroll
        for(int l = 0; l < D; ++l) uR += WR[1 + l] * n[l];
    }
    const T gm1 = g - one;
    const T aL = WL[0] != zero ? R::sqrt_(g * WL[D + 1] / WL[0]) : zero;
    const T aR = WR[0] != zero ? R::sqrt_(g * WR[D + 1] / WR[0]) : zero;
    if(WL[0] == zero || WR[0] == zero || two * (aL + aR) / gm1 <= uR - uL) {
        /* exact vacuum solution at x/t = 0 */
        T sol[S], vhalf = zero;
        const T tdgp1 = two / (g + one), gm1dgp1 = gm1 / (g + one);
        bool vac = false, fan = false;
        bool sright = false; /* the sampled state is the right one */
        if(WR[0] == zero) {
            if(aL > uL) {
                if(uL + two * aL / gm1 > zero) {
                    /* base > 0 in exact arithmetic on this branch */
                    const T base = R::max_(zero, tdgp1 + gm1dgp1 / aL * uL);
                    vhalf = tdgp1 * (aL + half * gm1 * uL) - uL;
#pragma unroll
                    for(int k = 0; k < S; ++k) sol[k] = WL[k];
                    sol[0] = WL[0] * R::pow_(base, two / gm1);
                    sol[D + 1] = WL[D + 1] * R::pow_(base, two * g / gm1);
                    fan = true;
                } else {
                    vac = true;
                }
            }
        } else if(WL[0] == zero) {
            sright = true;
            if(-uR < aR) {
                if(uR - two * aR / gm1 >= zero) {
                    vac = true;
                } else {
                    const T base = R::max_(zero, tdgp1 - gm1dgp1 / aR * uR);
                    vhalf = tdgp1 * (-aR + half * gm1 * uR) - uR;
#pragma unroll
                    for(int k = 0; k < S; ++k) sol[k] = WR[k];
                    sol[0] = WR[0] * R::pow_(base, two / gm1);
                    sol[D + 1] = WR[D + 1] * R::pow_(base, two * g / gm1);
                    fan = true;
                }
            }
        } else {
            const T SR = uR - two * aR / gm1, SL = uL + two * aL / gm1;
            if(SR > zero && SL < zero) {
                vac = true;
            } else if(SL >= zero) {
                if(aL > uL) {
                    const T base = R::max_(zero, tdgp1 + gm1dgp1 / aL * uL);
                    vhalf = tdgp1 * (aL + half * gm1 * uL) - uL;
#pragma unroll
                    for(int k = 0; k < S; ++k) sol[k] = WL[k];
                    sol[0] = WL[0] * R::pow_(base, two / gm1);
                    sol[D + 1] = WL[D + 1] * R::pow_(base, two * g / gm1);
                    fan = true;
                }
            } else {
                sright = true;
                if(-uR < aR) {
                    const T base = R::max_(zero, tdgp1 - gm1dgp1 / aR * uR);
                    vhalf = tdgp1 * (-aR + half * gm1 * uR) - uR;
#pragma unroll
                    for(int k = 0; k < S; ++k) sol[k] = WR[k];
                    sol[0] = WR[0] * R::pow_(base, two / gm1);
                    sol[D + 1] = WR[D + 1] * R::pow_(base, two * g / gm1);
                    fan = true;
                }
            }
        }
        if(vac) return;
        if(!fan) {
#pragma unroll
            for(int k = 0; k < S; ++k) sol[k] = sright ? WR[k] : WL[k];
        }
#pragma unroll
        for(int l = 0; l < D; ++l) sol[1 + l] += vhalf * n[l];
        if(sol[0] == zero) return;
        T vsol = zero, v2 = zero;
#pragma unroll
        for(int l = 0; l < D; ++l) {
            vsol += sol[1 + l] * n[l];
            v2 += sol[1 + l] * sol[1 + l];
        }
        F.m = sol[0] * vsol;
#pragma unroll
        for(int l = 0; l < D; ++l) F.mv[l] = F.m * sol[1 + l];
        F.P = sol[D + 1];
        const T e = sol[D + 1] / gm1 / sol[0] + half * v2;
        F.E = (sol[0] * e + sol[D + 1]) * vsol;
        return;
    }
    const T rhobar = half * (WL[0] + WR[0]);
    const T abar = half * (aL + aR);
    const T pstar = R::max_(zero, half * (WL[D + 1] + WR[D + 1]) - half * (uR - uL) * rhobar * abar);
    const T gp = half * (g + one) / g;
    /* a_K q_K */
    const T wL = pstar > WL[D + 1] ? R::sqrt_(g * (WL[D + 1] + gp * (pstar - WL[D + 1])) / WL[0])
                                   : aL;
    const T wR = pstar > WR[D + 1] ? R::sqrt_(g * (WR[D + 1] + gp * (pstar - WR[D + 1])) / WR[0])
                                   : aR;
    const T SL = uL - wL;
    const T SR = uR + wR;
    const T Sstar = (WR[D + 1] - WL[D + 1] + WL[0] * uL * (SL - uL) - WR[0] * uR * (SR - uR)) /
                    (WL[0] * (SL - uL) - WR[0] * (SR - uR));
    const bool left = Sstar >= zero;
    T Wk[S];
#pragma unroll
    for(int k = 0; k < S; ++k) Wk[k] = left ? WL[k] : WR[k];
    const T uk = left ? uL : uR;
    const T Sk = left ? SL : SR;
    T v2 = zero;
#pragma unroll
    for(int l = 0; l < D; ++l) v2 += Wk[1 + l] * Wk[1 + l];
    const T ek = Wk[D + 1] / gm1 / Wk[0] + half * v2;
    /* momentum flux = (mass flux) v + P n with P the star pressure
     * p_K + S_K fac (S* - u_K) when the star state is used */
    T mk = Wk[0] * uk;
    F.P = Wk[D + 1];
    F.E = (Wk[0] * ek + Wk[D + 1]) * uk;
    if(left ? (SL < zero) : (SR > zero)) {
        const T fac = Wk[0] * (Sk - uk) / (Sk - Sstar);
        const T ds = Sstar - uk;
        mk += Sk * (fac - Wk[0]);
        F.P += Sk * fac * ds;
        const T Ue = ek + ds * (Sstar + Wk[D + 1] / (Wk[0] * (Sk - uk)));
        F.E += Sk * (Ue * fac - Wk[0] * ek);
    }
    F.m = mk;
#pragma unroll
    for(int l = 0; l < D; ++l) F.mv[l] = mk * Wk[1 + l];
}

__device__ __forceinline__ bool finite4(float a, float b, float c, float d) {
    return isfinite(a) && isfinite(b) && isfinite(c) && isfinite(d);
}

/* the two face states and the normal, passed by value to the out-of-line
 * FP64 re-solve so that nothing goes through local memory on the hot path */
template <int D>
struct FaceStates {
    float L[D + 2], R[D + 2], n[D];
};

template <int D>
__device__ __noinline__ SFlux<D> shllc_fp64(float g, FaceStates<D> in, bool reflective) {
    constexpr int S = D + 2;
    double dL[S], dR[S], dn[D];
    for(int k = 0; k < S; ++k) {
        dL[k] = in.L[k];
        dR[k] = in.R[k];
    }
    for(int l = 0; l < D; ++l) dn[l] = in.n[l];
    TFlux<D, double> H;
    thllc<D, double>((double)g, dL, dR, dn, reflective, H);
    SFlux<D> F;
    F.m = (float)H.m;
    for(int l = 0; l < D; ++l) F.mv[l] = (float)H.mv[l];
    F.P = (float)H.P;
    F.E = (float)H.E;
    return F;
}

/* HLLC on the predicted FP32 states.  kSolveDefer: in FP32; false when
 * that flux is not finite, and the face is then queued for the FP64 solve
 * (k_group_sfaces_slow).  kSolveInline: in FP64 (the queued faces).  The
 * FP64 solve stays out of the FP32 kernel: a call from it, or its code
 * inline, costs that kernel a stack frame and spills on every face. */
template <int D, int MODE>
__device__ __forceinline__ bool shllc(float g, const float* WL, const float* WR, const float* n,
                                      bool reflective, SFlux<D>& F) {
    if(MODE == kSolveInline) {
        FaceStates<D> in;
#pragma unroll
        for(int k = 0; k < D + 2; ++k) {
            in.L[k] = WL[k];
            in.R[k] = WR[k];
        }
#pragma unroll
        for(int l = 0; l < D; ++l) in.n[l] = n[l];
        F = shllc_fp64<D>(g, in, reflective);
        return true;
    }
    TFlux<D, float> G;
    thllc<D, float>(g, WL, WR, n, reflective, G);
    float mvs = 0.f;
#pragma unroll
    for(int l = 0; l < D; ++l) mvs += G.mv[l];
    if(__builtin_expect(!finite4(G.m, G.P, G.E, mvs), 0)) return false;
    F.m = G.m;
#pragma unroll
    for(int l = 0; l < D; ++l) F.mv[l] = G.mv[l];
    F.P = G.P;
    F.E = G.E;
    return true;
}

/* exact solver half state in FP64 (ExactRiemannSolver.cpp:108-446, 644-673,
 * 462-546) with the device pow; returns 0 or SFX_ERR_* */
/* pow for the exact solver: the library's plain-double power (sfx_pow.h,
 * a few ulp, which the p* iteration's 1e-8 tolerance needs far less than),
 * out of line so that the face kernel carries one copy of its code (the
 * kernel stalled on instruction fetch with copies inlined at every site) */
__device__ __noinline__ double xpow(double x, double y) {
    return sfx_pow_fast(x, y);
}

template <int D>
struct XS {
    const sfx_solver_params& s;
    __device__ double fb(double p, const double* Wb, double a) const {
        if(p > Wb[D + 1]) {
            const double A = s.tdgp1 / Wb[0], B = s.gm1dgp1 * Wb[D + 1];
            return (p - Wb[D + 1]) * sqrt(A / (p + B));
        }
        return s.tdgm1 * a * (xpow(p / Wb[D + 1], s.gm1d2g) - 1.);
    }
    /* f_K, f_K' and, on the rarefaction side, z = (p/p_K)^e, e = (g-1)/(2g),
     * at one pressure: f_K' = r^(-(g+1)/(2g)) / (rho_K a_K) = z / (r rho_K a_K)
     * with r = p/p_K, so one power serves both; z = q ik with q = p^e shared
     * by the two sides and ik = p_K^-e computed once per face (ik = 0: the
     * power of the ratio instead) */
    __device__ void side(double p, const double* Wb, double a, double ik, double q,
                         double& f, double& fp, double& z) const {
        if(p > Wb[D + 1]) {
            const double A = s.tdgp1 / Wb[0], B = s.gm1dgp1 * Wb[D + 1];
            const double q = sqrt(A / (p + B));
            f = (p - Wb[D + 1]) * q;
            fp = (1. - 0.5 * (p - Wb[D + 1]) / (B + p)) * q;
            z = 0.;
        } else {
            const double r = p / Wb[D + 1];
            z = ik > 0. ? q * ik : xpow(r, s.gm1d2g);
            f = s.tdgm1 * a * (z - 1.);
            fp = r > 0. ? z / (r * (Wb[0] * a)) : 1. / (Wb[0] * a) * xpow(r, -s.gp1d2g);
        }
    }
};

/* p* for the face kernel: Newton's method in FP32 from the reference's
 * initial guess, then one FP64 Newton step from the FP32 root.  The face's
 * states are FP32 values; the FP32 root is within about 1e-6 of p*, and the
 * FP64 step (quadratic convergence) takes it to about 1e-12, inside the
 * iteration's 1e-8 tolerance.  f_K and the rarefaction powers z_K at the
 * final pressure are the FP64 values at the FP32 root carried along the
 * step to first order (error of the order of the step squared).  Two FP64
 * powers at most instead of one per FP64 iteration plus two per face.
 * Returns false, and the FP64 iteration runs from the start, outside the
 * range where FP32 is safe, when the FP32 iteration does not converge or
 * takes a Newton step to (nearly) zero pressure (where the reference's
 * iteration can stop at p = 0), when the FP64 step is not small, or when it
 * moves a side between shock and rarefaction. */
/* x^(1/5) for normal x > 0 without a division or a power: w ~ x^(-1/5) from
 * the FP32 hardware log2/exp2, two Newton steps for w^-5 = x, w <- w (6 -
 * x w^5) / 5 (quadratic convergence from ~1e-7 to below 1e-16), then
 * x w^4 = x^(1/5) */
__device__ __forceinline__ double fifth_root(double x) {
    double w = (double)exp2f(-0.2f * __log2f((float)x));
#pragma unroll
    for(int it = 0; it < 2; ++it) {
        const double w2 = w * w;
        w = w * (6. - x * (w2 * w2 * w)) * 0.2;
    }
    const double w2 = w * w;
    return x * (w2 * w2);
}

/* f_K, f_K' and z_K = (p/p_K)^((g-1)/(2g)) (rarefaction side) of one side in
 * FP64 (XS::side without the shared power); G53: gamma = 5/3, where the
 * exponent is 1/5 and z_K is a fifth root */
template <bool G53 = false>
__device__ __forceinline__ void side64(const sfx_solver_params& s, double p, double rho,
                                       double pK, double a, double& f, double& fp, double& z) {
    if(p > pK) {
        const double A = s.tdgp1 / rho, B = s.gm1dgp1 * pK;
        const double q = sqrt(A / (p + B));
        f = (p - pK) * q;
        fp = (1. - 0.5 * (p - pK) / (B + p)) * q;
        z = 0.;
    } else {
        /* p is a positive FP32 root and p_K < 1e12 (fast_root's range), so
         * r > 1e-57: no zero-pressure branch (and no power call for it) */
        const double r = p / pK;
        z = G53 ? fifth_root(r) : xpow(r, s.gm1d2g);
        f = s.tdgm1 * a * (z - 1.);
        fp = z / (r * (rho * a));
    }
}

/* p* for the face kernel: Newton's method in FP32 from the reference's
 * initial guess, then one FP64 Newton step from the FP32 root.  The face's
 * states are FP32 values; the FP32 root is within about 1e-6 of p*, and the
 * FP64 step (quadratic convergence) takes it to about 1e-12, inside the
 * iteration's 1e-8 tolerance.  f_K and the rarefaction powers z_K at the
 * final pressure are the FP64 values at the FP32 root carried along the
 * step to first order (error of the order of the step squared).  Two FP64
 * powers at most instead of one per FP64 iteration plus two per face.
 * Returns false, and the FP64 iteration runs from the start, outside the
 * range where FP32 is safe, when the FP32 iteration does not converge or
 * takes a Newton step to (nearly) zero pressure (where the reference's
 * iteration can stop at p = 0), when the FP64 step is not small, or when it
 * moves a side between shock and rarefaction. */
template <bool G53 = false>
__device__ __forceinline__ bool fast_root(const sfx_solver_params& s, double rL, double pL,
                                          double rR, double pR, double aL, double aR, double vL,
                                          double vR, double& p, double& fL, double& fR,
                                          double& zL, double& zR) {
    constexpr double lo = 1e-12, hi = 1e12;
    if(!(pL > lo && pL < hi && pR > lo && pR < hi && rL > lo && rL < hi && rR > lo &&
         rR < hi && fabs(vR - vL) < hi))
        return false;
    const float e = (float)s.gm1d2g, tdgm1 = (float)s.tdgm1;
    const float fpL = (float)pL, fpR = (float)pR, frL = (float)rL, frR = (float)rR;
    const float faL = (float)aL, faR = (float)aR, dv = (float)(vR - vL);
    const float AL = (float)s.tdgp1 / frL, BL = (float)s.gm1dgp1 * fpL;
    const float AR = (float)s.tdgp1 / frR, BR = (float)s.gm1dgp1 * fpR;
    auto side = [&](float q, float pK, float A, float B, float a, float rho, float& f,
                    float& fp) {
        if(q > pK) {
            const float w = sqrtf(A / (q + B));
            f = (q - pK) * w;
            fp = (1.f - 0.5f * (q - pK) / (B + q)) * w;
        } else {
            const float r = q / pK;
            const float z = exp2f(e * __log2f(r));
            f = tdgm1 * a * (z - 1.f);
            fp = z / (r * rho * a);
        }
    };
    /* the reference's guess (two-rarefaction, two-shock or PVRS) */
    const float pmin = fminf(fpL, fpR), pmax = fmaxf(fpL, fpR);
    const float floorp = (float)s.tol * 0.5f * (fpL + fpR);
    const float ppv = fmaxf(floorp, 0.5f * (fpL + fpR) - 0.125f * dv * (frL + frR) * (faL + faR));
    float pg;
    if(pmax / pmin <= 2.f && pmin <= ppv && ppv <= pmax) {
        pg = ppv;
    } else if(ppv < pmin) {
        const float num = faL + faR - (float)s.gm1d2 * dv;
        const float den = faL * exp2f(-e * __log2f(fpL)) + faR * exp2f(-e * __log2f(fpR));
        pg = exp2f(__log2f(num / den) / e);
    } else {
        const float gL = sqrtf(AL / (ppv + BL)), gR = sqrtf(AR / (ppv + BR));
        pg = (gL * fpL + gR * fpR - dv) / (gL + gR);
    }
    pg = fmaxf(floorp, pg);
    if(!(pg > 0.f && pg < 3e38f)) return false;
    for(int it = 0;; ++it) {
        float f1, g1, f2, g2;
        side(pg, fpL, AL, BL, faL, frL, f1, g1);
        side(pg, fpR, AR, BR, faR, frR, f2, g2);
        const float pn = pg - (f1 + f2 + dv) / (g1 + g2);
        if(!(pn > 1e-3f * pg && pn < 3e38f) || it >= 16) return false;
        const bool conv = fabsf(pn - pg) <= 1e-6f * pg;
        pg = pn;
        if(conv) break;
    }
    const double p0 = (double)pg;
    double fpl, fpr;
    side64<G53>(s, p0, rL, pL, aL, fL, fpl, zL);
    side64<G53>(s, p0, rR, pR, aR, fR, fpr, zR);
    const double dp = -(fL + fR + (vR - vL)) / (fpl + fpr);
    const double p1 = p0 + dp;
    if(!(fabs(dp) <= 1e-5 * p0) || (p0 > pL) != (p1 > pL) || (p0 > pR) != (p1 > pR))
        return false;
    fL += fpl * dp;
    fR += fpr * dp;
    zL *= 1. + s.gm1d2g * dp / p0;
    zR *= 1. + s.gm1d2g * dp / p0;
    p = p1;
    return true;
}

template <int D, int MODE>
__device__ int sexact(const sfx_solver_params& s, double* WL, double* WR, const double* n,
                      bool reflective, double* sol) {
    constexpr int S = D + 2;
    double vL = 0., vR = 0.;
#pragma unroll
    for(int l = 0; l < D; ++l) {
        vL += WL[1 + l] * n[l];
        vR += WR[1 + l] * n[l];
    }
    if(reflective) {
#pragma unroll
        for(int k = 0; k < S; ++k) WR[k] = WL[k];
        vR = -vL;
    }
    const double g = s.gamma;
    const double aL = WL[0] != 0. ? sqrt(g * WL[D + 1] / WL[0]) : 0.;
    const double aR = WR[0] != 0. ? sqrt(g * WR[D + 1] / WR[0]) : 0.;
    double vhalf = 0.;
    if(WL[0] == 0. || WR[0] == 0. || s.tdgm1 * (aL + aR) <= vR - vL) {
        /* vacuum cases (ExactRiemannSolver.cpp:304-446) */
#pragma unroll
        for(int k = 0; k < S; ++k) sol[k] = 0.;
        if(WL[0] == 0. && WR[0] == 0.) return SFX_OK;
        const double SR = vR - s.tdgm1 * aR, SL = vL + s.tdgm1 * aL;
        int side; /* 0 vacuum, 1 left state, 2 left fan, 3 right state, 4 right fan */
        if(WR[0] == 0.)
            side = vL < aL ? (SL > 0. ? 2 : 0) : 1;
        else if(WL[0] == 0.)
            side = -aR < vR ? (SR >= 0. ? 0 : 4) : 3;
        else if(SR > 0. && SL < 0.)
            side = 0;
        else if(SL >= 0.)
            side = aL > vL ? 2 : 1;
        else
            side = -aR < vR ? 4 : 3;
        if(side == 0) return SFX_OK;
#pragma unroll
        for(int k = 0; k < S; ++k) sol[k] = side <= 2 ? WL[k] : WR[k];
        if(side == 2) {
            const double base = s.tdgp1 + s.gm1dgp1 / aL * vL;
            sol[0] = WL[0] * xpow(base, s.tdgm1);
            vhalf = s.tdgp1 * (aL + s.gm1d2 * vL) - vL;
            sol[D + 1] = WL[D + 1] * xpow(base, s.tgdgm1);
        } else if(side == 4) {
            const double base = s.tdgp1 - s.gm1dgp1 / aR * vR;
            sol[0] = WR[0] * xpow(base, s.tdgm1);
            vhalf = s.tdgp1 * (-aR + s.gm1d2 * vR) - vR;
            sol[D + 1] = WR[D + 1] * xpow(base, s.tgdgm1);
        }
    } else {
        XS<D> x{s};
        const double pL = WL[D + 1], pR = WR[D + 1];
        double p = 0., fL = 0., zL = 0., fR = 0., zR = 0.;
        if(MODE != kSolveDefer ||
           !fast_root(s, WL[0], pL, WR[0], pR, aL, aR, vL, vR, p, fL, fR, zL, zR)) {
        /* p_K^-e (e = (g-1)/(2g)): (p/p_K)^e = p^e p_K^-e, one pow per
         * evaluation for both sides (0: not finite, pow of the ratio) */
        double iL = xpow(pL, -s.gm1d2g), iR = xpow(pR, -s.gm1d2g);
        if(!(iL > 0. && iL < 1e300)) iL = 0.;
        if(!(iR > 0. && iR < 1e300)) iR = 0.;
        const double pmin = fmin(pL, pR), pmax = fmax(pL, pR);
        double ppv = 0.5 * (pL + pR) - 0.125 * (vR - vL) * (WL[0] + WR[0]) * (aL + aR);
        const double floorp = s.tol * 0.5 * (pL + pR);
        ppv = fmax(floorp, ppv);
        double pg;
        if(pmax / pmin <= 2. && pmin <= ppv && ppv <= pmax) {
            pg = ppv;
        } else if(ppv < pmin) {
            pg = xpow((aL + aR - s.gm1d2 * (vR - vL)) /
                         (iL > 0. && iR > 0. ? aL * iL + aR * iR
                                             : aL / xpow(pL, s.gm1d2g) + aR / xpow(pR, s.gm1d2g)),
                     s.tgdgm1);
        } else {
            const double gL = sqrt(s.tdgp1 / WL[0] / (ppv + s.gm1dgp1 * pL));
            const double gR = sqrt(s.tdgp1 / WR[0] / (ppv + s.gm1dgp1 * pR));
            pg = (gL * pL + gR * pR - vR + vL) / (gL + gR);
        }
        pg = fmax(floorp, pg);
        auto f = [&](double p) { return x.fb(p, WL, aL) + x.fb(p, WR, aR) + (vR - vL); };
        /* f and f' at one pressure, the per-side values kept for the wave
         * velocity and the sampling below */
        double fpL = 0., fpR = 0.;
        auto eval = [&](double p, double& fv, double& fpv) {
            const bool need = (!(p > pL) && iL > 0.) || (!(p > pR) && iR > 0.);
            const double q = need ? xpow(p, s.gm1d2g) : 0.;
            x.side(p, WL, aL, iL, q, fL, fpL, zL);
            x.side(p, WR, aR, iR, q, fR, fpR, zR);
            fv = fL + fR + (vR - vL);
            fpv = fpL + fpR;
        };
        /* f(0): the rarefaction branch at p = 0 is -2 a_K / (g - 1) */
        const double f0 = pL > 0. && pR > 0. ? -s.tdgm1 * aL + -s.tdgm1 * aR + (vR - vL) : f(0.);
        double fg, fpg;
        eval(pg, fg, fpg);
        bool at_p = true; /* fL, fR, zL, zR hold the values at the final p */
        int it = 0;
        /* Newton stops when its next step is below the tolerance: the
         * current iterate, whose f values are at hand, is then within the
         * tolerance of the root (the reference takes that step and
         * evaluates f once more) */
        bool conv = false;
        if(f0 < s.cutoff) {
            for(;;) {
                const double pn = fmax(0., pg - fg / fpg);
                if(!(fabs(pn - pg) > s.tol * 0.5 * (pn + pg))) break;
                if(++it > SFX_MAX_ITER) return SFX_ERR_NOCONV;
                pg = pn;
                eval(pg, fg, fpg);
            }
            p = pg;
        } else {
            if(f0 * fg >= 0.) {
                while(fg < 0.) {
                    const double pn = pg - fg / fpg;
                    if(!(fabs(pn - pg) > s.tol * 0.5 * (pn + pg))) {
                        conv = true;
                        break;
                    }
                    if(++it > SFX_MAX_ITER) return SFX_ERR_NOCONV;
                    pg = pn;
                    eval(pg, fg, fpg);
                }
            }
            if(!conv && fg > 0.) {
                if(MODE == kSolveDefer) return kDefer;
                /* f(0) < 0 < f(pg).  The reference runs Brent's method on
                 * [0, pg] (ExactRiemannSolver.cpp:462-546), tens of
                 * iterations in one lane.  f is increasing and concave, so a
                 * Newton step from the right of the root lands on its left,
                 * and Newton iterates started on the left rise monotonically
                 * to it: a few iterations to the same root and tolerance
                 * (bisection keeps the iterate inside (0, pg)). */
                if(!(f0 < 0.)) {
                    /* no bracket (Brent's fa * fb >= 0 exit) */
                    p = f0 < fg ? 0. : pg;
                    at_p = false;
                } else {
                double lo = 0., hi = pg, x = pg - fg / fpg, fx, fpx;
                if(!(x > lo && x < hi)) x = 0.5 * (lo + hi);
                eval(x, fx, fpx);
                while(fx > 0.) {
                    if(++it > SFX_MAX_ITER) return SFX_ERR_NOCONV;
                    hi = x;
                    x = x - fx / fpx;
                    if(!(x > lo && x < hi)) x = 0.5 * (lo + hi);
                    eval(x, fx, fpx);
                }
                for(;;) {
                    const double xn = fx < 0. ? x - fx / fpx : x;
                    if(!(fabs(xn - x) > s.tol * 0.5 * (xn + x))) break;
                    if(++it > SFX_MAX_ITER) return SFX_ERR_NOCONV;
                    x = xn;
                    eval(x, fx, fpx);
                }
                p = x;
                }
            } else {
                p = pg;
            }
        }
        if(!at_p) {
            double t0, t1;
            eval(p, t0, t1);
        }
        }
        const double u = 0.5 * (vL + vR) + 0.5 * (fR - fL);
        if(u < 0.) {
#pragma unroll
            for(int k = 0; k < S; ++k) sol[k] = WR[k];
            const double r = p / pR;
            if(p > pR) {
                if(vR + aR * sqrt(s.gp1d2g * r + s.gm1d2g) > 0.) {
                    sol[0] = WR[0] * (r + s.gm1dgp1) / (s.gm1dgp1 * r + 1.);
                    sol[D + 1] = p;
                    vhalf = u - vR;
                }
            } else if(vR + aR > 0.) {
                if(u + aR * zR <= 0.) {
                    const double base = s.tdgp1 - s.gm1dgp1 / aR * vR;
                    sol[0] = WR[0] * xpow(base, s.tdgm1);
                    vhalf = s.tdgp1 * (-aR + s.gm1d2 * vR) - vR;
                    sol[D + 1] = pR * xpow(base, s.tgdgm1);
                } else {
                    /* r^(1/g) = z^(2/(g-1)) with z = r^((g-1)/(2g)) */
                    sol[0] = WR[0] * xpow(r, s.ginv);
                    sol[D + 1] = p;
                    vhalf = u - vR;
                }
            }
        } else {
#pragma unroll
            for(int k = 0; k < S; ++k) sol[k] = WL[k];
            const double r = p / pL;
            if(p > pL) {
                if(vL - aL * sqrt(s.gp1d2g * r + s.gm1d2g) < 0.) {
                    sol[0] = WL[0] * (r + s.gm1dgp1) / (s.gm1dgp1 * r + 1.);
                    sol[D + 1] = p;
                    vhalf = u - vL;
                }
            } else if(vL - aL < 0.) {
                if(u - aL * zL > 0.) {
                    const double base = s.tdgp1 + s.gm1dgp1 / aL * vL;
                    sol[0] = WL[0] * xpow(base, s.tdgm1);
                    vhalf = s.tdgp1 * (aL + s.gm1d2 * vL) - vL;
                    sol[D + 1] = pL * xpow(base, s.tgdgm1);
                } else {
                    sol[0] = WL[0] * xpow(r, s.ginv);
                    sol[D + 1] = p;
                    vhalf = u - vL;
                }
            }
        }
    }
#pragma unroll
    for(int l = 0; l < D; ++l) sol[1 + l] += vhalf * n[l];
    bool bad = !(sol[0] >= 0.) || !(sol[D + 1] >= 0.);
#pragma unroll
    for(int l = 0; l < D; ++l) bad |= sol[1 + l] != sol[1 + l];
    return bad ? SFX_ERR_RIEMANN : SFX_OK;
}

/* Phase one of every face kernel: a face's two predicted states (MUSCL-
 * Hancock half step with the pairwise limiter, VorFace.cpp:670-838), its unit
 * normal and what its dQ needs.  The over-flux limits lim_K = A / total_area_K
 * * Q.m_K (VorFace.cpp:837-866) are formed here once. */
/* ------------------- left-cell tiles staged by bulk copies -------------------
 * A 256-face block of the face list references a short range of left cells:
 * the builder emits each cell's faces together, in ascending cell order, and
 * cells are in spatial (Morton) order, so a block's left cells are about 33
 * consecutive cells in 3D and 85 in 2D on the random-field meshes.  The
 * staged face kernels (variant 4) copy the records of the block's left-cell
 * range -- state, position - centroid, gradients, and dW/dt where the kernel
 * reads it -- into shared memory with one 1D bulk copy per array
 * (cp.async.bulk, completion counted on an mbarrier, no multicast), and
 * face_work reads a left cell from there.  Any face order is valid: the range
 * is the block's lowest to highest left cell, capped at kTileCells cells, and
 * a left cell outside it is read from global memory.  Every array is 256-byte
 * aligned and a record is a whole number of 16-byte units, so each copy
 * starts and ends on a 16-byte boundary. */
constexpr int kTileCells = 128;

template <int D>
struct LeftTile {
    int c0 = 0, n = 0;          /* staged cells [c0, c0 + n); n = 0: none */
    const float4* cw = nullptr; /* [2 n] */
    const float4* cx = nullptr; /* [n] */
    const float4* cg = nullptr; /* [GradVec4 n] */
    const float4* cdw = nullptr; /* [DwdtVec4 n] (when staged) */
    __device__ bool has(int i) const { return (unsigned)(i - c0) < (unsigned)n; }
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

/* one 1D bulk copy global -> shared, completion on mbar (16-byte aligned
 * addresses, size a multiple of 16) */
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* mbar) {
    asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(smem_addr(dst)),
            "l"(src), "r"(bytes), "r"(smem_addr(mbar))
            : "memory");
}

/* wait for phase 0 of mbar with an iteration limit; false: gave up */
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, int limit) {
    const uint32_t a = smem_addr(mbar);
    for(int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
                "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; "
                "selp.u32 %0, 1, 0, p; }"
                : "=r"(done)
                : "r"(a)
                : "memory");
        if(done) return true;
    }
    return false;
}

constexpr int kTileWaitLimit = 1 << 16;

template <int D>
struct FaceWork {
    float WL[D + 2], WR[D + 2], n[D];
    float A, limL, limR;
    float dt; /* the face's time step (the step's dt; the shorter cell step with local steps) */
    float v[D]; /* face velocity (moving mesh; 0 on a static one) */
    bool mirror;
};

/* false: nothing to solve (a face past the end, or of zero area, whose dQ is
 * written as zero here) */
template <int D, bool STORED, bool MOVING = false, bool TILE = false>
__device__ __forceinline__ bool face_work(const sfx_dmesh& m, const float gamma, const float dt,
                                          const int f, FaceWork<D>& w,
                                          const LeftTile<D>& tile = LeftTile<D>{}) {
    constexpr int S = D + 2;
    float c[D], r[D], rn;
    geom<D>(m.fg, f, w.A, c, r, rn);
    const int2 fi = __ldg(m.fi + f);
    const int iL = fi.x;
    w.mirror = fi.y < 0;
    const int iR = w.mirror ? 0 : (fi.y & kIndexMask);
    /* local time steps (VorFace.cpp:672-697): a face is computed when either
     * of its cells is active, with the shorter of the two cells' steps;
     * timefac = that step / the longer one scales the over-flux limits */
    w.dt = dt;
    float timefac = 1.f;
    bool active = true;
    if(m.local) {
        const bool aL = m.tstart[iL] == m.t_now;
        const bool aR = !w.mirror && m.tstart[iR] == m.t_now;
        active = aL || aR;
        if(active) {
            double dtf = sfx_realtime(m.t_total, m.tend[iL] - m.tstart[iL]), dtmax = dtf;
            if(!w.mirror) {
                const double dtR = sfx_realtime(m.t_total, m.tend[iR] - m.tstart[iR]);
                dtf = fmin(dtf, dtR);
                dtmax = fmax(dtmax, dtR);
                timefac = (float)(dtf / dtmax);
            }
            w.dt = (float)dtf;
        }
    }
    if(w.A == 0.f || !active) {
        m.dqm[f] = make_float2(0.f, 0.f);
#pragma unroll
        for(int l = 0; l < D; ++l) m.dqv[(size_t)l * m.n_faces + f] = 0.;
        return false;
    }
    const float hdt = 0.5f * w.dt;
    const float irn = 1.f / rn;
#pragma unroll
    for(int l = 0; l < D; ++l) w.n[l] = -r[l] * irn;
    /* the left cell from the block's staged tile when it holds it */
    const bool tL = TILE && tile.has(iL);
    const int jL = tL ? iL - tile.c0 : iL;
    const Cell<D> cL = tL ? load_cell<D, false>(tile.cw, jL) : load_cell<D>(m.cw, iL);
    const float4 xL = tL ? tile.cx[jL] : __ldg(m.cx + iL);
    const float xmcL[3] = {xL.x, xL.y, xL.z};
    float WLr[S], WRr[S];
#pragma unroll
    for(int k = 0; k < S; ++k) {
        w.WL[k] = cL.W[k];
        w.WR[k] = 0.f;
        WRr[k] = 0.f;
    }
    /* a moving mesh: both states in the face's frame (WL -= v, WR -= v,
     * VorFace.cpp:703-710); dW/dt then at the boosted states, per face */
    constexpr bool moving = MOVING;
#pragma unroll
    for(int l = 0; l < D; ++l) {
        w.v[l] = MOVING ? (float)__ldg(m.vel + (size_t)l * m.n_faces + f) : 0.f;
        if(MOVING) w.WL[1 + l] -= w.v[l];
    }
    w.limL = w.A / cL.tarea * timefac * cL.Qm;
    w.limR = 0.f;
    float rr = 1.f;
    if(!w.mirror) {
        const Cell<D> cR = load_cell<D>(m.cw, iR);
        const float4 xR = __ldg(m.cx + iR);
        const float xmcR[3] = {xR.x, xR.y, xR.z};
#pragma unroll
        for(int k = 0; k < S; ++k) w.WR[k] = cR.W[k];
        if(MOVING) {
#pragma unroll
            for(int l = 0; l < D; ++l) w.WR[1 + l] -= w.v[l];
        }
        w.limR = w.A / cR.tarea * timefac * cR.Qm;
        /* centroid difference (unshifted centroids, as the reference) */
        float sh[D];
#pragma unroll
        for(int l = 0; l < D; ++l) sh[l] = 0.f;
        if(fi.y & kPeriodicBit) {
            const unsigned code = __ldg(m.fsh + f);
#pragma unroll
            for(int l = 0; l < D; ++l) {
                const unsigned cc = (code >> (2 * l)) & 3u;
                sh[l] = cc == 1u ? 1.f : (cc == 2u ? -1.f : 0.f);
            }
        }
        float cd2 = 0.f, dR[D];
#pragma unroll
        for(int l = 0; l < D; ++l) {
            const float cd = r[l] + sh[l] - xmcL[l] + xmcR[l];
            cd2 += cd * cd;
            dR[l] = c[l] + xmcR[l] + 0.5f * r[l];
        }
        rr = sqrtf(cd2);
        float gR[D][S], dWR[S];
        load_grad<D, STORED>(m.cg, m.cdw, iR, gamma, w.WR, gR, dWR, moving);
#pragma unroll
        for(int k = 0; k < S; ++k) WRr[k] = w.WR[k];
        spredict<D>(hdt, WRr, w.WR, w.WL, gR, dWR, dR, true, rr);
    }
    {
        float dL[D], gL[D][S], dWL[S];
#pragma unroll
        for(int l = 0; l < D; ++l) dL[l] = c[l] + xmcL[l] - 0.5f * r[l];
        if(tL)
            load_grad<D, STORED, false>(tile.cg, tile.cdw, jL, gamma, w.WL, gL, dWL, moving);
        else
            load_grad<D, STORED>(m.cg, m.cdw, iL, gamma, w.WL, gL, dWL, moving);
#pragma unroll
        for(int k = 0; k < S; ++k) WLr[k] = w.WL[k];
        spredict<D>(hdt, WLr, w.WL, w.WR, gL, dWL, dL, !w.mirror, rr);
    }
    if(w.WL[0] != 0.f) {
#pragma unroll
        for(int k = 0; k < S; ++k) w.WL[k] = WLr[k];
    }
    if(w.WR[0] != 0.f) {
#pragma unroll
        for(int k = 0; k < S; ++k) w.WR[k] = WRr[k];
    }
    return true;
}

/* the exact solver's flux contracted with n (ExactRiemannSolver::get_flux,
 * :815-880) from its half state */
template <int D>
__device__ __forceinline__ void exact_flux(double gamma, const double* h, const double* dn,
                                           const float* v, bool moving, SFlux<D>& F) {
    /* h is the half state in the face's frame; the lab-frame velocity is
     * h + v: mass flux rho (h.n), momentum (rho h.n)(h + v) + p n, energy
     * (h.n) e_lab + p (h + v).n (ExactRiemannSolver::get_flux with the face
     * velocity) */
    F.m = 0.f;
    F.P = 0.f;
    F.E = 0.f;
#pragma unroll
    for(int l = 0; l < D; ++l) F.mv[l] = 0.f;
    if(h[0] != 0.) {
        double un = 0., v2 = 0., vn = 0.;
        double hl[D];
#pragma unroll
        for(int l = 0; l < D; ++l) {
            hl[l] = h[1 + l] + (double)v[l];
            un += h[1 + l] * dn[l];
            vn += (double)v[l] * dn[l];
            v2 += hl[l] * hl[l];
        }
        const double e = 0.5 * h[0] * v2 + h[D + 1] / (gamma - 1.);
        const double mf = h[0] * un;
        F.m = (float)mf;
#pragma unroll
        for(int l = 0; l < D; ++l) F.mv[l] = (float)(mf * hl[l]);
        F.P = (float)h[D + 1];
        F.E = moving ? (float)(e * un + h[D + 1] * (un + vn)) : (float)((e + h[D + 1]) * un);
    }
}

/* the reference's HLLC de-boost (HLLCRiemannSolver.cpp:392-400): the
 * momentum flux gains v F_m, then the energy flux gains v . (the updated
 * momentum flux) + v^2 F_m / 2 */
template <int D>
__device__ __forceinline__ void hllc_deboost_split(const float* v, const float* n,
                                                   SFlux<D>& F) {
    float vm = 0.f, v2 = 0.f;
#pragma unroll
    for(int l = 0; l < D; ++l) {
        F.mv[l] += v[l] * F.m;
        vm += v[l] * (F.mv[l] + F.P * n[l]);
        v2 += v[l] * v[l];
    }
    F.E += vm + 0.5f * v2 * F.m;
}

/* Last phase of every face kernel: dt A flux with the over-flux limiter, the
 * face's dQ records and its status. */
template <int D>
__device__ __forceinline__ void face_dq(const sfx_dmesh& m, const int f, const FaceWork<D>& w,
                                        SFlux<D> F, int status) {
    const float dt = w.dt;
    if(w.mirror) {
        /* the reflective Riemann problem has zero normal velocity at the wall:
         * no mass, energy or advected momentum crosses it, only the pressure
         * force (the FP32 solver would leave a round-off-sized leak) */
        F.m = 0.f;
        F.E = 0.f;
#pragma unroll
        for(int l = 0; l < D; ++l) F.mv[l] = 0.f;
    }
    const float dtA = dt * w.A;
    float dm = dtA * F.m, dE = dtA * F.E;
    /* momentum: advective part in FP32, pressure force dt P (A n) in FP64 */
    double dv[D];
    const double dtP = (double)dt * (double)F.P;
    const int FF = m.n_faces;
#pragma unroll
    for(int l = 0; l < D; ++l)
        dv[l] = (double)(dtA * F.mv[l]) + dtP * __ldg(m.an + (size_t)l * FF + f);
    /* over-flux limiter (VorFace.cpp:837-866) */
    if(dm > w.limL) {
        const float cf = fabsf(w.limL / dm);
        dm *= cf;
        dE *= cf;
#pragma unroll
        for(int l = 0; l < D; ++l) dv[l] *= (double)cf;
    }
    if(!w.mirror) {
        if(-dm > w.limR) {
            const float cf = fabsf(w.limR / dm);
            dm *= cf;
            dE *= cf;
#pragma unroll
            for(int l = 0; l < D; ++l) dv[l] *= (double)cf;
        }
    }
    m.dqm[f] = make_float2(dm, dE);
#pragma unroll
    for(int l = 0; l < D; ++l) m.dqv[(size_t)l * FF + f] = dv[l];
    if(status == SFX_OK && F.m != F.m) status = SFX_ERR_NAN_FLUX;
    if(status != SFX_OK) report_face(m.err, f, status);
}

/* shared-memory copy of a block's left-cell records (DW: with dW/dt) */
template <int D, bool DW>
struct TileStore {
    float4 cw[2 * kTileCells];
    float4 cx[kTileCells];
    float4 cg[GradVec4<D>::value * kTileCells];
    float4 cdw[DW ? DwdtVec4<D>::value * kTileCells : 1];
    uint64_t mbar;
    int lo[32], hi[32];
    int c0, n;
};

/* stage the left cells of the block's faces (face f for this thread; every
 * thread of the block calls this): the block's lowest and highest left cell
 * by warp reductions, then thread 0 starts one bulk copy per array and
 * every thread waits for them, up to kTileWaitLimit tries.  ok = false: the
 * copies did not complete in time; the tile is then empty (every cell read
 * from global memory) and the caller reports the error and waits for the
 * copies again before it exits. */
template <int D, bool DW>
__device__ __forceinline__ LeftTile<D> stage_left_cells(const sfx_dmesh& m, int f,
                                                        TileStore<D, DW>& ts, bool& ok) {
    constexpr int G = GradVec4<D>::value, H = DwdtVec4<D>::value;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int lo = 0x7fffffff, hi = -1;
    if(f < sfx_flux_faces(m)) lo = hi = __ldg(m.fi + f).x;
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if(lane == 0) {
        ts.lo[warp] = lo;
        ts.hi[warp] = hi;
    }
    __syncthreads();
    if(threadIdx.x == 0) {
        int a = 0x7fffffff, b = -1;
        for(int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a = min(a, ts.lo[w]);
            b = max(b, ts.hi[w]);
        }
        const int n = b >= a ? min(b - a + 1, kTileCells) : 0;
        ts.c0 = a;
        ts.n = n;
        if(n) {
            const uint32_t bar = smem_addr(&ts.mbar);
            const uint32_t bytes = (uint32_t)n * (32u + 16u + 16u * G + (DW ? 16u * H : 0u));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"(bytes)
                         : "memory");
            bulk_copy(ts.cw, m.cw + 2 * (size_t)a, 32u * n, &ts.mbar);
            bulk_copy(ts.cx, m.cx + a, 16u * n, &ts.mbar);
            bulk_copy(ts.cg, m.cg + (size_t)G * a, 16u * G * n, &ts.mbar);
            if(DW) bulk_copy(ts.cdw, m.cdw + (size_t)H * a, 16u * H * n, &ts.mbar);
        }
    }
    __syncthreads();
    LeftTile<D> t;
    ok = true;
    if(ts.n) {
        ok = mbar_wait(&ts.mbar, kTileWaitLimit);
        if(ok) {
            t.c0 = ts.c0;
            t.n = ts.n;
            t.cw = ts.cw;
            t.cx = ts.cx;
            t.cg = ts.cg;
            t.cdw = ts.cdw;
        }
    }
    return t;
}

/* one face; true when the face is left for the queued-face kernel (HLLC in
 * kSolveDefer mode whose FP32 flux is not finite) */
template <int D, int SOLVER, int MODE, bool STORED_DW = SOLVER != SFX_SOLVER_HLLC,
          bool MOVING = false, bool TILE = false>
__device__ __forceinline__ bool sfaces_body(const sfx_dmesh& m, const sfx_solver_params& sp,
                                            const float dt, const int f,
                                            const LeftTile<D>& tile = LeftTile<D>{}) {
    constexpr int S = D + 2;
    if(f >= sfx_flux_faces(m) || failed(m.err)) return false;
    FaceWork<D> w;
    /* by default HLLC forms dW/dt itself and the exact solver's kernels read
     * it (STORED_DW: from the per-cell record) */
    if(!face_work<D, STORED_DW, MOVING, TILE>(m, (float)sp.gamma, dt, f, w, tile)) return false;
    SFlux<D> F;
    int status = SFX_OK;
    if constexpr(SOLVER == SFX_SOLVER_HLLC) {
        if(!shllc<D, MODE>((float)sp.gamma, w.WL, w.WR, w.n, w.mirror, F)) return true;
        if(MOVING) hllc_deboost_split<D>(w.v, w.n, F);
    } else {
        double dWL[S], dWR[S], dn[D], h[S];
#pragma unroll
        for(int l = 0; l < D; ++l) dn[l] = w.n[l];
#pragma unroll
        for(int k = 0; k < S; ++k) {
            dWL[k] = w.WL[k];
            dWR[k] = w.WR[k];
        }
        static_assert(MODE == kSolveInline, "queued faces come from k_group_sfaces_exact");
        status = sexact<D, MODE>(sp, dWL, dWR, dn, w.mirror, h);
        exact_flux<D>(sp.gamma, h, dn, w.v, MOVING, F);
    }
    face_dq<D>(m, f, w, F, status);
    return false;
}

/* -------------------- exact solver: faces sorted by wave pattern --------------------
 * The exact face kernel works in three phases per block of 256 faces:
 *   1. every thread forms its face's predicted states (face_work) and
 *      classifies the face's wave pattern in FP32 from the signs of
 *      f(p_min) and f(p_max) (f increasing in p*): two rarefactions, two
 *      shocks, or a shock on the lower-pressure side and a rarefaction on the
 *      other (two classes, by which side that is).  Faces outside the range
 *      where the FP32 iteration is safe, and vacuum faces, go to the queue
 *      solved by k_group_sfaces_slow;
 *   2. a counting sort of the block's faces by class (warp ballots, one scan
 *      of the 4 x 8 per-warp counts) through shared memory;
 *   3. thread t solves the block's t-th face in class order: p* by Newton in
 *      FP32 from the reference's guess plus one FP64 Newton step (fast_root),
 *      then the sampled half state in FP64.  A warp now takes one branch of
 *      the per-side shock/rarefaction code in every iteration.  A face whose
 *      FP32 iteration is refused, or whose state turns out to be a vacuum
 *      case in FP64, goes to the queue (warp-aggregated push).
 * Which thread solves a face changes nothing in its arithmetic, so reruns are
 * bitwise identical. */
constexpr int kClassRR = 0, kClassSS = 1, kClassSR = 2, kClassRS = 3, kNClass = 4;
constexpr int kClassQueue = 4, kClassNone = 5;
constexpr int kExactBlock = 256;

template <int D>
__device__ __forceinline__ int wave_class(const sfx_solver_params& s, const FaceWork<D>& w) {
    const float rL = w.WL[0], pL = w.WL[D + 1];
    const float rR = w.mirror ? rL : w.WR[0], pR = w.mirror ? pL : w.WR[D + 1];
    constexpr float lo = 1e-12f, hi = 1e12f;
    if(!(rL > lo && rL < hi && rR > lo && rR < hi && pL > lo && pL < hi && pR > lo && pR < hi))
        return kClassQueue;
    float vL = 0.f, vR = 0.f;
#pragma unroll
    for(int l = 0; l < D; ++l) {
        vL += w.WL[1 + l] * w.n[l];
        vR += w.WR[1 + l] * w.n[l];
    }
    if(w.mirror) vR = -vL;
    const float g = (float)s.gamma, tdgm1 = (float)s.tdgm1, e = (float)s.gm1d2g;
    const float aL = sqrtf(g * pL / rL), aR = sqrtf(g * pR / rR);
    const float dv = vR - vL;
    /* vacuum generation (and states near it, FP32 being coarse): the queue */
    if(!(tdgm1 * (aL + aR) > 1.0001f * dv)) return kClassQueue;
    const bool lowL = pL <= pR;
    const float pmin = lowL ? pL : pR, pmax = lowL ? pR : pL;
    /* f(p_min): the lower side contributes 0, the other one rarefies */
    const float ahi = lowL ? aR : aL;
    const float fmin = tdgm1 * ahi * (exp2f(e * __log2f(pmin / pmax)) - 1.f) + dv;
    if(fmin >= 0.f) return kClassRR;
    /* f(p_max): the lower side is a shock, the other one contributes 0 */
    const float rlo = lowL ? rL : rR;
    const float A = (float)s.tdgp1 / rlo, B = (float)s.gm1dgp1 * pmin;
    const float fmax = (pmax - pmin) * sqrtf(A / (pmax + B)) + dv;
    if(fmax <= 0.f) return kClassSS;
    return lowL ? kClassSR : kClassRS;
}

/* phase 3: p* by fast_root and the sampled half state; kDefer when the face
 * needs the FP64 iteration or is a vacuum case, SFX_ERR_RIEMANN for an
 * unphysical half state, SFX_OK otherwise */
/* G53: gamma = 5/3, where the sampling's powers are integers in z_K or in
 * the fan's base: (p/p_K)^(1/g) = z_K^3, base^(2/(g-1)) = base^3,
 * base^(2g/(g-1)) = base^5 */
/* phase 3 reads its face from the block's class-ordered lists in shared
 * memory where each value is used, not all at once into registers: the
 * FP64 solve then fits 64 registers with fewer spills */
template <int D, bool MOVING>
struct SortedFace {
    const float (*W)[kExactBlock]; /* [2 S][block]: left states, then right ones */
    const float (*n)[kExactBlock]; /* [D][block] */
    const float (*v)[kExactBlock]; /* [D][block] (MOVING) */
    int t;
    bool mirror;
    __device__ float WL(int k) const { return W[k][t]; }
    /* a reflective right state is the left state (its normal velocity
     * reversed by the caller) */
    __device__ float WR(int k) const { return W[mirror ? k : D + 2 + k][t]; }
    __device__ float N(int l) const { return n[l][t]; }
    __device__ float V(int l) const { return MOVING ? v[l][t] : 0.f; }
};

template <int D, bool G53 = false, bool MOVING = false>
__device__ __forceinline__ int exact_fast(const sfx_solver_params& s,
                                          const SortedFace<D, MOVING>& w, SFlux<D>& F) {
    /* of a reflective face's flux only the pressure survives (face_dq) */
    constexpr bool moving = MOVING;
    double vL = 0., vR = 0.;
#pragma unroll
    for(int l = 0; l < D; ++l) {
        vL += (double)w.WL(1 + l) * (double)w.N(l);
        vR += (double)w.WR(1 + l) * (double)w.N(l);
    }
    if(w.mirror) vR = -vL;
    const double rL = w.WL(0), pL = w.WL(D + 1), rR = w.WR(0), pR = w.WR(D + 1);
    const double g = s.gamma;
    const double aL = sqrt(g * pL / rL);
    const double aR = sqrt(g * pR / rR);
    if(s.tdgm1 * (aL + aR) <= vR - vL) return kDefer;
    double p, fL, fR, zL, zR;
    if(!fast_root<G53>(s, rL, pL, rR, pR, aL, aR, vL, vR, p, fL, fR, zL, zR)) return kDefer;
    /* sampling at x/t = 0 (ExactRiemannSolver.cpp:178-265): the side, the
     * half state's density and pressure, and its velocity shift along n */
    const double u = 0.5 * (vL + vR) + 0.5 * (fR - fL);
    const bool right = u < 0.;
    double srho = right ? rR : rL, spr = right ? pR : pL, vhalf = 0.;
    if(right) {
        const double r = p / pR;
        if(p > pR) {
            if(vR + aR * sqrt(s.gp1d2g * r + s.gm1d2g) > 0.) {
                srho = rR * (r + s.gm1dgp1) / (s.gm1dgp1 * r + 1.);
                spr = p;
                vhalf = u - vR;
            }
        } else if(vR + aR > 0.) {
            if(u + aR * zR <= 0.) {
                const double base = s.tdgp1 - s.gm1dgp1 / aR * vR;
                const double b3 = base * base * base;
                srho = rR * (G53 ? b3 : xpow(base, s.tdgm1));
                vhalf = s.tdgp1 * (-aR + s.gm1d2 * vR) - vR;
                spr = pR * (G53 ? b3 * base * base : xpow(base, s.tgdgm1));
            } else {
                srho = rR * (G53 ? zR * zR * zR : xpow(r, s.ginv));
                spr = p;
                vhalf = u - vR;
            }
        }
    } else {
        const double r = p / pL;
        if(p > pL) {
            if(vL - aL * sqrt(s.gp1d2g * r + s.gm1d2g) < 0.) {
                srho = rL * (r + s.gm1dgp1) / (s.gm1dgp1 * r + 1.);
                spr = p;
                vhalf = u - vL;
            }
        } else if(vL - aL < 0.) {
            if(u - aL * zL > 0.) {
                const double base = s.tdgp1 + s.gm1dgp1 / aL * vL;
                const double b3 = base * base * base;
                srho = rL * (G53 ? b3 : xpow(base, s.tdgm1));
                vhalf = s.tdgp1 * (aL + s.gm1d2 * vL) - vL;
                spr = pL * (G53 ? b3 * base * base : xpow(base, s.tgdgm1));
            } else {
                srho = rL * (G53 ? zL * zL * zL : xpow(r, s.ginv));
                spr = p;
                vhalf = u - vL;
            }
        }
    }
    /* the half state's velocity (in the face's frame; + v in the lab frame)
     * and its flux (ExactRiemannSolver::get_flux contracted with n,
     * :815-880) */
    double hv[D], un = 0., v2 = 0., vn = 0.;
    bool bad = !(srho >= 0.) || !(spr >= 0.);
#pragma unroll
    for(int l = 0; l < D; ++l) {
        const double nl = (double)w.N(l);
        hv[l] = (double)(right ? w.WR(1 + l) : w.WL(1 + l)) + vhalf * nl;
        bad |= hv[l] != hv[l];
        un += hv[l] * nl;
        hv[l] += (double)w.V(l);
        vn += (double)w.V(l) * nl;
        v2 += hv[l] * hv[l];
    }
    F.m = 0.f;
    F.P = 0.f;
    F.E = 0.f;
#pragma unroll
    for(int l = 0; l < D; ++l) F.mv[l] = 0.f;
    if(srho != 0.) {
        const double e = 0.5 * srho * v2 + spr / (g - 1.);
        const double mf = srho * un;
        F.m = (float)mf;
#pragma unroll
        for(int l = 0; l < D; ++l) F.mv[l] = (float)(mf * hv[l]);
        F.P = (float)spr;
        F.E = moving ? (float)(e * un + spr * (un + vn)) : (float)((e + spr) * un);
    }
    return bad ? SFX_ERR_RIEMANN : SFX_OK;
}

/* queue face f of the block's mesh for the lanes with `push` set: one
 * atomic per warp (all 32 lanes call this) */
__device__ __forceinline__ void queue_faces(const sfx_dmesh& m, bool push, int f) {
    const unsigned q = __ballot_sync(0xffffffffu, push);
    if(!q) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(q) - 1;
    int base = 0;
    if(lane == leader) base = atomicAdd(m.slowq_n, __popc(q));
    base = __shfl_sync(0xffffffffu, base, leader);
    const int at = base + __popc(q & ((1u << lane) - 1u));
    /* the queue has room for every face and each face is queued at most once
     * per step (the gradient launch empties it); a full queue is reported */
    if(push) {
        if(at < m.slowq_cap)
            m.slowq[at] = f;
        else
            report_face(m.err, f, SFX_ERR_INVALID);
    }
}

/* ------------------------------- update ------------------------------- */
template <int D, int LPC>
__device__ __forceinline__ void sapply_body(const sfx_dmesh& m, const double gamma,
                                            const int t) {
    constexpr int S = D + 2;
    const int i = t / LPC, lane = t % LPC;
    const bool live = i < sfx_update_cells(m) && !failed(m.err);
    const int n = m.n_cells, F = m.n_faces;
    double dQ[S];
#pragma unroll
    for(int k = 0; k < S; ++k) dQ[k] = 0.;
    const int beg = live ? __ldg(m.off + i) : 0;
    const int end = live ? __ldg(m.off + i + 1) : 0;
    /* each lane sums every LPC-th face in FP64; the group then adds the lanes'
     * partial sums in a fixed tree, so reruns are bitwise identical */
    for(int j = beg + lane; j < end; j += LPC) {
        const unsigned e = (unsigned)__ldg(m.idx + j);
        const int f = (int)(e & ~kRightBit);
        const float2 me = __ldg(m.dqm + f);
        double v[S];
        v[0] = me.x;
#pragma unroll
        for(int l = 0; l < D; ++l) v[1 + l] = __ldg(m.dqv + (size_t)l * F + f);
        v[D + 1] = me.y;
        if(e & kRightBit) {
#pragma unroll
            for(int k = 0; k < S; ++k) dQ[k] -= v[k];
        } else {
#pragma unroll
            for(int k = 0; k < S; ++k) dQ[k] += v[k];
        }
    }
#pragma unroll
    for(int k = 0; k < S; ++k) dQ[k] = seg_sum<LPC>(dQ[k]);
    if(!live || lane != 0) return;
    double Q[S];
#pragma unroll
    for(int k = 0; k < S; ++k) Q[k] = m.Q[(size_t)k * n + i] - dQ[k];
    if(Q[0] < 0. || Q[D + 1] < 0.) {
        report_cell(m.err, i, SFX_ERR_NEG_STATE);
        return;
    }
    if(m.local && m.tend[i] != m.t_next) {
        /* local time steps: a cell in the middle of its step takes its
         * active neighbours' flux into Q; its W waits for the end of its
         * step (src/Simulation.cpp:791-836); the record's mass (the
         * over-flux limit) follows Q */
#pragma unroll
        for(int k = 0; k < S; ++k) m.Q[(size_t)k * n + i] = Q[k];
        const Cell<D> c = load_cell<D>(m.cw, i);
        store_cell<D>(m.cw, i, c.W, (float)Q[0], c.tarea);
        return;
    }
    /* get_W (ExactRiemannSolver.cpp:716-766 / HLLCRiemannSolver.cpp:495-535) */
    const double V = m.vol[i];
    double W[S];
#pragma unroll
    for(int k = 0; k < S; ++k) W[k] = 0.;
    if(Q[0] != 0.) {
        const double im = 1. / Q[0];
        double p2 = 0.;
        W[0] = Q[0] / V;
#pragma unroll
        for(int l = 0; l < D; ++l) {
            W[1 + l] = Q[1 + l] * im;
            p2 += Q[1 + l] * Q[1 + l];
        }
        W[D + 1] = (gamma - 1.) * (Q[D + 1] - 0.5 * p2 * im) / V;
        if(W[D + 1] < 1e-30) {
            W[D + 1] = 1e-30;
            Q[D + 1] = 0.5 * p2 * im + W[D + 1] * V / (gamma - 1.);
        }
        if(W[0] < 1e-30) {
#pragma unroll
            for(int k = 0; k < S; ++k) W[k] = 0.;
        }
    }
#pragma unroll
    for(int k = 0; k < S; ++k) m.Q[(size_t)k * n + i] = Q[k];
    float Wf[S];
#pragma unroll
    for(int k = 0; k < S; ++k) Wf[k] = (float)W[k];
    store_cell<D>(m.cw, i, Wf, (float)Q[0], (float)m.tarea[i]);
}

/* ------------------------- grouped (batched) launches -------------------------
 * One launch per phase covers every mesh of a group: block b works on the
 * mesh whose block range [pre[mi], pre[mi+1]) contains b.  A mesh stepped on
 * its own is a group of one, so it runs the same kernels. */
__device__ __forceinline__ int group_mesh_of_block(const int* __restrict__ pre, int nm) {
    __shared__ int s_mesh;
    if(threadIdx.x == 0) {
        const int b = blockIdx.x;
        int lo = 0, hi = nm; /* largest mi with pre[mi] <= b */
        while(hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if(__ldg(pre + mid) <= b)
                lo = mid;
            else
                hi = mid;
        }
        s_mesh = lo;
    }
    __syncthreads();
    return s_mesh;
}

/* a member whose step counter reached 0 is done: all its blocks return */
__device__ __forceinline__ bool member_done(const sfx_group_entry* tab, int mi) {
    const int32_t* sl = tab[mi].steps_left;
    return sl && *(volatile const int32_t*)sl <= 0;
}

template <int D, int MINB, bool MOVING = false, bool G53 = false, bool TILE = false>
__global__ void __launch_bounds__(kExactBlock, MINB)
        k_group_sfaces_exact(const sfx_group_entry* tab, const int* pre, int nm,
                             sfx_solver_params sp) {
    constexpr int S = D + 2;
    constexpr int NW = kExactBlock / 32;
    /* the block's faces in class order: states, normals, area, limits, face id
     * (bit 31: mirror) */
    __shared__ float sW[2 * S][kExactBlock];
    __shared__ float sn[D][kExactBlock];
    __shared__ float sv[MOVING ? D : 1][kExactBlock]; /* one unused row when static */
    __shared__ float sA[kExactBlock], sLL[kExactBlock], sLR[kExactBlock], sdt[kExactBlock];
    __shared__ int sf[kExactBlock];
    __shared__ int sbase[kNClass][NW];
    __shared__ int stotal;
    const int mi = group_mesh_of_block(pre, nm);
    if(member_done(tab, mi)) return; /* the same for every thread of the block */
    const sfx_dmesh& m = tab[mi].m;
    const float dt = tab[mi].dt;
    const int f = (blockIdx.x - __ldg(pre + mi)) * kExactBlock + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    /* phase 1 (no thread leaves before the block's barriers); TILE: the
     * block's left cells staged in shared memory first */
    LeftTile<D> tile;
    bool tile_ok = true;
    uint64_t* tile_bar = nullptr;
    if constexpr(TILE) {
        __shared__ __align__(16) TileStore<D, true> ts;
        tile = stage_left_cells<D, true>(m, f, ts, tile_ok);
        tile_bar = &ts.mbar;
        if(!tile_ok && threadIdx.x == 0) report_face(m.err, f, SFX_ERR_CUDA);
    }
    FaceWork<D> w;
    int cls = kClassNone;
    if(f < sfx_flux_faces(m) && !failed(m.err) &&
       face_work<D, true, MOVING, TILE>(m, (float)sp.gamma, dt, f, w, tile))
        cls = wave_class<D>(sp, w);
    queue_faces(m, cls == kClassQueue, f);
    if(TILE && !tile_ok) mbar_wait(tile_bar, kTileWaitLimit); /* copies still in flight */
    /* phase 2: counting sort by class */
    unsigned mine = 0; /* the ballot of this thread's class */
#pragma unroll
    for(int c = 0; c < kNClass; ++c) {
        const unsigned b = __ballot_sync(0xffffffffu, cls == c);
        if(lane == c) sbase[c][warp] = __popc(b);
        if(cls == c) mine = b;
    }
    __syncthreads();
    if(warp == 0) {
        /* exclusive scan of the counts in (class, warp) order: lane l holds
         * entry l of the 4 x 8 table */
        const int c0 = lane / NW, w0 = lane % NW;
        const int v = sbase[c0][w0];
        int x = v;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if(lane >= o) x += y;
        }
        __syncwarp();
        sbase[c0][w0] = x - v;
        if(lane == 31) stotal = x;
    }
    __syncthreads();
    if(cls < kNClass) {
        const int slot = sbase[cls][warp] + __popc(mine & ((1u << lane) - 1u));
#pragma unroll
        for(int k = 0; k < S; ++k) {
            sW[k][slot] = w.WL[k];
            sW[S + k][slot] = w.WR[k];
        }
#pragma unroll
        for(int l = 0; l < D; ++l) {
            sn[l][slot] = w.n[l];
            if(MOVING) sv[MOVING ? l : 0][slot] = w.v[l];
        }
        sA[slot] = w.A;
        sdt[slot] = w.dt;
        sLL[slot] = w.limL;
        sLR[slot] = w.limR;
        sf[slot] = f | (w.mirror ? (int)kRightBit : 0);
    }
    __syncthreads();
    /* phase 3 */
    const int t = threadIdx.x;
    bool push = false;
    int fq = 0;
    if(t < stotal) {
        const int e = sf[t];
        fq = e & 0x7fffffff;
        const SortedFace<D, MOVING> face{sW, sn, sv, t, e < 0};
        SFlux<D> F;
        const int st = exact_fast<D, G53, MOVING>(sp, face, F);
        if(st == kDefer) {
            push = true;
        } else {
            /* what face_dq reads of the face */
            FaceWork<D> v;
            v.A = sA[t];
            v.dt = sdt[t];
            v.limL = sLL[t];
            v.limR = sLR[t];
            v.mirror = e < 0;
            face_dq<D>(m, fq, v, F, st);
        }
    }
    queue_faces(m, push, fq);
}

template <int D, int LPC>
__global__ void __launch_bounds__(256, 4) k_group_sgrad(const sfx_group_entry* tab, const int* pre,
                                                     int nm, float gamma) {
    const int mi = group_mesh_of_block(pre, nm);
    if(member_done(tab, mi)) return;
    sgrad_body<D, LPC>(tab[mi].m, gamma,
                       (blockIdx.x - __ldg(pre + mi)) * blockDim.x + threadIdx.x);
}

template <int D, int SOLVER, int MINB, bool STORED_DW = SOLVER != SFX_SOLVER_HLLC,
          bool MOVING = false, bool TILE = false>
__global__ void __launch_bounds__(256, MINB)
        k_group_sfaces(const sfx_group_entry* tab, const int* pre, int nm,
                       sfx_solver_params sp) {
    static_assert(SOLVER == SFX_SOLVER_HLLC, "the exact solver has k_group_sfaces_exact");
    const int mi = group_mesh_of_block(pre, nm);
    if(member_done(tab, mi)) return; /* the same for every thread of the block */
    const sfx_dmesh& m = tab[mi].m;
    const int f = (blockIdx.x - __ldg(pre + mi)) * blockDim.x + threadIdx.x;
    if constexpr(TILE) {
        /* the block's left cells staged in shared memory first */
        __shared__ __align__(16) TileStore<D, STORED_DW> ts;
        bool ok;
        const LeftTile<D> tile = stage_left_cells<D, STORED_DW>(m, f, ts, ok);
        if(!ok && threadIdx.x == 0) report_face(m.err, f, SFX_ERR_CUDA);
        const bool push = sfaces_body<D, SOLVER, kSolveDefer, STORED_DW, MOVING, true>(
                m, sp, tab[mi].dt, f, tile);
        queue_faces(m, push, f);
        if(!ok) mbar_wait(&ts.mbar, kTileWaitLimit); /* copies still in flight */
    } else {
        const bool push =
                sfaces_body<D, SOLVER, kSolveDefer, STORED_DW, MOVING>(m, sp, tab[mi].dt, f);
        queue_faces(m, push, f);
    }
}

/* The queued faces of every member, one per thread.  Exact solver: the
 * FP64 iteration from the reference's guess (the monotone Newton search
 * where the reference runs Brent's method) and the vacuum cases.  HLLC: the
 * FP64 solve of faces whose FP32 flux was not finite.  Each block reads
 * the members' queue lengths (kSlowChunk members at a time, in parallel),
 * forms their prefix sums in shared memory and strides over the flattened
 * list, finding a slot's member by binary search: no thread walks the
 * member list. */
constexpr int kSlowBlock = 128, kSlowChunk = 2048, kSlowPer = kSlowChunk / kSlowBlock;

template <int D, bool MOVING = false, int SOLVER = SFX_SOLVER_EXACT,
          bool STORED_DW = SOLVER == SFX_SOLVER_EXACT>
__global__ void __launch_bounds__(kSlowBlock) k_group_sfaces_slow(const sfx_group_entry* tab,
                                                                 int nm, sfx_solver_params sp) {
    __shared__ int spre[kSlowChunk + 1];
    __shared__ int swarp[kSlowBlock / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for(int base = 0; base < nm; base += kSlowChunk) {
        const int cnt = min(nm - base, kSlowChunk);
        /* thread t sums the queue lengths of members [t kSlowPer, (t+1) kSlowPer) */
        int loc[kSlowPer];
        int sum = 0;
#pragma unroll
        for(int k = 0; k < kSlowPer; ++k) {
            const int mi = t * kSlowPer + k;
            int c = 0;
            if(mi < cnt && !member_done(tab, base + mi)) {
                const sfx_dmesh& m = tab[base + mi].m;
                c = min(*(volatile const int32_t*)m.slowq_n, m.slowq_cap);
            }
            loc[k] = c;
            sum += c;
        }
        /* exclusive block scan of the per-thread sums */
        int x = sum;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if(lane >= o) x += y;
        }
        if(lane == 31) swarp[warp] = x;
        __syncthreads();
        int woff = 0, total = 0;
#pragma unroll
        for(int w = 0; w < kSlowBlock / 32; ++w) {
            if(w < warp) woff += swarp[w];
            total += swarp[w];
        }
        int run = woff + x - sum;
#pragma unroll
        for(int k = 0; k < kSlowPer; ++k) {
            spre[t * kSlowPer + k] = run;
            run += loc[k];
        }
        if(t == kSlowBlock - 1) spre[kSlowChunk] = run;
        __syncthreads();
        for(int j = blockIdx.x * kSlowBlock + t; j < total; j += gridDim.x * kSlowBlock) {
            int lo = 0, hi = cnt; /* the last member whose prefix is <= j */
            while(hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if(spre[mid] <= j)
                    lo = mid;
                else
                    hi = mid;
            }
            const sfx_group_entry& e = tab[base + lo];
            sfaces_body<D, SOLVER, kSolveInline, STORED_DW, MOVING>(
                    e.m, sp, e.dt, __ldg(e.m.slowq + (j - spre[lo])));
        }
        __syncthreads(); /* spre and swarp are rewritten by the next chunk */
    }
}

template <int D, int LPC>
__global__ void __launch_bounds__(256) k_group_sapply(const sfx_group_entry* tab, const int* pre,
                                                      int nm, double gamma) {
    const int mi = group_mesh_of_block(pre, nm);
    if(member_done(tab, mi)) return;
    sapply_body<D, LPC>(tab[mi].m, gamma, (blockIdx.x - __ldg(pre + mi)) * blockDim.x + threadIdx.x);
}

/* after a step: count the members' remaining steps down */
__global__ void k_group_tick(const sfx_group_entry* tab, int nm) {
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    if(mi >= nm) return;
    int32_t* sl = tab[mi].steps_left;
    if(sl && *sl > 0) *sl -= 1;
}

__global__ void k_group_reset_err(const sfx_group_entry* tab, int nm) {
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    if(mi >= nm) return;
    tab[mi].m.err->face_key = ~0ull;
    tab[mi].m.err->cell_key = ~0ull;
}

__global__ void k_group_collect_err(const sfx_group_entry* tab, int nm, sfx_dev_error* out) {
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    if(mi >= nm) return;
    out[mi] = *tab[mi].m.err;
}

template <int D, int LPC>
int group_phase(const sfx_group_dev* g, int phase, const sfx_solver_params* sp,
                cudaStream_t s) {
    const int nm = g->n_meshes;
    if(phase == 0) {
        if(g->blocks[0])
            k_group_sgrad<D, LPC><<<g->blocks[0], 256, 0, s>>>(g->tab, g->pre, nm,
                                                                (float)sp->gamma);
    } else if(phase == 1) {
        if(g->blocks[1]) {
            const int* pre1 = g->pre + (nm + 1);
            if(g->moving) {
                /* a moving mesh stepped alone: the face kernels with the boost */
                if(sp->kind == SFX_SOLVER_EXACT) {
                    k_group_sfaces_exact<D, 4, true><<<g->blocks[1], kExactBlock, 0, s>>>(
                            g->tab, pre1, nm, *sp);
                    k_group_sfaces_slow<D, true><<<kSlowGroupBlocks, kSlowBlock, 0, s>>>(
                            g->tab, nm, *sp);
                } else {
                    k_group_sfaces<D, SFX_SOLVER_HLLC, 4, false, true>
                            <<<g->blocks[1], 256, 0, s>>>(g->tab, pre1, nm, *sp);
                    k_group_sfaces_slow<D, true, SFX_SOLVER_HLLC>
                            <<<kSlowGroupBlocks, kSlowBlock, 0, s>>>(g->tab, nm, *sp);
                }
                sfx_count_launches(1);
            } else if(sp->kind == SFX_SOLVER_EXACT) {
                const int v = sfx_split_face_variant_kernel(sp, g->face_variant);
                if(v == 4 && sp->gamma == 5. / 3.)
                    k_group_sfaces_exact<D, 4, false, true, true>
                            <<<g->blocks[1], kExactBlock, 0, s>>>(g->tab, pre1, nm, *sp);
                else if(v == 4)
                    k_group_sfaces_exact<D, 4, false, false, true>
                            <<<g->blocks[1], kExactBlock, 0, s>>>(g->tab, pre1, nm, *sp);
                else if(v == 3)
                    k_group_sfaces_exact<D, 3, false, true><<<g->blocks[1], kExactBlock, 0, s>>>(
                            g->tab, pre1, nm, *sp);
                else if(v == 2)
                    k_group_sfaces_exact<D, 4, false, true><<<g->blocks[1], kExactBlock, 0, s>>>(
                            g->tab, pre1, nm, *sp);
                else if(v == 1)
                    k_group_sfaces_exact<D, 3><<<g->blocks[1], kExactBlock, 0, s>>>(
                            g->tab, pre1, nm, *sp);
                else
                    k_group_sfaces_exact<D, 4><<<g->blocks[1], kExactBlock, 0, s>>>(
                            g->tab, pre1, nm, *sp);
                k_group_sfaces_slow<D><<<kSlowGroupBlocks, kSlowBlock, 0, s>>>(g->tab, nm, *sp);
                sfx_count_launches(1);
            } else {
                /* HLLC; then the faces whose FP32 flux was not finite, in FP64 */
                const int v = sfx_split_face_variant_kernel(sp, g->face_variant);
                if(v == 2) {
                    k_group_sfaces<D, SFX_SOLVER_HLLC, 4, true><<<g->blocks[1], 256, 0, s>>>(
                            g->tab, pre1, nm, *sp);
                    k_group_sfaces_slow<D, false, SFX_SOLVER_HLLC, true>
                            <<<kSlowGroupBlocks, kSlowBlock, 0, s>>>(g->tab, nm, *sp);
                } else {
                    if(v == 4)
                        k_group_sfaces<D, SFX_SOLVER_HLLC, 5, false, false, true>
                                <<<g->blocks[1], 256, 0, s>>>(g->tab, pre1, nm, *sp);
                    else if(v == 3)
                        k_group_sfaces<D, SFX_SOLVER_HLLC, 5><<<g->blocks[1], 256, 0, s>>>(
                                g->tab, pre1, nm, *sp);
                    else if(v == 1)
                        k_group_sfaces<D, SFX_SOLVER_HLLC, 3><<<g->blocks[1], 256, 0, s>>>(
                                g->tab, pre1, nm, *sp);
                    else
                        k_group_sfaces<D, SFX_SOLVER_HLLC, 4><<<g->blocks[1], 256, 0, s>>>(
                                g->tab, pre1, nm, *sp);
                    k_group_sfaces_slow<D, false, SFX_SOLVER_HLLC>
                            <<<kSlowGroupBlocks, kSlowBlock, 0, s>>>(g->tab, nm, *sp);
                }
                sfx_count_launches(1);
            }
        }
    } else {
        if(g->blocks[2])
            k_group_sapply<D, LPC><<<g->blocks[2], 256, 0, s>>>(g->tab, g->pre + 2 * (nm + 1),
                                                                 nm, sp->gamma);
    }
    if(g->blocks[phase]) sfx_count_launches(1);
    return cudaGetLastError() == cudaSuccess ? SFX_OK : SFX_ERR_CUDA;
}

inline int grid_for(long long n, int b) {
    return (int)((n + b - 1) / b);
}
/* status of the n kernel launches just made, counted for sfx_launch_count */
inline int launched(int n) {
    sfx_count_launches(n);
    return cudaGetLastError() == cudaSuccess ? SFX_OK : SFX_ERR_CUDA;
}

}  // namespace

int sfx_split_prepare(const sfx_dmesh* m, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if(m->n_faces) {
        if(m->dim == 3)
            k_prep_faces<3><<<grid_for(m->n_faces, 256), 256, 0, s>>>(*m);
        else
            k_prep_faces<2><<<grid_for(m->n_faces, 256), 256, 0, s>>>(*m);
    }
    if(m->dim == 3)
        k_prep_cells<3><<<grid_for(m->n_cells, 256), 256, 0, s>>>(*m);
    else
        k_prep_cells<2><<<grid_for(m->n_cells, 256), 256, 0, s>>>(*m);
    return launched(m->n_faces ? 2 : 1);
}

int sfx_split_load_state(const sfx_dmesh* m, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if(m->dim == 3)
        k_load_state<3><<<grid_for(m->n_cells, 256), 256, 0, s>>>(*m);
    else
        k_load_state<2><<<grid_for(m->n_cells, 256), 256, 0, s>>>(*m);
    return launched(1);
}

int sfx_split_export_W(const sfx_dmesh* m, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if(m->dim == 3)
        k_export_W<3><<<grid_for(m->n_cells, 256), 256, 0, s>>>(*m);
    else
        k_export_W<2><<<grid_for(m->n_cells, 256), 256, 0, s>>>(*m);
    return launched(1);
}

int sfx_split_export_dQ(const sfx_dmesh* m, void* stream) {
    if(!m->n_faces) return SFX_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if(m->dim == 3)
        k_export_dQ<3><<<grid_for(m->n_faces, 256), 256, 0, s>>>(*m);
    else
        k_export_dQ<2><<<grid_for(m->n_faces, 256), 256, 0, s>>>(*m);
    return launched(1);
}

int sfx_split_face_variant_kernel(const sfx_solver_params* sp, int variant) {
    if(variant < 0 || variant >= SFX_FACE_VARIANTS) return 0;
    if(sp->kind == SFX_SOLVER_EXACT) {
        /* the gamma = 5/3 forms (2: 64 registers, 3: 80) exist for that gamma
         * only; 4 (left cells staged) is the gamma = 5/3 form at that gamma
         * and the generic one at others */
        if(sp->gamma != 5. / 3. && (variant == 2 || variant == 3)) return variant - 2;
        return variant;
    }
    return variant; /* HLLC: 3 is the 48-register kernel, 4 that with staged left cells */
}

int sfx_split_pack_cells(const sfx_dmesh* m, const int32_t* idx, int count, double* out,
                         void* stream) {
    if(count <= 0) return SFX_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const long long t = (long long)count * (m->S + 1);
    if(m->dim == 3)
        k_pack_cells_split<3><<<grid_for(t, 256), 256, 0, s>>>(*m, idx, count, out);
    else
        k_pack_cells_split<2><<<grid_for(t, 256), 256, 0, s>>>(*m, idx, count, out);
    return launched(1);
}

int sfx_split_unpack_cells(const sfx_dmesh* m, const int32_t* idx, int count, const double* in,
                           void* stream) {
    if(count <= 0) return SFX_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if(m->dim == 3)
        k_unpack_cells_split<3><<<grid_for(count, 256), 256, 0, s>>>(*m, idx, count, in);
    else
        k_unpack_cells_split<2><<<grid_for(count, 256), 256, 0, s>>>(*m, idx, count, in);
    return launched(1);
}

int sfx_split_blocks(int dim, int lanes, int n_cells, int n_faces, int32_t* out) {
    (void)dim;
    out[0] = grid_for((long long)n_cells * lanes, 256);
    out[1] = grid_for(n_faces, 256);
    out[2] = out[0];
    return SFX_OK;
}

int sfx_split_group_phase(const sfx_group_dev* g, int phase, const sfx_solver_params* sp,
                          void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if(g->dim == 3) {
        switch(g->lanes) {
        case 1: return group_phase<3, 1>(g, phase, sp, s);
        case 2: return group_phase<3, 2>(g, phase, sp, s);
        case 4: return group_phase<3, 4>(g, phase, sp, s);
        case 8: return group_phase<3, 8>(g, phase, sp, s);
        case 16: return group_phase<3, 16>(g, phase, sp, s);
        default: return SFX_ERR_INVALID;
        }
    }
    switch(g->lanes) {
    case 1: return group_phase<2, 1>(g, phase, sp, s);
    case 2: return group_phase<2, 2>(g, phase, sp, s);
    case 4: return group_phase<2, 4>(g, phase, sp, s);
    case 8: return group_phase<2, 8>(g, phase, sp, s);
    case 16: return group_phase<2, 16>(g, phase, sp, s);
    default: return SFX_ERR_INVALID;
    }
}

int sfx_split_group_tick(const sfx_group_dev* g, void* stream) {
    k_group_tick<<<grid_for(g->n_meshes, 128), 128, 0, (cudaStream_t)stream>>>(g->tab,
                                                                            g->n_meshes);
    return launched(1);
}

int sfx_split_group_reset(const sfx_group_dev* g, void* stream) {
    k_group_reset_err<<<grid_for(g->n_meshes, 128), 128, 0, (cudaStream_t)stream>>>(g->tab,
                                                                                  g->n_meshes);
    return launched(1);
}

int sfx_split_group_collect(const sfx_group_dev* g, sfx_dev_error* d_out, void* stream) {
    k_group_collect_err<<<grid_for(g->n_meshes, 128), 128, 0, (cudaStream_t)stream>>>(
            g->tab, g->n_meshes, d_out);
    return launched(1);
}
