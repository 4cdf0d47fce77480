/*
 * Host Voronoi face-list builder for static meshes.
 *
 * Produces the face-list contract that Shadowfax's VorTess/VorFace export to
 * the flux pass (src/VorTess.cpp:153-396, src/VorFace.cpp:293-404,
 * src/VorCell.cpp:257-411): per face the area, midpoint, left (owner) cell,
 * right neighbour (real cell, periodic image of a cell, or reflective
 * mirror) and the right generator's position; per cell the centroid, volume,
 * total face area and the list of its faces.
 *
 * Shadowfax builds the mesh by incremental Delaunay insertion with exact
 * predicates (DelTess + ExArith) and keeps it on the host; this builder is an
 * independent cell-by-cell construction used to produce inputs for the flux
 * pass (tests, benchmarks, the request server's mesh pool).  Each Voronoi
 * cell is the generator's bounding box clipped by the bisector planes of its
 * neighbours, visited in rings of a uniform bucket grid until the security
 * radius criterion (no unvisited generator is closer than twice the farthest
 * cell vertex) holds.  Cells are independent, so the build is split over
 * threads and the result does not depend on the thread count.
 *
 * Conventions, as in the reference:
 *  - faces are owned by the lower-index cell of a real pair (the cell that
 *    the reference's construct() loop meets first); a face to a periodic
 *    image or a reflective mirror is owned by the real cell, so the physical
 *    face between two cells across a periodic boundary appears twice, once
 *    from each side (src/DelTess_mpi.cpp:150-186, src/VorFace.cpp:913-955);
 *  - a reflective mirror sits at the generator reflected in the wall;
 *  - faces whose polygon degenerates get area 0 (src/VorTess.cpp:253-264,
 *    349-351, 382-384) and stay in the list.
 * Face order: by owner cell, then by (kind, neighbour, image).  Each cell's
 * face list is ascending in face index.
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/sfxflux.h"

namespace {

struct FaceRec {
    int32_t nb;    /* neighbour cell, or wall id (0..2D-1) for mirrors */
    int8_t kind;   /* 0 real, 1 periodic image, 2 mirror */
    int8_t sh[3];  /* periodic image shift in box units */
    double area;
    double mid[3];
};

struct CellOut {
    std::vector<FaceRec> faces;
    double volume = 0.;
    double centroid[3] = {0., 0., 0.};
    int ok = 1;
};

/* label encoding during clipping: >= 0 -> neighbour slot in a per-cell
 * table; -1-w -> wall / box face w */
struct Nb {
    int32_t j;
    int8_t sh[3];
};

struct Grid {
    int dim;
    int g;          /* buckets per axis */
    double h;       /* bucket size */
    std::vector<int32_t> start, items;
};

inline int bucket_of(double x, int g) {
    int b = (int)(x * g);
    if(b < 0) b = 0;
    if(b >= g) b = g - 1;
    return b;
}

Grid build_grid(int dim, int64_t n, const double* pos) {
    Grid G;
    G.dim = dim;
    double per = std::pow((double)n / 2.0, 1.0 / dim);
    G.g = std::max(1, (int)per);
    G.h = 1.0 / G.g;
    int64_t nb = 1;
    for(int d = 0; d < dim; ++d) nb *= G.g;
    std::vector<int32_t> cnt(nb + 1, 0);
    std::vector<int64_t> bid(n);
    for(int64_t i = 0; i < n; ++i) {
        int64_t b = 0;
        for(int d = dim; d--;) b = b * G.g + bucket_of(pos[i * dim + d], G.g);
        bid[i] = b;
        cnt[b + 1]++;
    }
    for(int64_t b = 0; b < nb; ++b) cnt[b + 1] += cnt[b];
    G.start = cnt;
    G.items.resize(n);
    std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
    for(int64_t i = 0; i < n; ++i) G.items[fill[bid[i]]++] = (int32_t)i;
    return G;
}

/* ------------------------------- 2D cell ------------------------------- */

struct Poly2 {
    std::vector<double> x, y; /* vertices in counter-clockwise order */
    std::vector<int> lab;     /* lab[k] labels edge (k, k+1) */
};

/* clip by {p : (p - m).u <= 0}; returns false if nothing changed */
bool clip2(Poly2& P, Poly2& tmp, double mx, double my, double ux, double uy,
           int label) {
    const int n = (int)P.x.size();
    double smax = -1.;
    static thread_local std::vector<double> s;
    s.resize(n);
    for(int k = 0; k < n; ++k) {
        s[k] = (P.x[k] - mx) * ux + (P.y[k] - my) * uy;
        smax = std::max(smax, s[k]);
    }
    if(smax <= 0.) return false;
    tmp.x.clear();
    tmp.y.clear();
    tmp.lab.clear();
    for(int k = 0; k < n; ++k) {
        int k1 = (k + 1) % n;
        bool in0 = s[k] <= 0., in1 = s[k1] <= 0.;
        if(in0) {
            tmp.x.push_back(P.x[k]);
            tmp.y.push_back(P.y[k]);
            tmp.lab.push_back(in1 ? P.lab[k] : P.lab[k]);
        }
        if(in0 != in1) {
            double t = s[k] / (s[k] - s[k1]);
            tmp.x.push_back(P.x[k] + t * (P.x[k1] - P.x[k]));
            tmp.y.push_back(P.y[k] + t * (P.y[k1] - P.y[k]));
            /* leaving the half-plane: the new edge runs along the bisector;
             * entering: continue the old edge */
            tmp.lab.push_back(in0 ? label : P.lab[k]);
        }
    }
    std::swap(P, tmp);
    return true;
}

void cell2(int64_t i, const double* pos, int64_t n, int periodic,
           const Grid& G, CellOut& out) {
    const double xi = pos[2 * i], yi = pos[2 * i + 1];
    Poly2 P, tmp;
    double lo[2], hi[2];
    if(periodic) {
        lo[0] = xi - 0.5;
        hi[0] = xi + 0.5;
        lo[1] = yi - 0.5;
        hi[1] = yi + 0.5;
    } else {
        lo[0] = lo[1] = 0.;
        hi[0] = hi[1] = 1.;
    }
    /* walls: 0 x=lo, 1 x=hi, 2 y=lo, 3 y=hi */
    P.x = {lo[0], hi[0], hi[0], lo[0]};
    P.y = {lo[1], lo[1], hi[1], hi[1]};
    P.lab = {-1 - 2, -1 - 1, -1 - 3, -1 - 0};
    std::vector<Nb> nbs;
    const int g = G.g;
    const int bx = bucket_of(xi, g), by = bucket_of(yi, g);
    const int kmax = periodic ? 2 * g + 2 : g + 1;
    for(int k = 0; k <= kmax; ++k) {
        for(int oy = -k; oy <= k; ++oy) {
            for(int ox = -k; ox <= k; ++ox) {
                if(std::max(std::abs(ox), std::abs(oy)) != k) continue;
                int cx = bx + ox, cy = by + oy;
                int sx = 0, sy = 0;
                if(periodic) {
                    sx = (int)std::floor((double)cx / g);
                    sy = (int)std::floor((double)cy / g);
                    cx -= sx * g;
                    cy -= sy * g;
                } else if(cx < 0 || cy < 0 || cx >= g || cy >= g) {
                    continue;
                }
                int64_t b = (int64_t)cy * g + cx;
                for(int32_t t = G.start[b]; t < G.start[b + 1]; ++t) {
                    int32_t j = G.items[t];
                    if(j == i && sx == 0 && sy == 0) continue;
                    double xj = pos[2 * j] + sx, yj = pos[2 * j + 1] + sy;
                    double ux = xj - xi, uy = yj - yi;
                    double mx = 0.5 * (xi + xj), my = 0.5 * (yi + yj);
                    int label = (int)nbs.size();
                    if(clip2(P, tmp, mx, my, ux, uy, label)) {
                        Nb nb;
                        nb.j = j;
                        nb.sh[0] = (int8_t)sx;
                        nb.sh[1] = (int8_t)sy;
                        nb.sh[2] = 0;
                        nbs.push_back(nb);
                    }
                }
            }
        }
        double r2 = 0.;
        for(size_t v = 0; v < P.x.size(); ++v) {
            double dx = P.x[v] - xi, dy = P.y[v] - yi;
            r2 = std::max(r2, dx * dx + dy * dy);
        }
        double reach = k * G.h;
        if(4. * r2 <= reach * reach) break;
        if(k == kmax) out.ok = 0;
    }
    /* faces */
    const int nv = (int)P.x.size();
    double vol = 0., cx = 0., cy = 0.;
    for(int v = 0; v < nv; ++v) {
        int v1 = (v + 1) % nv;
        int lab = P.lab[v];
        FaceRec fr;
        std::memset(&fr, 0, sizeof fr);
        if(lab >= 0) {
            const Nb& nb = nbs[lab];
            fr.nb = nb.j;
            fr.sh[0] = nb.sh[0];
            fr.sh[1] = nb.sh[1];
            fr.kind = (nb.sh[0] || nb.sh[1]) ? 1 : 0;
        } else {
            if(periodic) out.ok = 0; /* a box face survived: too few points */
            fr.nb = -1 - lab;
            fr.kind = 2;
        }
        double dx = P.x[v] - P.x[v1], dy = P.y[v] - P.y[v1];
        double len = std::sqrt(dx * dx + dy * dy);
        fr.area = len < 1e-13 ? 0. : len;
        fr.mid[0] = 0.5 * (P.x[v] + P.x[v1]);
        fr.mid[1] = 0.5 * (P.y[v] + P.y[v1]);
        out.faces.push_back(fr);
        /* triangle (generator, v, v1): VorCell::calculate_volume/centroid */
        double ax = P.x[v] - xi, ay = P.y[v] - yi;
        double qx = P.x[v1] - xi, qy = P.y[v1] - yi;
        double A = 0.5 * std::fabs(ax * qy - ay * qx);
        vol += A;
        cx += A * ((P.x[v] + P.x[v1] + xi) / 3.);
        cy += A * ((P.y[v] + P.y[v1] + yi) / 3.);
    }
    out.volume = vol;
    out.centroid[0] = cx / vol;
    out.centroid[1] = cy / vol;
}

/* ------------------------------- 3D cell ------------------------------- */

struct Poly3 {
    std::vector<double> v;        /* xyz triples */
    std::vector<int> fstart, flen, flab, idx;
};

struct Cross {
    int a, b, v;
};

bool clip3(Poly3& P, Poly3& T, const double* m, const double* u, int label,
           bool& bad) {
    const int nv = (int)P.v.size() / 3;
    static thread_local std::vector<double> s;
    s.resize(nv);
    double smax = -1.;
    for(int k = 0; k < nv; ++k) {
        s[k] = (P.v[3 * k] - m[0]) * u[0] + (P.v[3 * k + 1] - m[1]) * u[1] +
               (P.v[3 * k + 2] - m[2]) * u[2];
    }
    /* only vertices referenced by faces matter */
    for(int t : P.idx) smax = std::max(smax, s[t]);
    if(smax <= 0.) return false;
    static thread_local std::vector<Cross> cr;
    static thread_local std::vector<int> capnext, remap;
    cr.clear();
    T.v.clear();
    T.fstart.clear();
    T.flen.clear();
    T.flab.clear();
    T.idx.clear();
    remap.assign(nv, -1);
    auto keep = [&](int a) {
        if(remap[a] < 0) {
            remap[a] = (int)T.v.size() / 3;
            T.v.push_back(P.v[3 * a]);
            T.v.push_back(P.v[3 * a + 1]);
            T.v.push_back(P.v[3 * a + 2]);
        }
        return remap[a];
    };
    auto cross = [&](int a, int b) { /* a inside, b outside */
        int lo = std::min(a, b), hi = std::max(a, b);
        for(const Cross& c : cr)
            if(c.a == lo && c.b == hi) return c.v;
        double t = s[a] / (s[a] - s[b]);
        int vi = (int)T.v.size() / 3;
        for(int d = 0; d < 3; ++d)
            T.v.push_back(P.v[3 * a + d] + t * (P.v[3 * b + d] - P.v[3 * a + d]));
        cr.push_back({lo, hi, vi});
        return vi;
    };
    capnext.clear();
    const int nf = (int)P.fstart.size();
    for(int f = 0; f < nf; ++f) {
        const int* L = &P.idx[P.fstart[f]];
        const int n = P.flen[f];
        int nin = 0;
        for(int k = 0; k < n; ++k) nin += s[L[k]] <= 0.;
        if(nin == 0) continue;
        int st = (int)T.idx.size();
        if(nin == n) {
            for(int k = 0; k < n; ++k) T.idx.push_back(keep(L[k]));
        } else {
            int xin = -1, xout = -1;
            for(int k = 0; k < n; ++k) {
                int a = L[k], b = L[(k + 1) % n];
                bool ia = s[a] <= 0., ib = s[b] <= 0.;
                if(ia) T.idx.push_back(keep(a));
                if(ia && !ib) {
                    xout = cross(a, b);
                    T.idx.push_back(xout);
                } else if(!ia && ib) {
                    xin = cross(b, a);
                    T.idx.push_back(xin);
                }
            }
            if(xin < 0 || xout < 0) {
                bad = true;
                return true;
            }
            /* the clipped face runs xout -> (plane) -> xin; the cap runs
             * the other way */
            if((int)capnext.size() < (int)T.v.size() / 3)
                capnext.resize(T.v.size() / 3, -1);
            capnext[xin] = xout;
        }
        int len = (int)T.idx.size() - st;
        if(len >= 3) {
            T.fstart.push_back(st);
            T.flen.push_back(len);
            T.flab.push_back(P.flab[f]);
        } else {
            T.idx.resize(st);
        }
    }
    capnext.resize(T.v.size() / 3, -1);
    if(cr.empty()) {
        bad = true;
        return true;
    }
    int start = cr[0].v;
    int st = (int)T.idx.size();
    int cur = start, count = 0;
    do {
        T.idx.push_back(cur);
        cur = capnext[cur];
        ++count;
        if(cur < 0 || count > (int)cr.size()) {
            bad = true;
            return true;
        }
    } while(cur != start);
    if(count != (int)cr.size()) {
        bad = true;
        return true;
    }
    T.fstart.push_back(st);
    T.flen.push_back(count);
    T.flab.push_back(label);
    std::swap(P, T);
    return true;
}

void box3(Poly3& P, const double* lo, const double* hi) {
    P.v.clear();
    for(int c = 0; c < 8; ++c) {
        P.v.push_back((c & 1) ? hi[0] : lo[0]);
        P.v.push_back((c & 2) ? hi[1] : lo[1]);
        P.v.push_back((c & 4) ? hi[2] : lo[2]);
    }
    /* faces counter-clockwise seen from outside; walls 0 x-,1 x+,2 y-,3 y+,
     * 4 z-, 5 z+ */
    static const int F[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4},
                                {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
    P.idx.clear();
    P.fstart.clear();
    P.flen.clear();
    P.flab.clear();
    for(int f = 0; f < 6; ++f) {
        P.fstart.push_back((int)P.idx.size());
        for(int k = 0; k < 4; ++k) P.idx.push_back(F[f][k]);
        P.flen.push_back(4);
        P.flab.push_back(-1 - f);
    }
}

void cell3(int64_t i, const double* pos, int64_t n, int periodic,
           const Grid& G, CellOut& out) {
    const double* xi = pos + 3 * i;
    double lo[3], hi[3];
    for(int d = 0; d < 3; ++d) {
        lo[d] = periodic ? xi[d] - 0.5 : 0.;
        hi[d] = periodic ? xi[d] + 0.5 : 1.;
    }
    Poly3 P, T;
    box3(P, lo, hi);
    std::vector<Nb> nbs;
    const int g = G.g;
    int bc[3];
    for(int d = 0; d < 3; ++d) bc[d] = bucket_of(xi[d], g);
    const int kmax = periodic ? 2 * g + 2 : g + 1;
    bool bad = false;
    for(int k = 0; k <= kmax && !bad; ++k) {
        for(int oz = -k; oz <= k && !bad; ++oz) {
            for(int oy = -k; oy <= k && !bad; ++oy) {
                for(int ox = -k; ox <= k && !bad; ++ox) {
                    if(std::max(std::abs(ox), std::max(std::abs(oy), std::abs(oz))) != k)
                        continue;
                    int c[3] = {bc[0] + ox, bc[1] + oy, bc[2] + oz};
                    int sh[3] = {0, 0, 0};
                    bool skip = false;
                    for(int d = 0; d < 3; ++d) {
                        if(periodic) {
                            sh[d] = (int)std::floor((double)c[d] / g);
                            c[d] -= sh[d] * g;
                        } else if(c[d] < 0 || c[d] >= g) {
                            skip = true;
                        }
                    }
                    if(skip) continue;
                    int64_t b = ((int64_t)c[2] * g + c[1]) * g + c[0];
                    for(int32_t t = G.start[b]; t < G.start[b + 1]; ++t) {
                        int32_t j = G.items[t];
                        if(j == i && !sh[0] && !sh[1] && !sh[2]) continue;
                        double xj[3], u[3], m[3];
                        for(int d = 0; d < 3; ++d) {
                            xj[d] = pos[3 * j + d] + sh[d];
                            u[d] = xj[d] - xi[d];
                            m[d] = 0.5 * (xi[d] + xj[d]);
                        }
                        int label = (int)nbs.size();
                        if(clip3(P, T, m, u, label, bad)) {
                            Nb nb;
                            nb.j = j;
                            for(int d = 0; d < 3; ++d) nb.sh[d] = (int8_t)sh[d];
                            nbs.push_back(nb);
                            if(bad) break;
                        }
                    }
                }
            }
        }
        double r2 = 0.;
        for(int t : P.idx) {
            double dx = P.v[3 * t] - xi[0], dy = P.v[3 * t + 1] - xi[1],
                   dz = P.v[3 * t + 2] - xi[2];
            r2 = std::max(r2, dx * dx + dy * dy + dz * dz);
        }
        double reach = k * G.h;
        if(4. * r2 <= reach * reach) break;
        if(k == kmax) out.ok = 0;
    }
    if(bad) {
        out.ok = 0;
        return;
    }
    double vol = 0., C[3] = {0., 0., 0.};
    const int nf = (int)P.fstart.size();
    for(int f = 0; f < nf; ++f) {
        const int* L = &P.idx[P.fstart[f]];
        const int nvf = P.flen[f];
        FaceRec fr;
        std::memset(&fr, 0, sizeof fr);
        int lab = P.flab[f];
        if(lab >= 0) {
            const Nb& nb = nbs[lab];
            fr.nb = nb.j;
            for(int d = 0; d < 3; ++d) fr.sh[d] = nb.sh[d];
            fr.kind = (nb.sh[0] || nb.sh[1] || nb.sh[2]) ? 1 : 0;
        } else {
            if(periodic) out.ok = 0;
            fr.nb = -1 - lab;
            fr.kind = 2;
        }
        /* drop vertices closer than 1e-13 to the previous kept one, as the
         * reference's construct() does (src/VorTess.cpp:207-250) */
        int keepv[512];
        int nk = 0;
        for(int k = 0; k < nvf && nk < 512; ++k) {
            const double* a = &P.v[3 * L[k]];
            bool dup = false;
            if(nk) {
                const double* b = &P.v[3 * keepv[nk - 1]];
                const double* c0 = &P.v[3 * keepv[0]];
                double d1 = std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) +
                                      (a[2] - b[2]) * (a[2] - b[2]));
                double d2 = std::sqrt((a[0] - c0[0]) * (a[0] - c0[0]) +
                                      (a[1] - c0[1]) * (a[1] - c0[1]) +
                                      (a[2] - c0[2]) * (a[2] - c0[2]));
                dup = !(d1 > 1e-13 && d2 > 1e-13);
            }
            if(!dup) keepv[nk++] = L[k];
        }
        if(nk < 3) {
            fr.area = 0.;
        } else {
            /* VorFace::calculate_midpoint / calculate_area
             * (src/VorFace.cpp:293-404) */
            double area = 0., mid[3] = {0., 0., 0.};
            const double* v0 = &P.v[3 * keepv[0]];
            for(int k = 1; k < nk - 1; ++k) {
                const double* a = &P.v[3 * keepv[k]];
                const double* b = &P.v[3 * keepv[k + 1]];
                double ab[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
                double ac[3] = {a[0] - v0[0], a[1] - v0[1], a[2] - v0[2]};
                double ab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
                double ac2 = ac[0] * ac[0] + ac[1] * ac[1] + ac[2] * ac[2];
                double abac = ab[0] * ac[0] + ab[1] * ac[1] + ab[2] * ac[2];
                double ta = 0.5 * std::sqrt(std::fabs(ab2 * ac2 - abac * abac));
                area += ta;
                for(int d = 0; d < 3; ++d) mid[d] += (a[d] + b[d] + v0[d]) * ta;
            }
            for(int d = 0; d < 3; ++d) mid[d] /= 3. * area;
            if(mid[0] != mid[0]) {
                fr.area = 0.;
            } else {
                double ar = 0.;
                for(int k = 0; k < nk; ++k) {
                    const double* a = &P.v[3 * keepv[k]];
                    const double* b = &P.v[3 * keepv[(k + 1) % nk]];
                    double ab[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
                    double ac[3] = {a[0] - mid[0], a[1] - mid[1], a[2] - mid[2]};
                    double ab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
                    double ac2 = ac[0] * ac[0] + ac[1] * ac[1] + ac[2] * ac[2];
                    double abac = ab[0] * ac[0] + ab[1] * ac[1] + ab[2] * ac[2];
                    ar += 0.5 * std::sqrt(std::fabs(ab2 * ac2 - abac * abac));
                }
                fr.area = (ar != ar) ? 0. : ar;
                for(int d = 0; d < 3; ++d) fr.mid[d] = mid[d];
            }
        }
        out.faces.push_back(fr);
        /* tetrahedra (v0, vk, vk+1, generator): VorCell::calculate_volume /
         * calculate_centroid (src/VorCell.cpp:257-387) */
        const double* p0 = &P.v[3 * L[0]];
        for(int k = 1; k < nvf - 1; ++k) {
            const double* pj = &P.v[3 * L[k]];
            const double* pk = &P.v[3 * L[k + 1]];
            double r1[3], r2[3], r3[3];
            for(int d = 0; d < 3; ++d) {
                r1[d] = p0[d] - pj[d];
                r2[d] = pj[d] - pk[d];
                r3[d] = pk[d] - xi[d];
            }
            double A = std::fabs(r1[0] * r2[1] * r3[2] + r1[1] * r2[2] * r3[0] +
                                 r1[2] * r2[0] * r3[1] - r1[2] * r2[1] * r3[0] -
                                 r2[2] * r3[1] * r1[0] - r3[2] * r1[1] * r2[0]);
            A /= 6;
            for(int d = 0; d < 3; ++d)
                C[d] += 0.25 * (p0[d] + pj[d] + pk[d] + xi[d]) * A;
            vol += A;
        }
    }
    out.volume = vol;
    for(int d = 0; d < 3; ++d) out.centroid[d] = C[d] / vol;
}

}  // namespace

/* ----------------------------- assembly ----------------------------- */

struct sfx_voronoi {
    int dim = 0;
    int periodic = 0;
    int64_t ncell = 0;
    std::vector<double> cell_pos, centroid, volume, total_area;
    std::vector<int32_t> cell_off, cell_idx;
    std::vector<double> farea, fmid, frpos;
    std::vector<int32_t> fleft, fright, fkind;
};

static bool face_less(const FaceRec& a, const FaceRec& b) {
    if(a.kind != b.kind) return a.kind < b.kind;
    if(a.nb != b.nb) return a.nb < b.nb;
    for(int d = 0; d < 3; ++d)
        if(a.sh[d] != b.sh[d]) return a.sh[d] < b.sh[d];
    return false;
}

extern "C" int sfx_voronoi_build(int dim, int64_t n, const double* pos,
                                 int periodic, int nthreads,
                                 sfx_voronoi** out) {
    if(!out || !pos || (dim != 2 && dim != 3) || n < 2 || n > 0x7ffffff0)
        return SFX_ERR_INVALID;
    for(int64_t t = 0; t < n * dim; ++t) {
        if(!(pos[t] >= 0. && pos[t] < 1.)) return SFX_ERR_INVALID;
    }
    Grid G = build_grid(dim, n, pos);
    std::vector<CellOut> cells(n);
    if(nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int64_t> next(0);
    const int64_t chunk = 256;
    auto work = [&]() {
        for(;;) {
            int64_t b = next.fetch_add(chunk);
            if(b >= n) break;
            int64_t e = std::min(n, b + chunk);
            for(int64_t i = b; i < e; ++i) {
                if(dim == 2)
                    cell2(i, pos, n, periodic, G, cells[i]);
                else
                    cell3(i, pos, n, periodic, G, cells[i]);
            }
        }
    };
    std::vector<std::thread> th;
    for(int t = 1; t < nthreads; ++t) th.emplace_back(work);
    work();
    for(auto& t : th) t.join();
    for(int64_t i = 0; i < n; ++i)
        if(!cells[i].ok) return SFX_ERR_MESH;

    sfx_voronoi* V = new sfx_voronoi;
    V->dim = dim;
    V->periodic = periodic;
    V->ncell = n;
    V->cell_pos.assign(pos, pos + n * dim);
    V->centroid.resize(n * dim);
    V->volume.resize(n);
    for(int64_t i = 0; i < n; ++i) {
        std::sort(cells[i].faces.begin(), cells[i].faces.end(), face_less);
        V->volume[i] = cells[i].volume;
        for(int d = 0; d < dim; ++d) V->centroid[i * dim + d] = cells[i].centroid[d];
    }
    /* owner faces: real pairs from the lower index (or from the higher one
     * if only that side found the face), images and mirrors from the cell */
    for(int64_t i = 0; i < n; ++i) {
        for(const FaceRec& fr : cells[i].faces) {
            bool own;
            if(fr.kind != 0) {
                own = true;
            } else if(fr.nb > i) {
                own = true;
            } else {
                /* i is the higher index: own only if nb does not list i */
                own = true;
                for(const FaceRec& o : cells[fr.nb].faces)
                    if(o.kind == 0 && o.nb == i) {
                        own = false;
                        break;
                    }
            }
            if(!own) continue;
            int32_t L = (int32_t)i, R = fr.nb;
            if(fr.kind == 0 && R < L) std::swap(L, R);
            V->fleft.push_back(L);
            V->fkind.push_back(fr.kind);
            V->farea.push_back(fr.area);
            for(int d = 0; d < dim; ++d) V->fmid.push_back(fr.mid[d]);
            const double* xl = pos + (int64_t)L * dim;
            if(fr.kind == 0) {
                V->fright.push_back(R);
                for(int d = 0; d < dim; ++d) V->frpos.push_back(pos[(int64_t)R * dim + d]);
            } else if(fr.kind == 1) {
                V->fright.push_back(R);
                for(int d = 0; d < dim; ++d)
                    V->frpos.push_back(pos[(int64_t)R * dim + d] + (double)fr.sh[d]);
            } else {
                /* mirror of the owner in wall fr.nb: axis nb/2, side nb%2 */
                V->fright.push_back(-1);
                int ax = fr.nb / 2, side = fr.nb % 2;
                for(int d = 0; d < dim; ++d) {
                    double x = xl[d];
                    if(d == ax) x = side ? 2. - x : -x;
                    V->frpos.push_back(x);
                }
            }
        }
    }
    /* the owner loop visits faces with the lower index as owner in order of
     * the owner only when both sides agree; re-sort faces by left cell to keep
     * the owner-major order in the rare asymmetric case */
    const int64_t nf = (int64_t)V->fleft.size();
    std::vector<int64_t> perm(nf);
    for(int64_t f = 0; f < nf; ++f) perm[f] = f;
    std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) {
        return V->fleft[a] < V->fleft[b];
    });
    {
        auto P = [&](auto& vec, int w) {
            auto old = vec;
            for(int64_t f = 0; f < nf; ++f)
                for(int k = 0; k < w; ++k) vec[f * w + k] = old[perm[f] * w + k];
        };
        P(V->fleft, 1);
        P(V->fright, 1);
        P(V->fkind, 1);
        P(V->farea, 1);
        P(V->fmid, dim);
        P(V->frpos, dim);
    }
    /* cell face lists, ascending face index */
    V->cell_off.assign(n + 1, 0);
    for(int64_t f = 0; f < nf; ++f) {
        V->cell_off[V->fleft[f] + 1]++;
        if(V->fkind[f] == 0) V->cell_off[V->fright[f] + 1]++;
    }
    for(int64_t i = 0; i < n; ++i) V->cell_off[i + 1] += V->cell_off[i];
    V->cell_idx.resize(V->cell_off[n]);
    std::vector<int32_t> fill(V->cell_off.begin(), V->cell_off.end() - 1);
    for(int64_t f = 0; f < nf; ++f) {
        V->cell_idx[fill[V->fleft[f]]++] = (int32_t)f;
        if(V->fkind[f] == 0) V->cell_idx[fill[V->fright[f]]++] = (int32_t)f;
    }
    /* total area in the cell's face order (VorCell::calculate_total_area,
     * src/VorCell.cpp:396-411) */
    V->total_area.assign(n, 0.);
    for(int64_t i = 0; i < n; ++i) {
        double a = 0.;
        for(int32_t k = V->cell_off[i]; k < V->cell_off[i + 1]; ++k)
            a += V->farea[V->cell_idx[k]];
        V->total_area[i] = a;
    }
    *out = V;
    return SFX_OK;
}

extern "C" int sfx_voronoi_counts(const sfx_voronoi* V, int64_t* ncell,
                                  int64_t* nface, int64_t* nnz) {
    if(!V) return SFX_ERR_INVALID;
    *ncell = V->ncell;
    *nface = (int64_t)V->fleft.size();
    *nnz = (int64_t)V->cell_idx.size();
    return SFX_OK;
}

extern "C" int sfx_voronoi_export(const sfx_voronoi* V, double* cell_centroid,
                                  double* cell_volume, double* cell_total_area,
                                  int32_t* cell_face_offset,
                                  int32_t* cell_face_index, double* face_area,
                                  double* face_midpoint, int32_t* face_left,
                                  int32_t* face_right, int32_t* face_kind,
                                  double* face_right_pos) {
    if(!V) return SFX_ERR_INVALID;
    auto cp = [](auto* dst, const auto& src) {
        if(dst) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
    };
    cp(cell_centroid, V->centroid);
    cp(cell_volume, V->volume);
    cp(cell_total_area, V->total_area);
    cp(cell_face_offset, V->cell_off);
    cp(cell_face_index, V->cell_idx);
    cp(face_area, V->farea);
    cp(face_midpoint, V->fmid);
    cp(face_left, V->fleft);
    cp(face_right, V->fright);
    cp(face_kind, V->fkind);
    cp(face_right_pos, V->frpos);
    return SFX_OK;
}

extern "C" void sfx_voronoi_free(sfx_voronoi* V) {
    delete V;
}
