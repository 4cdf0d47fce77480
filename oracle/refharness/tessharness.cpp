/*
 * Reference tessellation harness (TEST INFRASTRUCTURE ONLY).
 *
 * Linked against the UNMODIFIED reference sources of the tessellation
 * (DelTess, DelTess_mpi, VorTess, Simplex, the exact predicates of ExArith
 * with the fixed-width integer stand-in under shim/boost, the particle Tree)
 * and of the hot path, compiled by oracle/build.py.  For a set of generator
 * positions in the unit box it
 *
 *   1. sets up the particles as the reference does: Hilbert keys from the
 *      box (ParticleVector::sort, src/utilities/ParticleVector.cpp:222-262),
 *      sorted by key, local ids in that order, an octtree of them;
 *   2. tessellates them with the reference's own VorTess (constructor,
 *      add_point per particle, complete with the tree for the reflective
 *      mirrors or periodic images, construct: src/VorTessManager.cpp:56-75);
 *   3. exports the face list in the sfxflux layout: per cell position,
 *      centroid, volume, total area and its faces in VorCell order; per face
 *      area, midpoint, left cell, right cell or -1, kind (real, periodic
 *      image: the neighbour generator has id 1 and a particle; reflective
 *      mirror: no particle, DelTess_mpi.cpp:150-186) and the right
 *      generator's position -- the exporter a Shadowfax maintainer adds
 *      beside VorTessManager::hydro;
 *   4. optionally runs the reference's per-step loop (gradients, face fluxes,
 *      update_Q, get_W; src/Simulation.cpp:414-483, 791-836) for a static
 *      mesh with one global time step on the objects VorTess built.
 *
 * The product library never links, loads or runs this program.
 *
 * Usage:  tessharness <in.bin> <out.bin>
 *   in:  int32 dim, n, periodic, solver (0 exact, 1 HLLC), nsteps, has_w;
 *        double gamma, tolerance, cutoff, dt, tessellation tolerance;
 *        double positions[n][dim]; double W0[n][S] when has_w (input order)
 *   out: int32 status, steps_done, n, nface, nnz; int32 order[n] (input index
 *        of the cell at each sorted position); the face list in sorted order:
 *        pos[n][dim], centroid[n][dim], volume[n], total_area[n],
 *        face_offset[n+1], face_index[nnz], area[F], midpoint[F][dim],
 *        left[F], right[F], kind[F], right_pos[F][dim]; when has_w, W[n][S]
 *        and Q[n][S] after nsteps (sorted order)
 */
#include "RectangularBox.hpp"
#include "StateVector.hpp"
#include "TimeLine.hpp"
#include "Vec.hpp"
#include "VorCell.hpp"
#include "VorFace.hpp"
#include "VorGen.hpp"
#include "VorTess.hpp"
#include "riemann/ExactRiemannSolver.hpp"
#include "riemann/HLLCRiemannSolver.hpp"
#include "utilities/GasParticle.hpp"
#include "utilities/Tree.hpp"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <map>
#include <vector>

#include "timeline_stub.hpp"

namespace {

const int S = ndim_ + 2;

enum { H_OK = 0, H_RIEMANN_EXC = 10, H_UPDATEQ_EXC = 11, H_FLUX_EXC = 12, H_OTHER_EXC = 13 };

template <typename T>
void read_or_die(FILE* f, T* dst, size_t n) {
    if(n && fread(dst, sizeof(T), n, f) != n) {
        fprintf(stderr, "tessharness: truncated input\n");
        exit(3);
    }
}

template <typename T>
void put(FILE* f, const std::vector<T>& v) {
    if(!v.empty()) fwrite(v.data(), sizeof(T), v.size(), f);
}

#if ndim_ == 3
Vec vec_of(const double* x) {
    return Vec(x[0], x[1], x[2]);
}
#else
Vec vec_of(const double* x) {
    return Vec(x[0], x[1]);
}
#endif

}  // namespace

int main(int argc, char** argv) {
    if(argc < 3) {
        fprintf(stderr, "usage: tessharness <in.bin> <out.bin>\n");
        return 1;
    }
    FILE* in = fopen(argv[1], "rb");
    if(!in) return 1;
    int32_t hdr[6];
    read_or_die(in, hdr, 6);
    const int dim = hdr[0], n = hdr[1], periodic = hdr[2], solverkind = hdr[3];
    const int nsteps = hdr[4], has_w = hdr[5];
    double prm[5];
    read_or_die(in, prm, 5);
    const double gamma = prm[0], tol = prm[1], cutoff = prm[2], dt = prm[3], tess_tol = prm[4];
    if(dim != ndim_ || n < 1) {
        fprintf(stderr, "tessharness built for %dD, input is %dD (n = %d)\n", ndim_, dim, n);
        return 2;
    }
    std::vector<double> pos((size_t)n * dim), W0;
    read_or_die(in, pos.data(), pos.size());
    if(has_w) {
        W0.resize((size_t)n * S);
        read_or_die(in, W0.data(), W0.size());
    }
    fclose(in);

    /* 1. particles in Hilbert order with local ids, and their octtree */
#if ndim_ == 3
    RectangularBox box(Vec(0.5, 0.5, 0.5), Vec(1., 1., 1.));
#else
    RectangularBox box(Vec(0.5, 0.5), Vec(1., 1.));
#endif
    std::vector<GasParticle*> parts(n);
    for(int i = 0; i < n; ++i) {
        parts[i] = new GasParticle(vec_of(&pos[(size_t)i * dim]));
        parts[i]->set_key(box.get_key(parts[i]->get_position()));
    }
    std::vector<int> order(n);
    for(int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return parts[a]->get_key() < parts[b]->get_key();
    });
    std::vector<GasParticle*> sorted(n);
    for(int j = 0; j < n; ++j) sorted[j] = parts[order[j]];
    /* equal keys: shifted within the lowest tree node, as the reference does */
    for(int j = 1; j < n; ++j) {
        if(sorted[j - 1]->get_key() == sorted[j]->get_key()) {
            const unsigned long last = (1ul << ndim_) - 1;
            if((sorted[j]->get_key() & last) == last)
                sorted[j - 1]->set_key(sorted[j - 1]->get_key() - 1);
            else
                sorted[j]->set_key(sorted[j]->get_key() + 1);
        }
    }
    for(int j = 0; j < n; ++j) sorted[j]->set_local_id(j);
    Tree tree(box.get_cuboid(), periodic != 0);
    for(int j = 0; j < n; ++j) tree.add_particle(sorted[j]);
    tree.finalize();

    /* 2. the reference's tessellation */
    VorTess* tess = new VorTess(&box, n, periodic != 0, tess_tol);
    for(int j = 0; j < n; ++j) tess->add_point(sorted[j], j);
    tess->complete(tree);
    tess->construct();

    /* 3. the face list */
    std::vector<VorFace*>& faces = tess->get_faces();
    const int F = (int)faces.size();
    std::map<VorFace*, int32_t> fid;
    for(int f = 0; f < F; ++f) fid[faces[f]] = f;
    std::vector<double> cpos((size_t)n * dim), ccen((size_t)n * dim), cvol(n), carea(n);
    std::vector<int32_t> coff(n + 1, 0), cidx;
    std::vector<VorCell*> cells(n);
    for(int j = 0; j < n; ++j) {
        VorCell* c = sorted[j]->get_cell();
        cells[j] = c;
        const Vec x = sorted[j]->get_position();
        const Vec cen = c->get_centroid();
        for(int l = 0; l < dim; ++l) {
            cpos[(size_t)j * dim + l] = x[l];
            ccen[(size_t)j * dim + l] = cen[l];
        }
        cvol[j] = c->get_volume();
        carea[j] = c->get_total_area();
        for(VorFace* face : c->get_faces()) cidx.push_back(fid.at(face));
        coff[j + 1] = (int32_t)cidx.size();
    }
    std::vector<double> farea(F), fmid((size_t)F * dim), frpos((size_t)F * dim);
    std::vector<int32_t> fleft(F), fright(F), fkind(F);
    for(int f = 0; f < F; ++f) {
        VorGen* L = faces[f]->get_left();
        VorGen* R = faces[f]->get_ngb();
        farea[f] = faces[f]->get_area();
        const Vec& mid = faces[f]->get_midpoint();
        const Vec rp = R->get_position();
        for(int l = 0; l < dim; ++l) {
            fmid[(size_t)f * dim + l] = mid[l];
            frpos[(size_t)f * dim + l] = rp[l];
        }
        fleft[f] = (int32_t)L->get_particle()->get_local_id();
        if(R->get_particle() == NULL) { /* reflective mirror */
            fkind[f] = 2;
            fright[f] = -1;
        } else if(R->get_id() == 1) { /* periodic image */
            fkind[f] = 1;
            fright[f] = (int32_t)R->get_particle()->get_local_id();
        } else {
            fkind[f] = 0;
            fright[f] = (int32_t)R->get_particle()->get_local_id();
        }
    }

    /* 4. the reference's step loop on the objects VorTess built */
    int status = H_OK, steps_done = 0;
    if(has_w) {
        RiemannSolver* solver;
        if(solverkind == 0)
            solver = new ExactRiemannSolver(gamma, tol, cutoff);
        else
            solver = new HLLCRiemannSolver(gamma);
        /* initial state: W given, Q = get_Q(V, W) (src/Simulation.cpp:1231-1251) */
        for(int j = 0; j < n; ++j) {
            StateVector W;
            for(int k = 0; k < S; ++k) W[k] = W0[(size_t)order[j] * S + k];
            sorted[j]->set_W(W);
            sorted[j]->set_Q(solver->get_Q(cvol[j], W));
            sorted[j]->set_centroid(cells[j]->get_centroid());
            sorted[j]->set_total_area(carea[j]);
            sorted[j]->set_soundspeed(solver->get_soundspeed(W));
            sorted[j]->set_starttime(0);
            sorted[j]->set_endtime(1ul << 60);
        }
        char dummy[64] = {0};
        TimeLine* tl = new TimeLine(dt, dt, 0.4, 0., *(ParticleVector*)dummy, "", "",
                                    *(UnitSet*)dummy, *(UnitSet*)dummy, false, false, NULL,
                                    false, 0., 0., 0, false);
        try {
            for(int step = 0; step < nsteps; ++step) {
                for(int j = 0; j < n; ++j) {
                    StateVector gradients[3];
                    cells[j]->estimate_gradient(gradients);
                    sorted[j]->set_gradients(gradients);
                }
                for(int f = 0; f < F; ++f) {
                    faces[f]->set_v();
                    faces[f]->calculate_flux(*tl, *solver);
                }
                for(int j = 0; j < n; ++j) sorted[j]->update_Q();
                for(int j = 0; j < n; ++j) {
                    StateVector W = solver->get_W(cvol[j], sorted[j]->get_Qvec());
                    sorted[j]->set_W(W);
                    sorted[j]->set_soundspeed(solver->get_soundspeed(W));
                }
                ++steps_done;
            }
        } catch(RiemannSolverException& e) {
            status = H_RIEMANN_EXC;
        } catch(UpdateQException& e) {
            status = H_UPDATEQ_EXC;
        } catch(FluxCalculationException& e) {
            status = H_FLUX_EXC;
        } catch(std::exception& e) {
            status = H_OTHER_EXC;
        }
    }

    FILE* out = fopen(argv[2], "wb");
    if(!out) return 4;
    const int32_t ohdr[5] = {status, steps_done, n, F, (int32_t)cidx.size()};
    fwrite(ohdr, sizeof(int32_t), 5, out);
    put(out, order);
    put(out, cpos);
    put(out, ccen);
    put(out, cvol);
    put(out, carea);
    put(out, coff);
    put(out, cidx);
    put(out, farea);
    put(out, fmid);
    put(out, fleft);
    put(out, fright);
    put(out, fkind);
    put(out, frpos);
    if(has_w) {
        std::vector<double> buf((size_t)n * S);
        for(int j = 0; j < n; ++j)
            for(int k = 0; k < S; ++k) buf[(size_t)j * S + k] = sorted[j]->get_Wvec()[k];
        put(out, buf);
        for(int j = 0; j < n; ++j)
            for(int k = 0; k < S; ++k) buf[(size_t)j * S + k] = sorted[j]->get_Qvec()[k];
        put(out, buf);
    }
    fclose(out);
    return 0;
}
