/*
 * Reference CPU flux-pass harness (TEST INFRASTRUCTURE ONLY).
 *
 * This translation unit is linked against the UNMODIFIED reference Shadowfax
 * sources of the hot path (VorFace, VorCell, VorGen, GasParticle, Particle and
 * the Exact/HLLC Riemann solvers), compiled from the reference tree by
 * oracle/build.py.  It reads a face-list mesh in the sfxflux binary
 * exchange format, builds the reference's own VorGen / VorCell / VorFace /
 * GasParticle objects from it and runs the reference's per-step loop for a
 * static mesh with one global time step:
 *
 *   for every cell:  VorCell::estimate_gradient -> GasParticle::set_gradients
 *                    (src/Simulation.cpp:414-420, src/VorCell.cpp:464-530)
 *   for every face:  VorFace::calculate_flux   (src/VorTessManager.cpp:198-212,
 *                                               src/VorFace.cpp:670-1024)
 *   for every cell:  GasParticle::update_Q      (src/Simulation.cpp:473-483)
 *   for every cell:  RiemannSolver::get_W, set_W (src/Simulation.cpp:791-836)
 *
 * Initial conserved quantities follow src/Simulation.cpp:1231-1251
 * (Q = solver->get_Q(V, W)).
 *
 * The product library never links, loads or runs this program; tests and the
 * CPU-baseline leg of bench.py do.
 *
 * Usage:  harness <mesh.bin> <out.bin> [mode]
 *   mode "step"    (default) run the step loop described by the input header
 *   mode "riemann" evaluate solve() / solve_for_flux() on the state pairs
 *                  stored in the input (golden-vector checks)
 */
#include "StateVector.hpp"
#include "TimeLine.hpp"
#include "Vec.hpp"
#include "VorCell.hpp"
#include "VorFace.hpp"
#include "VorGen.hpp"
#include "MPIGlobal.hpp"
#include "riemann/ExactRiemannSolver.hpp"
#include "riemann/HLLCRiemannSolver.hpp"
#include "utilities/GasParticle.hpp"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <vector>


#include "timeline_stub.hpp"

namespace {

struct Reader {
    FILE* f;
    template <typename T> void read(T* dst, size_t n) {
        if(n && fread(dst, sizeof(T), n, f) != n) {
            fprintf(stderr, "harness: truncated input\n");
            exit(3);
        }
    }
    template <typename T> std::vector<T> vec(size_t n) {
        std::vector<T> v(n);
        read(v.data(), n);
        return v;
    }
};

const int S = ndim_ + 2;

/* status codes mirrored by the host tooling */
enum { H_OK = 0, H_RIEMANN_EXC = 10, H_UPDATEQ_EXC = 11, H_FLUX_EXC = 12,
       H_OTHER_EXC = 13 };

int run_steps(Reader& in, const char* outpath) {
    int32_t hdr[8];
    in.read(hdr, 8);
    const int dim = hdr[0], ncell = hdr[1], nface = hdr[2], nnz = hdr[3];
    const int solverkind = hdr[4], nsteps = hdr[5];
    /* moving generators (builds without -DSTATIC only): per step the
     * generator velocities of VorCell::get_velocity with the reflective-box
     * check of src/Simulation.cpp:366-398, the face velocities of
     * VorFace::set_v, and the drift after the update (src/Simulation.cpp:
     * 473-481).  One step per tessellation, as in the reference, where the
     * mesh is rebuilt after every drift. */
    const int moving = hdr[6] == 1, periodic = hdr[7];
    /* local (hierarchical) time steps: mode 2, one system step [t_now,
     * t_next) with every particle's step bounds, and the stored gradients of
     * the inactive ones, given in the input (the static build) */
    const int local = hdr[6] == 2;
#ifndef STATIC
    if(local) {
        fprintf(stderr, "harness: local time steps use the static build\n");
        return 5;
    }
#endif
    if(local && nsteps != 1) {
        fprintf(stderr, "harness: local time steps take one system step\n");
        return 5;
    }
#ifdef STATIC
    if(moving) {
        fprintf(stderr, "harness: moving generators need a build without -DSTATIC\n");
        return 5;
    }
#else
    if(moving && nsteps != 1) {
        fprintf(stderr, "harness: moving generators take one step per tessellation\n");
        return 5;
    }
#endif
    double prm[4];
    in.read(prm, 4);
    const double gamma = prm[0], tol = prm[1], cutoff = prm[2], dt = prm[3];
    if(dim != ndim_) {
        fprintf(stderr, "harness built for %dD, mesh is %dD\n", ndim_, dim);
        return 2;
    }
    std::vector<double> cpos = in.vec<double>((size_t)ncell * dim);
    std::vector<double> ccen = in.vec<double>((size_t)ncell * dim);
    std::vector<double> cvol = in.vec<double>(ncell);
    std::vector<double> carea = in.vec<double>(ncell);
    std::vector<int32_t> coff = in.vec<int32_t>(ncell + 1);
    std::vector<int32_t> cidx = in.vec<int32_t>(nnz);
    std::vector<double> farea = in.vec<double>(nface);
    std::vector<double> fmid = in.vec<double>((size_t)nface * dim);
    std::vector<int32_t> fleft = in.vec<int32_t>(nface);
    std::vector<int32_t> fright = in.vec<int32_t>(nface);
    std::vector<int32_t> fkind = in.vec<int32_t>(nface);
    std::vector<double> frpos = in.vec<double>((size_t)nface * dim);
    std::vector<double> fvel = in.vec<double>((size_t)nface * dim);
    std::vector<double> W0 = in.vec<double>((size_t)ncell * S);
    std::vector<uint64_t> tstart, tend;
    std::vector<double> grad0;
    uint64_t t_now = 0, t_next = 0;
    double t_total = dt;
    if(local) {
        tstart = in.vec<uint64_t>(ncell);
        tend = in.vec<uint64_t>(ncell);
        uint64_t tw[2];
        in.read(tw, 2);
        t_now = tw[0];
        t_next = tw[1];
        in.read(&t_total, 1);
        grad0 = in.vec<double>((size_t)ncell * dim * S);
    }

    RiemannSolver* solver;
    if(solverkind == 0) {
        solver = new ExactRiemannSolver(gamma, tol, cutoff);
    } else {
        solver = new HLLCRiemannSolver(gamma);
    }

    /* real generators and their particles */
    std::vector<GasParticle*> parts(ncell);
    std::vector<VorGen*> gens;
    gens.reserve(ncell + nface + 1);
    for(int i = 0; i < ncell; ++i) {
        const double* x = &cpos[(size_t)i * dim];
#if ndim_ == 3
        Vec p(x[0], x[1], x[2]);
        VorGen* g = new VorGen(x[0], x[1], x[2]);
#else
        Vec p(x[0], x[1]);
        VorGen* g = new VorGen(x[0], x[1]);
#endif
        GasParticle* gp = new GasParticle(p);
        gp->set_starttime(local ? tstart[i] : 0);
        gp->set_endtime(local ? tend[i] : 1ul << 60);
        g->set_particle(gp);
        g->set_particle_id(i);
        g->set_id(2);
        gp->set_vorgen(g);
        gp->set_local_id(i);
        parts[i] = gp;
        gens.push_back(g);
    }
    /* faces; the right generator is the real neighbour, a periodic image
     * (same particle, shifted position, id 1) or a reflective mirror
     * (no particle, id 1) as DelTess::add_mirrors builds them
     * (src/DelTess_mpi.cpp:150-186). */
    std::vector<VorFace*> faces(nface);
    std::vector<VorGen*> rgen(nface);
    for(int f = 0; f < nface; ++f) {
        std::vector<VorGen*> pts(1, gens[fleft[f]]);
        VorFace* face = new VorFace(0, pts);
        VorGen* r;
        if(fkind[f] == 0) {
            r = gens[fright[f]];
        } else {
            const double* x = &frpos[(size_t)f * dim];
#if ndim_ == 3
            r = new VorGen(x[0], x[1], x[2]);
#else
            r = new VorGen(x[0], x[1]);
#endif
            r->set_id(1);
            if(fkind[f] == 1) {
                r->set_particle(parts[fright[f]]);
                r->set_particle_id(fright[f]);
            } else {
                r->set_particle(NULL);
            }
        }
        rgen[f] = r;
        face->add_ngb(r);
        face->set_area(farea[f]);
        face->set_midpoint(&fmid[(size_t)f * dim]);
        /* STATIC build: VorFace::set_v is a no-op and _v stays zero */
        faces[f] = face;
    }
    /* cells: faces in the order of the cell's face list, neighbour j is the
     * generator on the other side of face j (src/VorTess.cpp:153-283) */
    std::vector<VorCell*> cells(ncell);
    for(int i = 0; i < ncell; ++i) {
        VorCell* c = new VorCell(gens[i]);
        for(int k = coff[i]; k < coff[i + 1]; ++k) {
            int f = cidx[k];
            c->add_face(faces[f]);
            c->add_ngb(fleft[f] == i ? rgen[f] : gens[fleft[f]]);
        }
#if ndim_ == 3
        c->set_centroid(Vec(ccen[(size_t)i * 3], ccen[(size_t)i * 3 + 1],
                            ccen[(size_t)i * 3 + 2]));
#else
        c->set_centroid(Vec(ccen[(size_t)i * 2], ccen[(size_t)i * 2 + 1]));
#endif
        c->set_volume(cvol[i]);
        gens[i]->set_cell(c);
        cells[i] = c;
    }
    /* initial state: W given, Q = get_Q(V, W) (src/Simulation.cpp:1231-1251) */
    for(int i = 0; i < ncell; ++i) {
        StateVector W;
        for(int k = 0; k < S; ++k) W[k] = W0[(size_t)i * S + k];
        parts[i]->set_W(W);
        parts[i]->set_Q(solver->get_Q(cvol[i], W));
        parts[i]->set_centroid(cells[i]->get_centroid());
        parts[i]->set_total_area(carea[i]);
        parts[i]->set_soundspeed(solver->get_soundspeed(W));
    }

    char dummy[64] = {0};
    TimeLine* tl = new TimeLine(local ? t_total : dt, local ? t_total : dt, 0.4, 0.,
                                *(ParticleVector*)dummy, "", "", *(UnitSet*)dummy,
                                *(UnitSet*)dummy, false, false, NULL, false, 0., 0., 0, false);
    if(local) tl->set_time((unsigned long)t_now);
    std::vector<double> vel_out((size_t)ncell * dim, 0.);

    std::vector<double> grad_last((size_t)ncell * dim * S, 0.);
    std::vector<double> dQ_last((size_t)ncell * S, 0.);
    int status = H_OK;
    double secs = 0.;
    std::vector<double> step_secs(nsteps > 0 ? nsteps : 1, 0.);
    int steps_done = 0;
    try {
        for(int step = 0; step < nsteps; ++step) {
            auto t0 = std::chrono::steady_clock::now();
#ifndef STATIC
            if(moving) {
                for(int i = 0; i < ncell; ++i) {
                    StateVector Wgas = parts[i]->get_Wvec();
                    Vec v = cells[i]->get_velocity();
                    if(!periodic) {
                        /* the unit box: centre 0.5, half side 0.5
                         * (RectangularBox::inside, src/RectangularBox.cpp:91-99) */
                        Vec newx = parts[i]->get_position() + dt * v;
                        bool inside = true;
                        for(unsigned int l = 0; l < ndim_; l++)
                            if(fabs(0.5 - newx[l]) > 1. / 2) inside = false;
                        if(!inside) {
                            v[0] -= Wgas[1];
                            v[1] -= Wgas[2];
#if ndim_ == 3
                            v[2] -= Wgas[3];
#endif
                        }
                    }
                    parts[i]->set_velocity(v);
                }
            }
#endif
            if(local) {
                /* the first kick (src/Simulation.cpp:366-398): the particles
                 * starting a step set their velocity; then gradients of the
                 * active particles, the stored ones of the others */
                for(int i = 0; i < ncell; ++i) {
                    if(parts[i]->get_starttime() != t_now) continue;
                    StateVector Wgas = parts[i]->get_Wvec();
                    Vec v = cells[i]->get_velocity();
                    if(!periodic) {
                        double dti = tl->get_realtime_interval(parts[i]->get_endtime() -
                                                              parts[i]->get_starttime());
                        Vec newx = parts[i]->get_position() + dti * v;
                        bool inside = true;
                        for(unsigned int l = 0; l < ndim_; l++)
                            if(fabs(0.5 - newx[l]) > 1. / 2) inside = false;
                        if(!inside) {
                            v[0] -= Wgas[1];
                            v[1] -= Wgas[2];
#if ndim_ == 3
                            v[2] -= Wgas[3];
#endif
                        }
                    }
                    parts[i]->set_velocity(v);
                    for(int l = 0; l < dim; ++l) vel_out[(size_t)i * dim + l] = v[l];
                }
                for(int i = 0; i < ncell; ++i) {
                    StateVector gradients[3];
                    if(parts[i]->get_starttime() == t_now) {
                        cells[i]->estimate_gradient(gradients);
                    } else {
                        for(int l = 0; l < dim; ++l)
                            for(int k = 0; k < S; ++k)
                                gradients[l][k] = grad0[((size_t)i * dim + l) * S + k];
                    }
                    parts[i]->set_gradients(gradients);
                }
            } else {
                for(int i = 0; i < ncell; ++i) {
                    StateVector gradients[3];
                    cells[i]->estimate_gradient(gradients);
                    parts[i]->set_gradients(gradients);
                }
            }
            for(int f = 0; f < nface; ++f) {
                faces[f]->set_v();
                faces[f]->calculate_flux(*tl, *solver);
            }
            if(step == nsteps - 1) {
                for(int i = 0; i < ncell; ++i) {
                    StateVector g[ndim_];
                    parts[i]->get_gradients(g);
                    for(int l = 0; l < dim; ++l)
                        for(int k = 0; k < S; ++k)
                            grad_last[((size_t)i * dim + l) * S + k] = g[l][k];
                    for(int k = 0; k < S; ++k)
                        dQ_last[(size_t)i * S + k] = parts[i]->get_dQvec()[k];
                }
            }
            for(int i = 0; i < ncell; ++i) {
#ifndef STATIC
                if(moving) parts[i]->drift(dt);
#endif
                parts[i]->update_Q();
            }
            for(int i = 0; i < ncell; ++i) {
                /* with local steps only the particles ending their step */
                if(local && parts[i]->get_endtime() != t_next) continue;
                StateVector W = solver->get_W(cvol[i], parts[i]->get_Qvec());
                parts[i]->set_W(W);
                parts[i]->set_soundspeed(solver->get_soundspeed(W));
            }
            auto t1 = std::chrono::steady_clock::now();
            step_secs[step] = std::chrono::duration<double>(t1 - t0).count();
            secs += step_secs[step];
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

    FILE* out = fopen(outpath, "wb");
    if(!out) return 4;
    int32_t ohdr[4] = {status, steps_done, ncell, dim};
    fwrite(ohdr, sizeof(int32_t), 4, out);
    fwrite(&secs, sizeof(double), 1, out);
    fwrite(step_secs.data(), sizeof(double), nsteps, out);
    std::vector<double> buf((size_t)ncell * S);
    for(int i = 0; i < ncell; ++i)
        for(int k = 0; k < S; ++k) buf[(size_t)i * S + k] = parts[i]->get_Wvec()[k];
    fwrite(buf.data(), sizeof(double), buf.size(), out);
    for(int i = 0; i < ncell; ++i)
        for(int k = 0; k < S; ++k) buf[(size_t)i * S + k] = parts[i]->get_Qvec()[k];
    fwrite(buf.data(), sizeof(double), buf.size(), out);
    fwrite(grad_last.data(), sizeof(double), grad_last.size(), out);
    fwrite(dQ_last.data(), sizeof(double), dQ_last.size(), out);
    if(local) fwrite(vel_out.data(), sizeof(double), vel_out.size(), out);
    if(moving) {
        /* generator positions after the drift */
        std::vector<double> pb((size_t)ncell * dim);
        for(int i = 0; i < ncell; ++i)
            for(int l = 0; l < dim; ++l) pb[(size_t)i * dim + l] = parts[i]->get_position()[l];
        fwrite(pb.data(), sizeof(double), pb.size(), out);
    }
    fclose(out);
    return 0;
}

/* Riemann golden-vector mode: for each of n state pairs evaluate
 * solve() (Exact only) and solve_for_flux() with normal n and zero face
 * velocity. */
int run_riemann(Reader& in, const char* outpath) {
    int32_t hdr[4];
    in.read(hdr, 4);
    const int n = hdr[0], solverkind = hdr[1], reflective = hdr[2];
    double prm[4];
    in.read(prm, 4);
    std::vector<double> WL = in.vec<double>((size_t)n * S);
    std::vector<double> WR = in.vec<double>((size_t)n * S);
    std::vector<double> nrm = in.vec<double>((size_t)n * ndim_);
    RiemannSolver* solver;
    if(solverkind == 0) {
        solver = new ExactRiemannSolver(prm[0], prm[1], prm[2]);
    } else {
        solver = new HLLCRiemannSolver(prm[0]);
    }
    std::vector<double> half((size_t)n * S, 0.), flux((size_t)n * S, 0.);
    std::vector<int32_t> st(n, 0);
    for(int i = 0; i < n; ++i) {
        StateVector L, R;
        for(int k = 0; k < S; ++k) {
            L[k] = WL[(size_t)i * S + k];
            R[k] = WR[(size_t)i * S + k];
        }
        Vec nv, v;
        for(int k = 0; k < ndim_; ++k) nv[k] = nrm[(size_t)i * ndim_ + k];
        try {
            if(solverkind == 0) {
                StateVector L2 = L, R2 = R;
                double mach = 0.;
                StateVector h = solver->solve(L2, R2, nv, mach, reflective != 0);
                for(int k = 0; k < S; ++k) half[(size_t)i * S + k] = h[k];
            }
            StateVector L3 = L, R3 = R;
            StateVector fl = solver->solve_for_flux(L3, R3, nv, v, reflective != 0);
            for(int k = 0; k < S; ++k) flux[(size_t)i * S + k] = fl[k];
        } catch(std::exception& e) {
            st[i] = H_RIEMANN_EXC;
        }
    }
    FILE* out = fopen(outpath, "wb");
    if(!out) return 4;
    fwrite(st.data(), sizeof(int32_t), n, out);
    fwrite(half.data(), sizeof(double), half.size(), out);
    fwrite(flux.data(), sizeof(double), flux.size(), out);
    fclose(out);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if(argc < 3) {
        fprintf(stderr, "usage: %s <in.bin> <out.bin> [step|riemann]\n", argv[0]);
        return 1;
    }
    MPIGlobal::rank = 0;
    MPIGlobal::size = 1;
    FILE* f = fopen(argv[1], "rb");
    if(!f) {
        fprintf(stderr, "cannot open %s\n", argv[1]);
        return 1;
    }
    char magic[8];
    if(fread(magic, 1, 8, f) != 8 || memcmp(magic, "SFXMESH1", 8)) {
        fprintf(stderr, "bad magic\n");
        return 1;
    }
    Reader in{f};
    std::string mode = argc > 3 ? argv[3] : "step";
    int rc = mode == "riemann" ? run_riemann(in, argv[2]) : run_steps(in, argv[2]);
    fclose(f);
    return rc;
}
