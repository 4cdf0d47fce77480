/*
 * Dimension-specific part of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 * Included twice by sfx_oracle.c with D = 2 and D = 3; FN(x) appends the
 * dimension to every name.  S = D + 2 hydro fields (rho, v[D], p).
 *
 * Expression order follows the reference literally (left-to-right
 * association of every C++ expression), because the goal is bit-identical
 * results.
 */

#define S (D + 2)

/* ---- Riemann solver state (src/riemann/ExactRiemannSolver.cpp:48-70) ---- */
typedef struct FN(solver) {
    int kind;
    double gamma, tol, cutoff;
    double gp1d2g, gm1d2g, gm1dgp1, tdgp1, tdgm1, gm1d2, tgdgm1, ginv;
} FN(solver);

static void FN(solver_init)(FN(solver) * s, const sfxo_params* p) {
    double g = p->gamma;
    s->kind = p->solver;
    s->gamma = g;
    s->tol = p->tolerance;
    s->cutoff = p->cutoff;
    s->gp1d2g = 0.5 * (g + 1.) / g;
    s->gm1d2g = 0.5 * (g - 1.) / g;
    s->gm1dgp1 = (g - 1.) / (g + 1.);
    s->tdgp1 = 2. / (g + 1.);
    s->tdgm1 = 2. / (g - 1.);
    s->gm1d2 = 0.5 * (g - 1.);
    s->tgdgm1 = 2. * g / (g - 1.);
    s->ginv = 1. / g;
}

/* ---- time derivative of the primitive variables ----
 * ExactRiemannSolver.cpp:892-934 and HLLCRiemannSolver.cpp:415-450 (same
 * arithmetic for the hydro fields).  g[l][k] = d W_k / d x_l.  The 2D row for
 * v_y uses g[1] twice, as the reference does (ExactRiemannSolver.cpp:920). */
static void FN(time_derivative)(const FN(solver) * s, const double* W,
                                const double g[D][S], double* dW) {
#if D == 3
    dW[0] = -W[0] * (g[0][1] + g[1][2] + g[2][3]) - W[1] * g[0][0] -
            W[2] * g[1][0] - W[3] * g[2][0];
    dW[1] = -W[1] * g[0][1] - W[2] * g[1][1] - W[3] * g[2][1] - g[0][4] / W[0];
    dW[2] = -W[1] * g[0][2] - W[2] * g[1][2] - W[3] * g[2][2] - g[1][4] / W[0];
    dW[3] = -W[1] * g[0][3] - W[2] * g[1][3] - W[3] * g[2][3] - g[2][4] / W[0];
    dW[4] = -s->gamma * W[4] * (g[0][1] + g[1][2] + g[2][3]) - W[1] * g[0][4] -
            W[2] * g[1][4] - W[3] * g[2][4];
#else
    dW[0] = -W[1] * g[0][0] - W[2] * g[1][0] - W[0] * (g[0][1] + g[1][2]);
    dW[1] = -W[1] * g[0][1] - W[2] * g[1][1] - g[0][3] / W[0];
    dW[2] = -W[1] * g[1][2] - W[2] * g[1][2] - g[1][3] / W[0];
    dW[3] = -s->gamma * W[3] * (g[0][1] + g[1][2]) - W[1] * g[0][3] -
            W[2] * g[1][3];
#endif
}

/* ---- reconstruction, src/VorFace.hpp:174-196 ---- */
static void FN(reconstruct)(double* W, const double g[D][S], const double* d) {
    for(int k = 0; k < S; ++k) {
#if D == 3
        W[k] += g[0][k] * d[0] + g[1][k] * d[1] + g[2][k] * d[2];
#else
        W[k] += g[0][k] * d[0] + g[1][k] * d[1];
#endif
    }
}

/* ---- pairwise slope limiter, src/VorFace.hpp:92-137 ---- */
static double FN(limit1)(double phimid0, double phiL, double phiR,
                         const double* d, double r) {
    double psi1 = 0.5;
    double psi2 = 0.25;
#if D == 3
    double dnrm = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
#else
    double dnrm = sqrt(d[0] * d[0] + d[1] * d[1]);
#endif
    double delta1 = psi1 * fabs(phiL - phiR);
    double delta2 = psi2 * fabs(phiL - phiR);
    double phimin = fmin(phiL, phiR);
    double phimax = fmax(phiL, phiR);
    double phibar = phiL + dnrm / r * (phiR - phiL);
    double phiplus, phiminus, phimid;
    if((phimax + delta1) * phimax > 0.) {
        phiplus = phimax + delta1;
    } else {
        phiplus = phimax / (1. + delta1 / fabs(phimax));
    }
    if((phimin - delta1) * phimin > 0.) {
        phiminus = phimin - delta1;
    } else {
        phiminus = phimin / (1. + delta1 / fabs(phimin));
    }
    if(phiL == phiR) {
        phimid = phiL;
    } else {
        if(phiL < phiR) {
            phimid = fmax(phiminus, fmin(phibar + delta2, phimid0));
        } else {
            phimid = fmin(phiplus, fmax(phibar - delta2, phimid0));
        }
    }
    return phimid;
}

/* StateVector limiter, src/VorFace.hpp:150-162 */
static void FN(limit)(double* W, const double* WL, const double* WR,
                      const double* d, double r) {
    for(int k = 0; k < S; ++k) W[k] = FN(limit1)(W[k], WL[k], WR[k], d, r);
}

/* ---- mirror of a state across a reflective face:
 * VorFace::transform / invtransform (src/VorFace.cpp:417-542) with the normal
 * velocity flipped in between (src/VorCell.cpp:479-485) ---- */
static void FN(mirror_state)(double* W, const double* left, const double* right) {
#if D == 3
    double n[4], o[4], p[3];
    n[0] = right[0] - left[0];
    n[1] = right[1] - left[1];
    n[2] = right[2] - left[2];
    n[3] = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    n[0] /= n[3];
    n[1] /= n[3];
    n[2] /= n[3];
    if(n[0] || n[1]) {
        o[0] = -n[1];
        o[1] = n[0];
        o[2] = 0.;
        o[3] = sqrt(o[0] * o[0] + o[1] * o[1]);
        o[0] /= o[3];
        o[1] /= o[3];
        p[0] = -n[2] * o[1];
        p[1] = n[2] * o[0];
        p[2] = o[3];
    } else {
        o[0] = 0.;
        o[1] = 1.;
        o[2] = 0.;
        o[3] = 1.;
        p[0] = -1.;
        p[1] = 0.;
        p[2] = 0.;
    }
    double v0 = W[1], v1 = W[2], v2 = W[3];
    W[1] = v0 * n[0] + v1 * n[1] + v2 * n[2];
    W[2] = v0 * o[0] + v1 * o[1];
    W[3] = v0 * p[0] + v1 * p[1] + v2 * p[2];
    W[1] = -W[1];
    v0 = W[1];
    v1 = W[2];
    v2 = W[3];
    W[1] = v0 * n[0] + v1 * o[0] + v2 * p[0];
    W[2] = v0 * n[1] + v1 * o[1] + v2 * p[1];
    W[3] = v0 * n[2] + v2 * p[2];
#else
    double d[3];
    d[0] = left[0] - right[0];
    d[1] = left[1] - right[1];
    d[2] = sqrt(d[0] * d[0] + d[1] * d[1]);
    double cost = -d[0] / d[2];
    double sint = -d[1] / d[2];
    double W1 = W[1] * cost + W[2] * sint;
    W[2] = -W[1] * sint + W[2] * cost;
    W[1] = W1;
    W[1] = -W[1];
    W1 = W[1] * cost - W[2] * sint;
    W[2] = W[1] * sint + W[2] * cost;
    W[1] = W1;
#endif
}

/* ---- gradients with the cell-wise slope limiter,
 * VorCell::estimate_gradient (src/VorCell.cpp:464-530) ---- */
static void FN(cell_gradient)(const sfxo_mesh* m, const double* Wall, int i,
                              double delta[D][S]) {
    const double* W = Wall + (size_t)i * S;
    const double* xi = m->cell_pos + (size_t)i * D;
    double Wmax[S], Wmin[S];
    for(int k = 0; k < S; ++k) {
        Wmax[k] = W[k];
        Wmin[k] = W[k];
        for(int l = 0; l < D; ++l) delta[l][k] = 0.;
    }
    int beg = m->cell_face_offset[i], end = m->cell_face_offset[i + 1];
    for(int j = end; j-- > beg;) {
        int f = m->cell_face_index[j];
        double Aij = m->face_area[f];
        if(!Aij) continue;
        const double* mid = m->face_midpoint + (size_t)f * D;
        const double* xj;
        double Wj[S];
        if(m->face_left[f] == i) {
            xj = m->face_right_pos + (size_t)f * D;
            if(m->face_kind[f] == 2) {
                for(int k = 0; k < S; ++k) Wj[k] = W[k];
                FN(mirror_state)(Wj, xi, xj);
            } else {
                const double* Wr = Wall + (size_t)m->face_right[f] * S;
                for(int k = 0; k < S; ++k) Wj[k] = Wr[k];
            }
        } else {
            int jl = m->face_left[f];
            xj = m->cell_pos + (size_t)jl * D;
            const double* Wl = Wall + (size_t)jl * S;
            for(int k = 0; k < S; ++k) Wj[k] = Wl[k];
        }
        double c[D], rij[D];
        for(int l = 0; l < D; ++l) c[l] = mid[l] - 0.5 * (xi[l] + xj[l]);
        for(int l = 0; l < D; ++l) rij[l] = xi[l] - xj[l];
#if D == 3
        double rnorm = sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
#else
        double rnorm = sqrt(rij[0] * rij[0] + rij[1] * rij[1]);
#endif
        for(int l = D; l--;) {
            for(int k = 0; k < S; ++k) {
                delta[l][k] += Aij * ((Wj[k] - W[k]) * c[l] / rnorm -
                                      0.5 * (W[k] + Wj[k]) * rij[l] / rnorm);
            }
        }
        for(int k = 0; k < S; ++k) {
            Wmax[k] = (Wmax[k] < Wj[k]) ? Wj[k] : Wmax[k]; /* std::max */
            Wmin[k] = (Wj[k] < Wmin[k]) ? Wj[k] : Wmin[k]; /* std::min */
        }
    }
    double V = m->cell_volume[i];
    for(int l = D; l--;)
        for(int k = 0; k < S; ++k) delta[l][k] /= V;
    const double* cen = m->cell_centroid + (size_t)i * D;
    double alpha[S];
    for(int k = 0; k < S; ++k) alpha[k] = 1.;
    for(int j = end; j-- > beg;) {
        int f = m->cell_face_index[j];
        if(!m->face_area[f]) continue;
        const double* mid = m->face_midpoint + (size_t)f * D;
        double d[D];
        for(int l = 0; l < D; ++l) d[l] = mid[l] - cen[l];
        for(int k = 0; k < S; ++k) {
            double dp = delta[0][k] * d[0] + delta[1][k] * d[1];
#if D == 3
            dp += delta[2][k] * d[2];
#endif
            /* StateVector::operator/= maps a zero divisor to 1
             * (src/StateVector.hpp:607-646) */
            double q1 = Wmax[k] - W[k];
            double q2 = Wmin[k] - W[k];
            if(dp) {
                q1 /= dp;
                q2 /= dp;
            } else {
                q1 = 1.;
                q2 = 1.;
            }
            double mx = (q1 < q2) ? q2 : q1;           /* std::max */
            alpha[k] = (mx < alpha[k]) ? mx : alpha[k]; /* std::min */
        }
    }
    for(int l = D; l--;)
        for(int k = 0; k < S; ++k) delta[l][k] *= alpha[k];
}

/* ======================= exact Riemann solver ======================= */

static double FN(sound)(const FN(solver) * s, const double* W) {
    /* ExactRiemannSolver.cpp:681-687 */
    if(W[0]) return sqrt(s->gamma * W[D + 1] / W[0]);
    return 0.;
}

static double FN(fb)(const FN(solver) * s, double p, const double* Wb, double a) {
    /* ExactRiemannSolver.cpp:556-567 */
    double fval;
    if(p > Wb[D + 1]) {
        double A = s->tdgp1 / Wb[0];
        double B = s->gm1dgp1 * Wb[D + 1];
        fval = (p - Wb[D + 1]) * sqrt(A / (p + B));
    } else {
        fval = s->tdgm1 * a * (opow(p / Wb[D + 1], s->gm1d2g) - 1.);
    }
    return fval;
}

static double FN(gb)(const FN(solver) * s, double p, const double* Wb) {
    /* ExactRiemannSolver.cpp:575-579 */
    double A = s->tdgp1 / Wb[0];
    double B = s->gm1dgp1 * Wb[D + 1];
    return sqrt(A / (p + B));
}

static double FN(fprimeb)(const FN(solver) * s, double p, const double* Wb,
                          double a) {
    /* ExactRiemannSolver.cpp:589-600 */
    double fval;
    if(p > Wb[D + 1]) {
        double A = s->tdgp1 / Wb[0];
        double B = s->gm1dgp1 * Wb[D + 1];
        fval = (1. - 0.5 * (p - Wb[D + 1]) / (B + p)) * sqrt(A / (p + B));
    } else {
        fval = 1. / (Wb[0] * a) * opow(p / Wb[D + 1], -s->gp1d2g);
    }
    return fval;
}

static double FN(f)(const FN(solver) * s, double p, const double* WL,
                    const double* WR, double vL, double vR, double aL,
                    double aR) {
    /* ExactRiemannSolver.cpp:628-631 */
    return FN(fb)(s, p, WL, aL) + FN(fb)(s, p, WR, aR) + (vR - vL);
}

static double FN(fprime)(const FN(solver) * s, double p, const double* WL,
                         const double* WR, double aL, double aR) {
    /* ExactRiemannSolver.cpp:611-614 */
    return FN(fprimeb)(s, p, WL, aL) + FN(fprimeb)(s, p, WR, aR);
}

static double FN(guess_p)(const FN(solver) * s, const double* WL,
                          const double* WR, double vL, double vR, double aL,
                          double aR) {
    /* ExactRiemannSolver.cpp:644-673; min/max are std::min/std::max */
    double pL = WL[D + 1], pR = WR[D + 1];
    double pguess;
    double pmin = (pR < pL) ? pR : pL;
    double pmax = (pL < pR) ? pR : pL;
    double qmax = pmax / pmin;
    double ppv = 0.5 * (pL + pR) - 0.125 * (vR - vL) * (WL[0] + WR[0]) * (aL + aR);
    double fl = s->tol * 0.5 * (pL + pR);
    ppv = (fl < ppv) ? ppv : fl;
    if(qmax <= 2. && pmin <= ppv && ppv <= pmax) {
        pguess = ppv;
    } else {
        if(ppv < pmin) {
            pguess = opow((aL + aR - s->gm1d2 * (vR - vL)) /
                                  (aL / opow(pL, s->gm1d2g) +
                                   aR / opow(pR, s->gm1d2g)),
                          s->tgdgm1);
        } else {
            pguess = (FN(gb)(s, ppv, WL) * pL + FN(gb)(s, ppv, WR) * pR - vR + vL) /
                     (FN(gb)(s, ppv, WL) + FN(gb)(s, ppv, WR));
        }
    }
    fl = s->tol * 0.5 * (pL + pR);
    pguess = (fl < pguess) ? pguess : fl;
    return pguess;
}

/* Brent's method, ExactRiemannSolver.cpp:462-546.  *iters counts function
 * evaluations inside the loop; the loop is capped at SFXO_MAX_ITER. */
static double FN(brent)(const FN(solver) * s, double lowerLimit,
                        double upperLimit, double errorTol, const double* WL,
                        const double* WR, double vL, double vR, double aL,
                        double aR, int* iters, int* errexit, int* noconv) {
    double a = lowerLimit;
    double b = upperLimit;
    double c = 0.;
    double d = 1e230;
    double fa = FN(f)(s, a, WL, WR, vL, vR, aL, aR);
    double fbv = FN(f)(s, b, WL, WR, vL, vR, aL, aR);
    double fc = 0.;
    double sv = 0.;
    double fs = 0.;
    *iters = 0;
    *errexit = 0;
    if(fa * fbv >= 0) {
        *errexit = 1;
        if(fa < fbv)
            return a;
        else
            return b;
    }
    if(fabs(fa) < fabs(fbv)) {
        double tmp = a;
        a = b;
        b = tmp;
        tmp = fa;
        fa = fbv;
        fbv = tmp;
    }
    c = a;
    fc = fa;
    int mflag = 1;
    while(!(fbv == 0) && (fabs(a - b) > errorTol * (a + b) * 0.5)) {
        if(*iters >= SFXO_MAX_ITER) {
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
        double tmp2 = (3. * a + b) / 4.;
        if(!(((sv > tmp2) && (sv < b)) || ((sv < tmp2) && (sv > b))) ||
           (mflag && (fabs(sv - b) >= (fabs(b - c) / 2.))) ||
           (!mflag && (fabs(sv - b) >= (fabs(c - d) / 2.))) ||
           (mflag && (fabs(b - c) < errorTol * (b + c) * 0.5)) ||
           (!mflag && (fabs(c - d) < errorTol * (c + d) * 0.5))) {
            sv = (a + b) / 2.;
            mflag = 1;
        } else {
            mflag = 0;
        }
        fs = FN(f)(s, sv, WL, WR, vL, vR, aL, aR);
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
            double tmp = a;
            a = b;
            b = tmp;
            tmp = fa;
            fa = fbv;
            fbv = tmp;
        }
    }
    return b;
}

/* vacuum Riemann problem, ExactRiemannSolver.cpp:304-446; returns 0 or an
 * error code, the half state in sol and the branch code in *code */
static int FN(solve_vacuum)(const FN(solver) * s, const double* WL,
                            const double* WR, double vL, double vR, double aL,
                            double aR, const double* n, double* sol, int* code) {
    double g = s->gamma;
    double vhalf;
    int k;
    if(!WR[0] && !WL[0]) {
        for(k = 0; k < S; ++k) sol[k] = 0.;
        *code = SFXB_VAC_BOTH;
        return SFXO_OK;
    }
    if(!WR[0]) {
        for(k = 0; k < S; ++k) sol[k] = WL[k];
        if(vL < aL) {
            double SL = vL + 2. * aL / (g - 1.);
            if(SL > 0.) {
                sol[0] = WL[0] * opow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * vL,
                                      2. / (g - 1.));
                vhalf = 2. / (g + 1.) * (aL + 0.5 * (g - 1.) * vL) - vL;
                sol[D + 1] = WL[D + 1] *
                             opow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * vL,
                                  2. * g / (g - 1.));
                *code = SFXB_VAC_RIGHT | SFXB_S_LFAN;
            } else {
                for(k = 0; k < S; ++k) sol[k] = 0.;
                vhalf = 0.;
                *code = SFXB_VAC_RIGHT | SFXB_S_VAC;
            }
        } else {
            vhalf = 0.;
            *code = SFXB_VAC_RIGHT | SFXB_S_LUP;
        }
    } else {
        if(!WL[0]) {
            for(k = 0; k < S; ++k) sol[k] = WR[k];
            if(-aR < vR) {
                double SR = vR - 2. * aR / (g - 1.);
                if(SR >= 0.) {
                    for(k = 0; k < S; ++k) sol[k] = 0.;
                    vhalf = 0.;
                    *code = SFXB_VAC_LEFT | SFXB_S_VAC;
                } else {
                    sol[0] = WR[0] *
                             opow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * vR,
                                  2. / (g - 1.));
                    vhalf = 2. / (g + 1.) * (-aR + 0.5 * (g - 1.) * vR) - vR;
                    sol[D + 1] = WR[D + 1] *
                                 opow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * vR,
                                      2. * g / (g - 1.));
                    *code = SFXB_VAC_LEFT | SFXB_S_RFAN;
                }
            } else {
                vhalf = 0.;
                *code = SFXB_VAC_LEFT | SFXB_S_RUP;
            }
        } else {
            double SR = vR - 2. * aR / (g - 1.);
            double SL = vL + 2. * aL / (g - 1.);
            if(SR > 0. && SL < 0.) {
                for(k = 0; k < S; ++k) sol[k] = 0.;
                vhalf = 0.;
                *code = SFXB_VAC_GEN | SFXB_S_VAC;
            } else {
                if(SL >= 0.) {
                    for(k = 0; k < S; ++k) sol[k] = WL[k];
                    if(aL > vL) {
                        sol[0] = WL[0] *
                                 opow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * vL,
                                      2. / (g - 1.));
                        vhalf = 2. / (g + 1.) * (aL + 0.5 * (g - 1.) * vL) - vL;
                        sol[D + 1] = WL[D + 1] *
                                     opow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * vL,
                                          2. * g / (g - 1.));
                        *code = SFXB_VAC_GEN | SFXB_S_LFAN;
                    } else {
                        vhalf = 0.;
                        *code = SFXB_VAC_GEN | SFXB_S_LUP;
                    }
                } else {
                    for(k = 0; k < S; ++k) sol[k] = WR[k];
                    if(-aR < vR) {
                        sol[0] = WR[0] *
                                 opow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * vR,
                                      2. / (g - 1.));
                        vhalf = 2. / (g + 1.) * (-aR + 0.5 * (g - 1.) * vR) - vR;
                        sol[D + 1] = WR[D + 1] *
                                     opow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * vR,
                                          2. * g / (g - 1.));
                        *code = SFXB_VAC_GEN | SFXB_S_RFAN;
                    } else {
                        vhalf = 0.;
                        *code = SFXB_VAC_GEN | SFXB_S_RUP;
                    }
                }
            }
        }
    }
    for(k = 0; k < D; ++k) sol[1 + k] += vhalf * n[k];
    int bad = (sol[0] < 0.) || (sol[0] != sol[0]);
    for(k = 0; k < D; ++k) bad |= (sol[1 + k] != sol[1 + k]);
    bad |= (sol[D + 1] < 0.) || (sol[D + 1] != sol[D + 1]);
    return bad ? SFXO_ERR_RIEMANN : SFXO_OK;
}

/* ExactRiemannSolver::solve (ExactRiemannSolver.cpp:108-290).  WR is
 * overwritten with WL for a reflective face, as in the reference. */
static int FN(exact_solve)(const FN(solver) * s, double* WL, double* WR,
                           const double* n, int reflective, double* sol,
                           int* code) {
    int k;
#if D == 3
    double vL = WL[1] * n[0] + WL[2] * n[1] + WL[3] * n[2];
    double vR = WR[1] * n[0] + WR[2] * n[1] + WR[3] * n[2];
#else
    double vL = WL[1] * n[0] + WL[2] * n[1];
    double vR = WR[1] * n[0] + WR[2] * n[1];
#endif
    if(reflective) {
        for(k = 0; k < S; ++k) WR[k] = WL[k];
        vR = -vL;
    }
    double aL = FN(sound)(s, WL);
    double aR = FN(sound)(s, WR);
    *code = 0;
    if(!WL[0] || !WR[0]) {
        return FN(solve_vacuum)(s, WL, WR, vL, vR, aL, aR, n, sol, code);
    }
    double g = s->gamma;
    if(2. * aL / (g - 1.) + 2. * aR / (g - 1.) <= vR - vL) {
        int rc = FN(solve_vacuum)(s, WL, WR, vL, vR, aL, aR, n, sol, code);
        *code = (*code & ~SFXB_VAC_MASK) | SFXB_VAC_SPEED;
        return rc;
    }
    double tol = s->tol;
    double p = 0.;
    double pguess = FN(guess_p)(s, WL, WR, vL, vR, aL, aR);
    double fp = FN(f)(s, p, WL, WR, vL, vR, aL, aR);
    double fpguess = FN(f)(s, pguess, WL, WR, vL, vR, aL, aR);
    int newton = 0, brent_it = 0, errexit = 0, noconv = 0, mode;
    if(fp < s->cutoff) {
        mode = SFXB_IT_NEWTON_ONLY;
        while(fabs(p - pguess) > tol * 0.5 * (p + pguess)) {
            if(newton >= SFXO_MAX_ITER) {
                noconv = 1;
                break;
            }
            ++newton;
            p = pguess;
            pguess = pguess - fpguess / FN(fprime)(s, pguess, WL, WR, aL, aR);
            if(pguess < 0.) {
                pguess = 0.;
            }
            fpguess = FN(f)(s, pguess, WL, WR, vL, vR, aL, aR);
        }
        p = pguess;
    } else {
        mode = SFXB_IT_NEWTON;
        if(fp * fpguess >= 0.) {
            while(fabs(p - pguess) > tol * 0.5 * (p + pguess) && fpguess < 0.) {
                if(newton >= SFXO_MAX_ITER) {
                    noconv = 1;
                    break;
                }
                ++newton;
                p = pguess;
                pguess = pguess - fpguess / FN(fprime)(s, pguess, WL, WR, aL, aR);
                fpguess = FN(f)(s, pguess, WL, WR, vL, vR, aL, aR);
            }
        }
        if(!noconv && fabs(p - pguess) > tol * 0.5 * (p + pguess) && fpguess > 0.) {
            mode = SFXB_IT_BRENT;
            p = 0.;
            p = FN(brent)(s, p, pguess, tol, WL, WR, vL, vR, aL, aR, &brent_it,
                          &errexit, &noconv);
        } else {
            p = pguess;
        }
    }
    double u = 0.5 * (vL + vR) + 0.5 * (FN(fb)(s, p, WR, aR) - FN(fb)(s, p, WL, aL));
    double vhalf;
    int region;
    if(u < 0) {
        for(k = 0; k < S; ++k) sol[k] = WR[k];
        double pdpR = p / WR[D + 1];
        if(p > WR[D + 1]) {
            double SR = vR + aR * sqrt(s->gp1d2g * pdpR + s->gm1d2g);
            if(SR > 0) {
                sol[0] = WR[0] * (pdpR + s->gm1dgp1) / (s->gm1dgp1 * pdpR + 1.);
                sol[D + 1] = p;
                vhalf = u - vR;
                region = SFXB_S_RSHOCK_STAR;
            } else {
                vhalf = 0.;
                region = SFXB_S_RUP_SHOCK;
            }
        } else {
            double SHR = vR + aR;
            if(SHR > 0) {
                double STR = u + aR * opow(pdpR, s->gm1d2g);
                if(STR <= 0) {
                    sol[0] = WR[0] * opow(s->tdgp1 - s->gm1dgp1 / aR * vR, s->tdgm1);
                    vhalf = s->tdgp1 * (-aR + s->gm1d2 * vR) - vR;
                    sol[D + 1] = WR[D + 1] *
                                 opow(s->tdgp1 - s->gm1dgp1 / aR * vR, s->tgdgm1);
                    region = SFXB_S_RFAN;
                } else {
                    sol[0] = WR[0] * opow(pdpR, s->ginv);
                    sol[D + 1] = p;
                    vhalf = u - vR;
                    region = SFXB_S_RRARE_STAR;
                }
            } else {
                vhalf = 0.;
                region = SFXB_S_RUP;
            }
        }
    } else {
        for(k = 0; k < S; ++k) sol[k] = WL[k];
        double pdpL = p / WL[D + 1];
        if(p > WL[D + 1]) {
            double SL = vL - aL * sqrt(s->gp1d2g * pdpL + s->gm1d2g);
            if(SL < 0) {
                sol[0] = WL[0] * (pdpL + s->gm1dgp1) / (s->gm1dgp1 * pdpL + 1.);
                sol[D + 1] = p;
                vhalf = u - vL;
                region = SFXB_S_LSHOCK_STAR;
            } else {
                vhalf = 0.;
                region = SFXB_S_LUP_SHOCK;
            }
        } else {
            double SHL = vL - aL;
            if(SHL < 0) {
                double STL = u - aL * opow(pdpL, s->gm1d2g);
                if(STL > 0) {
                    sol[0] = WL[0] * opow(s->tdgp1 + s->gm1dgp1 / aL * vL, s->tdgm1);
                    vhalf = s->tdgp1 * (aL + s->gm1d2 * vL) - vL;
                    sol[D + 1] = WL[D + 1] *
                                 opow(s->tdgp1 + s->gm1dgp1 / aL * vL, s->tgdgm1);
                    region = SFXB_S_LFAN;
                } else {
                    sol[0] = WL[0] * opow(pdpL, s->ginv);
                    vhalf = u - vL;
                    sol[D + 1] = p;
                    region = SFXB_S_LRARE_STAR;
                }
            } else {
                vhalf = 0.;
                region = SFXB_S_LUP;
            }
        }
    }
    for(k = 0; k < D; ++k) sol[1 + k] += vhalf * n[k];
    *code = mode | region | (newton > 127 ? 127 : newton) << SFXB_NEWTON_SHIFT |
            (brent_it > 127 ? 127 : brent_it) << SFXB_BRENT_SHIFT |
            (errexit ? SFXB_BRENT_ERREXIT : 0);
    if(noconv) return SFXO_ERR_NOCONV;
    int bad = (sol[0] < 0.) || (sol[0] != sol[0]);
    for(k = 0; k < D; ++k) bad |= (sol[1 + k] != sol[1 + k]);
    bad |= (sol[D + 1] < 0.) || (sol[D + 1] != sol[D + 1]);
    return bad ? SFXO_ERR_RIEMANN : SFXO_OK;
}

/* ExactRiemannSolver::get_flux (ExactRiemannSolver.cpp:815-836), hydro
 * fields only; get_energy is ExactRiemannSolver.cpp:695-704 */
static void FN(exact_get_flux)(const FN(solver) * s, const double* v, int index,
                               const double* W, double* F) {
    int k;
    for(k = 0; k < S; ++k) F[k] = 0.;
    if(!W[0]) return;
    F[0] = W[0] * (W[1 + index] - v[index]);
    F[1] = W[0] * (W[1 + index] - v[index]) * W[1];
    F[2] = W[0] * (W[1 + index] - v[index]) * W[2];
#if D == 3
    F[3] = W[0] * (W[1 + index] - v[index]) * W[3];
    double e = 0.5 * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) +
               W[4] / (s->gamma - 1.);
#else
    double e = 0.5 * W[0] * (W[1] * W[1] + W[2] * W[2]) + W[3] / (s->gamma - 1.);
#endif
    F[1 + index] += W[D + 1];
    F[D + 1] = (W[1 + index] - v[index]) * e + W[D + 1] * W[1 + index];
}

/* ExactRiemannSolver::solve_for_flux (ExactRiemannSolver.cpp:858-880) */
static int FN(exact_flux)(const FN(solver) * s, double* WL, double* WR,
                          const double* n, const double* v, int reflective,
                          double* flux, int* code) {
    double half[S];
    int rc = FN(exact_solve)(s, WL, WR, n, reflective, half, code);
    if(rc) return rc;
    int k;
    for(k = 0; k < D; ++k) half[1 + k] += v[k];
    double F0[S], F1[S];
    FN(exact_get_flux)(s, v, 0, half, F0);
    FN(exact_get_flux)(s, v, 1, half, F1);
#if D == 3
    double F2[S];
    FN(exact_get_flux)(s, v, 2, half, F2);
    for(k = 0; k < S; ++k) flux[k] = F0[k] * n[0] + F1[k] * n[1] + F2[k] * n[2];
#else
    for(k = 0; k < S; ++k) flux[k] = F0[k] * n[0] + F1[k] * n[1];
#endif
    return SFXO_OK;
}

/* ========================= HLLC Riemann solver ========================= */

/* de-boost to the lab frame, HLLCRiemannSolver.cpp:392-400 / 196-205 */
static void FN(hllc_deboost)(const double* v, double* flux) {
    flux[1] += v[0] * flux[0];
    flux[2] += v[1] * flux[0];
#if D == 3
    flux[3] += v[2] * flux[0];
    double nrm2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    flux[4] += v[0] * flux[1] + v[1] * flux[2] + v[2] * flux[3] + 0.5 * nrm2 * flux[0];
#else
    double nrm2 = v[0] * v[0] + v[1] * v[1];
    flux[3] += v[0] * flux[1] + v[1] * flux[2] + 0.5 * nrm2 * flux[0];
#endif
}

/* HLLCRiemannSolver::vacuum_flux (HLLCRiemannSolver.cpp:44-209) */
static void FN(hllc_vacuum_flux)(const FN(solver) * s, const double* WL,
                                 const double* WR, const double* n,
                                 const double* v, double uL, double uR,
                                 double aL, double aR, double* flux, int* code) {
    double g = s->gamma;
    double sol[S];
    double vhalf;
    int k;
    if(!WR[0]) {
        for(k = 0; k < S; ++k) sol[k] = WL[k];
        if(aL > uL) {
            double SL = uL + 2. * aL / (g - 1.);
            if(SL > 0.) {
                sol[0] = WL[0] * opow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * uL,
                                      2. / (g - 1.));
                vhalf = 2. / (g + 1.) * (aL + 0.5 * (g - 1.) * uL) - uL;
                sol[D + 1] = WL[D + 1] *
                             opow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * uL,
                                  2. * g / (g - 1.));
                *code = SFXB_VAC_RIGHT | SFXB_S_LFAN;
            } else {
                for(k = 0; k < S; ++k) sol[k] = 0.;
                vhalf = 0.;
                *code = SFXB_VAC_RIGHT | SFXB_S_VAC;
            }
        } else {
            vhalf = 0.;
            *code = SFXB_VAC_RIGHT | SFXB_S_LUP;
        }
    } else {
        if(!WL[0]) {
            for(k = 0; k < S; ++k) sol[k] = WR[k];
            if(-uR < aR) {
                double SR = uR - 2. * aR / (g - 1.);
                if(SR >= 0.) {
                    for(k = 0; k < S; ++k) sol[k] = 0.;
                    vhalf = 0.;
                    *code = SFXB_VAC_LEFT | SFXB_S_VAC;
                } else {
                    sol[0] = WR[0] *
                             opow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * uR,
                                  2. / (g - 1.));
                    vhalf = 2. / (g + 1.) * (-aR + 0.5 * (g - 1.) * uR) - uR;
                    sol[D + 1] = WR[D + 1] *
                                 opow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * uR,
                                      2. * g / (g - 1.));
                    *code = SFXB_VAC_LEFT | SFXB_S_RFAN;
                }
            } else {
                vhalf = 0.;
                *code = SFXB_VAC_LEFT | SFXB_S_RUP;
            }
        } else {
            double SR = uR - 2. * aR / (g - 1.);
            double SL = uL + 2. * aL / (g - 1.);
            if(SR > 0. && SL < 0.) {
                for(k = 0; k < S; ++k) sol[k] = 0.;
                vhalf = 0.;
                *code = SFXB_VAC_SPEED | SFXB_S_VAC;
            } else {
                if(SL >= 0.) {
                    for(k = 0; k < S; ++k) sol[k] = WL[k];
                    if(uL < aL) {
                        sol[0] = WL[0] *
                                 opow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * uL,
                                      2. / (g - 1.));
                        vhalf = 2. / (g + 1.) * (aL + 0.5 * (g - 1.) * uL) - uL;
                        sol[D + 1] = WL[D + 1] *
                                     opow(2. / (g + 1.) + (g - 1.) / (g + 1.) / aL * uL,
                                          2. * g / (g - 1.));
                        *code = SFXB_VAC_SPEED | SFXB_S_LFAN;
                    } else {
                        vhalf = 0.;
                        *code = SFXB_VAC_SPEED | SFXB_S_LUP;
                    }
                } else {
                    for(k = 0; k < S; ++k) sol[k] = WR[k];
                    if(-uR < aR) {
                        sol[0] = WR[0] *
                                 opow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * uR,
                                      2. / (g - 1.));
                        vhalf = 2. / (g + 1.) * (-aR + 0.5 * (g - 1.) * uR) - uR;
                        sol[D + 1] = WR[D + 1] *
                                     opow(2. / (g + 1.) - (g - 1.) / (g + 1.) / aR * uR,
                                          2. * g / (g - 1.));
                        *code = SFXB_VAC_SPEED | SFXB_S_RFAN;
                    } else {
                        vhalf = 0.;
                        *code = SFXB_VAC_SPEED | SFXB_S_RUP;
                    }
                }
            }
        }
    }
    for(k = 0; k < D; ++k) sol[1 + k] += vhalf * n[k];
    for(k = 0; k < S; ++k) flux[k] = 0.;
    if(!sol[0]) return;
    double vsol = sol[1] * n[0] + sol[2] * n[1];
    double v2 = sol[1] * sol[1] + sol[2] * sol[2];
#if D == 3
    vsol += sol[3] * n[2];
    v2 += sol[3] * sol[3];
#endif
    flux[0] = sol[0] * vsol;
    flux[1] = sol[0] * sol[1] * vsol + sol[D + 1] * n[0];
    flux[2] = sol[0] * sol[2] * vsol + sol[D + 1] * n[1];
#if D == 3
    flux[3] = sol[0] * sol[3] * vsol + sol[D + 1] * n[2];
#endif
    double e = sol[D + 1] / (g - 1.) / sol[0] + 0.5 * v2;
    flux[D + 1] = sol[0] * e * vsol + sol[D + 1] * vsol;
    FN(hllc_deboost)(v, flux);
}

/* HLLCRiemannSolver::solve_for_flux (HLLCRiemannSolver.cpp:258-403) */
static int FN(hllc_flux)(const FN(solver) * s, double* WL, double* WR,
                         const double* n, const double* v, int reflective,
                         double* flux, int* code) {
    int k;
    double g = s->gamma;
    *code = SFXB_HLLC;
    if(!WL[0] && (reflective || !WR[0])) {
        for(k = 0; k < S; ++k) flux[k] = 0.;
        *code |= SFXB_VAC_BOTH;
        return SFXO_OK;
    }
#if D == 3
    double uL = WL[1] * n[0] + WL[2] * n[1] + WL[3] * n[2];
    double uR = WR[1] * n[0] + WR[2] * n[1] + WR[3] * n[2];
#else
    double uL = WL[1] * n[0] + WL[2] * n[1];
    double uR = WR[1] * n[0] + WR[2] * n[1];
#endif
    if(reflective) {
        for(k = 0; k < S; ++k) WR[k] = WL[k];
        uR = -uL;
    }
    /* HLLCRiemannSolver::get_soundspeed (:458-460) has no vacuum guard */
    double aL = sqrt(g * WL[D + 1] / WL[0]);
    double aR = sqrt(g * WR[D + 1] / WR[0]);
    int vc;
    if(!WL[0] || !WR[0]) {
        FN(hllc_vacuum_flux)(s, WL, WR, n, v, uL, uR, aL, aR, flux, &vc);
        *code |= vc;
        return SFXO_OK;
    }
    if(2. * aL / (g - 1.) + 2. * aR / (g - 1.) <= uR - uL) {
        FN(hllc_vacuum_flux)(s, WL, WR, n, v, uL, uR, aL, aR, flux, &vc);
        *code |= (vc & ~SFXB_VAC_MASK) | SFXB_VAC_SPEED;
        return SFXO_OK;
    }
    double rhobar = 0.5 * (WL[0] + WR[0]);
    double abar = 0.5 * (aL + aR);
    double pPVRS = 0.5 * (WL[D + 1] + WR[D + 1]) - 0.5 * (uR - uL) * rhobar * abar;
    double pstar = (0. < pPVRS) ? pPVRS : 0.; /* std::max(0., pPVRS) */
    double qL = 1.;
    if(pstar > WL[D + 1]) {
        qL = sqrt(1. + 0.5 * (g + 1.) / g * (pstar / WL[D + 1] - 1.));
    }
    double qR = 1.;
    if(pstar > WR[D + 1]) {
        qR = sqrt(1. + 0.5 * (g + 1.) / g * (pstar / WR[D + 1] - 1.));
    }
    double SL = uL - aL * qL;
    double SR = uR + aR * qR;
    double Sstar = (WR[D + 1] - WL[D + 1] + WL[0] * uL * (SL - uL) -
                    WR[0] * uR * (SR - uR)) /
                   (WL[0] * (SL - uL) - WR[0] * (SR - uR));
    for(k = 0; k < S; ++k) flux[k] = 0.;
    if(Sstar >= 0.) {
        flux[0] = WL[0] * uL;
        flux[1] = WL[0] * WL[1] * uL + WL[D + 1] * n[0];
        flux[2] = WL[0] * WL[2] * uL + WL[D + 1] * n[1];
        double v2 = WL[1] * WL[1] + WL[2] * WL[2];
#if D == 3
        flux[3] = WL[0] * WL[3] * uL + WL[D + 1] * n[2];
        v2 += WL[3] * WL[3];
#endif
        double eL = WL[D + 1] / (g - 1.) / WL[0] + 0.5 * v2;
        flux[D + 1] = WL[0] * eL * uL + WL[D + 1] * uL;
        if(SL < 0.) {
            double U[S];
            U[0] = 1.;
            U[1] = WL[1] + (Sstar - uL) * n[0];
            U[2] = WL[2] + (Sstar - uL) * n[1];
#if D == 3
            U[3] = WL[3] + (Sstar - uL) * n[2];
#endif
            U[D + 1] = eL + (Sstar - uL) * (Sstar + WL[D + 1] / (WL[0] * (SL - uL)));
            double fac = WL[0] * (SL - uL) / (SL - Sstar);
            for(k = 0; k < S; ++k) U[k] *= fac;
            flux[0] += SL * (U[0] - WL[0]);
            flux[1] += SL * (U[1] - WL[0] * WL[1]);
            flux[2] += SL * (U[2] - WL[0] * WL[2]);
#if D == 3
            flux[3] += SL * (U[3] - WL[0] * WL[3]);
#endif
            flux[D + 1] += SL * (U[D + 1] - WL[0] * eL);
            *code |= SFXB_HLLC_LSTAR;
        } else {
            *code |= SFXB_HLLC_L;
        }
    } else {
        flux[0] = WR[0] * uR;
        flux[1] = WR[0] * WR[1] * uR + WR[D + 1] * n[0];
        flux[2] = WR[0] * WR[2] * uR + WR[D + 1] * n[1];
        double v2 = WR[1] * WR[1] + WR[2] * WR[2];
#if D == 3
        flux[3] = WR[0] * WR[3] * uR + WR[D + 1] * n[2];
        v2 += WR[3] * WR[3];
#endif
        double eR = WR[D + 1] / (g - 1.) / WR[0] + 0.5 * v2;
        flux[D + 1] = WR[0] * eR * uR + WR[D + 1] * uR;
        if(SR > 0.) {
            double U[S];
            U[0] = 1.;
            U[1] = WR[1] + (Sstar - uR) * n[0];
            U[2] = WR[2] + (Sstar - uR) * n[1];
#if D == 3
            U[3] = WR[3] + (Sstar - uR) * n[2];
#endif
            U[D + 1] = eR + (Sstar - uR) * (Sstar + WR[D + 1] / (WR[0] * (SR - uR)));
            double fac = WR[0] * (SR - uR) / (SR - Sstar);
            for(k = 0; k < S; ++k) U[k] *= fac;
            flux[0] += SR * (U[0] - WR[0]);
            flux[1] += SR * (U[1] - WR[0] * WR[1]);
            flux[2] += SR * (U[2] - WR[0] * WR[2]);
#if D == 3
            flux[3] += SR * (U[3] - WR[0] * WR[3]);
#endif
            flux[D + 1] += SR * (U[D + 1] - WR[0] * eR);
            *code |= SFXB_HLLC_RSTAR;
        } else {
            *code |= SFXB_HLLC_R;
        }
    }
    FN(hllc_deboost)(v, flux);
    return SFXO_OK;
}

/* ======================== per-face flux pipeline ======================== */

/* VorFace::calculate_flux (src/VorFace.cpp:670-1024) for a static mesh in
 * which every cell is active with the same global dt (so timefac = 1).
 * Writes the limited dQL (the left cell receives +dQL, a real right cell
 * receives -dQL, bit-identical to the reference's dQR). */
static int FN(face_flux)(const FN(solver) * s, const sfxo_mesh* m, int f,
                         double dt, const double* Wall, const double* Qall,
                         const double* grad, double* dQL, int* code) {
    int k;
    *code = 0;
    for(k = 0; k < S; ++k) dQL[k] = 0.;
    double A = m->face_area[f];
    if(!A) {
        *code = SFXB_SKIPPED;
        return SFXO_OK;
    }
    const int iL = m->face_left[f];
    const int kind = m->face_kind[f];
    const int has_right = kind != 2;
    const int iR = has_right ? m->face_right[f] : -1;
    const double* v = m->face_velocity + (size_t)f * D;
    const double* mid = m->face_midpoint + (size_t)f * D;
    const double* xL = m->cell_pos + (size_t)iL * D;
    const double* xRimg = m->face_right_pos + (size_t)f * D;
    double WL[S], WR[S], WLrec[S], WRrec[S], Wt[S], dW[S], d[D];
    for(k = 0; k < S; ++k) {
        WL[k] = Wall[(size_t)iL * S + k];
        WR[k] = has_right ? Wall[(size_t)iR * S + k] : 0.;
        WRrec[k] = 0.;
    }
    for(k = 0; k < D; ++k) {
        WL[1 + k] -= v[k];
        WR[1 + k] -= v[k];
    }
    const double(*gL)[S] = (const double(*)[S])(grad + (size_t)iL * D * S);
    const double* cenL = m->cell_centroid + (size_t)iL * D;
    if(has_right) {
        const double(*gR)[S] = (const double(*)[S])(grad + (size_t)iR * D * S);
        const double* cenR = m->cell_centroid + (size_t)iR * D;
        const double* xR = m->cell_pos + (size_t)iR * D;
        for(k = 0; k < S; ++k) Wt[k] = WR[k];
        for(int n = D; n--;) {
            double correction = xR[n] - xRimg[n];
            d[n] = mid[n] - cenR[n] + correction;
        }
        double dW0[S];
        FN(time_derivative)(s, Wt, gR, dW0);
        for(k = 0; k < S; ++k) dW[k] = 0.5 * dt * dW0[k];
        FN(reconstruct)(Wt, gR, d);
        double cd[D];
        for(k = 0; k < D; ++k) cd[k] = cenL[k] - cenR[k];
#if D == 3
        double r = sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
#else
        double r = sqrt(cd[0] * cd[0] + cd[1] * cd[1]);
#endif
        FN(limit)(Wt, WR, WL, d, r);
        if(Wt[0] < 0. || Wt[D + 1] < 0.) {
            for(k = 0; k < S; ++k) Wt[k] = WR[k];
        }
        for(int mm = S; mm--;) Wt[mm] += dW[mm];
        if(Wt[0] < 0. || Wt[D + 1] < 0.) {
            for(k = 0; k < S; ++k) Wt[k] -= dW[k];
        }
        for(k = 0; k < S; ++k) WRrec[k] = Wt[k];
    }
    /* left state */
    for(k = 0; k < S; ++k) Wt[k] = WL[k];
    for(int n = D; n--;) {
        double correction = xL[n] - xL[n];
        d[n] = mid[n] - cenL[n] + correction;
    }
    {
        double dW0[S];
        FN(time_derivative)(s, Wt, gL, dW0);
        for(k = 0; k < S; ++k) dW[k] = 0.5 * dt * dW0[k];
    }
    FN(reconstruct)(Wt, gL, d);
    if(has_right) {
        const double* cenR = m->cell_centroid + (size_t)iR * D;
        double cd[D];
        for(k = 0; k < D; ++k) cd[k] = cenL[k] - cenR[k];
#if D == 3
        double r = sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
#else
        double r = sqrt(cd[0] * cd[0] + cd[1] * cd[1]);
#endif
        FN(limit)(Wt, WL, WR, d, r);
    }
    if(Wt[0] < 0. || Wt[D + 1] < 0.) {
        for(k = 0; k < S; ++k) Wt[k] = WL[k];
    }
    for(int mm = S; mm--;) Wt[mm] += dW[mm];
    if(Wt[0] < 0. || Wt[D + 1] < 0.) {
        for(k = 0; k < S; ++k) Wt[k] -= dW[k];
    }
    for(k = 0; k < S; ++k) WLrec[k] = Wt[k];
    if(WL[0]) {
        for(k = 0; k < S; ++k) WL[k] = WLrec[k];
    }
    if(WR[0]) {
        for(k = 0; k < S; ++k) WR[k] = WRrec[k];
    }
    /* VorFace::get_normal (src/VorFace.cpp:553-571) */
    double nrm[D];
    {
        double dd[D + 1];
        for(k = 0; k < D; ++k) dd[k] = xL[k] - xRimg[k];
#if D == 3
        dd[3] = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
#else
        dd[2] = sqrt(dd[0] * dd[0] + dd[1] * dd[1]);
#endif
        for(k = 0; k < D; ++k) nrm[k] = -dd[k] / dd[D];
    }
    double flux[S];
    int rc;
    if(s->kind == 0) {
        rc = FN(exact_flux)(s, WL, WR, nrm, v, !has_right, flux, code);
    } else {
        rc = FN(hllc_flux)(s, WL, WR, nrm, v, !has_right, flux, code);
    }
    if(rc) return rc;
    double dQR[S];
    for(k = 0; k < S; ++k) {
        dQL[k] = dt * A * flux[k];
        dQR[k] = -dt * A * flux[k];
    }
    /* over-flux limiter, src/VorFace.cpp:837-866 (timefac == 1) */
    double timefac = 1.;
    if(has_right) {
        double dtmax = dt;
        dtmax = (dtmax < dt) ? dt : dtmax;
        timefac = dt / dtmax;
    }
    double areafac = A / m->cell_total_area[iL];
    areafac *= timefac;
    double QLm = Qall[(size_t)iL * S];
    if(dQL[0] > areafac * QLm) {
        double corfac = fabs(areafac * QLm / dQL[0]);
        for(k = 0; k < S; ++k) dQL[k] *= corfac;
        for(k = 0; k < S; ++k) dQR[k] = -1. * dQL[k];
        *code |= SFXB_LIMIT_L;
    }
    if(has_right) {
        double areafacR = A / m->cell_total_area[iR];
        areafacR *= timefac;
        double QRm = Qall[(size_t)iR * S];
        if(dQR[0] > areafacR * QRm) {
            double corfac = fabs(areafacR * QRm / dQR[0]);
            for(k = 0; k < S; ++k) dQR[k] *= corfac;
            for(k = 0; k < S; ++k) dQL[k] = -1. * dQR[k];
            *code |= SFXB_LIMIT_R;
        }
    }
    if(flux[0] != flux[0]) return SFXO_ERR_NAN_FLUX;
    return SFXO_OK;
}

/* conserved -> primitive, ExactRiemannSolver.cpp:716-766 (use_energy) and
 * HLLCRiemannSolver.cpp:495-535: identical arithmetic on the hydro fields.
 * May rewrite Q[D+1] (pressure floor). */
static void FN(get_W)(const FN(solver) * s, double V, double* Q, double* W) {
    int k;
    double g = s->gamma;
    for(k = 0; k < S; ++k) W[k] = 0.;
    if(!Q[0]) return;
    W[0] = Q[0] / V;
    W[1] = Q[1] / Q[0];
    W[2] = Q[2] / Q[0];
#if D == 3
    W[3] = Q[3] / Q[0];
    W[4] = (g - 1.) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / Q[0]) / V;
#else
    W[3] = (g - 1.) * (Q[3] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) / Q[0]) / V;
#endif
    if(W[D + 1] < 1.e-30) {
        W[D + 1] = 1.e-30;
#if D == 3
        Q[4] = 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / Q[0] +
               W[4] * V / (g - 1.);
#else
        Q[3] = 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) / Q[0] + W[3] * V / (g - 1.);
#endif
    }
    if(W[0] < 1.e-30) {
        for(k = 0; k < S; ++k) W[k] = 0.;
    }
}

/* primitive -> conserved: ExactRiemannSolver.cpp:776-804 or
 * HLLCRiemannSolver.cpp:471-483 (different energy expression order) */
static int FN(get_Q)(const FN(solver) * s, double V, const double* W, double* Q) {
    double g = s->gamma;
    Q[0] = W[0] * V;
    Q[1] = Q[0] * W[1];
    Q[2] = Q[0] * W[2];
#if D == 3
    Q[3] = Q[0] * W[3];
#endif
    if(s->kind == 0) {
#if D == 3
        Q[4] = (0.5 * W[0] * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) +
                W[4] / (g - 1.)) * V;
#else
        Q[3] = (0.5 * W[0] * (W[1] * W[1] + W[2] * W[2]) + W[3] / (g - 1.)) * V;
#endif
        if(Q[0] < 0. || Q[D + 1] < 0.) return SFXO_ERR_NEG_STATE;
    } else {
        double v2 = W[1] * W[1] + W[2] * W[2];
#if D == 3
        v2 += W[3] * W[3];
#endif
        Q[D + 1] = V * W[D + 1] / (g - 1.) + 0.5 * Q[0] * v2;
    }
    return SFXO_OK;
}

static int FN(init_Q)(const sfxo_mesh* m, const sfxo_params* p, const double* W,
                      double* Q) {
    FN(solver) s;
    FN(solver_init)(&s, p);
    for(int i = 0; i < m->ncell; ++i) {
        int rc = FN(get_Q)(&s, m->cell_volume[i], W + (size_t)i * S, Q + (size_t)i * S);
        if(rc) return rc;
    }
    return SFXO_OK;
}

static int FN(gradients)(const sfxo_mesh* m, const double* W, double* grad) {
    for(int i = 0; i < m->ncell; ++i) {
        double g[D][S];
        FN(cell_gradient)(m, W, i, g);
        memcpy(grad + (size_t)i * D * S, g, sizeof g);
    }
    return SFXO_OK;
}

static int FN(face_fluxes)(const sfxo_mesh* m, const sfxo_params* p, double dt,
                           const double* W, const double* Q, const double* grad,
                           double* dQL, int* code, int* bad_face) {
    FN(solver) s;
    FN(solver_init)(&s, p);
    for(int f = 0; f < m->nface; ++f) {
        int c = 0;
        int rc = FN(face_flux)(&s, m, f, dt, W, Q, grad, dQL + (size_t)f * S, &c);
        if(code) code[f] = c;
        if(rc) {
            if(bad_face) *bad_face = f;
            return rc;
        }
    }
    return SFXO_OK;
}

/* scatter in face order (src/VorTessManager.cpp:205-209 with the rules of
 * src/VorFace.cpp:913-955), GasParticle::update_Q (GasParticle.cpp:617-624)
 * and get_W (src/Simulation.cpp:791-836) */
static int FN(apply)(const sfxo_mesh* m, const sfxo_params* p, const double* dQL,
                     double* Q, double* W, double* dQcell, int* bad_cell) {
    FN(solver) s;
    FN(solver_init)(&s, p);
    int k;
    size_t ncs = (size_t)m->ncell * S;
    for(size_t t = 0; t < ncs; ++t) dQcell[t] = 0.;
    for(int f = 0; f < m->nface; ++f) {
        if(!m->face_area[f]) continue;
        const double* q = dQL + (size_t)f * S;
        double* a = dQcell + (size_t)m->face_left[f] * S;
        for(k = 0; k < S; ++k) a[k] += q[k];
        if(m->face_kind[f] == 0) {
            double* b = dQcell + (size_t)m->face_right[f] * S;
            for(k = 0; k < S; ++k) b[k] += -1. * q[k];
        }
    }
    for(int i = 0; i < m->ncell; ++i) {
        double* Qi = Q + (size_t)i * S;
        for(k = 0; k < S; ++k) Qi[k] -= dQcell[(size_t)i * S + k];
        if(Qi[0] < 0. || Qi[D + 1] < 0.) {
            if(bad_cell) *bad_cell = i;
            return SFXO_ERR_NEG_STATE;
        }
    }
    for(int i = 0; i < m->ncell; ++i) {
        FN(get_W)(&s, m->cell_volume[i], Q + (size_t)i * S, W + (size_t)i * S);
    }
    return SFXO_OK;
}

static int FN(riemann)(const sfxo_params* p, int n, const double* WLa,
                       const double* WRa, const double* normal, int reflective,
                       double* half, double* flux, int* code) {
    FN(solver) s;
    FN(solver_init)(&s, p);
    double zero[D];
    for(int k = 0; k < D; ++k) zero[k] = 0.;
    int worst = SFXO_OK;
    for(int i = 0; i < n; ++i) {
        double L[S], R[S];
        int c = 0, rc;
        if(p->solver == 0) {
            memcpy(L, WLa + (size_t)i * S, sizeof L);
            memcpy(R, WRa + (size_t)i * S, sizeof R);
            rc = FN(exact_solve)(&s, L, R, normal + (size_t)i * D, reflective,
                                 half + (size_t)i * S, &c);
            if(rc && !worst) worst = rc;
        }
        memcpy(L, WLa + (size_t)i * S, sizeof L);
        memcpy(R, WRa + (size_t)i * S, sizeof R);
        if(p->solver == 0)
            rc = FN(exact_flux)(&s, L, R, normal + (size_t)i * D, zero, reflective,
                                flux + (size_t)i * S, &c);
        else
            rc = FN(hllc_flux)(&s, L, R, normal + (size_t)i * D, zero, reflective,
                               flux + (size_t)i * S, &c);
        if(code) code[i] = rc ? -rc : c;
        if(rc && !worst) worst = rc;
    }
    return worst;
}


/* ---- moving generators (the reference built without -DSTATIC) ----
 * Generator velocities: VorCell::get_velocity (src/VorCell.cpp:966-1008)
 * from the state W and the stored sound speed sqrt(gamma p / rho), then the
 * reflective-box check of src/Simulation.cpp:366-398 (a generator that would
 * leave the unit box, RectangularBox::inside, src/RectangularBox.cpp:91-99,
 * loses the fluid velocity).  Face velocities: VorFace::set_v
 * (src/VorFace.cpp:586-660).  vgen [ncell][D], vface [nface][D]. */
static void FN(move_velocities)(const sfxo_mesh* m, const sfxo_params* p, double dt,
                                int periodic, const double* Wall, double* vgen,
                                double* vface) {
    for(int i = 0; i < m->ncell; ++i) {
        const double* W = Wall + (size_t)i * S;
        const double* x = m->cell_pos + (size_t)i * D;
        double vel[D];
        for(int l = 0; l < D; ++l) vel[l] = 0.;
        if(W[0]) {
            double d[D];
            for(int l = 0; l < D; ++l) d[l] = m->cell_centroid[(size_t)i * D + l] - x[l];
            double Ri = m->cell_volume[i];
            double csnd = sqrt(p->gamma * W[D + 1] / W[0]);
#if D == 3
            Ri = sfx_cbrt(3. * Ri / 4. / SFXO_PI);
            double dn = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
#else
            Ri = sqrt(Ri / SFXO_PI);
            double dn = sqrt(d[0] * d[0] + d[1] * d[1]);
#endif
            double check = 4. * dn / Ri;
            if(check > 0.9) {
                if(check < 1.1) {
                    double fac = csnd / dn * (dn - 0.9 * 0.25 * Ri) / (0.2 * 0.25 * Ri);
                    for(int l = 0; l < D; ++l) vel[l] = fac * d[l];
                } else {
                    double fac = csnd / dn;
                    for(int l = 0; l < D; ++l) vel[l] = fac * d[l];
                }
            }
        }
        double v[D];
        for(int l = 0; l < D; ++l) v[l] = W[1 + l] + vel[l];
        if(W[0] < 1.e-10) {
            double fac = W[0] * 1.e10;
            for(int l = 0; l < D; ++l) v[l] = fac * v[l];
        }
        if(!periodic) {
            int inside = 1;
            for(int l = 0; l < D; ++l)
                if(fabs(0.5 - (x[l] + dt * v[l])) > 0.5) inside = 0;
            if(!inside)
                for(int l = 0; l < D; ++l) v[l] -= W[1 + l];
        }
        for(int l = 0; l < D; ++l) vgen[(size_t)i * D + l] = v[l];
    }
    for(int f = 0; f < m->nface; ++f) {
        const int L = m->face_left[f];
        const double* xl = m->cell_pos + (size_t)L * D;
        const double* xr = m->face_right_pos + (size_t)f * D;
        const double* mid = m->face_midpoint + (size_t)f * D;
        const double* vl = vgen + (size_t)L * D;
        double vr[D];
        double* out = vface + (size_t)f * D;
        if(m->face_kind[f] != 2) {
            for(int l = 0; l < D; ++l) vr[l] = vgen[(size_t)m->face_right[f] * D + l];
        } else {
#if D == 3
            for(int l = 0; l < D; ++l) out[l] = 0.;
            continue;
#else
            double Wd[4] = {0., vl[0], vl[1], 0.};
            FN(mirror_state)(Wd, xl, xr);
            vr[0] = Wd[1];
            vr[1] = Wd[2];
#endif
        }
        double rRL[D + 1];
        for(int l = 0; l < D; ++l) rRL[l] = xr[l] - xl[l];
#if D == 3
        rRL[3] = rRL[0] * rRL[0] + rRL[1] * rRL[1] + rRL[2] * rRL[2];
#else
        rRL[2] = rRL[0] * rRL[0] + rRL[1] * rRL[1];
#endif
        double fac = (vl[0] - vr[0]) * (mid[0] - 0.5 * (xl[0] + xr[0]));
        for(int l = 1; l < D; ++l) fac += (vl[l] - vr[l]) * (mid[l] - 0.5 * (xl[l] + xr[l]));
        fac /= rRL[D];
        for(int l = 0; l < D; ++l) out[l] = 0.5 * (vl[l] + vr[l]) + fac * rRL[l];
    }
}

/* ---- local time steps: TimeLine::calculate_timestep (src/TimeLine.cpp:
 * 233-317) for the gas cells whose step ends at t_next, on the timeline of
 * 2^60 ticks spanning t_total: h (VorCell::get_h, src/VorCell.cpp:948-956),
 * the CFL step h / (|v - v_gen| + c), S = cfl x that; max_step when that is
 * shorter than S, otherwise the largest power-of-two number of ticks not
 * longer than S, halved until 2^60 - end is a multiple of it, clamped to
 * [min_step, max_step]; the cell's next step is [end, end + step).  *smin
 * receives the smallest new step (max_step when no cell ends at t_next). */
static int FN(timestep_bins)(const sfxo_mesh* m, const sfxo_params* p, const double* Wall,
                             const double* vgen, uint64_t* start, uint64_t* end,
                             uint64_t t_next, double t_total, double cfl, uint64_t max_step,
                             uint64_t min_step, uint64_t* smin) {
    const uint64_t ticks = (uint64_t)1 << 60;
    uint64_t best = max_step;
    for(int i = 0; i < m->ncell; ++i) {
        if(end[i] != t_next) continue;
        const double* W = Wall + (size_t)i * S;
        const double V = m->cell_volume[i];
#if D == 3
        const double h = sfx_cbrt(V * 3. / 4. / SFXO_PI);
#else
        const double h = sqrt(V / SFXO_PI);
#endif
        double v[D];
        for(int l = 0; l < D; ++l) v[l] = W[1 + l] - vgen[(size_t)i * D + l];
#if D == 3
        const double vi = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
#else
        const double vi = sqrt(v[0] * v[0] + v[1] * v[1]);
#endif
        const double ci = W[0] ? sqrt(p->gamma * W[D + 1] / W[0]) : 0.;
        const double Sreal = cfl * (h / (vi + ci));
        uint64_t S2;
        if(t_total * ((double)max_step / (double)ticks) < Sreal) {
            S2 = max_step;
        } else {
            S2 = ticks;
            while(S2 && t_total * ((double)S2 / (double)ticks) > Sreal) S2 >>= 1;
            if(!S2) return 15; /* SFX_ERR_TIMESTEP */
            while((ticks - end[i]) % S2) S2 >>= 1;
            if(S2 < min_step) S2 = min_step;
            if(S2 > max_step) S2 = max_step;
        }
        start[i] = end[i];
        end[i] = end[i] + S2;
        if(S2 < best) best = S2;
    }
    *smin = best;
    return SFXO_OK;
}

#undef S
