/*
 * sfx_pow: a deterministic double-precision power function for host (C/C++)
 * and device (CUDA) code.
 *
 * Why: the exact Riemann solver of Shadowfax (src/riemann/ExactRiemannSolver.cpp
 * :556-631 fb/fprimeb, :644-673 guess_p, :178-265 sampling) calls pow() with
 * exponents fixed by gamma.  glibc's pow and CUDA's pow are different
 * implementations and can differ in the last bit, which can flip an iteration
 * count or a wave-pattern branch.  Both the GPU flux pass and the CPU oracle
 * therefore call this one routine, which uses only IEEE-754 basic operations
 * (+ - * / and fused multiply-add), each correctly rounded on both sides, so
 * the two produce bit-identical results.
 *
 * Method (textbook double-double evaluation, see J.-M. Muller et al.,
 * "Handbook of Floating-Point Arithmetic", ch. on elementary functions, and
 * T. J. Dekker, "A floating-point technique for extending the available
 * precision", 1971, for the error-free transformations):
 *   x = 2^e * m,  m in [sqrt(1/2), sqrt(2))
 *   ln m = 2 atanh(s),  s = (m - 1) / (m + 1),  series in s^2 (|s| < 0.172)
 *   ln x = e ln2 + ln m                             (double-double)
 *   t    = y ln x                                   (double-double)
 *   exp t = 2^k exp(r),  r = t - k ln2,  exp(r) = (exp(r / 256))^256
 *           with a Taylor series for exp(r/256) - 1 and eight exact-form
 *           squarings  e1 <- e1 (2 + e1)            (double-double)
 * The final sum 1 + e1 is rounded once.  The relative error before that
 * rounding is below 2^-90 for |t| < 710, so the result is the correctly
 * rounded power except when the exact value lies within 2^-90 of a rounding
 * boundary.  Special values follow C99 Annex F (pow).  Results that fall in
 * the subnormal range are rounded twice (documented limitation; the flux pass
 * never produces them for physical states).
 *
 * Host builds must not contract a*b+c into an FMA (-ffp-contract=off), and
 * CUDA builds must use -fmad=false for the same reason.
 */
#ifndef SFX_POW_H
#define SFX_POW_H

#if defined(__CUDACC__)
#define SFX_HD __host__ __device__ __forceinline__
#else
#define SFX_HD static inline
#endif

#if !defined(__CUDACC__)
#include <math.h>
#include <stdint.h>
#include <string.h>
#else
#include <stdint.h>
#endif

SFX_HD uint64_t sfx_d2u(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, sizeof u);
    return u;
#endif
}

SFX_HD double sfx_u2d(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, sizeof x);
    return x;
#endif
}

SFX_HD double sfx_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

/* double-double helpers: value = hi + lo, |lo| <= ulp(hi)/2 */
SFX_HD void sfx_two_sum(double a, double b, double* s, double* e) {
    double ss = a + b;
    double bb = ss - a;
    *e = (a - (ss - bb)) + (b - bb);
    *s = ss;
}

SFX_HD void sfx_fast_two_sum(double a, double b, double* s, double* e) {
    double ss = a + b;
    *e = b - (ss - a);
    *s = ss;
}

/* (ah, al) * (bh, bl) */
SFX_HD void sfx_dd_mul(double ah, double al, double bh, double bl, double* rh,
                       double* rl) {
    double p = ah * bh;
    double e = sfx_fma(ah, bh, -p);
    e = e + (ah * bl + al * bh);
    sfx_fast_two_sum(p, e, rh, rl);
}

/* (ah, al) + (bh, bl) */
SFX_HD void sfx_dd_add(double ah, double al, double bh, double bl, double* rh,
                       double* rl) {
    double s, e;
    sfx_two_sum(ah, bh, &s, &e);
    e = e + (al + bl);
    sfx_fast_two_sum(s, e, rh, rl);
}

/* ln(x) as double-double for finite x > 0 */
SFX_HD void sfx_log_dd(double x, double* rh, double* rl) {
    int e = 0;
    uint64_t u = sfx_d2u(x);
    if((u >> 52) == 0) { /* subnormal: scale by 2^54 */
        x = x * 0x1p54;
        u = sfx_d2u(x);
        e = -54;
    }
    e += (int)(u >> 52) - 1023;
    /* mantissa in [1, 2) */
    double m = sfx_u2d((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    if(m > 0x1.6a09e667f3bcdp+0) { /* > sqrt(2): use m/2 in [0.707, 1) */
        m = m * 0.5;
        e += 1;
    }
    /* s = (m - 1) / (m + 1) in double-double; m - 1 is exact */
    double f = m - 1.0;
    double gh, gl;
    sfx_two_sum(m, 1.0, &gh, &gl);
    double sh = f / gh;
    double rem = sfx_fma(-sh, gh, f);
    rem = rem - sh * gl;
    double sl = rem / gh;
    sfx_fast_two_sum(sh, sl, &sh, &sl);
    /* z = s^2 */
    double zh, zl;
    sfx_dd_mul(sh, sl, sh, sl, &zh, &zl);
    /* tail: sum_{k>=4} z^(k-4) / (2k+1), k = 4..18, in double */
    double z = zh;
    double t = 1.0 / 37.0;
    t = t * z + 1.0 / 35.0;
    t = t * z + 1.0 / 33.0;
    t = t * z + 1.0 / 31.0;
    t = t * z + 1.0 / 29.0;
    t = t * z + 1.0 / 27.0;
    t = t * z + 1.0 / 25.0;
    t = t * z + 1.0 / 23.0;
    t = t * z + 1.0 / 21.0;
    t = t * z + 1.0 / 19.0;
    t = t * z + 1.0 / 17.0;
    t = t * z + 1.0 / 15.0;
    t = t * z + 1.0 / 13.0;
    t = t * z + 1.0 / 11.0;
    t = t * z + 1.0 / 9.0;
    /* P = 1/3 + z(1/5 + z(1/7 + z t)), leading levels in double-double */
    double ph, pl;
    sfx_dd_mul(zh, zl, t, 0.0, &ph, &pl);
    sfx_dd_add(0x1.2492492492492p-3, 0x1.2492492492492p-57, ph, pl, &ph, &pl);
    sfx_dd_mul(zh, zl, ph, pl, &ph, &pl);
    sfx_dd_add(0x1.999999999999ap-3, -0x1.999999999999ap-57, ph, pl, &ph, &pl);
    sfx_dd_mul(zh, zl, ph, pl, &ph, &pl);
    sfx_dd_add(0x1.5555555555555p-2, 0x1.5555555555555p-56, ph, pl, &ph, &pl);
    /* ln m = 2 s (1 + z P) = 2s + 2s z P */
    double qh, ql;
    sfx_dd_mul(zh, zl, ph, pl, &qh, &ql);
    sfx_dd_mul(sh, sl, qh, ql, &qh, &ql);
    double lh, ll;
    sfx_dd_add(sh, sl, qh, ql, &lh, &ll);
    lh = lh * 2.0;
    ll = ll * 2.0;
    /* + e ln2; e*ln2_hi is exact (ln2_hi has 42 significant bits) */
    double de = (double)e;
    double ah = de * 0x1.62e42fefa3800p-1;
    double mh = de * 0x1.ef35793c76730p-45;
    double me = sfx_fma(de, 0x1.ef35793c76730p-45, -mh);
    me = me + de * 0x1.f97b57a079a19p-103;
    double bh, bl;
    sfx_two_sum(ah, mh, &bh, &bl);
    bl = bl + me;
    sfx_fast_two_sum(bh, bl, &bh, &bl);
    sfx_dd_add(bh, bl, lh, ll, rh, rl);
}

/* exp(th + tl) for |th| <= 709 (caller handles overflow/underflow) */
SFX_HD double sfx_exp_dd(double th, double tl) {
    /* k = nearest integer to t / ln2 (round-half-even via the 1.5*2^52 trick,
     * identical on host and device) */
    double kd = th * 0x1.71547652b82fep+0;
    kd = (kd + 0x1.8p52) - 0x1.8p52;
    int k = (int)kd;
    /* r = t - k ln2 in double-double */
    double a = th - kd * 0x1.62e42fefa3800p-1; /* exact: Sterbenz-like */
    double mh = kd * 0x1.ef35793c76730p-45;
    double me = sfx_fma(kd, 0x1.ef35793c76730p-45, -mh);
    me = me + kd * 0x1.f97b57a079a19p-103;
    double rh, rl;
    sfx_two_sum(a, -mh, &rh, &rl);
    rl = rl + (tl - me);
    sfx_fast_two_sum(rh, rl, &rh, &rl);
    /* u = r / 256, exact scaling */
    double uh = rh * 0x1p-8, ul = rl * 0x1p-8;
    /* e1 = exp(u) - 1 = u + u^2 (1/2 + u (1/6 + u q)), q in double */
    double q = 1.0 / 40320.0;
    q = q * uh + 1.0 / 5040.0;
    q = q * uh + 1.0 / 720.0;
    q = q * uh + 1.0 / 120.0;
    q = q * uh + 1.0 / 24.0;
    double ph, pl;
    sfx_dd_mul(uh, ul, q, 0.0, &ph, &pl);
    sfx_dd_add(0x1.5555555555555p-3, 0x1.5555555555555p-57, ph, pl, &ph, &pl);
    sfx_dd_mul(uh, ul, ph, pl, &ph, &pl);
    sfx_dd_add(0.5, 0.0, ph, pl, &ph, &pl);
    double u2h, u2l;
    sfx_dd_mul(uh, ul, uh, ul, &u2h, &u2l);
    sfx_dd_mul(u2h, u2l, ph, pl, &ph, &pl);
    double eh, el;
    sfx_dd_add(uh, ul, ph, pl, &eh, &el);
    /* (1 + e1)^256 - 1 by eight squarings e1 <- e1 (2 + e1) */
    for(int i = 0; i < 8; ++i) {
        double sh2, sl2;
        sfx_dd_add(2.0, 0.0, eh, el, &sh2, &sl2);
        sfx_dd_mul(eh, el, sh2, sl2, &eh, &el);
    }
    /* 1 + e1, rounded once */
    double s, e;
    sfx_two_sum(1.0, eh, &s, &e);
    e = e + el;
    double res = s + e;
    /* scale by 2^k; split so that intermediate exponents stay in range */
    if(k > 1000) {
        res = res * 0x1p1000;
        k -= 1000;
    } else if(k < -1000) {
        res = res * 0x1p-1000;
        k += 1000;
    }
    return res * sfx_u2d((uint64_t)(k + 1023) << 52);
}

SFX_HD int sfx_is_integer(double y) {
    /* |y| >= 2^52 is always an integer */
    double ay = y < 0 ? -y : y;
    if(ay >= 0x1p52) return 1;
    double r = (ay + 0x1p52) - 0x1p52;
    return r == ay;
}

SFX_HD int sfx_is_odd_integer(double y) {
    double ay = y < 0 ? -y : y;
    if(ay >= 0x1p53) return 0;
    if(!sfx_is_integer(ay)) return 0;
    double h = ay * 0.5;
    return !sfx_is_integer(h);
}

/* pow(x, y) with C99 Annex F special cases */
SFX_HD double sfx_pow(double x, double y) {
    const double inf = sfx_u2d(0x7ff0000000000000ull);
    const double nan = sfx_u2d(0x7ff8000000000000ull);
    if(y == 0.0) return 1.0;
    if(x == 1.0) return 1.0;
    if(x != x || y != y) return nan;
    double ax = x < 0 ? -x : x;
    double ay = y < 0 ? -y : y;
    if(ay == inf) {
        if(ax == 1.0) return 1.0;
        if((ax < 1.0) == (y > 0)) return 0.0;
        return inf;
    }
    int negate = 0;
    if(x < 0.0 || (x == 0.0 && (sfx_d2u(x) >> 63))) {
        /* negative base (or -0): only integer exponents give real results */
        if(x != 0.0 && ax != inf && !sfx_is_integer(y)) return nan;
        negate = sfx_is_odd_integer(y);
    }
    if(ax == 0.0) {
        double r = y < 0 ? inf : 0.0;
        return negate ? -r : r;
    }
    if(ax == inf) {
        double r = y < 0 ? 0.0 : inf;
        return negate ? -r : r;
    }
    double lh, ll;
    sfx_log_dd(ax, &lh, &ll);
    double th = y * lh;
    double tl = sfx_fma(y, lh, -th) + y * ll;
    double s, e;
    sfx_fast_two_sum(th, tl, &s, &e);
    double r;
    if(s > 709.8) {
        r = inf;
    } else if(s < -745.2) {
        r = 0.0;
    } else {
        r = sfx_exp_dd(s, e);
    }
    return negate ? -r : r;
}

/*
 * sfx_pow_fast: x^y in plain double arithmetic, for the split pass's exact
 * solver, whose p* iteration needs about 1e-14 and no correct rounding.  The
 * method of sfx_pow without the double-double parts:
 *   x = 2^e m, m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s), s = (m-1)/(m+1),
 *   by the odd series s (1 + s^2/3 + ... + s^20/21)   (|s| < 0.1716);
 *   t = y log2 x = y (e + ln m / ln 2);
 *   2^t = 2^n exp(f ln 2), n the nearest integer to t, |f| <= 1/2, with the
 *   Taylor series of exp to degree 13 (remainder below 1e-17).
 * Relative error a few ulp, growing with |t| (about 2|t| ulp from the rounding
 * of t).  Arguments outside x > 0 normal, |t| < 1000 go to SFX_POW_FAST_RARE
 * (sfx_pow unless the includer names an out-of-line wrapper of it).
 */
#ifndef SFX_POW_FAST_RARE
#define SFX_POW_FAST_RARE sfx_pow
#endif
SFX_HD double sfx_pow_fast(double x, double y) {
    const uint64_t u = sfx_d2u(x);
    const uint64_t ex = u >> 52; /* includes the sign bit */
    if(ex == 0 || ex >= 0x7ff || y != y) return SFX_POW_FAST_RARE(x, y);
    int e = (int)ex - 1023;
    double m = sfx_u2d((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    if(m > 0x1.6a09e667f3bcdp+0) {
        m = m * 0.5;
        e += 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double z = s * s;
    double p = 1.0 / 21.0;
    p = sfx_fma(p, z, 1.0 / 19.0);
    p = sfx_fma(p, z, 1.0 / 17.0);
    p = sfx_fma(p, z, 1.0 / 15.0);
    p = sfx_fma(p, z, 1.0 / 13.0);
    p = sfx_fma(p, z, 1.0 / 11.0);
    p = sfx_fma(p, z, 1.0 / 9.0);
    p = sfx_fma(p, z, 1.0 / 7.0);
    p = sfx_fma(p, z, 1.0 / 5.0);
    p = sfx_fma(p, z, 1.0 / 3.0);
    p = sfx_fma(p, z, 1.0);
    const double lnm = 2.0 * s * p;
    /* log2 e and ln 2 rounded to double */
    const double t = y * sfx_fma(lnm, 1.4426950408889634, (double)e);
    if(!(t > -1000.0 && t < 1000.0)) return SFX_POW_FAST_RARE(x, y);
    const double n = rint(t);
    const double f = (t - n) * 0.6931471805599453;
    double q = 1.0 / 6227020800.0; /* 1/13! */
    q = sfx_fma(q, f, 1.0 / 479001600.0);
    q = sfx_fma(q, f, 1.0 / 39916800.0);
    q = sfx_fma(q, f, 1.0 / 3628800.0);
    q = sfx_fma(q, f, 1.0 / 362880.0);
    q = sfx_fma(q, f, 1.0 / 40320.0);
    q = sfx_fma(q, f, 1.0 / 5040.0);
    q = sfx_fma(q, f, 1.0 / 720.0);
    q = sfx_fma(q, f, 1.0 / 120.0);
    q = sfx_fma(q, f, 1.0 / 24.0);
    q = sfx_fma(q, f, 1.0 / 6.0);
    q = sfx_fma(q, f, 0.5);
    q = sfx_fma(q, f, 1.0);
    q = sfx_fma(q, f, 1.0);
    const int ni = (int)n;
    if(ni < -1022 || ni > 1023) return SFX_POW_FAST_RARE(x, y);
    return q * sfx_u2d((uint64_t)(ni + 1023) << 52);
}


/*
 * sfx_cbrt: a deterministic cube root for host and device code (the moving
 * mesh's generator velocity, VorCell::get_velocity, src/VorCell.cpp:966-1008,
 * takes the cube root of the cell volume; glibc's and CUDA's cbrt can differ
 * in the last bit).  Only IEEE basic operations and FMA:
 *   |x| = 2^(3k) t, t in [1, 8) (subnormals scaled by 2^162 first);
 *   Newton's iteration y <- (2 y + t / y^2) / 3 from y = (t + 2) / 3, which is
 *   never below t^(1/3) (arithmetic-geometric mean inequality), so the
 *   iterates fall monotonically to the root: six steps reach double
 *   precision on [1, 8);
 *   one more step with the residual y^3 - t formed exactly to first order
 *   (products split by FMA), then 2^k and the sign.
 * Special values: +-0, +-inf and NaN are returned as they are.
 */
SFX_HD double sfx_cbrt(double x) {
    if(x == 0.0 || x != x || x - x != 0.0) return x; /* 0, NaN, inf */
    const double ax = x < 0.0 ? -x : x;
    uint64_t u = sfx_d2u(ax);
    int adj = 0;
    double a = ax;
    if((u >> 52) == 0) { /* subnormal */
        a = ax * 0x1p162;
        u = sfx_d2u(a);
        adj = -54;
    }
    const int e = (int)(u >> 52) - 1023;
    /* e = 3k + r, r in {0, 1, 2} */
    int k = e >= 0 ? e / 3 : -((-e + 2) / 3);
    const int r = e - 3 * k;
    const double t = sfx_u2d((u & 0x000fffffffffffffull) | ((uint64_t)(1023 + r) << 52));
    double y = (t + 2.0) / 3.0;
    for(int i = 0; i < 6; ++i) y = (2.0 * y + t / (y * y)) / 3.0;
    /* y^3 - t with the rounding errors of y*y and (y*y)*y kept */
    const double p = y * y;
    const double pe = sfx_fma(y, y, -p);
    const double q = p * y;
    const double qe = sfx_fma(p, y, -q) + pe * y;
    const double res = (q - t) + qe;
    y = y - res / (3.0 * p);
    k += adj;
    /* y * 2^k, k within the normal exponent range for every double x */
    const double sc = sfx_u2d((uint64_t)(1023 + k) << 52);
    const double out = y * sc;
    return x < 0.0 ? -out : out;
}

#endif /* SFX_POW_H */
