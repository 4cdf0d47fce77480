/*
 * The slope limiter's quotient for one face, plain-FP64 gradients
 * (VorCell::estimate_gradient, src/VorCell.cpp:486-530), for device code and
 * for host-side tests of the same source.
 *
 * The reference forms q1 = a / dp and q2 = b / dp with a = W_max - W and
 * b = W_min - W (q1 = q2 = 1 where dp == 0) and keeps mx = (q1 < q2) ? q2 : q1.
 * sfx_limiter_ratio returns the same value bit for bit with one division
 * where the signs decide the select: for finite a >= 0 >= b and finite
 * dp > 0, q1 >= +0 >= q2 (b = +0 gives q2 = +0, which does not compare below
 * q1), so mx = q1; for finite dp < 0, q1 <= -0 and q2 >= -0, so mx = q2
 * unless q2 is zero, where q1 is zero too and the select keeps q1.  Any
 * other input (dp == 0, a non-finite or misordered operand) takes the
 * reference's two divisions.
 */
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define SFX_LIM_HD __host__ __device__ __forceinline__
#else
#define SFX_LIM_HD static inline
#endif

/* the reference's two divisions and select */
SFX_LIM_HD double sfx_limiter_ratio_ref(double a, double b, double dp) {
    double q1 = a, q2 = b;
    if(dp != 0.) {
        q1 = q1 / dp;
        q2 = q2 / dp;
    } else {
        q1 = 1.;
        q2 = 1.;
    }
    return (q1 < q2) ? q2 : q1;
}

SFX_LIM_HD double sfx_limiter_ratio(double a, double b, double dp) {
    const double big = 1.7976931348623157e308;
    const bool fin = a >= 0. && a <= big && b <= 0. && b >= -big && fabs(dp) <= big;
    if(fin && dp > 0.) return a / dp;
    if(fin && dp < 0.) {
        const double q2 = b / dp;
        if(q2 != 0.) return q2;
        const double q1 = a / dp;
        return (q1 < q2) ? q2 : q1;
    }
    return sfx_limiter_ratio_ref(a, b, dp);
}
