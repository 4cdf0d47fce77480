/*
 * Replaces libm's pow() and cbrt() in the "sfxpow" builds of the reference
 * harness (TEST INFRASTRUCTURE ONLY).  The reference sources call them
 * through <cmath>; linking these definitions into the executable routes
 * those calls to sfx_pow and sfx_cbrt, the deterministic functions shared by
 * the GPU pass and the CPU oracle, so the harness, the oracle and the GPU
 * agree bit for bit.  The "libm" build of the harness leaves glibc's in place.
 */
#include "../../shadowfax_b200/csrc/sfx_pow.h"

double pow(double x, double y) {
    return sfx_pow(x, y);
}

double cbrt(double x) {
    return sfx_cbrt(x);
}
