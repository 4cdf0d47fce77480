/*
 * Replaces libm's pow() in the "sfxpow" build of the reference harness
 * (TEST INFRASTRUCTURE ONLY).  The reference sources call pow() through
 * <cmath>; linking this definition into the executable routes those calls to
 * sfx_pow, the deterministic power function shared by the GPU pass and the
 * CPU oracle, so the harness, the oracle and the GPU agree bit for bit.
 * The "libm" build of the harness leaves glibc's pow in place.
 */
#include "../../shadowfax_b200/csrc/sfx_pow.h"

double pow(double x, double y) {
    return sfx_pow(x, y);
}
