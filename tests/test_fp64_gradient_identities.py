"""The two identities the plain-FP64 gradient kernels rest on, checked on the
CPU (IEEE double arithmetic, no contraction):

* the first gradient loop's term of a face seen from its right cell is the
  exact negation of the term seen from its left cell (up to the sign of a
  zero, which a sum starting at +0 cannot tell apart), so one evaluation per
  face serves both cells;
* the limiter quotient with one division (sfx_limiter.h, compiled here from
  the same source as the device code) equals the reference's two divisions
  and select bit for bit, special values included."""
import ctypes as C
import itertools
import subprocess
from pathlib import Path

import numpy as np
import pytest

CSRC = Path(__file__).resolve().parent.parent / "shadowfax_b200" / "csrc"


def _term(W, Wj, xi, xj, mid, A):
    """A ((Wj - W) c / |r| - 0.5 (W + Wj) r / |r|) per direction, in the
    kernels' operation order: c = mid - 0.5 (xi + xj), r = xi - xj"""
    D = xi.shape[1]
    c = mid - 0.5 * (xi + xj)
    r = xi - xj
    dot = r[:, 0] * r[:, 0] + r[:, 1] * r[:, 1]
    if D == 3:
        dot = dot + r[:, 2] * r[:, 2]
    rn = np.sqrt(dot)
    out = np.empty_like(r)
    for l in range(D):
        out[:, l] = A * ((Wj - W) * c[:, l] / rn - 0.5 * (W + Wj) * r[:, l] / rn)
    return out


def _values(rng, n):
    """magnitudes over many decades, signs, exact repeats and zeros"""
    v = rng.standard_normal(n) * 10.0 ** rng.integers(-30, 30, n)
    v[rng.random(n) < 0.05] = 0.0
    v[rng.random(n) < 0.02] = -0.0
    return v


@pytest.mark.parametrize("D", [2, 3])
def test_face_term_is_negated_for_the_right_cell(D):
    rng = np.random.default_rng(40 + D)
    n = 200_000
    W = _values(rng, n)
    Wj = np.where(rng.random(n) < 0.1, W, _values(rng, n))          # equal states too
    xi = rng.random((n, D))
    xj = xi + rng.standard_normal((n, D)) * 10.0 ** rng.integers(-6, 0, (n, 1))
    same = rng.random((n, D)) < 0.05                                 # coincident coordinates
    xj[same] = xi[same]
    ok = np.any(xi != xj, axis=1)
    W, Wj, xi, xj = W[ok], Wj[ok], xi[ok], xj[ok]
    mid = 0.5 * (xi + xj) + rng.standard_normal(xi.shape) * 1e-3
    A = rng.random(len(W)) * 10.0 ** rng.integers(-8, 2, len(W))
    left = _term(W, Wj, xi, xj, mid, A)
    right = _term(Wj, W, xj, xi, mid, A)
    neg = -left
    same_bits = right.view(np.uint64) == neg.view(np.uint64)
    zeros = (right == 0) & (left == 0)
    assert np.all(same_bits | zeros)
    assert zeros.sum() > 0          # the zero case is exercised
    # a running sum from +0: adding the right cell's term equals subtracting
    # the left cell's, bit for bit, signed zeros included
    m = 64
    s1 = np.zeros(len(W) // m)
    s2 = np.zeros(len(W) // m)
    for q in range(m):
        sl = slice(q * (len(W) // m), (q + 1) * (len(W) // m))
        s1 = s1 + right[sl, 0]
        s2 = s2 - left[sl, 0]
        assert np.array_equal(s1.view(np.uint64), s2.view(np.uint64))


_SRC = r"""
#include "sfx_limiter.h"
extern "C" void lim(const double* a, const double* b, const double* dp, long n,
                    double* fast, double* ref) {
    for(long i = 0; i < n; ++i) {
        fast[i] = sfx_limiter_ratio(a[i], b[i], dp[i]);
        ref[i] = sfx_limiter_ratio_ref(a[i], b[i], dp[i]);
    }
}
"""


@pytest.fixture(scope="module")
def limlib(tmp_path_factory):
    d = tmp_path_factory.mktemp("lim")
    src = d / "lim.cpp"
    src.write_text(_SRC)
    so = d / "liblim.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                    "-shared", "-I", str(CSRC), str(src), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))
    p = C.POINTER(C.c_double)
    lib.lim.argtypes = [p, p, p, C.c_long, p, p]
    return lib


def _run(lib, a, b, dp):
    a, b, dp = (np.ascontiguousarray(x, dtype=np.float64) for x in (a, b, dp))
    fast = np.empty_like(a)
    ref = np.empty_like(a)
    p = C.POINTER(C.c_double)
    lib.lim(a.ctypes.data_as(p), b.ctypes.data_as(p), dp.ctypes.data_as(p), len(a),
            fast.ctypes.data_as(p), ref.ctypes.data_as(p))
    return fast, ref


def _same(fast, ref):
    return np.all((fast.view(np.uint64) == ref.view(np.uint64)) | (np.isnan(fast) & np.isnan(ref)))


def test_limiter_ratio_special_values(limlib):
    tiny, small = 5e-324, 2.2250738585072014e-308
    big = 1.7976931348623157e308
    v = [0.0, -0.0, tiny, -tiny, small, -small, 1e-300, -1e-300, 1e-160, -1e-160, 0.5, -0.5,
         1.0, -1.0, 3.0, -3.0, 1e160, -1e160, 1e300, -1e300, big, -big, np.inf, -np.inf, np.nan]
    a, b, dp = (np.array(t) for t in zip(*itertools.product(v, v, v)))
    fast, ref = _run(limlib, a, b, dp)
    assert _same(fast, ref)


def test_limiter_ratio_random_and_underflow(limlib):
    rng = np.random.default_rng(7)
    n = 2_000_000
    a = np.abs(rng.standard_normal(n)) * 10.0 ** rng.integers(-320, 308, n)
    b = -np.abs(rng.standard_normal(n)) * 10.0 ** rng.integers(-320, 308, n)
    dp = rng.standard_normal(n) * 10.0 ** rng.integers(-320, 308, n)
    a[rng.random(n) < 0.1] = 0.0
    b[rng.random(n) < 0.1] = 0.0
    fast, ref = _run(limlib, a, b, dp)
    assert _same(fast, ref)
    # quotients that underflow to a signed zero on either side
    k = 200_000
    a2 = np.abs(rng.standard_normal(k)) * 1e-300
    b2 = -np.abs(rng.standard_normal(k)) * 1e-300
    dp2 = rng.choice([-1.0, 1.0], k) * 1e300 * (1 + rng.random(k))
    fast, ref = _run(limlib, a2, b2, dp2)
    assert _same(fast, ref)
    assert np.any(ref == 0)
