/*
 * Stand-in for Boost.Multiprecision's fixed-width integers (TEST
 * INFRASTRUCTURE ONLY): the reference's exact geometric predicates
 * (src/ExArith.cpp) need int128_t, int256_t and a 278-bit signed-magnitude
 * cpp_int, used only as values built from 64-bit integers and combined by
 * +, -, * and comparisons; the reference bounds every intermediate below 278
 * bits.  One 320-bit two's-complement type serves all three.  Written for the
 * oracle's reference-tessellation harness; Boost is not installed here.
 */
#ifndef SFX_SHIM_BOOST_MP_CPP_INT_HPP
#define SFX_SHIM_BOOST_MP_CPP_INT_HPP

#include <cstdint>

namespace boost {
namespace multiprecision {

enum cpp_integer_type { unsigned_magnitude = 0, signed_magnitude = 1 };
enum cpp_int_check_type { unchecked = 0, checked = 1 };

namespace shim {

/* two's complement, little-endian 64-bit limbs */
class Int320 {
public:
    static const int L = 5;
    uint64_t w[L];

    Int320() {
        for(int i = 0; i < L; ++i) w[i] = 0;
    }
    Int320(long long v) { set(v); }
    Int320(long v) { set((long long)v); }
    Int320(int v) { set((long long)v); }
    Int320(unsigned long v) {
        w[0] = v;
        for(int i = 1; i < L; ++i) w[i] = 0;
    }
    Int320(unsigned int v) {
        w[0] = v;
        for(int i = 1; i < L; ++i) w[i] = 0;
    }

    bool negative() const { return (w[L - 1] >> 63) != 0; }
    bool zero() const {
        for(int i = 0; i < L; ++i)
            if(w[i]) return false;
        return true;
    }

    Int320 operator-() const {
        Int320 r;
        unsigned __int128 c = 1;
        for(int i = 0; i < L; ++i) {
            c += (unsigned __int128)(~w[i]);
            r.w[i] = (uint64_t)c;
            c >>= 64;
        }
        return r;
    }
    friend Int320 operator+(const Int320& a, const Int320& b) {
        Int320 r;
        unsigned __int128 c = 0;
        for(int i = 0; i < L; ++i) {
            c += (unsigned __int128)a.w[i] + b.w[i];
            r.w[i] = (uint64_t)c;
            c >>= 64;
        }
        return r;
    }
    friend Int320 operator-(const Int320& a, const Int320& b) { return a + (-b); }
    friend Int320 operator*(const Int320& a, const Int320& b) {
        const bool neg = a.negative() != b.negative();
        const Int320 x = a.negative() ? -a : a, y = b.negative() ? -b : b;
        Int320 r;
        for(int i = 0; i < L; ++i) {
            unsigned __int128 c = 0;
            for(int j = 0; i + j < L; ++j) {
                c += (unsigned __int128)x.w[i] * y.w[j] + r.w[i + j];
                r.w[i + j] = (uint64_t)c;
                c >>= 64;
            }
        }
        return neg ? -r : r;
    }
    Int320& operator+=(const Int320& b) { return *this = *this + b; }
    Int320& operator-=(const Int320& b) { return *this = *this - b; }
    Int320& operator*=(const Int320& b) { return *this = *this * b; }

    friend bool operator==(const Int320& a, const Int320& b) {
        for(int i = 0; i < L; ++i)
            if(a.w[i] != b.w[i]) return false;
        return true;
    }
    friend bool operator!=(const Int320& a, const Int320& b) { return !(a == b); }
    friend bool operator<(const Int320& a, const Int320& b) {
        if(a.negative() != b.negative()) return a.negative();
        for(int i = L - 1; i >= 0; --i)
            if(a.w[i] != b.w[i]) return a.w[i] < b.w[i];
        return false;
    }
    friend bool operator>(const Int320& a, const Int320& b) { return b < a; }
    friend bool operator<=(const Int320& a, const Int320& b) { return !(b < a); }
    friend bool operator>=(const Int320& a, const Int320& b) { return !(a < b); }

private:
    void set(long long v) {
        w[0] = (uint64_t)v;
        const uint64_t ext = v < 0 ? ~(uint64_t)0 : 0;
        for(int i = 1; i < L; ++i) w[i] = ext;
    }
};

}  // namespace shim

template <unsigned MinBits, unsigned MaxBits, cpp_integer_type SignType,
          cpp_int_check_type Checked, class Allocator>
struct cpp_int_backend {};

template <class Backend, int ExpressionTemplates = 0>
using number = shim::Int320;

typedef shim::Int320 int128_t;
typedef shim::Int320 int256_t;

}  // namespace multiprecision
}  // namespace boost

#endif
