// Test infrastructure only: a stand-in for the small part of GMP's C++
// interface (<gmpxx.h>) that the reference's GMP-based programs use, so that
// oracle/Makefile can compile those programs unmodified from their own sources
// (fourcore_cls5_gpu_v4.cu, fourcore_find_v4.cu, fourcore_hunt_v3.cpp) on a
// machine without the GMP development headers.  Nothing in the product links
// or includes it.
//
// The reference uses GMP only for exact sixth powers and their sums,
// differences, exact quotients and remainders (fourcore_gmp.hpp:15-123), and
// for moving results into 64-bit words with mpz_export / mpz_import and
// mpz_sizeinbase(·, 2) (fourcore_cls5_gpu_v4.cu:52-60,257-258;
// fourcore_hunt_v3.cpp:71-74,97-102).  Every value it forms is below 2^200
// (B^6 with B < 2^32 is below 2^192), so this header keeps a sign and a
// fixed 512-bit magnitude and aborts, rather than wrapping, if a result
// would not fit.  Division and remainder truncate toward zero, as
// mpz_class's operators do.
//
// Only the members and functions that those programs call are provided:
//   mpz_class(integer), copy, = += -= *=, binary + - * / %, == != < <= > >=
//   (against mpz_class or a built-in integer), get_mpz_t(),
//   mpz_sizeinbase(op, 2), mpz_export(..., order -1, size 8, endian 0, nails 0),
//   mpz_import(..., order -1, size 8, endian 0, nails 0).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace gmpshim {

constexpr int kWords = 8;   // 512-bit magnitude

struct Num {
    bool neg = false;                 // sign; zero is never negative
    std::uint64_t w[kWords] = {};     // magnitude, least significant word first
};

[[noreturn]] inline void fail(const char* what) {
    std::fprintf(stderr, "gmpshim: %s\n", what);
    std::abort();
}

inline bool is_zero(const Num& a) {
    for (int i = 0; i < kWords; ++i)
        if (a.w[i]) return false;
    return true;
}

inline void normalize(Num& a) {
    if (is_zero(a)) a.neg = false;
}

// Compare magnitudes: -1, 0, 1.
inline int cmp_mag(const Num& a, const Num& b) {
    for (int i = kWords - 1; i >= 0; --i) {
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
    }
    return 0;
}

inline int cmp(const Num& a, const Num& b) {
    if (a.neg != b.neg) return a.neg ? -1 : 1;
    const int m = cmp_mag(a, b);
    return a.neg ? -m : m;
}

// |r| = |a| + |b|
inline void add_mag(Num& r, const Num& a, const Num& b) {
    unsigned __int128 carry = 0;
    for (int i = 0; i < kWords; ++i) {
        carry += (unsigned __int128)a.w[i] + b.w[i];
        r.w[i] = (std::uint64_t)carry;
        carry >>= 64;
    }
    if (carry) fail("sum exceeds 512 bits");
}

// |r| = |a| - |b|, requires |a| >= |b|
inline void sub_mag(Num& r, const Num& a, const Num& b) {
    std::uint64_t borrow = 0;
    for (int i = 0; i < kWords; ++i) {
        const std::uint64_t x = a.w[i], y = b.w[i];
        const std::uint64_t d = x - y - borrow;
        borrow = (x < y) || (x == y && borrow) ? 1 : 0;
        r.w[i] = d;
    }
}

inline Num add(const Num& a, const Num& b) {
    Num r;
    if (a.neg == b.neg) {
        add_mag(r, a, b);
        r.neg = a.neg;
    } else if (cmp_mag(a, b) >= 0) {
        sub_mag(r, a, b);
        r.neg = a.neg;
    } else {
        sub_mag(r, b, a);
        r.neg = b.neg;
    }
    normalize(r);
    return r;
}

inline Num negate(Num a) {
    a.neg = !a.neg;
    normalize(a);
    return a;
}

inline Num mul(const Num& a, const Num& b) {
    std::uint64_t t[2 * kWords] = {};
    for (int i = 0; i < kWords; ++i) {
        if (!a.w[i]) continue;
        unsigned __int128 carry = 0;
        for (int j = 0; j < kWords; ++j) {
            carry += (unsigned __int128)a.w[i] * b.w[j] + t[i + j];
            t[i + j] = (std::uint64_t)carry;
            carry >>= 64;
        }
        t[i + kWords] = (std::uint64_t)carry;
    }
    for (int i = kWords; i < 2 * kWords; ++i)
        if (t[i]) fail("product exceeds 512 bits");
    Num r;
    std::memcpy(r.w, t, sizeof r.w);
    r.neg = a.neg != b.neg;
    normalize(r);
    return r;
}

inline int bit_length(const Num& a) {
    for (int i = kWords - 1; i >= 0; --i) {
        if (a.w[i]) return 64 * i + 64 - __builtin_clzll(a.w[i]);
    }
    return 0;
}

// Magnitude division: |a| = q·|b| + r with 0 <= r < |b|.
inline void divmod_mag(const Num& a, const Num& b, Num& q, Num& r) {
    if (is_zero(b)) fail("division by zero");
    q = Num{};
    r = Num{};
    if (bit_length(b) <= 64) {           // one-word divisor: schoolbook short division
        const std::uint64_t d = b.w[0];
        unsigned __int128 rem = 0;
        for (int i = kWords - 1; i >= 0; --i) {
            rem = (rem << 64) | a.w[i];
            q.w[i] = (std::uint64_t)(rem / d);
            rem %= d;
        }
        r.w[0] = (std::uint64_t)rem;
        return;
    }
    // Restoring binary long division, most significant bit first.
    for (int bit = bit_length(a) - 1; bit >= 0; --bit) {
        // r = 2r + bit
        for (int i = kWords - 1; i > 0; --i) r.w[i] = (r.w[i] << 1) | (r.w[i - 1] >> 63);
        r.w[0] = (r.w[0] << 1) | ((a.w[bit / 64] >> (bit % 64)) & 1);
        if (cmp_mag(r, b) >= 0) {
            sub_mag(r, r, b);
            q.w[bit / 64] |= 1ULL << (bit % 64);
        }
    }
}

inline Num from_u64(std::uint64_t v) {
    Num r;
    r.w[0] = v;
    return r;
}

inline Num from_i64(long long v) {
    Num r;
    if (v < 0) {
        r.neg = true;
        r.w[0] = (std::uint64_t)0 - (std::uint64_t)v;
    } else {
        r.w[0] = (std::uint64_t)v;
    }
    return r;
}

}  // namespace gmpshim

typedef gmpshim::Num* mpz_ptr;
typedef const gmpshim::Num* mpz_srcptr;

class mpz_class {
public:
    mpz_class() = default;
    mpz_class(int v) : v_(gmpshim::from_i64(v)) {}
    mpz_class(long v) : v_(gmpshim::from_i64(v)) {}
    mpz_class(long long v) : v_(gmpshim::from_i64(v)) {}
    mpz_class(unsigned v) : v_(gmpshim::from_u64(v)) {}
    mpz_class(unsigned long v) : v_(gmpshim::from_u64(v)) {}
    mpz_class(unsigned long long v) : v_(gmpshim::from_u64(v)) {}

    mpz_ptr get_mpz_t() { return &v_; }
    mpz_srcptr get_mpz_t() const { return &v_; }

    mpz_class& operator+=(const mpz_class& o) { v_ = gmpshim::add(v_, o.v_); return *this; }
    mpz_class& operator-=(const mpz_class& o) { v_ = gmpshim::add(v_, gmpshim::negate(o.v_)); return *this; }
    mpz_class& operator*=(const mpz_class& o) { v_ = gmpshim::mul(v_, o.v_); return *this; }
    mpz_class& operator/=(const mpz_class& o) { *this = div_(*this, o, false); return *this; }
    mpz_class& operator%=(const mpz_class& o) { *this = div_(*this, o, true); return *this; }

    friend mpz_class operator+(mpz_class a, const mpz_class& b) { return a += b; }
    friend mpz_class operator-(mpz_class a, const mpz_class& b) { return a -= b; }
    friend mpz_class operator*(mpz_class a, const mpz_class& b) { return a *= b; }
    friend mpz_class operator/(const mpz_class& a, const mpz_class& b) { return div_(a, b, false); }
    friend mpz_class operator%(const mpz_class& a, const mpz_class& b) { return div_(a, b, true); }
    friend mpz_class operator-(const mpz_class& a) {
        mpz_class r;
        r.v_ = gmpshim::negate(a.v_);
        return r;
    }

    friend bool operator==(const mpz_class& a, const mpz_class& b) { return gmpshim::cmp(a.v_, b.v_) == 0; }
    friend bool operator!=(const mpz_class& a, const mpz_class& b) { return gmpshim::cmp(a.v_, b.v_) != 0; }
    friend bool operator<(const mpz_class& a, const mpz_class& b) { return gmpshim::cmp(a.v_, b.v_) < 0; }
    friend bool operator<=(const mpz_class& a, const mpz_class& b) { return gmpshim::cmp(a.v_, b.v_) <= 0; }
    friend bool operator>(const mpz_class& a, const mpz_class& b) { return gmpshim::cmp(a.v_, b.v_) > 0; }
    friend bool operator>=(const mpz_class& a, const mpz_class& b) { return gmpshim::cmp(a.v_, b.v_) >= 0; }

private:
    // Truncating division (quotient rounds toward zero; the remainder takes
    // the dividend's sign), the rule of mpz_class's / and %.
    static mpz_class div_(const mpz_class& a, const mpz_class& b, bool want_rem) {
        gmpshim::Num q, r;
        gmpshim::divmod_mag(a.v_, b.v_, q, r);
        mpz_class out;
        if (want_rem) {
            r.neg = a.v_.neg;
            gmpshim::normalize(r);
            out.v_ = r;
        } else {
            q.neg = a.v_.neg != b.v_.neg;
            gmpshim::normalize(q);
            out.v_ = q;
        }
        return out;
    }

    gmpshim::Num v_;
};

// Number of base-2 digits of |op| (1 for zero, as GMP returns).
inline std::size_t mpz_sizeinbase(mpz_srcptr op, int base) {
    if (base != 2) gmpshim::fail("mpz_sizeinbase: only base 2 is provided");
    const int n = gmpshim::bit_length(*op);
    return n ? (std::size_t)n : 1;
}

// Writes |op| as 64-bit words, least significant first (order -1, size 8,
// native endian, no nails); *countp gets the number of words (0 for zero).
inline void* mpz_export(void* rop, std::size_t* countp, int order, std::size_t size, int endian,
                        std::size_t nails, mpz_srcptr op) {
    if (order != -1 || size != sizeof(std::uint64_t) || endian != 0 || nails != 0)
        gmpshim::fail("mpz_export: only order -1, 8-byte words, native endian, no nails");
    const int bits = gmpshim::bit_length(*op);
    const std::size_t words = (std::size_t)(bits + 63) / 64;
    if (words) std::memcpy(rop, op->w, words * sizeof(std::uint64_t));
    if (countp) *countp = words;
    return rop;
}

// Sets rop from count 64-bit words, least significant first (same forms as
// mpz_export); the result is non-negative.
inline void mpz_import(mpz_ptr rop, std::size_t count, int order, std::size_t size, int endian,
                       std::size_t nails, const void* op) {
    if (order != -1 || size != sizeof(std::uint64_t) || endian != 0 || nails != 0)
        gmpshim::fail("mpz_import: only order -1, 8-byte words, native endian, no nails");
    if (count > (std::size_t)gmpshim::kWords) gmpshim::fail("mpz_import: more than 512 bits");
    gmpshim::Num r;
    std::memcpy(r.w, op, count * sizeof(std::uint64_t));
    *rop = r;
}
