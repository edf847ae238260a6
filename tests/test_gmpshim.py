"""The test-only GMP stand-in (oracle/gmpshim/gmpxx.h) against Python integers.

The reference's GMP programs are compiled against that header to produce
fixtures, so its arithmetic must be exact on every operation they use
(fourcore_gmp.hpp:15-123; fourcore_cls5_gpu_v4.cu:52-60): products of sixth
powers, sums, differences, truncating quotients and remainders, comparisons,
mpz_sizeinbase(., 2) and mpz_export / mpz_import of 64-bit words.
"""
import os
import random
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "gmpshim")

PROG = r"""
#include <gmpxx.h>
#include <cstdio>
#include <cstdlib>
#include <cstdint>

static void put(const mpz_class& z) {
    mpz_class a = z < 0 ? -z : z;
    uint64_t w[8] = {0};
    size_t n = 0;
    mpz_export(w, &n, -1, 8, 0, 0, a.get_mpz_t());
    std::printf("%s%zu", z < 0 ? "-" : "+", n);
    for (size_t i = 0; i < n; ++i) std::printf(":%llx", (unsigned long long)w[i]);
    std::printf(" %zu\n", mpz_sizeinbase(z.get_mpz_t(), 2));
}

static mpz_class pow6(unsigned long long x) {
    mpz_class z(x);
    z *= z;
    mpz_class z2 = z;
    z *= z;
    z *= z2;
    return z;
}

int main() {
    unsigned long long a, b, c;
    long long s;
    while (std::scanf("%llu %llu %llu %lld", &a, &b, &c, &s) == 4) {
        mpz_class A = pow6(a), B = pow6(b), C = pow6(c);
        mpz_class diff = A - B - C;            // may be negative
        put(A);
        put(diff);
        put(A * mpz_class(s) + B);             // signed product
        mpz_class den = pow6(c % 50 + 2);
        put(diff / den);                       // truncating division
        put(diff % den);
        put(A / (B + 1));                      // multi-word divisor
        put(A % (B + 1));
        std::printf("%d %d %d\n", (int)(diff < 0), (int)(diff == 0), (int)(A >= B));
        uint64_t w[2] = {a * 0x9E3779B97F4A7C15ULL, b};
        mpz_class T;
        mpz_import(T.get_mpz_t(), 2, -1, 8, 0, 0, w);
        put(T);
    }
    return 0;
}
"""


def words(v):
    m = abs(v)
    out = []
    while m:
        out.append(m & (2**64 - 1))
        m >>= 64
    return out


def fmt(v):
    w = words(v)
    return f"{'-' if v < 0 else '+'}{len(w)}" + "".join(f":{x:x}" for x in w) + \
        f" {max(abs(v).bit_length(), 1)}"


def tdiv(a, b):
    q = abs(a) // abs(b)
    q = -q if (a < 0) != (b < 0) else q
    return q, a - q * b


@pytest.fixture(scope="module")
def shim_prog(tmp_path_factory):
    d = tmp_path_factory.mktemp("gmpshim")
    src, exe = d / "t.cpp", d / "t"
    src.write_text(PROG)
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{SHIM}", "-o", str(exe), str(src)], check=True)
    return str(exe)


def test_gmpshim_matches_python_ints(shim_prog):
    rng = random.Random(615)
    cases = [(1, 1, 1, 1), (42, 1, 1, -3), (2353975, 85710, 2353974, 7), (2752470, 2, 3, -1),
             (100003, 17646, 9 * 21, 5)]
    for _ in range(400):
        cases.append((rng.randrange(1, 2**32), rng.randrange(1, 2**32), rng.randrange(1, 2**31),
                      rng.randrange(-2**40, 2**40)))
    inp = "".join(f"{a} {b} {c} {s}\n" for a, b, c, s in cases)
    out = subprocess.run([shim_prog], input=inp, capture_output=True, text=True, check=True)
    lines = out.stdout.splitlines()
    per = 9
    assert len(lines) == per * len(cases)
    for k, (a, b, c, s) in enumerate(cases):
        A, B, Cc = a**6, b**6, c**6
        diff = A - B - Cc
        den = (c % 50 + 2) ** 6
        q, r = tdiv(diff, den)
        q2, r2 = tdiv(A, B + 1)
        T = ((a * 0x9E3779B97F4A7C15) % 2**64) | (b << 64)
        want = [fmt(A), fmt(diff), fmt(A * s + B), fmt(q), fmt(r), fmt(q2), fmt(r2),
                f"{int(diff < 0)} {int(diff == 0)} {int(A >= B)}", fmt(T)]
        got = lines[per * k: per * (k + 1)]
        assert got == want, (a, b, c, s)
