#!/usr/bin/env python
"""Writes crmath_tables.h: the constants and tables of the correctly rounded transcendentals in
crmath.cuh, each value computed with mpmath at 400 bits and split into doubles.

    python gen_crmath_tables.py > crmath_tables.h

Double-double values are (hi, lo) with hi = RN(v) and lo = RN(v - hi). The tables:
  kSinCos[i]   sin(i/128), cos(i/128) for i = 0..103 (hi, lo each)
  kAtan[i]     atan(i/128) for i = 0..128
  kExp2[j]     2^(j/64) and 2^(j/64) - 1 for j = 0..63
  kTwoOverPi   2/pi as a binary fraction in 64-bit words, most significant first
and the split constants of the Cody-Waite reductions by pi/2 and ln2/64 and the Taylor
coefficients (1/n!, 1/(2n+1)) of the polynomial phases.
"""
import mpmath as mp

mp.mp.prec = 400


def split(v, n):
    """v as n doubles, each the rounded remainder of the previous ones."""
    out = []
    for _ in range(n):
        d = float(v)
        out.append(d)
        v = v - mp.mpf(d)
    return out


def trunc_bits(v, bits):
    """v rounded toward zero to `bits` significant bits (a double)."""
    m, e = mp.frexp(v)
    q = mp.floor(m * 2 ** bits)
    return float(mp.ldexp(q, e - bits))


def dd(v):
    return split(v, 2)


def hexd(x):
    return float.hex(float(x))


def emit_array(name, rows, per):
    print("CR_TABLE double %s[%d] = {" % (name, len(rows) * per))
    for r in rows:
        print("    " + ", ".join(hexd(x) for x in r) + ",")
    print("};")


def main():
    print("// crmath_tables.h -- generated by gen_crmath_tables.py (mpmath, 400 bits); do not edit.")
    print("#pragma once")
    print("#include <stdint.h>")
    print("#if defined(__CUDACC__)")
    print("#define CR_TABLE static __device__ const")
    print("#define CR_TABLE_U64 static __device__ const uint64_t")
    print("#else")
    print("#define CR_TABLE static const")
    print("#define CR_TABLE_U64 static const uint64_t")
    print("#endif")
    print("namespace bmadgpu {\nnamespace cr {")
    pi = mp.pi
    # pi/2 for the Cody-Waite reduction: P1 with 33 significant bits (k * P1 exact for k < 2^20),
    # then three full doubles
    p1 = trunc_bits(pi / 2, 33)
    rest = split(pi / 2 - mp.mpf(p1), 3)
    print("constexpr double kPio2_1 = %s, kPio2_2 = %s, kPio2_3 = %s, kPio2_4 = %s;" % (hexd(p1), *map(hexd, rest)))
    print("constexpr double kPio2H = %s, kPio2L = %s;" % tuple(map(hexd, dd(pi / 2))))
    print("constexpr double kPiH = %s, kPiL = %s;" % tuple(map(hexd, dd(pi))))
    print("constexpr double kPio4H = %s, kPio4L = %s;" % tuple(map(hexd, dd(pi / 4))))
    print("constexpr double k3Pio4H = %s, k3Pio4L = %s;" % tuple(map(hexd, dd(3 * pi / 4))))
    print("constexpr double kTwoOverPi = %s;" % hexd(2 / pi))
    # ln2/64: L1 with 36 significant bits (k * L1 exact for |k| < 2^17), then two doubles
    l = mp.log(2) / 64
    l1 = trunc_bits(l, 36)
    lr = split(l - mp.mpf(l1), 2)
    print("constexpr double kLn2o64_1 = %s, kLn2o64_2 = %s, kLn2o64_3 = %s;" % (hexd(l1), *map(hexd, lr)))
    print("constexpr double kInvLn2o64 = %s;" % hexd(64 / mp.log(2)))
    # Taylor coefficients as double-doubles (phase 2) -- index n holds the coefficient of the
    # n-th term of each series
    fact = lambda n: mp.factorial(n)
    emit_array("kSinCoef", [dd((-1) ** n / fact(2 * n + 1)) for n in range(1, 8)], 2)   # d^2n/(2n+1)!
    emit_array("kCosCoef", [dd((-1) ** n / fact(2 * n)) for n in range(1, 9)], 2)       # d^2n/(2n)!
    emit_array("kAtanCoef", [dd(mp.mpf((-1) ** n) / (2 * n + 1)) for n in range(1, 9)], 2)  # u^2n/(2n+1)
    emit_array("kExpCoef", [dd(1 / fact(n)) for n in range(2, 14)], 2)                  # r^n/n!, n = 2..13
    emit_array("kSinCos", [dd(mp.sin(mp.mpf(i) / 128)) + dd(mp.cos(mp.mpf(i) / 128)) for i in range(104)], 4)
    emit_array("kAtan", [dd(mp.atan(mp.mpf(i) / 128)) for i in range(129)], 2)
    emit_array("kExp2", [dd(mp.mpf(2) ** (mp.mpf(j) / 64)) + dd(mp.mpf(2) ** (mp.mpf(j) / 64) - 1)
                         for j in range(64)], 4)
    # 2/pi as a binary fraction: word w holds bits 64w+1 .. 64w+64 after the binary point
    words = []
    with mp.workprec(2200):  # 24 words = 1536 bits of 2/pi, plus guard bits
        f = 2 / mp.pi
        for _ in range(24):
            f = f * 2 ** 64
            w = int(mp.floor(f))
            words.append(w)
            f = f - w
    print("CR_TABLE_U64 kTwoOverPiBits[24] = {")
    for i in range(0, 24, 4):
        print("    " + ", ".join("0x%016xull" % w for w in words[i:i + 4]) + ",")
    print("};")
    print("}  // namespace cr\n}  // namespace bmadgpu")


if __name__ == "__main__":
    main()
