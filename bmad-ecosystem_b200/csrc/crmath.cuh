// crmath.cuh -- correctly rounded sin, cos, asin, atan2, sinh and cosh in FP64 for the device
// (and, for the tests and the oracle's correctly rounded mode, the host).
//
// Why: the tracking maps call these six functions thousands of times per particle and turn, and
// long-term tracking amplifies a one-ulp difference in any of them to ~1e-8 after 1000 turns. A
// correctly rounded (CR) result is unique, so any two CR implementations -- this one on the GPU,
// the same source on the host, or an independent one -- give the same bits, and the device then
// reproduces bit for bit a CPU run of the reference's algorithm with a correctly rounded libm.
//
// Method: Ziv's two-phase evaluation (A. Ziv, "Fast evaluation of elementary mathematical
// functions with correctly rounded last bit", ACM TOMS 17 (1991) 410-423). Phase 1 evaluates
// the function as a double-double h + l with a relative error below kErr1; if h + (l - e) and
// h + (l + e) (e = kErr1 |h|) round to the same double, that double is the correctly rounded
// result. Otherwise phase 2 evaluates in double-double throughout (error below kErr2) and
// repeats the test; the rare argument whose value lies closer than kErr2 to a rounding boundary
// gets the phase-2 rounding (faithful, and correct unless the boundary is that close).
//
// Double-double arithmetic (Dekker, "A floating-point technique for extending the available
// precision", Numer. Math. 18 (1971) 224-242; Knuth's two-sum): exact sums and products of two
// doubles by the error-free transformations two_sum and two_prod (the latter by one FMA).
//
// Argument reductions and series (own code; tables from gen_crmath_tables.py):
//  - sin, cos: x = k pi/2 + r by Cody-Waite with pi/2 in four parts (the first of 33 bits, so
//    k P1 is exact) for |x| < 2^20, else Payne-Hanek with 2/pi in 64-bit words; then r = i/128
//    + d, |d| <= 1/256, sin(r) = S_i cos(d) + C_i sin(d) and cos(r) = C_i cos(d) - S_i sin(d)
//    with S_i, C_i tabulated as double-doubles and Taylor series in d.
//  - atan2 (and asin through atan2(x, sqrt(1 - x^2))): t = min/max of |y|, |x| as a
//    double-double quotient, t = i/128 + ..., atan t = atan(i/128) + atan(u) with
//    u = (t - i/128)/(1 + t i/128), |u| <= 1/256, Taylor series in u; quadrants by pi/2, pi.
//  - sinh, cosh: e^x = 2^m 2^(j/64) e^r, r = x - (64m + j) ln2/64 by Cody-Waite (ln2/64 in three
//    parts, the first of 36 bits), e^r by its Taylor series; cosh = (E + 1/E)/2, and sinh
//    = (E - 1/E)/2 for |x| >= 1/4, else (E1 + E1/(E1 + 1))/2 with E1 = e^x - 1 formed from the
//    tabulated 2^(j/64) - 1 without cancellation.
// Each function is compiled without FMA contraction like the rest of the library; the FMAs it
// needs are explicit. Special values follow C99 Annex F (NaN in, NaN out; signed zeros; the
// infinities of atan2; overflow to infinity).
// Known exception: atan2 results below 2^-500 in magnitude are the correctly rounded quotient
// y/x, which differs from the correctly rounded arctangent only when y/x is exactly halfway
// between two doubles.
#pragma once
#include <math.h>
#include <stdint.h>

#include "crmath_tables.h"

// CR_API: how the six entry points (and the fused pairs) are compiled: inlined, or on the device
// one out-of-line copy each with CR_DEVICE_NOINLINE.
#if defined(__CUDACC__) && defined(CR_DEVICE_NOINLINE)
#define CR_API static __device__ __noinline__
#else
#define CR_API CR_HD
#endif

#if defined(__CUDACC__)
#define CR_HD __device__ __forceinline__
#define CR_SLOW static __device__ __noinline__
#define CR_LD(p) __ldg(p)
#else
#define CR_HD inline
#define CR_SLOW static __attribute__((noinline)) inline
#define CR_LD(p) (*(p))
#endif

namespace bmadgpu {
namespace cr {

constexpr double kErr1 = 0x1p-64;   // phase-1 relative error bound (>= 8x the largest seen)
constexpr double kErr2 = 0x1p-95;   // phase-2 relative error bound

struct dd {
  double h, l;
};

CR_HD dd two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
CR_HD dd fast_two_sum(double a, double b) {  // |a| >= |b| or a == 0
  const double s = a + b;
  return {s, b - (s - a)};
}
CR_HD dd two_prod(double a, double b) {
  const double p = a * b;
  return {p, fma(a, b, -p)};
}
CR_HD dd dd_add(dd a, dd b) {  // accurate sum, also under cancellation
  dd s = two_sum(a.h, b.h);
  const dd t = two_sum(a.l, b.l);
  s.l = s.l + t.h;
  s = fast_two_sum(s.h, s.l);
  s.l = s.l + t.l;
  return fast_two_sum(s.h, s.l);
}
CR_HD dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.h, b.h);
  p.l = p.l + (a.h * b.l + a.l * b.h);
  return fast_two_sum(p.h, p.l);
}
// 1/b to about an ulp for |b| in [2^-120, 2^120]: the device's approximate reciprocal (or the
// host's division), then two Newton steps y += y (1 - b y) by FMA. The quotients built on it are
// double-doubles whose low part absorbs the last-bit differences, so host and device round the
// same functions to the same doubles.
CR_HD double rcp(double b) {
#if defined(__CUDACC__)
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));  // about 20 good bits
#else
  double y = 1.0 / b;
#endif
  y = fma(y, fma(-b, y, 1.0), y);
  return fma(y, fma(-b, y, 1.0), y);
}

// rint(v) (ties to even) and its value as an int, for |v| < 2^31, by adding 1.5 2^52: the sum
// holds the rounded integer in its low mantissa bits (no conversion instructions).
CR_HD double round_int(double v, int& k) {
  const double t = v + 0x1.8p52;
#if defined(__CUDACC__)
  k = __double2loint(t);
#else
  uint64_t u;
  __builtin_memcpy(&u, &t, 8);
  k = (int)(uint32_t)u;
#endif
  return t - 0x1.8p52;
}
// a / b as a double-double: q = a.h y, the exact residual a.h - q b.h by two_prod, and the
// correction r y (|b.h| in the float normal range).
CR_HD dd dd_div(dd a, dd b) {
  const double y = rcp(b.h);
  const double q = a.h * y;
  const dd p = two_prod(q, b.h);
  const double r = (((a.h - p.h) - p.l) + a.l) - q * b.l;
  return fast_two_sum(q, r * y);
}
// 2^e for -1022 <= e <= 1023, exactly.
CR_HD double pow2(int e) {
  const uint64_t u = (uint64_t)(e + 1023) << 52;
#if defined(__CUDACC__)
  return __longlong_as_double((long long)u);
#else
  double d;
  __builtin_memcpy(&d, &u, 8);
  return d;
#endif
}
CR_HD dd dd_neg(dd a) { return {-a.h, -a.l}; }
CR_HD dd dd_ld(const double* t) { return {CR_LD(t), CR_LD(t + 1)}; }

// The correctly rounded value of v = h + l known to |v - (h + l)| <= err, if one rounding fits.
CR_HD bool rounds(double h, double l, double err, double* out) {
  const double u = h + (l + err), v = h + (l - err);
  if (u == v) {
    *out = u;
    return true;
  }
  return false;
}

CR_HD double bits_to_double(uint64_t u) {
#if defined(__CUDACC__)
  return __longlong_as_double((long long)u);
#else
  double d;
  __builtin_memcpy(&d, &u, 8);
  return d;
#endif
}
CR_HD uint64_t double_to_bits(double d) {
#if defined(__CUDACC__)
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t u;
  __builtin_memcpy(&u, &d, 8);
  return u;
#endif
}

// ---- sin and cos -------------------------------------------------------------------------------

// Payne-Hanek reduction for |x| >= 2^20 (finite): x 2/pi = k + f with |f| <= 1/2 from the
// bits of 2/pi around x's exponent (integer arithmetic), r = f pi/2 as a double-double.
CR_HD void mul64(uint64_t a, uint64_t b, uint64_t& hi, uint64_t& lo) {
#if defined(__CUDACC__)
  lo = a * b;
  hi = __umul64hi(a, b);
#else
  const unsigned __int128 p = (unsigned __int128)a * b;
  lo = (uint64_t)p;
  hi = (uint64_t)(p >> 64);
#endif
}

CR_SLOW int reduce_large(double x, double& rh, double& rl) {
  const uint64_t ux = double_to_bits(x);
  const int ex = (int)((ux >> 52) & 0x7ff);
  const uint64_t mant = (ux & ((1ull << 52) - 1)) | (1ull << 52);
  const int E = ex - 1075;  // |x| = mant 2^E, E >= -32 here
  // product mant * W[j0 .. j0+4] (320 bits of 2/pi); bit b of the 384-bit product weighs
  // 2^(E - 64 (j0 + 5) + b): choose j0 so the units bit b0 = 64 (j0 + 5) - E is in [192, 256)
  int j0 = (E + 192 + 63) / 64 - 5;
  if (j0 < 0) j0 = 0;
  const int b0 = 64 * (j0 + 5) - E;
  uint64_t p[6] = {0, 0, 0, 0, 0, 0};  // little-endian 64-bit limbs
  for (int w = 0; w < 5; w++) {
    // word j0 + w has weight 2^(-64 (j0 + w + 1)), i.e. limb 4 - w of the 320-bit integer
    uint64_t hi, lo;
    mul64(mant, CR_LD(&kTwoOverPiBits[j0 + w]), hi, lo);
    const int at = 4 - w;
    uint64_t s = p[at] + lo;
    uint64_t c = s < lo;
    p[at] = s;
    const uint64_t t = p[at + 1] + hi;
    const uint64_t c1 = t < hi;
    s = t + c;
    c = c1 | (s < t);
    p[at + 1] = s;
    for (int q = at + 2; c && q < 6; q++) {
      p[q] += 1;
      c = p[q] == 0;
    }
  }
  // shift right by b0 - 192 so the units bit lands on bit 192 (limb 3, bit 0)
  const int sh = b0 - 192;
  uint64_t f[4];  // f[3] bit 0..1: k mod 4; f[2], f[1], f[0]: 192 fraction bits
  for (int q = 0; q < 4; q++) {
    const int src = q + sh / 64, bit = sh % 64;
    const uint64_t a = src < 6 ? p[src] : 0, b = src + 1 < 6 ? p[src + 1] : 0;
    f[q] = bit ? (a >> bit) | (b << (64 - bit)) : a;
  }
  int k = (int)(f[3] & 3);
  // fraction in [0, 1) as 192 bits; take [-1/2, 1/2)
  bool neg = (f[2] >> 63) != 0;
  if (neg) {
    k = (k + 1) & 3;
    // f - 1: two's complement of the 192-bit fraction, magnitude 1 - f
    f[0] = ~f[0];
    f[1] = ~f[1];
    f[2] = ~f[2];
    if (++f[0] == 0 && ++f[1] == 0) ++f[2];
  }
  // magnitude as a sum of six 32-bit pieces (exact doubles), largest first, accumulated exactly
  double acc_h = 0, acc_l = 0;
  for (int q = 2; q >= 0; q--) {
    const double hi32 = (double)(f[q] >> 32), lo32 = (double)(f[q] & 0xffffffffull);
    const double w1 = ldexp(hi32, 64 * (q - 3) + 32), w2 = ldexp(lo32, 64 * (q - 3));
    dd s = two_sum(acc_h, w1);
    acc_l = acc_l + s.l;
    acc_h = s.h;
    s = two_sum(acc_h, w2);
    acc_l = acc_l + s.l;
    acc_h = s.h;
  }
  const dd fr = fast_two_sum(acc_h, acc_l);
  dd r = dd_mul(fr, dd{kPio2H, kPio2L});
  if (neg) r = dd_neg(r);
  if (x < 0) {
    r = dd_neg(r);
    k = (4 - k) & 3;
  }
  rh = r.h;
  rl = r.l;
  return k;
}

// x = k pi/2 + rh + rl with |r| <= pi/4 (+ a rounding). Returns k mod 4.
CR_HD int reduce_pio2(double x, double& rh, double& rl) {
  const double ax = fabs(x);
  if (ax <= 0x1.921fb54442d18p-1) {
    rh = x;
    rl = 0;
    return 0;
  }
  if (ax < 0x1p20) {
    int k;
    const double kd = round_int(x * kTwoOverPi, k);
    const double t1 = x - kd * kPio2_1;  // exact (Sterbenz; kd kPio2_1 exact)
    const dd p2 = two_prod(kd, kPio2_2);
    const dd s = two_sum(t1, -p2.h);
    const dd p3 = two_prod(kd, kPio2_3);
    const double lo = ((s.l - p2.l) - p3.h) - (p3.l + kd * kPio2_4);
    const dd r = two_sum(s.h, lo);
    if (fabs(r.h) >= 0x1p-20) {
      rh = r.h;
      rl = r.l;
      return k & 3;
    }
  }
  return reduce_large(x, rh, rl);
}

// Split of r >= 0: r = i/128 + d, |d| <= 1/256 (+ a rounding).
CR_HD int sc_split(double rh, double rl, double& dh, double& dl) {
  int i;
  const double c = round_int(rh * 128.0, i) * (1.0 / 128);
  const dd d = fast_two_sum(rh - c, rl);  // rh - i/128 exact
  dh = d.h;
  dl = d.l;
  return i;
}

// The parts of sin(d) = dh + sd_lo and cos(d) = 1 + c_hi + c_lo shared by both functions.
struct ScPoly {
  double sd_lo, c_hi, c_lo;
};
CR_HD ScPoly sc_poly1(double dh, double dl) {
  const double d2 = dh * dh;
  ScPoly q;
  q.c_hi = -0.5 * d2;                                      // exact
  q.c_lo = fma(-0.5, fma(dh, dh, -d2), -dh * dl) + (d2 * d2) * fma(d2, -1.0 / 720, 1.0 / 24);
  q.sd_lo = fma(dh, d2 * fma(d2, fma(d2, -1.0 / 5040, 1.0 / 120), -1.0 / 6), dl);
  return q;
}

// Phase 1 of A cos(d) + B sin(d) with (A, B) = (S_i, C_i) for sin(r) and (C_i, -S_i) for cos(r).
// |A| >= 1/128 > |B d| unless A = S_0 = 0, and |A c_hi| <= |A| 2^-17: the two-sums are ordered.
CR_HD dd sc_phase1(int i, double dh, const ScPoly& q, bool want_cos) {
  const double* t = kSinCos + 4 * i;
  const double Ah = CR_LD(t + (want_cos ? 2 : 0)), Al = CR_LD(t + (want_cos ? 3 : 1));
  double Bh = CR_LD(t + (want_cos ? 0 : 2)), Bl = CR_LD(t + (want_cos ? 1 : 3));
  if (want_cos) {
    Bh = -Bh;
    Bl = -Bl;
  }
  const dd a = two_prod(Bh, dh);
  const dd u = fast_two_sum(Ah, a.h);
  const dd b = two_prod(Ah, q.c_hi);
  const dd w = fast_two_sum(u.h, b.h);
  double lo = (u.l + w.l) + (a.l + b.l);
  lo = fma(Ah, q.c_lo, lo + Al);
  lo = fma(Al, q.c_hi, lo);
  lo = fma(Bh, q.sd_lo, lo);
  lo = fma(Bl, dh, lo);
  return {w.h, lo};
}

// Phase 2 of the same in double-double throughout.
CR_HD dd sc_phase2(int i, double dh, double dl, bool want_cos) {
  const dd d{dh, dl};
  const dd d2 = dd_mul(d, d);
  dd ps = dd_ld(kSinCoef + 12);
  for (int n = 5; n >= 0; n--) ps = dd_add(dd_ld(kSinCoef + 2 * n), dd_mul(ps, d2));
  ps = dd_mul(ps, d2);                          // sin(d)/d - 1
  dd pc = dd_ld(kCosCoef + 14);
  for (int n = 6; n >= 0; n--) pc = dd_add(dd_ld(kCosCoef + 2 * n), dd_mul(pc, d2));
  pc = dd_mul(pc, d2);                          // cos(d) - 1
  const dd sd = dd_add(d, dd_mul(d, ps));
  const dd cd = dd_add(dd{1.0, 0.0}, pc);
  const double* t = kSinCos + 4 * i;
  const dd S = dd_ld(t), C = dd_ld(t + 2);
  return want_cos ? dd_add(dd_mul(C, cd), dd_neg(dd_mul(S, sd))) : dd_add(dd_mul(S, cd), dd_mul(C, sd));
}

// Phase 2 and the rounding of its result.
CR_SLOW double sc_slow(int i, double dh, double dl, bool want_cos) {
  const dd v = sc_phase2(i, dh, dl, want_cos);
  double out;
  if (!rounds(v.h, v.l, fabs(v.h) * kErr2, &out)) out = v.h + v.l;
  return out;
}

// sin(r) (want_cos false) or cos(r) of r = rh + rl, |r| <= pi/4 + a rounding, correctly rounded.
CR_HD double sc_eval(double rh, double rl, bool want_cos) {
  const bool neg = rh < 0;
  if (neg) {
    rh = -rh;
    rl = -rl;
  }
  double dh, dl;
  const int i = sc_split(rh, rl, dh, dl);
  const dd v = sc_phase1(i, dh, sc_poly1(dh, dl), want_cos);
  double out;
  if (!rounds(v.h, v.l, fabs(v.h) * kErr1, &out)) out = sc_slow(i, dh, dl, want_cos);
  return (neg && !want_cos) ? -out : out;
}

// sin(x + q pi/2): the reduced argument's sine or cosine with the quadrant's sign.
CR_HD double sin_quadrant(double x, int q) {
  double rh, rl;
  const int k = (reduce_pio2(x, rh, rl) + q) & 3;
  const double v = sc_eval(rh, rl, (k & 1) != 0);
  return (k & 2) ? -v : v;
}

// Entry points. The arguments the tracking maps pass (|x| <= pi/4 for sin and cos, small |x|
// for asin, moderate ratios for atan2, 1/4 <= |x| <= 20 for the pair sinh, cosh) take a short
// inline path; every other argument (tiny, large, infinite, NaN) one out-of-line call.
CR_SLOW double sin_cold(double x) {
  const double ax = fabs(x);
  if (!(ax <= 1.79769313486231570815e308)) return x - x;  // NaN, +-inf -> NaN
  if (ax < 0x1p-26) return x;                            // sin x = x (1 - x^2/6 ...) rounds to x
  return sin_quadrant(x, 0);
}
CR_SLOW double cos_cold(double x) {
  const double ax = fabs(x);
  if (!(ax <= 1.79769313486231570815e308)) return x - x;
  if (ax < 0x1p-27) return 1.0;  // cos x = 1 - x^2/2 ... rounds to 1
  return sin_quadrant(x, 1);
}
CR_SLOW void sincos_cold(double x, double* s, double* c) {
  *s = sin_cold(x);
  *c = cos_cold(x);
}

CR_API double sin(double x) {
  const double ax = fabs(x);
  if (ax >= 0x1p-26 && ax <= 0x1.921fb54442d18p-1) return sc_eval(x, 0.0, false);
  return sin_cold(x);
}

CR_API double cos(double x) {
  const double ax = fabs(x);
  if (ax >= 0x1p-27 && ax <= 0x1.921fb54442d18p-1) return sc_eval(x, 0.0, true);
  return cos_cold(x);
}

// Both, from one split of x and one set of series in d; the same bits as sin(x) and cos(x).
CR_API void sincos(double x, double* s, double* c) {
  const double ax = fabs(x);
  if (!(ax >= 0x1p-26 && ax <= 0x1.921fb54442d18p-1)) {
    sincos_cold(x, s, c);
    return;
  }
  double dh, dl;
  const int i = sc_split(ax, 0.0, dh, dl);
  const ScPoly q = sc_poly1(dh, dl);
  const dd vs = sc_phase1(i, dh, q, false), vc = sc_phase1(i, dh, q, true);
  double sr, cr;
  if (!rounds(vs.h, vs.l, vs.h * kErr1, &sr)) sr = sc_slow(i, dh, dl, false);
  if (!rounds(vc.h, vc.l, vc.h * kErr1, &cr)) cr = sc_slow(i, dh, dl, true);
  *s = x < 0 ? -sr : sr;
  *c = cr;
}

// ---- tan ---------------------------------------------------------------------------------------

// tan of r = rh + rl, |r| <= pi/4 + a rounding (odd: -1/tan r, the cotangent branch of the
// quadrants k = 1, 3): sin and cos of |r| as double-doubles and their double-double quotient. The
// quotient's relative error is below the sum of the two phase errors and the division's (< 2^-100),
// so the rounding test takes 3 times the phase bound.
CR_SLOW double tan_slow(int i, double dh, double dl, bool odd) {
  const dd s2 = sc_phase2(i, dh, dl, false), c2 = sc_phase2(i, dh, dl, true);
  const dd s = fast_two_sum(s2.h, s2.l), c = fast_two_sum(c2.h, c2.l);
  const dd v = odd ? dd_div(c, s) : dd_div(s, c);
  double out;
  if (!rounds(v.h, v.l, v.h * (3 * kErr2), &out)) out = v.h + v.l;
  return out;
}
CR_HD double tan_reduced(double rh, double rl, bool odd) {
  const bool neg = rh < 0;
  if (neg) {
    rh = -rh;
    rl = -rl;
  }
  double dh, dl;
  const int i = sc_split(rh, rl, dh, dl);
  const ScPoly q = sc_poly1(dh, dl);
  // phase 1 leaves low parts up to 2^-26 of the high ones: normalised before the division, whose
  // correction step assumes both operands' low parts below an ulp
  const dd s1 = sc_phase1(i, dh, q, false), c1 = sc_phase1(i, dh, q, true);
  const dd s = fast_two_sum(s1.h, s1.l), c = fast_two_sum(c1.h, c1.l);
  const dd v = odd ? dd_div(c, s) : dd_div(s, c);
  double out;
  if (!rounds(v.h, v.l, v.h * (3 * kErr1), &out)) out = tan_slow(i, dh, dl, odd);
  return (neg != odd) ? -out : out;
}

// tan x = x (1 + x^2/3 + ...) rounds to x below 2^-27; beyond pi/4 the reduction by pi/2 (the
// nearest multiple of pi/2 to any double is more than 2^-70 away, so sin r stays far inside the
// range of the reciprocal).
CR_SLOW double tan_cold(double x) {
  const double ax = fabs(x);
  if (!(ax <= 1.79769313486231570815e308)) return x - x;  // NaN, +-inf -> NaN
  if (ax < 0x1p-27) return x;
  double rh, rl;
  const int k = reduce_pio2(x, rh, rl);
  return tan_reduced(rh, rl, (k & 1) != 0);
}

CR_API double tan(double x) {
  const double ax = fabs(x);
  if (ax >= 0x1p-27 && ax <= 0x1.921fb54442d18p-1) return tan_reduced(x, 0.0, false);
  return tan_cold(x);
}

// ---- atan2 and asin ----------------------------------------------------------------------------

// The octant: mode 0 atan(t), 1 pi/2 - atan(t), 2 pi - atan(t), 3 pi/2 + atan(t).
CR_HD dd atan_octant(dd a, int mode) {
  if (mode == 0) return a;
  const dd base = mode == 2 ? dd{kPiH, kPiL} : dd{kPio2H, kPio2L};
  return dd_add(base, mode == 3 ? a : dd_neg(a));
}

// Phase 1 of atan(a/b), 0 <= a <= b (double-doubles, b.h in the float range): with c = i/128 the
// nearest to a/b, atan(a/b) = atan(c) + atan(u), u = (a - c b)/(b + c a), |u| <= 1/256 + a
// rounding, atan(u) = u (1 - u^2/3 + u^4/5 - u^6/7 + u^8/9). a.h - (c b).h is exact (Sterbenz,
// i >= 1) and |atan(c)| >= 1/128 > |u| unless c = 0.
CR_HD dd atan_phase1(dd a, dd b) {
  int i;
  const double c = round_int(a.h * rcp(b.h) * 128.0, i) * (1.0 / 128);
  const dd cb = two_prod(c, b.h);
  const dd n = two_sum(a.h - cb.h, fma(-c, b.l, a.l - cb.l));
  const dd ca = two_prod(c, a.h);
  dd m = two_sum(b.h, ca.h);
  m.l = m.l + (fma(c, a.l, ca.l) + b.l);
  const double y = rcp(m.h);
  const double uh = n.h * y;
  const dd q = two_prod(uh, m.h);
  const double ul = fma(-uh, m.l, ((n.h - q.h) - q.l) + n.l) * y;
  const double u2 = uh * uh;
  const double pa = u2 * fma(u2, fma(u2, fma(u2, 1.0 / 9, -1.0 / 7), 1.0 / 5), -1.0 / 3);
  const double* A = kAtan + 2 * i;
  const dd s = fast_two_sum(CR_LD(A), uh);
  return {s.h, fma(uh, pa, (s.l + CR_LD(A + 1)) + ul)};
}

// Phase 2 (t = a/b, u = (t - c)/(1 + t c) and the series in double-double) and its rounding.
CR_SLOW double atan_slow(dd a, dd b, int mode) {
  const dd t = dd_div(a, b);
  const int i = (int)(t.h * 128.0 + 0.5);
  const double c = i * (1.0 / 128);
  const dd n = dd_add(t, dd{-c, 0.0});
  const dd D = dd_add(dd{1.0, 0.0}, dd_mul(t, dd{c, 0.0}));
  const dd u = dd_div(n, D);
  const dd u2 = dd_mul(u, u);
  dd pa = dd_ld(kAtanCoef + 14);
  for (int k = 6; k >= 0; k--) pa = dd_add(dd_ld(kAtanCoef + 2 * k), dd_mul(pa, u2));
  pa = dd_mul(pa, u2);
  const dd v = atan_octant(dd_add(dd_ld(kAtan + 2 * i), dd_add(u, dd_mul(u, pa))), mode);
  double out;
  if (!rounds(v.h, v.l, fabs(v.h) * kErr2, &out)) out = v.h + v.l;
  return out;
}

CR_HD double atan_finish(dd a, dd b, int mode, double sign) {
  const dd v = atan_octant(atan_phase1(a, b), mode);
  double out;
  if (!rounds(v.h, v.l, fabs(v.h) * kErr1, &out)) out = atan_slow(a, b, mode);
  return sign * out;
}

// atan2 of positive finite num, den given as double-doubles (den_l, num_l may be 0).
CR_HD double atan2_pos(dd num, dd den, bool x_neg, double sign) {
  const bool swap = num.h > den.h;
  const dd a = swap ? den : num, b = swap ? num : den;  // a <= b
  int mode;
  if (!swap) mode = x_neg ? 2 : 0;
  else mode = x_neg ? 3 : 1;
  return atan_finish(a, b, mode, sign);
}

// atan2 of finite nonzero y, x whose magnitudes or ratio are extreme: both scaled by a power of
// two so that the larger lies in [1, 2) (exact unless the smaller falls below the normal range,
// where the quotient is far below 2^-500 anyway).
CR_SLOW double atan2_far(double y, double x) {
  const double ax = fabs(x), ay = fabs(y);
  const bool x_neg = signbit(x);
  const double sy = signbit(y) ? -1.0 : 1.0;
  const double big = ax > ay ? ax : ay;
  const int e = ilogb(big);
  const double sx = ldexp(ax, -e), syy = ldexp(ay, -e);
  const double small = ax > ay ? syy : sx;
  if (small < 0x1p-500) {
    // the quotient is below 2^-500: atan q rounds as q does, except exactly halfway between
    // two doubles; the octant constants absorb it entirely
    if (ay < ax) return x_neg ? sy * kPiH : y / ax;
    return sy * kPio2H;
  }
  return atan2_pos(dd{syy, 0.0}, dd{sx, 0.0}, x_neg, sy);
}

CR_SLOW double atan2_cold(double y, double x) {
  if (x != x || y != y) return x + y;
  const double ax = fabs(x), ay = fabs(y);
  const bool x_neg = signbit(x);
  const double sy = signbit(y) ? -1.0 : 1.0;
  const double kInf = 1.79769313486231570815e308;
  if (ay == 0) return x_neg ? sy * kPiH : y;
  if (ax == 0) return sy * kPio2H;
  if (ax > kInf) {
    if (ay > kInf) return sy * (x_neg ? k3Pio4H : kPio4H);
    return x_neg ? sy * kPiH : sy * 0.0;
  }
  if (ay > kInf) return sy * kPio2H;
  return atan2_far(y, x);
}

CR_API double atan2(double y, double x) {
  const double ax = fabs(x), ay = fabs(y);
  const double big = ax > ay ? ax : ay, small = ax > ay ? ay : ax;
  // finite, nonzero, the divisor of the quotient in the reciprocal's range (atan2_pos)
  if (big >= 0x1p-120 && big <= 0x1p120 && small >= big * 0x1p-500)
    return atan2_pos(dd{ay, 0.0}, dd{ax, 0.0}, signbit(x), signbit(y) ? -1.0 : 1.0);
  return atan2_cold(y, x);
}

// asin of 2^-7 <= |x| < 1 (and of smaller |x| whose series phase could not round): atan2(x, s)
// with s = sqrt(1 - x^2) as a double-double; 1 - x^2 exact as (1 - p.h) - p.l.
CR_SLOW double asin_general(double x) {
  const double ax = fabs(x);
  const dd p = two_prod(ax, ax);
  const dd w0 = two_sum(1.0, -p.h);
  const dd w = fast_two_sum(w0.h, w0.l - p.l);
  const double sh = sqrt(w.h);
  const double sl = (fma(-sh, sh, w.h) + w.l) * (0.5 * rcp(sh));
  return atan2_pos(dd{ax, 0.0}, fast_two_sum(sh, sl), false, x < 0 ? -1.0 : 1.0);
}

CR_SLOW double asin_cold(double x) {
  const double ax = fabs(x);
  if (!(ax <= 1.0)) return (x - x) / (x - x);  // NaN (also for NaN in)
  if (ax == 1.0) return x * kPio2H;
  if (ax < 0x1p-26) return x;                 // asin x = x (1 + x^2/6 ...) rounds to x
  return asin_general(x);
}

CR_API double asin(double x) {
  const double ax = fabs(x);
  if (ax >= 0x1p-26 && ax < 0x1p-7) {
    // asin x = x + x^3 (1/6 + 3/40 x^2 + 5/112 x^4 + 35/1152 x^6 + 63/2816 x^8 + ...): the tail
    // is below 2^-16.5 of x, its rounding below 2^-68 of the result, the truncation 2^-90
    const double x2 = x * x;
    const double t = (x * x2) * fma(x2, fma(x2, fma(x2, fma(x2, 63.0 / 2816, 35.0 / 1152), 5.0 / 112), 3.0 / 40), 1.0 / 6);
    const dd v = fast_two_sum(x, t);
    double out;
    if (rounds(v.h, v.l, fabs(v.h) * kErr1, &out)) return out;
    return asin_general(x);
  }
  return asin_cold(x);
}

// ---- sinh and cosh -----------------------------------------------------------------------------

// x >= 0, x < 711: x = (64 m + j) ln2/64 + r, |r| <= ln2/128 (+ a rounding).
CR_HD void exp_reduce(double x, int& m, int& j, double& rh, double& rl) {
  int k;
  const double kd = round_int(x * kInvLn2o64, k);
  const double t1 = x - kd * kLn2o64_1;  // exact
  const dd p2 = two_prod(kd, kLn2o64_2);
  const dd s = two_sum(t1, -p2.h);
  const dd r = two_sum(s.h, (s.l - p2.l) - kd * kLn2o64_3);
  m = k >> 6;
  j = k & 63;
  rh = r.h;
  rl = r.l;
}

// Phase 1 of e^r - 1 = rh + rl + qh + ql.
CR_HD void expm1_r1(double rh, double rl, double& qh, double& ql) {
  const double sq = rh * rh;
  qh = 0.5 * sq;
  const double p = fma(rh, fma(rh, fma(rh, fma(rh, 1.0 / 5040, 1.0 / 720), 1.0 / 120), 1.0 / 24), 1.0 / 6);
  ql = fma(0.5, fma(rh, rh, -sq), rh * rl) + (rh * sq) * p;
}

// Phase 1: F = 2^(j/64) e^r (in [1, 2.02)) or, with em1, E1 = 2^(j/64) e^r - 1 (m = 0). The
// two-sums are ordered: |base| >= |T r| unless base = 0, and |T q| <= |T r| 2^-7.
CR_HD dd exp_phase1(int j, double rh, double rl, bool em1) {
  double qh, ql;
  expm1_r1(rh, rl, qh, ql);
  const double* T = kExp2 + 4 * j;
  const double Th = CR_LD(T), Tl = CR_LD(T + 1);
  const double base = em1 ? CR_LD(T + 2) : Th, base_l = em1 ? CR_LD(T + 3) : Tl;
  const dd a = two_prod(Th, rh);
  const dd s = fast_two_sum(base, a.h);
  const dd b = two_prod(Th, qh);
  const dd w = fast_two_sum(s.h, b.h);
  double lo = ((s.l + w.l) + (a.l + b.l)) + base_l;
  lo = fma(Th, rl + ql, lo);
  lo = fma(Tl, rh + qh, lo);
  return fast_two_sum(w.h, lo);
}

CR_SLOW dd exp_phase2(int j, double rh, double rl, bool em1) {
  const dd r{rh, rl};
  dd q = dd_ld(kExpCoef + 22);  // r^13/13!
  for (int n = 10; n >= 0; n--) q = dd_add(dd_ld(kExpCoef + 2 * n), dd_mul(q, r));
  q = dd_mul(dd_mul(q, r), r);  // e^r - 1 - r
  const dd em = dd_add(r, q);
  const double* T = kExp2 + 4 * j;
  const dd Tv = dd_ld(T);
  return dd_add(em1 ? dd_ld(T + 2) : Tv, dd_mul(Tv, em));
}

// v 2^e for v in [0.5, 4), -1 <= e <= 1024: exact, or overflow to infinity.
CR_HD double scale_up(double v, int e) { return e <= 1023 ? v * pow2(e) : (v * pow2(1023)) * 2.0; }

// F + G (cosh) and F - G (sinh) with G = 2^-2m / F, F = 2^(j/64) e^r (F >= 1.28 > G for x >= 1/4:
// the two-sums are ordered); G is dropped when below 2^-110 of F.
CR_HD void hyp_pair(dd F, int m, dd* vs, dd* vc) {
  if (2 * m > 110) {
    *vs = F;
    *vc = F;
    return;
  }
  const double s2 = pow2(-2 * m);
  const double g = rcp(F.h);
  const double gl = fma(-g, F.l, fma(-g, F.h, 1.0)) * g;
  const double Gh = g * s2, Gl = gl * s2;
  dd c = fast_two_sum(F.h, Gh);
  *vc = {c.h, c.l + (F.l + Gl)};
  c = fast_two_sum(F.h, -Gh);
  *vs = {c.h, c.l + (F.l - Gl)};
}

// sinh of 2^-26 <= x < 1/4 (m = 0): (E1 + E1/(E1 + 1))/2 with E1 = e^x - 1, unscaled.
CR_HD dd sinh_small(dd e1) {
  const dd D = fast_two_sum(1.0, e1.h);
  const double y = rcp(D.h);
  const double qh = e1.h * y;
  const dd p = two_prod(qh, D.h);
  const double ql = fma(-qh, D.l + e1.l, ((e1.h - p.h) - p.l) + e1.l) * y;
  const dd s = fast_two_sum(e1.h, qh);
  return {s.h, s.l + (e1.l + ql)};
}

// cosh (want_sinh = false) or sinh of ax (2^-26 <= ax <= 711) as 2^scale v, v a double-double
// from the given exponential phase.
template <int PHASE>
CR_HD dd hyp_value(double ax, bool want_sinh, int& scale) {
  int m, j;
  double rh, rl;
  exp_reduce(ax, m, j, rh, rl);
  if (want_sinh && ax < 0.25) {
    scale = -1;
    return sinh_small(PHASE == 1 ? exp_phase1(j, rh, rl, true) : exp_phase2(j, rh, rl, true));
  }
  const dd F = PHASE == 1 ? exp_phase1(j, rh, rl, false) : exp_phase2(j, rh, rl, false);
  scale = m - 1;
  dd vs, vc;
  hyp_pair(F, m, &vs, &vc);
  return want_sinh ? vs : vc;
}

// Phase 2 and its rounding (unscaled; the scale is phase 1's).
CR_SLOW double hyp_slow(double ax, bool want_sinh) {
  int scale;
  const dd v = hyp_value<2>(ax, want_sinh, scale);
  double out;
  if (!rounds(v.h, v.l, v.h * kErr2, &out)) out = v.h + v.l;
  return out;
}

// cosh x = 1 + x^2/2 + eps, 0 < eps < 2^-100, for 2^-27 <= x < 2^-24: 1 + x^2/2 (exact: x^2 by
// two_prod) is a midpoint between two doubles for x = 2^-26 and 3 2^-26, and eps decides those
// upwards.
CR_SLOW double cosh_tiny(double ax) {
  dd q = two_prod(ax, ax);
  q.h = 0.5 * q.h;
  q.l = 0.5 * q.l;
  const dd s = two_sum(1.0, q.h);
  const double lo = s.l + q.l;
  const double eps = (q.h * q.h) * (1.0 / 6);  // x^4/24
  double out;
  if (rounds(s.h, lo + 0.5 * eps, 0.5 * eps + 0x1p-104, &out)) return out;
  return lo > 0 ? s.h + 2 * lo : s.h;          // lo is half an ulp of s.h
}

CR_SLOW double hyp_cold(double x, bool want_sinh) {
  const double ax = fabs(x);
  if (x != x) return x + x;
  if (want_sinh ? ax < 0x1p-26 : ax < 0x1p-27) return want_sinh ? x : 1.0;  // x (1 + x^2/6), 1 + x^2/2
  if (ax > 711.0) return want_sinh ? x * 0x1p1023 * 2.0 : ax * 0x1p1023 * 2.0;  // overflow (inf -> inf)
  if (!want_sinh && ax < 0x1p-24) return cosh_tiny(ax);
  int scale;
  const dd v = hyp_value<1>(ax, want_sinh, scale);
  double out;
  if (!rounds(v.h, v.l, v.h * kErr1, &out)) out = hyp_slow(ax, want_sinh);
  out = scale_up(out, scale);
  return (want_sinh && x < 0) ? -out : out;
}

// sinh, cosh of 1/4 <= |x| <= 20 (2m <= 58, no overflow): the shared inline path.
CR_HD double hyp_mid(double x, bool want_sinh) {
  const double ax = fabs(x);
  int m, j;
  double rh, rl;
  exp_reduce(ax, m, j, rh, rl);
  dd vs, vc;
  hyp_pair(exp_phase1(j, rh, rl, false), m, &vs, &vc);
  const dd v = want_sinh ? vs : vc;
  double out;
  if (!rounds(v.h, v.l, v.h * kErr1, &out)) out = hyp_slow(ax, want_sinh);
  out = out * pow2(m - 1);
  return (want_sinh && x < 0) ? -out : out;
}

CR_API double sinh(double x) {
  const double ax = fabs(x);
  return (ax >= 0.25 && ax <= 20.0) ? hyp_mid(x, true) : hyp_cold(x, true);
}
CR_API double cosh(double x) {
  const double ax = fabs(x);
  return (ax >= 0.25 && ax <= 20.0) ? hyp_mid(x, false) : hyp_cold(x, false);
}

CR_SLOW void sinhcosh_cold(double x, double* sh, double* ch) {
  *sh = hyp_cold(x, true);
  *ch = hyp_cold(x, false);
}

// Both, sharing e^x and its reciprocal (1/4 <= |x| <= 20); the same bits as sinh(x), cosh(x).
CR_API void sinhcosh(double x, double* sh, double* ch) {
  const double ax = fabs(x);
  if (!(ax >= 0.25 && ax <= 20.0)) {
    sinhcosh_cold(x, sh, ch);
    return;
  }
  int m, j;
  double rh, rl;
  exp_reduce(ax, m, j, rh, rl);
  dd vs, vc;
  hyp_pair(exp_phase1(j, rh, rl, false), m, &vs, &vc);
  double os, oc;
  if (!rounds(vs.h, vs.l, vs.h * kErr1, &os)) os = hyp_slow(ax, true);
  if (!rounds(vc.h, vc.l, vc.h * kErr1, &oc)) oc = hyp_slow(ax, false);
  const double sc = pow2(m - 1);
  os = os * sc;
  *sh = x < 0 ? -os : os;
  *ch = oc * sc;
}

// ---- exp ---------------------------------------------------------------------------------------

// e^x below 2^-1022 (x < -708.3): F 2^m rounded on the grid of 2^-1074 that the subnormals and the
// lowest binade share, as the integer nearest to W = F 2^(m+1074) < 2^53 (exact scaling), decided
// by the same error test as the rounding to a double.
CR_SLOW double exp_tiny(double x) {
  if (x < -746.0) return 0.0;  // e^x < 2^-1076 rounds to +0
  int m, j;
  double rh, rl;
  exp_reduce(x, m, j, rh, rl);
  for (int phase = 1; phase <= 2; phase++) {
    const dd F = phase == 1 ? exp_phase1(j, rh, rl, false) : exp_phase2(j, rh, rl, false);
    const double sc = pow2(m + 1074);
    const double wh = F.h * sc, wl = F.l * sc;
    const double n = rint(wh);
    const double f = wh - n;             // exact, |f| <= 1/2
    const double up = (f - 0.5) + wl, down = (f + 0.5) + wl;  // distances to the midpoints
    const double err = wh * (phase == 1 ? kErr1 : kErr2);
    if (phase == 1 && (fabs(up) <= err || fabs(down) <= err)) continue;  // too close to decide
    const double adj = up > 0 ? 1 : (down < 0 ? -1 : 0);
    return (n + adj) * 0x1p-1074;
  }
  return 0.0;  // not reached
}

// e^x for |x| < 2^-26: D = e^x - 1 = x + x^2/2 + x^3/6 + x^4/24 (the rest below 2^-130) as a
// double-double, rounded on the grid of the doubles next to 1 (2^-52 above, 2^-53 below) as the
// integer nearest to D / grid. Near x = 2^-53 the value lies 2^-107 above a midpoint, which this
// form resolves and a phase working to 2^-95 of the value would not.
CR_SLOW double exp_small(double x) {
  const dd q = two_prod(x, x);
  const double c3 = x * (x * x) * (1.0 / 6), c4 = (q.h * q.h) * (1.0 / 24);
  const dd D = two_sum(x, 0.5 * q.h);
  const double dl = D.l + ((0.5 * q.l + c4) + c3);
  const double grid = D.h >= 0 ? 0x1p52 : 0x1p53;
  const double uh = D.h * grid, ul = dl * grid;
  const double n = rint(uh);
  const double f = uh - n;                  // exact, |f| <= 1/2
  // the side of the midpoints n +- 1/2 (f -+ 1/2 exact for |f| >= 1/4; elsewhere far from them)
  const double k = ((f - 0.5) + ul > 0) ? n + 1 : (((f + 0.5) + ul < 0) ? n - 1 : n);
  return 1.0 + k / grid;
}

CR_SLOW double exp_cold(double x) {
  if (x != x) return x + x;
  if (x > 709.79) return 0x1p1023 * 2.0;  // overflow (and +inf)
  if (x < -708.3) return exp_tiny(x);
  return exp_small(x);                    // |x| < 2^-26
}

// e^x = 2^m 2^(j/64) e^r for -708.3 <= x <= 709.79 (a normal result): phase 1 of F, the rounding
// test, phase 2 on failure, then the exact scaling (overflow to infinity at the top).
CR_API double exp(double x) {
  const double ax = fabs(x);
  if (!(ax >= 0x1p-26 && x >= -708.3 && x <= 709.79)) return exp_cold(x);
  int m, j;
  double rh, rl;
  exp_reduce(x, m, j, rh, rl);
  const dd F = exp_phase1(j, rh, rl, false);
  double out;
  if (!rounds(F.h, F.l, F.h * kErr1, &out)) {
    const dd G = exp_phase2(j, rh, rl, false);
    if (!rounds(G.h, G.l, G.h * kErr2, &out)) out = G.h + G.l;
  }
  return scale_up(out, m);
}

}  // namespace cr
}  // namespace bmadgpu
