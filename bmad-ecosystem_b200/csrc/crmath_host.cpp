// crmath_host.cpp -- TEST-ONLY host build of the correctly rounded functions (crmath.cuh).
//
// The CPU tests check them against mpmath; the oracle's correctly rounded mode takes its libm
// from here. Built into _build/libbmadgpu_crmath.so, which the product never loads.
#include <quadmath.h>

#include "crmath.cuh"

extern "C" {
double bmadgpu_cr_sin(double x) { return bmadgpu::cr::sin(x); }
double bmadgpu_cr_cos(double x) { return bmadgpu::cr::cos(x); }
double bmadgpu_cr_asin(double x) { return bmadgpu::cr::asin(x); }
double bmadgpu_cr_atan2(double y, double x) { return bmadgpu::cr::atan2(y, x); }
double bmadgpu_cr_sinh(double x) { return bmadgpu::cr::sinh(x); }
double bmadgpu_cr_cosh(double x) { return bmadgpu::cr::cosh(x); }
double bmadgpu_cr_exp(double x) { return bmadgpu::cr::exp(x); }
double bmadgpu_cr_tan(double x) { return bmadgpu::cr::tan(x); }
void bmadgpu_cr_sincos(double x, double* s, double* c) { bmadgpu::cr::sincos(x, s, c); }
void bmadgpu_cr_sinhcosh(double x, double* s, double* c) { bmadgpu::cr::sinhcosh(x, s, c); }

// An independent correctly rounded set for cross-checks: libquadmath's 113-bit functions rounded
// once to double (a wrong rounding needs a value within 2^-112 of a midpoint between doubles).
double bmadgpu_q_sin(double x) { return (double)sinq((__float128)x); }
double bmadgpu_q_cos(double x) { return (double)cosq((__float128)x); }
double bmadgpu_q_asin(double x) { return (double)asinq((__float128)x); }
double bmadgpu_q_atan2(double y, double x) { return (double)atan2q((__float128)y, (__float128)x); }
double bmadgpu_q_sinh(double x) { return (double)sinhq((__float128)x); }
double bmadgpu_q_cosh(double x) { return (double)coshq((__float128)x); }
double bmadgpu_q_exp(double x) { return (double)expq((__float128)x); }
double bmadgpu_q_tan(double x) { return (double)tanq((__float128)x); }

// Vector forms for the tests: fn 0 sin, 1 cos, 2 asin, 3 atan2(y = a, x = b), 4 sinh, 5 cosh,
// 8 exp, 9 tan.
void bmadgpu_cr_eval_host(int fn, const double* a, const double* b, double* out, long n) {
  for (long i = 0; i < n; i++) {
    switch (fn) {
      case 0: out[i] = bmadgpu::cr::sin(a[i]); break;
      case 1: out[i] = bmadgpu::cr::cos(a[i]); break;
      case 2: out[i] = bmadgpu::cr::asin(a[i]); break;
      case 3: out[i] = bmadgpu::cr::atan2(a[i], b[i]); break;
      case 4: out[i] = bmadgpu::cr::sinh(a[i]); break;
      case 8: out[i] = bmadgpu::cr::exp(a[i]); break;
      case 9: out[i] = bmadgpu::cr::tan(a[i]); break;
      default: out[i] = bmadgpu::cr::cosh(a[i]); break;
    }
  }
}
}
