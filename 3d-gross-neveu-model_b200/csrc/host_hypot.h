// host_hypot.h -- |z| of a complex double exactly as the host C library
// computes it (cabs / hypot of glibc 2.35 and later on x86-64, the libm the
// reference's conjugategradient.c:65 runs on), for the exact-order mode.
//
// That libm's hypot is not correctly rounded: it is the corrected algorithm
// without fused multiply-add of C. F. Borges, "An Improved Algorithm for
// hypot(a, b)", ACM Trans. Math. Softw. 47(1), 2021 (arXiv:1904.09481).  With
// a >= b >= 0, h = sqrt(a^2 + b^2) is refined by one Newton step,
// h -= r / (2h), where r = h^2 - a^2 - b^2 is evaluated without FMA from the
// exact difference d = h - b (when h <= 2b) or d = h - a (otherwise):
//   h <= 2b:  r = a (2d - a) + (d - 2(a - b)) d
//   h >  2b:  r = 2d (a - 2b) + ((4d - b) b + d^2)
// The evaluation order above reproduces the library's results (checked against
// it on 2e8 random pairs spanning 2^-60 .. 2^20, tests/test_host_hypot.py).
// The scaling the library applies near overflow and underflow is not needed
// for the magnitudes of a solver's vectors and is left out.
// Must be compiled without floating-point contraction (--fmad=false /
// -ffp-contract=off).
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define GN_HD __host__ __device__ __forceinline__
#else
#define GN_HD static inline
#endif

GN_HD double gn_host_hypot(double x, double y) {
  double a = fabs(x), b = fabs(y);
  if (a < b) {
    const double t = a;
    a = b;
    b = t;
  }
  if (b == 0.0) return a;
  const double h = sqrt(a * a + b * b);
  double r;
  if (h <= 2.0 * b) {
    const double d = h - b;
    r = a * (2.0 * d - a) + (d - 2.0 * (a - b)) * d;
  } else {
    const double d = h - a;
    r = 2.0 * d * (a - 2.0 * b) + ((4.0 * d - b) * b + d * d);
  }
  return h - r / (2.0 * h);
}

#undef GN_HD
