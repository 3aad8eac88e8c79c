// Deterministic FP64 elementary functions for the FELIS slice loop.
//
// Every function here is written with +, -, *, /, sqrt, rint and explicit
// fma() only, in a fixed evaluation order.  IEEE-754 gives those operations a
// single correctly rounded result, so the same source evaluated by the host
// compiler (g++ with -ffp-contract=off) and by nvcc for sm_100a (with
// --fmad=false) returns bit-identical values.  That is what lets the FP64
// plain GPU path reproduce the CPU restatement of the reference bit for bit:
// the reference evaluates std::exp(I*phase), std::atan and std::atan2 on every
// particle of every step (particlePush.cpp:274-278,334,361;
// solveField.cpp:261-266,301,336,344) and SASE amplifies last-bit
// differences in those calls.
//
// Methods (all public textbook material, constants derived from pi to 300 bits
// with mpmath; none is taken from any vendor library):
//   * sin/cos: Cody & Waite three-part reduction by pi/2 (two 33-bit parts,
//     so k*P1 and k*P2 are exact for |k| < 2^20), then Taylor series of
//     sin (through r^19) and cos (through r^20) on |r| <= pi/4 + eps, which
//     truncate below 2^-60 relative.  Quadrant from k mod 4.
//   * atan: reciprocal reduction atan(x) = pi/2 - atan(1/x) for |x| > 1,
//     then the addition formula atan(x) = atan(c) + atan((x-c)/(1+x c)) with
//     c = k/8 nearest to x, so |u| <= 1/16, then the odd Taylor series of
//     atan(u) through u^17.  atan(k/8) is stored as a hi+lo pair.
//   * atan2: quadrant logic on top of atan(y/x) (C99 Annex F special cases
//     for zeros; infinities are not expected on this path).
// Accuracy against glibc: <= 2 ulp on the ranges the slice loop uses
// (checked by tests/test_detmath.py); for |x| >= 2^20*pi/2 the sin/cos
// reduction loses accuracy but stays deterministic.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define FM_HD __host__ __device__ __forceinline__
#else
#define FM_HD static inline
#endif

namespace fm {

// pi/2 = P1 + P2 + P3 (P1, P2 carry 33 significant bits each).
#define FM_PIO2_1 0x1.921fb544p+0
#define FM_PIO2_2 0x1.0b4611a6p-34
#define FM_PIO2_3 0x1.3198a2e037073p-69
#define FM_2_OVER_PI 0x1.45f306dc9c883p-1
#define FM_PIO2_HI 0x1.921fb54442d18p+0
#define FM_PIO2_LO 0x1.1a62633145c07p-54

// sin(r) and cos(r) for |r| <= pi/4 (+ a few ulp).
FM_HD void sincos_kernel(double r, double* s, double* c) {
  const double z = r * r;
  // sin: r + r*z*(-1/3! + z*(1/5! + z*(-1/7! + ...)))
  double ps = -0x1.2f49b46814157p-57;       // -1/19!
  ps = fma(ps, z, 0x1.952c77030ad4ap-49);   // +1/17!
  ps = fma(ps, z, -0x1.ae7f3e733b81fp-41);  // -1/15!
  ps = fma(ps, z, 0x1.6124613a86d09p-33);   // +1/13!
  ps = fma(ps, z, -0x1.ae64567f544e4p-26);  // -1/11!
  ps = fma(ps, z, 0x1.71de3a556c734p-19);   // +1/9!
  ps = fma(ps, z, -0x1.a01a01a01a01ap-13);  // -1/7!
  ps = fma(ps, z, 0x1.1111111111111p-7);    // +1/5!
  ps = fma(ps, z, -0x1.5555555555555p-3);   // -1/3!
  *s = fma(r * z, ps, r);
  // cos: 1 - z/2 + z*z*(1/4! + z*(-1/6! + ...))
  double pc = 0x1.e542ba4020225p-62;        // +1/20!
  pc = fma(pc, z, -0x1.6827863b97d97p-53);  // -1/18!
  pc = fma(pc, z, 0x1.ae7f3e733b81fp-45);   // +1/16!
  pc = fma(pc, z, -0x1.93974a8c07c9dp-37);  // -1/14!
  pc = fma(pc, z, 0x1.1eed8eff8d898p-29);   // +1/12!
  pc = fma(pc, z, -0x1.27e4fb7789f5cp-22);  // -1/10!
  pc = fma(pc, z, 0x1.a01a01a01a01ap-16);   // +1/8!
  pc = fma(pc, z, -0x1.6c16c16c16c17p-10);  // -1/6!
  pc = fma(pc, z, 0x1.5555555555555p-5);    // +1/4!
  const double hz = 0.5 * z;
  const double w = 1.0 - hz;
  // (1 - w) - hz recovers the rounding error of w exactly (Sterbenz).
  *c = w + (((1.0 - w) - hz) + z * z * pc);
}

// sin(x), cos(x) for finite x.
FM_HD void sincos(double x, double* s, double* c) {
  const double k = rint(x * FM_2_OVER_PI);
  double r = x - k * FM_PIO2_1;  // exact: k*P1 exact, Sterbenz for the difference
  r = r - k * FM_PIO2_2;         // k*P2 exact
  r = r - k * FM_PIO2_3;
  double sr, cr;
  sincos_kernel(r, &sr, &cr);
  const long long q = ((long long)k) & 3;
  if (q == 0) { *s = sr;  *c = cr; }
  else if (q == 1) { *s = cr;  *c = -sr; }
  else if (q == 2) { *s = -sr; *c = -cr; }
  else { *s = -cr; *c = sr; }
}

// atan(u) for |u| <= 1/16 (odd Taylor series through u^17).
FM_HD double atan_kernel(double u) {
  const double z = u * u;
  double p = 1.0 / 17.0;
  p = fma(p, z, -1.0 / 15.0);
  p = fma(p, z, 1.0 / 13.0);
  p = fma(p, z, -1.0 / 11.0);
  p = fma(p, z, 1.0 / 9.0);
  p = fma(p, z, -1.0 / 7.0);
  p = fma(p, z, 1.0 / 5.0);
  p = fma(p, z, -1.0 / 3.0);
  return fma(u * z, p, u);
}

FM_HD double atan_table_hi(int k) {
  switch (k) {
    case 1: return 0x1.fd5ba9aac2f6ep-4;
    case 2: return 0x1.f5b75f92c80ddp-3;
    case 3: return 0x1.6f61941e4def1p-2;
    case 4: return 0x1.dac670561bb4fp-2;
    case 5: return 0x1.1e00babdefeb4p-1;
    case 6: return 0x1.4978fa3269ee1p-1;
    case 7: return 0x1.700a7c5784634p-1;
    case 8: return 0x1.921fb54442d18p-1;
    default: return 0.0;
  }
}
FM_HD double atan_table_lo(int k) {
  switch (k) {
    case 1: return -0x1.cd37686760c17p-59;
    case 2: return 0x1.8ab6e3cf7afbdp-57;
    case 3: return -0x1.c63aae6f6e918p-56;
    case 4: return 0x1.a2b7f222f65e2p-56;
    case 5: return -0x1.928df287a668fp-58;
    case 6: return 0x1.2419a87f2a458p-56;
    case 7: return -0x1.8c34d25aadef6p-56;
    case 8: return 0x1.1a62633145c07p-55;
    default: return 0.0;
  }
}

// atan(t) for 0 <= t <= 1.
FM_HD double atan_unit(double t) {
  const int k = (int)rint(t * 8.0);
  if (k == 0) return atan_kernel(t);
  const double c = 0.125 * (double)k;
  const double u = (t - c) / (1.0 + t * c);
  return atan_table_hi(k) + (atan_table_lo(k) + atan_kernel(u));
}

FM_HD double atan(double x) {
  if (x != x) return x;
  const double ax = fabs(x);
  double r;
  if (ax <= 1.0) {
    r = atan_unit(ax);
  } else {
    const double t = 1.0 / ax;
    r = FM_PIO2_HI - (atan_unit(t) - FM_PIO2_LO);
  }
  return x < 0.0 ? -r : r;
}

FM_HD double atan2(double y, double x) {
  if (x != x || y != y) return x + y;
  const double pi_hi = 0x1.921fb54442d18p+1, pi_lo = 0x1.1a62633145c07p-53;
  if (y == 0.0) {
    if (signbit(x)) return signbit(y) ? -pi_hi : pi_hi;
    return y;  // +-0
  }
  if (x == 0.0) return y > 0.0 ? FM_PIO2_HI : -FM_PIO2_HI;
  const double ay = fabs(y), ax = fabs(x);
  double r;
  if (ay <= ax) {
    r = atan_unit(ay / ax);
  } else {
    r = FM_PIO2_HI - (atan_unit(ax / ay) - FM_PIO2_LO);
  }
  if (x < 0.0) r = pi_hi - (r - pi_lo);
  return y < 0.0 ? -r : r;
}

}  // namespace fm
