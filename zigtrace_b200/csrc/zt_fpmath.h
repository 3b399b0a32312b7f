/*
 * zt_fpmath.h -- f64 transcendental routines shared by the CUDA renderer and
 * the CPU oracle.
 *
 * The reference calls Zig's `@sin`/`@cos` (src/rng.zig:62, src/light.zig:295)
 * and `std.math.pow(f64, x, 5)` (src/material.zig:69).  Those come from the
 * Zig 0.14 standard library / compiler-rt, which is not available here.  To
 * make the device path and the CPU oracle agree bit for bit, both evaluate the
 * functions below with the same sequence of IEEE-754 double operations
 * (compile with FMA contraction off: `-ffp-contract=off` on the host,
 * `-fmad=false` on the device).
 *
 * sin/cos: Cody-Waite reduction by pi/2 with a three-part split of pi/2
 * (P1 and P2 carry 33 significant bits, so k*P1 and k*P2 are exact for
 * |k| < 2^20), followed by the Maclaurin series of sin and cos on
 * [-pi/4, pi/4] in Horner form.  The truncation error of the series there is
 * below 2^-60 relative; the evaluation error is about one ulp.  Domain:
 * |x| < 2^19 (the renderer only passes angles in [0, 2*pi)).
 *
 * pow5: std.math.pow for a positive integer exponent is binary exponentiation
 * on the frexp significand (the Go math.Pow algorithm that Zig's pow.zig
 * restates).  For y = 5 that is m * ((m*m)*(m*m)) with the power-of-two
 * rescalings exact, i.e. x * ((x*x)*(x*x)) for every normal result, and
 * pow(1, 5) = 1, pow(0, 5) = 0 from its special cases.
 */
#ifndef ZT_FPMATH_H
#define ZT_FPMATH_H

#include <math.h>

#if defined(__CUDACC__)
#define ZT_FPM_HD __host__ __device__ __forceinline__
#else
#define ZT_FPM_HD static inline
#endif

/* pi/2 = ZT_PIO2_1 + ZT_PIO2_2 + ZT_PIO2_3 (+ 1e-37). */
#define ZT_PIO2_1 1.5707963267341256      /* 0x1.921fb544p+0, 33 bits */
#define ZT_PIO2_2 6.077100506303966e-11   /* 0x1.0b4611a6p-34, 33 bits */
#define ZT_PIO2_3 2.0222662487959506e-21  /* 0x1.3198a2e037073p-69 */
#define ZT_2_OVER_PI 0.6366197723675814   /* 0x1.45f306dc9c883p-1 */

/* sin(r) = r + r^3 * S(r^2), S(z) = -1/3! + z/5! - ... + z^8/19! */
ZT_FPM_HD double zt_sin_poly(double r) {
  const double z = r * r;
  double p = -8.22063524662433e-18;        /* -1/19! */
  p = p * z + 2.8114572543455206e-15;      /*  1/17! */
  p = p * z + -7.647163731819816e-13;      /* -1/15! */
  p = p * z + 1.6059043836821613e-10;      /*  1/13! */
  p = p * z + -2.505210838544172e-08;      /* -1/11! */
  p = p * z + 2.7557319223985893e-06;      /*  1/9!  */
  p = p * z + -0.0001984126984126984;      /* -1/7!  */
  p = p * z + 0.008333333333333333;        /*  1/5!  */
  p = p * z + -0.16666666666666666;        /* -1/3!  */
  return r + (r * z) * p;
}

/* cos(r) = (1 - r^2/2) + r^4 * C(r^2), C(z) = 1/4! - z/6! + ... - z^7/18! */
ZT_FPM_HD double zt_cos_poly(double r) {
  const double z = r * r;
  double p = -1.5619206968586225e-16;      /* -1/18! */
  p = p * z + 4.779477332387385e-14;       /*  1/16! */
  p = p * z + -1.1470745597729725e-11;     /* -1/14! */
  p = p * z + 2.08767569878681e-09;        /*  1/12! */
  p = p * z + -2.755731922398589e-07;      /* -1/10! */
  p = p * z + 2.48015873015873e-05;        /*  1/8!  */
  p = p * z + -0.001388888888888889;       /* -1/6!  */
  p = p * z + 0.041666666666666664;        /*  1/4!  */
  const double hz = 0.5 * z;
  return (1.0 - hz) + (z * z) * p;
}

/* Reduces x to r in [-pi/4, pi/4] and returns the quadrant k mod 4. */
ZT_FPM_HD int zt_reduce_pio2(double x, double* r) {
  const double kd = floor(x * ZT_2_OVER_PI + 0.5);
  double t = x - kd * ZT_PIO2_1;
  t = t - kd * ZT_PIO2_2;
  t = t - kd * ZT_PIO2_3;
  *r = t;
  long long k = (long long)kd;
  return (int)(k & 3);
}

ZT_FPM_HD void zt_sincos(double x, double* s, double* c) {
  double r;
  const int q = zt_reduce_pio2(x, &r);
  const double sr = zt_sin_poly(r);
  const double cr = zt_cos_poly(r);
  switch (q) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
  }
}

ZT_FPM_HD double zt_sin(double x) {
  double s, c;
  zt_sincos(x, &s, &c);
  return s;
}

ZT_FPM_HD double zt_cos(double x) {
  double s, c;
  zt_sincos(x, &s, &c);
  return c;
}

/* std.math.pow(f64, x, 5) for the Schlick term (x = 1 - cos in [0, 2]). */
ZT_FPM_HD double zt_pow5(double x) {
  if (x == 1.0) return 1.0;
  const double x2 = x * x;
  const double x4 = x2 * x2;
  return x * x4;
}

#endif /* ZT_FPMATH_H */
