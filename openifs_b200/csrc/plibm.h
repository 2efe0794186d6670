/*
 * plibm.h -- portable double-precision exp and pow for CLOUDSC.
 *
 * Why this exists: CLOUDSC's outputs are sensitive to the last bit of its
 * exp/pow results (the sink-truncation sort and the MIN() limiters are
 * discontinuous at ties, and several process rates are differences such as
 * 1-EXP(x) with |x| tiny).  Two correct libms that differ by one or two ulp
 * (glibc vs CUDA, or glibc vs Intel's libimf) therefore give CLOUDSC results
 * that differ by up to ~1e-10 element-wise.  These functions use only IEEE
 * correctly-rounded +, -, *, /, and fused multiply-add, in a fixed order, so
 * they return bit-identical results on the host (C/C++, -ffp-contract=off)
 * and on the GPU (CUDA, --fmad=false): the B200 kernels and a CPU build of
 * the reference's algorithm linked against this file agree bit for bit.
 *
 * Methods (textbook, written for this project):
 *   exp(x): Cody-Waite reduction x = k*ln2 + r, |r| <= ln2/2, with a fused
 *           multiply-add and a two-part ln2; exp(r) = 1 + (r + r^2 P(r)) with
 *           P the Taylor series 1/2! .. 1/13! (truncation < 5e-18); scaling
 *           by 2^k through the exponent field.
 *   log(x) (double-double, for pow): x = m 2^e with m in [sqrt(1/2), sqrt(2)),
 *           s = (m-1)/(m+1) carried as s_hi + s_lo, log m = 2 atanh(s) =
 *           2s + s^3 T(s^2) with T the atanh series 2/3, 2/5, .. 2/23
 *           (|s| <= 0.1716, truncation < 1e-19), plus e*ln2 in two parts.
 *   pow(x,y) = exp(y * log(x)) with y*log(x) formed as a double-double and
 *           its low part added to the reduced argument.
 * Accuracy (tests/test_plibm.py, against glibc): exp within 1 ulp, pow within
 * 2 ulp over the argument ranges CLOUDSC uses.
 * Domain: pow is evaluated for x >= 0 (every CLOUDSC base is >= 0); x < 0
 * returns NaN, x = 0 returns 0 for y > 0, +inf for y < 0, 1 for y = 0.
 */
#ifndef CLOUDSC_PLIBM_H
#define CLOUDSC_PLIBM_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define PLIBM_FN static __host__ __device__ __forceinline__
#else
#define PLIBM_FN static inline
#endif

PLIBM_FN uint64_t plibm_bits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  memcpy(&u, &x, 8);
  return u;
#endif
}
PLIBM_FN double plibm_from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x;
  memcpy(&x, &u, 8);
  return x;
#endif
}
PLIBM_FN double plibm_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}

#define PLIBM_INV_LN2 0x1.71547652b82fep+0
#define PLIBM_LN2_HI 0x1.62e42fefa39efp-1
#define PLIBM_LN2_LO 0x1.abc9e3b39803fp-56
#define PLIBM_LN2_HI42 0x1.62e42fefa3800p-1 /* 42 significant bits: e*HI42 exact */
#define PLIBM_LN2_LO42 0x1.ef35793c76730p-45
#define PLIBM_SHIFT 0x1.8p52

/* 2^k for -1022 <= k <= 1023 */
PLIBM_FN double plibm_pow2i(int k) { return plibm_from_bits((uint64_t)(k + 1023) << 52); }

/* exp(hi + lo) for |lo| <= ~1e-16 |hi|; the kernel of both exp and pow. */
PLIBM_FN double plibm_exp_dd(double hi, double lo) {
  if (hi != hi) return hi + hi;
  if (hi > 709.8) return HUGE_VAL;
  if (hi < -745.2) return 0.0;
  double kd = plibm_fma(hi, PLIBM_INV_LN2, PLIBM_SHIFT);
  int k = (int)((int64_t)(plibm_bits(kd) & 0xfffffffffffffULL) - (int64_t)(1LL << 51));
  kd = kd - PLIBM_SHIFT;
  double r = plibm_fma(-kd, PLIBM_LN2_HI, hi);
  r = plibm_fma(-kd, PLIBM_LN2_LO, r);
  r = r + lo;
  double p = 0x1.6124613a86d09p-33;          /* 1/13! */
  p = plibm_fma(p, r, 0x1.1eed8eff8d898p-29); /* 1/12! */
  p = plibm_fma(p, r, 0x1.ae64567f544e4p-26); /* 1/11! */
  p = plibm_fma(p, r, 0x1.27e4fb7789f5cp-22); /* 1/10! */
  p = plibm_fma(p, r, 0x1.71de3a556c734p-19); /* 1/9!  */
  p = plibm_fma(p, r, 0x1.a01a01a01a01ap-16); /* 1/8!  */
  p = plibm_fma(p, r, 0x1.a01a01a01a01ap-13); /* 1/7!  */
  p = plibm_fma(p, r, 0x1.6c16c16c16c17p-10); /* 1/6!  */
  p = plibm_fma(p, r, 0x1.1111111111111p-7);  /* 1/5!  */
  p = plibm_fma(p, r, 0x1.5555555555555p-5);  /* 1/4!  */
  p = plibm_fma(p, r, 0x1.5555555555555p-3);  /* 1/3!  */
  p = plibm_fma(p, r, 0x1.0000000000000p-1);  /* 1/2!  */
  double q = r * r;
  double e = 1.0 + plibm_fma(q, p, r);
  if (k >= -1021 && k <= 1023) return e * plibm_pow2i(k);
  /* near the overflow / underflow thresholds: scale in two exact steps */
  if (k > 1023) return (e * plibm_pow2i(k - 512)) * plibm_pow2i(512);
  return (e * plibm_pow2i(k + 512)) * plibm_pow2i(-512);
}

PLIBM_FN double plibm_exp(double x) { return plibm_exp_dd(x, 0.0); }

/* log(x) as hi + lo for finite x > 0. */
PLIBM_FN void plibm_log_dd(double x, double *hi, double *lo) {
  uint64_t u = plibm_bits(x);
  int e = 0;
  if ((u >> 52) == 0) { /* subnormal */
    x = x * 0x1p54;
    u = plibm_bits(x);
    e = -54;
  }
  e += (int)(u >> 52) - 1023;
  double m = plibm_from_bits((u & 0xfffffffffffffULL) | 0x3ff0000000000000ULL); /* [1,2) */
  if (m > 0x1.6a09e667f3bcdp+0) { /* > sqrt(2): use m/2 */
    m = m * 0.5;
    e += 1;
  }
  double f = m - 1.0; /* exact */
  /* d = m + 1 as d_hi + d_lo (two-sum) */
  double d_hi = m + 1.0;
  double bb = d_hi - m;
  double d_lo = (m - (d_hi - bb)) + (1.0 - bb);
  double rcp = 1.0 / d_hi;
  double s_hi = f * rcp;
  double rem = plibm_fma(-s_hi, d_hi, f);
  rem = plibm_fma(-s_hi, d_lo, rem);
  double s_lo = rem * rcp;
  double z = s_hi * s_hi;
  double t = 0x1.642c8590b2164p-4;   /* 2/23 */
  t = plibm_fma(t, z, 0x1.8618618618618p-4); /* 2/21 */
  t = plibm_fma(t, z, 0x1.af286bca1af28p-4); /* 2/19 */
  t = plibm_fma(t, z, 0x1.e1e1e1e1e1e1ep-4); /* 2/17 */
  t = plibm_fma(t, z, 0x1.1111111111111p-3); /* 2/15 */
  t = plibm_fma(t, z, 0x1.3b13b13b13b14p-3); /* 2/13 */
  t = plibm_fma(t, z, 0x1.745d1745d1746p-3); /* 2/11 */
  t = plibm_fma(t, z, 0x1.c71c71c71c71cp-3); /* 2/9  */
  t = plibm_fma(t, z, 0x1.2492492492492p-2); /* 2/7  */
  t = plibm_fma(t, z, 0x1.999999999999ap-2); /* 2/5  */
  t = plibm_fma(t, z, 0x1.5555555555555p-1); /* 2/3  */
  double tail = (z * s_hi) * t;
  double ed = (double)e;
  double a_hi = ed * PLIBM_LN2_HI42; /* exact */
  double b_hi = 2.0 * s_hi;          /* exact */
  double sum = a_hi + b_hi;          /* two-sum */
  double bv = sum - a_hi;
  double err = (a_hi - (sum - bv)) + (b_hi - bv);
  double low = err + (ed * PLIBM_LN2_LO42 + (2.0 * s_lo + tail));
  double h = sum + low; /* fast two-sum renormalisation */
  *lo = low - (h - sum);
  *hi = h;
}

PLIBM_FN double plibm_pow(double x, double y) {
  if (x != x || y != y) return x + y;
  if (y == 0.0) return 1.0;
  if (x < 0.0) return (x - x) / (x - x); /* NaN: CLOUDSC never raises a negative base */
  if (x == 0.0) return y > 0.0 ? 0.0 : HUGE_VAL;
  if (x == HUGE_VAL) return y > 0.0 ? HUGE_VAL : 0.0;
  double lhi, llo;
  plibm_log_dd(x, &lhi, &llo);
  double t_hi = y * lhi;
  double t_lo = plibm_fma(y, lhi, -t_hi) + y * llo;
  return plibm_exp_dd(t_hi, t_lo);
}

/* pow with a precomputed double-double log of the base (shared-base calls). */
PLIBM_FN double plibm_pow_log(double lhi, double llo, double y) {
  double t_hi = y * lhi;
  double t_lo = plibm_fma(y, lhi, -t_hi) + y * llo;
  return plibm_exp_dd(t_hi, t_lo);
}

#endif /* CLOUDSC_PLIBM_H */
