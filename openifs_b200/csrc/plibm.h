/*
 * plibm.h -- portable double-precision exp and pow for CLOUDSC.
 *
 * Why this exists: CLOUDSC's outputs are sensitive to the last bit of its
 * exp/pow results (the sink-truncation sort and the MIN() limiters are
 * discontinuous at ties, and several process rates are differences such as
 * 1-EXP(x) with |x| tiny).  Two correct libms that differ by one or two ulp
 * (glibc vs CUDA, or glibc vs Intel's libimf) therefore give CLOUDSC results
 * that differ by up to ~1e-10 element-wise.  These functions use only IEEE
 * correctly-rounded +, -, *, /, sqrt and fused multiply-add, in a fixed order,
 * so they return bit-identical results on the host (C/C++, -ffp-contract=off)
 * and on the GPU (CUDA, --fmad=false): the B200 kernels and a CPU build of
 * the reference's algorithm linked against this file agree bit for bit.
 *
 * Methods (textbook, written for this project; tables in plibm_tables.h,
 * generated exactly by make_plibm_tables.py):
 *   exp(x): x = (128 m + j) ln2/128 + r, |r| <= ln2/256, with a two-part
 *           ln2/128 and fused multiply-adds; exp(x) = 2^m (T_j + T_j p(r))
 *           where T_j = 2^(j/128) is stored as hi + lo and p(r) = expm1(r) is
 *           its Taylor polynomial to degree 5 (truncation < 6e-19).
 *   log(x) (double-double, for pow): x = 2^e m, m in [1,2); with the top 7
 *           mantissa bits j, m*INVC_j = 1 + r, |r| <= 2^-8, formed exactly
 *           with a fused multiply-add; ln x = e ln2 + (-ln INVC_j) + ln(1+r),
 *           ln(1+r) by its series to r^7/7 (absolute truncation < 2^-64),
 *           summed as a double-double.
 *   log(x) = the high part of that double-double (for the one LOG CLOUDSC calls).
 *   pow(x,y) = exp(y ln x) with y ln x a double-double whose low part enters
 *           the reduced exp argument; exponents 0.5, 1.5, 2 and 3 are
 *           evaluated from sqrt(x) and products, the last two with their
 *           rounding errors carried (fused multiply-adds) so that each
 *           result is rounded once.
 * The code paths are branch-free (special inputs are fixed up with selects),
 * so a compiler can interleave independent calls.
 * Accuracy (tests/test_plibm.py, against glibc): exp within 1 ulp, pow within
 * 2 ulp over the argument ranges CLOUDSC uses.
 * Domain: CLOUDSC raises only non-negative bases; pow returns NaN for x < 0,
 * 0 / +inf / 1 for x = 0 and y > 0 / y < 0 / y = 0, and 1 for y = 0.
 */
#ifndef CLOUDSC_PLIBM_H
#define CLOUDSC_PLIBM_H

#include <stdint.h>
#include <string.h>
#include <math.h>
#include "plibm_tables.h"

#if defined(__CUDACC__)
#define PLIBM_FN static __host__ __device__ __forceinline__
#if defined(PLIBM_DEVICE_NOINLINE)
#define PLIBM_FN_HEAVY static __host__ __device__ __noinline__
#else
#define PLIBM_FN_HEAVY PLIBM_FN
#endif
#else
#define PLIBM_FN static inline
#define PLIBM_FN_HEAVY static inline
#endif
/* The rarely taken full paths (extreme arguments, special values) are kept
 * out of line on the device, so each inlined call site carries only the
 * common path. */
#if defined(__CUDACC__)
#define PLIBM_FN_COLD static __host__ __device__ __noinline__
#else
#define PLIBM_FN_COLD static
#endif

/* The tables: one copy for host code, one in device global memory (read
 * through the read-only data cache). */
static const double plibm_exp_tbl[256] = PLIBM_EXP_TBL_INIT;
static const double plibm_log_tbl[384] = PLIBM_LOG_TBL_INIT;
#if defined(__CUDACC__)
static __device__ const double plibm_exp_tbl_d[256] = PLIBM_EXP_TBL_INIT;
static __device__ const double plibm_log_tbl_d[384] = PLIBM_LOG_TBL_INIT;
#endif

/* With PLIBM_SMEM_TABLES, device code reads per-CTA shared-memory copies of
 * the tables, which every kernel that calls plibm fills first with
 * plibm_load_tables() (all threads of the CTA, then a CTA barrier). */
#if defined(__CUDACC__) && defined(PLIBM_SMEM_TABLES)
static __shared__ double plibm_exp_tbl_s[256];
static __shared__ double plibm_log_tbl_s[384];
static __device__ __forceinline__ void plibm_load_tables() {
  for (int i = threadIdx.x; i < 256; i += blockDim.x) plibm_exp_tbl_s[i] = plibm_exp_tbl_d[i];
  for (int i = threadIdx.x; i < 384; i += blockDim.x) plibm_log_tbl_s[i] = plibm_log_tbl_d[i];
  __syncthreads();
}
#endif

PLIBM_FN double plibm_exp_t(int i) {
#if defined(__CUDA_ARCH__) && defined(PLIBM_SMEM_TABLES)
  return plibm_exp_tbl_s[i];
#elif defined(__CUDA_ARCH__)
  return __ldg(&plibm_exp_tbl_d[i]);
#else
  return plibm_exp_tbl[i];
#endif
}
PLIBM_FN double plibm_log_t(int i) {
#if defined(__CUDA_ARCH__) && defined(PLIBM_SMEM_TABLES)
  return plibm_log_tbl_s[i];
#elif defined(__CUDA_ARCH__)
  return __ldg(&plibm_log_tbl_d[i]);
#else
  return plibm_log_tbl[i];
#endif
}

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
PLIBM_FN double plibm_sqrt(double x) {
#if defined(__CUDA_ARCH__)
  return __dsqrt_rn(x);
#else
  return sqrt(x);
#endif
}

#define PLIBM_INV_LN2_128 0x1.71547652b82fep+7 /* 128/ln2 */
#define PLIBM_LN2_128_HI 0x1.62e42fefa39efp-8  /* ln2/128 in two parts */
#define PLIBM_LN2_128_LO 0x1.abc9e3b39803fp-63
#define PLIBM_LN2_HI42 0x1.62e42fefa3800p-1 /* ln2, 42 significant bits: e*HI42 is exact */
#define PLIBM_LN2_LO42 0x1.ef35793c76730p-45
#define PLIBM_SHIFT 0x1.8p52
#define PLIBM_INF (plibm_from_bits(0x7ff0000000000000ULL))
#define PLIBM_NAN (plibm_from_bits(0x7ff8000000000000ULL))

/* 2^k for -1022 <= k <= 1023 */
PLIBM_FN double plibm_pow2i(int k) { return plibm_from_bits((uint64_t)(int64_t)(k + 1023) << 52); }

/* exp(hi + lo) for |lo| <= ~1e-15 |hi|, every hi; the kernel of both exp and
 * pow.  Straight-line code (no branch), so that a compiler can interleave
 * independent calls: the argument is clamped to [-746, 709.9] (the result
 * then overflows or underflows as it should) and the scale 2^m is applied as
 * two exact factors 2^(m>>1) 2^(m-(m>>1)), each a normal number for every m
 * the clamped argument gives; NaN is passed through by a select.  The table
 * index j is in [0, 127] for every input, NaN included.  (For -700 < hi <
 * 700, 2^m e is normal and the two factors give exactly the bits of adding m
 * to e's exponent field.)  use_lo = 0 skips the addition of lo = 0, which
 * changes r only for r = -0, where expm1(-0) and expm1(+0) give the same
 * sum s. */
PLIBM_FN_HEAVY double plibm_exp_core(double hi, double lo, int use_lo) {
  double hc = hi > 709.9 ? 709.9 : hi;
  hc = hc < -746.0 ? -746.0 : hc;
  double kd = plibm_fma(hc, PLIBM_INV_LN2_128, PLIBM_SHIFT);
  int64_t ki = (int64_t)(plibm_bits(kd) & 0xfffffffffffffULL) - (int64_t)(1LL << 51);
  kd = kd - PLIBM_SHIFT;
  double r = plibm_fma(-kd, PLIBM_LN2_128_HI, hc);
  r = plibm_fma(-kd, PLIBM_LN2_128_LO, r);
  if (use_lo) r = r + lo;
  int j = (int)(ki & 127);
  int m = (int)(ki >> 7);
  double thi = plibm_exp_t(2 * j), tlo = plibm_exp_t(2 * j + 1);
  double p = plibm_fma(r, 0x1.1111111111111p-7, 0x1.5555555555555p-5); /* 1/120, 1/24 */
  p = plibm_fma(p, r, 0x1.5555555555555p-3);                          /* 1/6 */
  p = plibm_fma(p, r, 0x1.0000000000000p-1);                          /* 1/2 */
  p = plibm_fma(p, r * r, r);                                         /* expm1(r) */
  double s = plibm_fma(thi, p, tlo);
  double e = thi + s;
  int m1 = m >> 1, m2 = m - (m >> 1);
  double res = (e * plibm_pow2i(m1)) * plibm_pow2i(m2);
  return hi != hi ? hi : res;
}
PLIBM_FN double plibm_exp_dd(double hi, double lo) { return plibm_exp_core(hi, lo, 1); }

/* exp(x): lo = 0 needs no addition. */
PLIBM_FN double plibm_exp(double x) { return plibm_exp_core(x, 0.0, 0); }

/* ln(x) as hi + lo for finite x > 0. */
PLIBM_FN_HEAVY void plibm_log_dd(double x, double *hi, double *lo) {
  uint64_t u = plibm_bits(x);
  int e = -1023;
  if ((u >> 52) == 0) { /* subnormal (or zero): scale into the normal range */
    u = plibm_bits(x * 0x1p54);
    e -= 54;
  }
  e += (int)(u >> 52);
  uint64_t mant = u & 0xfffffffffffffULL;
  int j = (int)(mant >> 45);
  double m = plibm_from_bits(mant | 0x3ff0000000000000ULL);
  double invc = plibm_log_t(3 * j), lchi = plibm_log_t(3 * j + 1), lclo = plibm_log_t(3 * j + 2);
  double p = m * invc;
  double perr = plibm_fma(m, invc, -p); /* m*invc = p + perr exactly */
  double r1 = p - 1.0;                  /* exact */
  double q = plibm_fma(r1, 0x1.2492492492492p-3, -0x1.5555555555555p-3); /* 1/7, -1/6 */
  q = plibm_fma(q, r1, 0x1.999999999999ap-3);                           /* 1/5 */
  q = plibm_fma(q, r1, -0x1.0000000000000p-2);                          /* -1/4 */
  q = plibm_fma(q, r1, 0x1.5555555555555p-2);                           /* 1/3 */
  q = plibm_fma(q, r1, -0x1.0000000000000p-1);                          /* -1/2 */
  double poly = q * (r1 * r1);
  double corr = plibm_fma(-perr, r1, perr);
  double ed = (double)e;
  double a = ed * PLIBM_LN2_HI42; /* exact */
  /* a + lchi exactly as s1 + err1: |a| >= ln2 > lchi for e != 0 and a = 0
   * for e = 0, so the fast two-sum is exact (and equal to the full one) */
  double s1 = a + lchi;
  double err1 = lchi - (s1 - a);
  double s2 = s1 + r1; /* two-sum */
  double b2 = s2 - s1;
  double err2 = (s1 - (s2 - b2)) + (r1 - b2);
  double low = ((err1 + err2) + (lclo + ed * PLIBM_LN2_LO42)) + (corr + poly);
  double h = s2 + low;
  *lo = low - (h - s2);
  *hi = h;
}

/* x^y given ln(x) = lhi + llo for finite x > 0 (shared-base calls). */
PLIBM_FN double plibm_pow_log(double lhi, double llo, double y) {
  double t_hi = y * lhi;
  double t_lo = plibm_fma(y, lhi, -t_hi) + y * llo;
  return plibm_exp_dd(t_hi, t_lo);
}

/* ln of a base for pow: the log of x for finite x > 0, else of 1 (pow's
 * special values are fixed up from x itself). */
PLIBM_FN void plibm_log_base(double x, double *lhi, double *llo) {
  int ok = (x > 0.0) && (x < PLIBM_INF);
  plibm_log_dd(ok ? x : 1.0, lhi, llo);
}

/* x^3 rounded once: x*x = h + l and h*x = p + pe exactly (fused
 * multiply-adds), so p + (pe + l*x) carries the exact cube to within
 * 2^-104 relative before its one rounding -- the correctly rounded cube
 * except at near-ties, as a correctly rounded pow(x, 3) gives.  (x*x)*x,
 * two roundings, differs from that in about a quarter of all arguments.
 * Outside 1e-90 < |x| < 1e90 (where the exact splits could under- or
 * overflow) and for NaN the plain product. */
PLIBM_FN double plibm_cube(double x) {
  double ax = x < 0.0 ? -x : x;
  if (!(ax > 1e-90 && ax < 1e90)) return (x * x) * x;
  double h = x * x;
  double l = plibm_fma(x, x, -h);
  double p = h * x;
  double pe = plibm_fma(h, x, -p);
  return p + (pe + l * x);
}

/* x^1.5 rounded once: s = sqrt(x) (correctly rounded) and x - s^2 = e
 * exactly, so sqrt(x) = s + e/(2s) to 2^-105 relative, and
 * x*e/(2s) = (s^2 + e)*e/(2s) = e*s/2 + e^2/(2s), whose last term is below
 * 2^-104 of the result; x*s = p + pe exactly.  p + (pe + (e*s)*0.5) thus
 * rounds the product with the exact root once, without a division.
 * x*sqrt(x) rounds twice and differs from the correctly rounded x^1.5 in
 * about a quarter of all arguments.  Outside 1e-290 < x < 1e300 (and for
 * x <= 0 or NaN) the plain product. */
PLIBM_FN double plibm_pow1p5(double x) {
  double s = plibm_sqrt(x);
  if (!(x > 1e-290 && x < 1e300)) return x * s;
  double e = plibm_fma(-s, s, x);
  double p = x * s;
  double pe = plibm_fma(x, s, -p);
  return p + (pe + (e * s) * 0.5);
}

/* x^y given plibm_log_base(x) = lhi + llo; pow(x, y) is exactly this, so
 * calls that share a base can share its logarithm. */
PLIBM_FN_COLD double plibm_pow_special(double x, double y, double res);
PLIBM_FN double plibm_pow_with_log(double x, double y, double lhi, double llo) {
  /* exponents with exact-operation forms (uniform branches for constant y):
   * sqrt and x*x are correctly rounded, the cube and x^1.5 as good as */
  if (y == 0.5) return plibm_sqrt(x);
  if (y == 1.5) return plibm_pow1p5(x);
  if (y == 2.0) return x * x;
  if (y == 3.0) return plibm_cube(x);
  double res = plibm_pow_log(lhi, llo, y);
  if (x > 0.0 && x < PLIBM_INF && y != 0.0 && y == y) return res;
  return plibm_pow_special(x, y, res);
}

/* x^y given plibm_log_base(x) = lhi + llo, for an exponent that is none of
 * 0.5, 1.5, 2 and 3: the same bits as plibm_pow_with_log without its tests
 * of the exponent (the kernels use it where the exponent is a parameter the
 * host has checked). */
PLIBM_FN double plibm_pow_with_log_gen(double x, double y, double lhi, double llo) {
  double res = plibm_pow_log(lhi, llo, y);
  if (x > 0.0 && x < PLIBM_INF && y != 0.0 && y == y) return res;
  return plibm_pow_special(x, y, res);
}

/* pow's special values: x = 0, +inf, negative or NaN; y = 0 or NaN. */
PLIBM_FN_COLD double plibm_pow_special(double x, double y, double res) {
  int ok = (x > 0.0) && (x < PLIBM_INF);
  double spec_zero = y > 0.0 ? 0.0 : (y < 0.0 ? PLIBM_INF : 1.0);
  double spec_inf = y > 0.0 ? PLIBM_INF : (y < 0.0 ? 0.0 : 1.0);
  double spec = x == 0.0 ? spec_zero : (x == PLIBM_INF ? spec_inf : PLIBM_NAN);
  res = ok ? res : spec;
  res = y == 0.0 ? 1.0 : res;
  return y != y ? y : res;
}

/* True when pow(x, y) does not need ln x (an exact-operation exponent). */
PLIBM_FN int plibm_pow_is_direct(double y) { return y == 0.5 || y == 1.5 || y == 2.0 || y == 3.0; }

/* ln(x) for finite x > 0: the rounded sum of plibm_log_dd's double-double
 * (within 1 ulp).  CLOUDSC's cloud-inhomogeneity path calls it with
 * arguments >= 1 (cloudsc.F90:2096). */
PLIBM_FN double plibm_log(double x) {
  double h, l;
  plibm_log_dd(x, &h, &l);
  return h;
}

PLIBM_FN double plibm_pow(double x, double y) {
  double lhi = 0.0, llo = 0.0;
  if (!plibm_pow_is_direct(y)) plibm_log_base(x, &lhi, &llo);
  return plibm_pow_with_log(x, y, lhi, llo);
}

#endif /* CLOUDSC_PLIBM_H */
