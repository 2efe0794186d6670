// One CLOUDSC column, top to bottom, on one GPU thread.
//
// This is the per-column body shared by the FP64 kernel (Real = double) and
// the FP32-mixed kernel (Real = float).  It restates, for a single column, the
// whole of ifs-source/arpifs/phys_ec/cloudsc.F90 in its default configuration:
//   first guess and tidy-up          :982-1199
//   level loop JK=NCLDTOP..KLEV       :1219-4128
//   DDH flux recurrences              :4218-4303
//   CLOUD_SUPERSATCHECK               cloud_supersatcheck.F90:111-226
// fused into ONE pass over the levels: every pre-loop quantity is computed for
// level JK when the pass reaches it, the quantities the reference reads from
// level JK-1 (ZA, ZQX(R/S), ZTP1, PAP) or JK+1 (PAPH, PLU, PMFU, PMFD) are
// carried in registers, and the flux prefix sums are accumulated as the pass
// goes, so every input element is read once and every output element written
// once.
//
// FP64 parity: with Real = double every floating-point operation is the
// reference's, in the reference's order (the file is compiled with
// --fmad=false so nothing is contracted).  The explicit (ZSOLQA) and implicit
// (ZSOLQB) 5x5 process matrices are held in registers using their structural
// sparsity in this configuration -- ZSOLQA has 18 entries that any process can
// touch, ZSOLQB has 5: (L,L), (I,I), (R,L), (S,I), (S,L).  The skipped entries
// are exact zeros, and every skipped operation on them (x - 0, x + 0,
// x - 0*y with finite y) returns x unchanged, so the sparse forms below give
// the dense reference results bit for bit (up to the sign of a zero).  The
// LHS matrix is lower triangular (its only off-diagonal entries are
// -ZSOLQB(R,L), -ZSOLQB(S,I), -ZSOLQB(S,L)), so the reference's non-pivoting
// LU (:3600-3628) reduces to three multipliers and forward/back substitution
// performed in the same order.
//
// Saturation exponentials: FOEEWM, FOEELIQ, FOEEICE and FOEEW share the two
// exponentials exp(R3LES*(T-RTT)/(T-R4LES)) and exp(R3IES*(T-RTT)/(T-R4IES));
// a term whose weight is exactly zero (FOEALFA = 1, FOEDELTA = 0/1) is
// skipped, which again leaves the result bit-identical.
//
// FP32-mixed (template flag F32M): the exponentials and powers of the
// microphysical processes and of the level's saturation values are evaluated
// in FP32; the state, every other operation, the sink truncation, the 5x5
// solve, CLOUD_SUPERSATCHECK (with its FP64 exponentials) and the tendency and
// flux (budget) accumulations stay in FP64.  Keeping the state and the
// threshold tests in FP64 is what keeps the tendencies within 1e-5 of the FP64
// result: with an FP32 state the scheme's thresholds and MIN() limiters flip
// (a measured 5-7 % RMS error on the T tendency).
#pragma once
#include <cstdint>
#include <cstring>
#include <type_traits>

#include "cloudsc_common.cuh"
#include "plibm.h"

#ifndef CSC_DEV
#define CSC_DEV __device__ __forceinline__
#endif

namespace cloudsc {

template <typename T>
CSC_DEV T mn(T a, T b) { return a < b ? a : b; }
template <typename T>
CSC_DEV T mx(T a, T b) { return a > b ? a : b; }

// What the fast division reports, accumulated over every division of a
// column.  acc ORs, for each dividend a and divisor b, the offsets
// (2 * hi(x)) - kDivBase, whose top bits are clear exactly when x's biased
// exponent lies in [767, 1278], i.e. 2^-256 <= |x| < 2^256 (a zero dividend
// adds 0).  bad(): some operand left that window.
constexpr unsigned kDivBase = 767u << 21, kDivRange = 1u << 30;
struct DivCheck {
  unsigned acc = 0u;
  CSC_DEV bool bad() const { return acc >= kDivRange; }
};

#if !defined(__CUDA_ARCH__)
// The window offset of x on the host (the GPU code takes hi(x) with
// __double2hiint): host builds report the operands the GPU kernels report.
inline unsigned div_offset_host(double x) {
  uint64_t u;
  std::memcpy(&u, &x, sizeof u);
  return (unsigned)(u >> 32) * 2u - kDivBase;
}
#endif

// Branch-free double division for the column code.  A reciprocal estimate
// (rcp.approx.ftz.f64) is refined by three Newton-Raphson steps
// y <- y + y(1 - by), each error term and update one fused multiply-add; the
// last step returns y = RN(1/b), the correctly rounded reciprocal, for every
// divisor whose significand is not all ones (Markstein, IBM J. Res. Dev.
// 34(1), 1990; Muller et al., Handbook of Floating-Point Arithmetic, ch. 5).
// For b = (2 - 2^-52) 2^E the step ends on the tie 2^(-E-1) while
// 1/b = 2^(-E-1) (1 + 2^-53 + 2^-106 + ...): the low significand bit of y is
// then set, which gives RN(1/b) = 2^(-E-1) (1 + 2^-52).  The quotient of |a|,
// q0 = RN(|a| y), within 1.5 ulp of |a|/b, is corrected twice with its
// residual, q <- RN(q + RN(|a| - b q) y): the first correction brings it
// within one ulp, where the residual is exact, and by Markstein's theorem the
// second then returns RN(|a|/b).  The sign of a is put back by flipping the
// sign bit, so that the result equals IEEE a/b bit for bit, zeros included,
// when no step under- or overflows: that holds for 2^-256 <= |b| < 2^256 and
// a = 0 or 2^-256 <= |a| < 2^256 (the quotient and every residual then stay
// normal).  Operands outside that window (zeros, subnormals, infinities and
// NaNs among them, a zero dividend excepted) are recorded in dc, and a column
// with any is rerun with IEEE division.  The GPU tests compare it with IEEE
// division on random operands and on hard ones (significands of all ones or
// all zeros, quotients next to a rounding tie).  The host build divides with
// IEEE division and reports the operands the GPU would report
// (CLOUDSC_HOST_FORCE_REDO makes every call report, to drive the caller's
// rerun in host tests).
CSC_DEV double fast_div(double a, double b, DivCheck &dc) {
#if defined(__CUDA_ARCH__)
  const int ha = __double2hiint(a), hb = __double2hiint(b);
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  // all-ones significand of b: w == 0, and the clamped shift gives 1 (else 0)
  const unsigned w = ~(((unsigned)hb | 0xfff00000u) & (unsigned)__double2loint(b));
  y = __hiloint2double(__double2hiint(y), __double2loint(y) | (int)__funnelshift_rc(1u, 0u, w));
  const double aa = fabs(a);
  const double q0 = __dmul_rn(aa, y);
  double r = __fma_rn(-b, q0, aa);
  const double q1 = __fma_rn(r, y, q0);
  r = __fma_rn(-b, q1, aa);
  const double q = __fma_rn(r, y, q1);
  const unsigned da = a == 0.0 ? 0u : (unsigned)ha * 2u - kDivBase;
  dc.acc |= da | ((unsigned)hb * 2u - kDivBase);
  return __hiloint2double(__double2hiint(q) ^ (ha & (int)0x80000000), __double2loint(q));
#else
#if defined(CLOUDSC_HOST_FORCE_REDO)
  dc.acc = ~0u;
#else
  dc.acc |= (a == 0.0 ? 0u : div_offset_host(a)) | div_offset_host(b);
#endif
  return a / b;
#endif
}

// The reciprocal half of fast_div on its own: y = RN(1/b), the correctly
// rounded reciprocal (IEEE 1/b), for 2^-256 <= |b| < 2^256; b outside that
// window is recorded in dc.  Used for the quotients 1/b and, through
// fast_div_k, for several dividends over one divisor.
CSC_DEV double fast_rcp(double b, DivCheck &dc) {
#if defined(__CUDA_ARCH__)
  const int hb = __double2hiint(b);
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  const unsigned w = ~(((unsigned)hb | 0xfff00000u) & (unsigned)__double2loint(b));
  y = __hiloint2double(__double2hiint(y), __double2loint(y) | (int)__funnelshift_rc(1u, 0u, w));
  dc.acc |= (unsigned)hb * 2u - kDivBase;
  return y;
#else
#if defined(CLOUDSC_HOST_FORCE_REDO)
  dc.acc = ~0u;
#else
  dc.acc |= div_offset_host(b);
#endif
  return 1.0 / b;
#endif
}

// fast_div for a literal divisor b, given y = RN(1/b) folded at compile
// time (IEEE division of two constants): only the two residual corrections
// and the dividend's window test remain.  Exact as fast_div is: every such
// divisor lies in the window and has no all-ones significand, so y is the
// correctly rounded reciprocal Markstein's theorem needs.
CSC_DEV double fast_div_k(double a, double b, double y, DivCheck &dc) {
#if defined(__CUDA_ARCH__)
  const int ha = __double2hiint(a);
  const double aa = fabs(a);
  const double q0 = __dmul_rn(aa, y);
  double r = __fma_rn(-b, q0, aa);
  const double q1 = __fma_rn(r, y, q0);
  r = __fma_rn(-b, q1, aa);
  const double q = __fma_rn(r, y, q1);
  dc.acc |= a == 0.0 ? 0u : (unsigned)ha * 2u - kDivBase;
  return __hiloint2double(__double2hiint(q) ^ (ha & (int)0x80000000), __double2loint(q));
#else
  (void)y;
#if defined(CLOUDSC_HOST_FORCE_REDO)
  dc.acc = ~0u;
#else
  dc.acc |= a == 0.0 ? 0u : div_offset_host(a);
#endif
  return a / b;
#endif
}

// a / b for a literal b (y = 1/b folded): fast_div_k when FAST and the
// quotient is a double; IEEE otherwise.
template <bool FAST, typename A>
CSC_DEV auto cdivk(A a, double b, double y, DivCheck &dc) -> decltype(a / A(b)) {
  typedef decltype(a / A(b)) T;
  if constexpr (FAST && std::is_same<T, double>::value) {
    return fast_div_k(double(a), b, y, dc);
  } else {
    (void)dc;
    (void)y;
    return a / A(b);
  }
}

// 1 / b: fast_rcp when FAST and b is a double; IEEE otherwise.
template <bool FAST, typename B>
CSC_DEV B crcp(B b, DivCheck &dc) {
  if constexpr (FAST && std::is_same<B, double>::value) {
    return fast_rcp(b, dc);
  } else {
    (void)dc;
    return B(1) / b;
  }
}

// Passes of the column code (cloudsc_column's PASS): plain, IEEE division
// throughout; fast, the branch-free fast_div, recording operands outside its
// exact window; redo, the rerun with IEEE division of a column whose fast
// pass recorded one.
enum { kPassPlain = 0, kPassFast = 1, kPassRedo = 2 };

// a / b, by fast_div when FAST and the quotient is a double; IEEE otherwise.
template <bool FAST, typename A, typename B>
CSC_DEV auto cdiv(A a, B b, DivCheck &dc) -> decltype(a / b) {
  typedef decltype(a / b) T;
  if constexpr (FAST && std::is_same<T, double>::value) {
    return fast_div(double(a), double(b), dc);
  } else {
    (void)dc;
    return a / b;
  }
}

// Double precision uses the portable exp/pow of plibm.h (bit-identical on the
// host and the GPU).
#if defined(CLOUDSC_HOST_LIBM_GLIBC) && !defined(__CUDA_ARCH__)
// host test builds only: the system libm, to measure libm sensitivity
CSC_DEV double xexp(double x) { return exp(x); }
CSC_DEV double xpow(double x, double y) { return pow(x, y); }
CSC_DEV double xlog(double x) { return log(x); }
#else
CSC_DEV double xexp(double x) { return plibm_exp(x); }
CSC_DEV double xpow(double x, double y) { return plibm_pow(x, y); }
CSC_DEV double xlog(double x) { return plibm_log(x); }
#endif
// FP32 transcendentals of the FP32-mixed kernel: on the GPU the special-
// function-unit forms (__expf, __powf: one ex2 / lg2 each, relative error of a
// few 1e-7 times the size of the exponent's argument), on the host the C
// library; exponents 0.5, 1.5, 2 and 3 are evaluated exactly as roots and
// products, as plibm does in double.
CSC_DEV float xexp(float x) {
#if defined(__CUDA_ARCH__)
  return __expf(x);
#else
  return expf(x);
#endif
}
CSC_DEV float xpow(float x, float y) {
  if (y == 0.5f) return sqrtf(x);
  if (y == 1.5f) return x * sqrtf(x);
  if (y == 2.0f) return x * x;
  if (y == 3.0f) return x * x * x;
#if defined(__CUDA_ARCH__)
  return __powf(x, y);
#else
  return powf(x, y);
#endif
}

// Transcendentals of the microphysics: FP64 (plibm) in the FP64 kernel,
// FP32 (xexp/xpow above, on the argument rounded to float) in the FP32-mixed
// kernel.  Everything else in both kernels is FP64.
template <bool F32>
CSC_DEV double mexp(double x) {
  if (F32) return (double)xexp((float)x);
  return xexp(x);
}
template <bool F32>
CSC_DEV double mpow(double x, double y) {
  if (F32) return (double)xpow((float)x, (float)y);
  return xpow(x, y);
}

// A pow base whose logarithm several calls share (FP64: plibm's double-double
// ln, computed once; FP32-mixed: nothing is precomputed).  mpowb(b, y) equals
// mpow(b.x, y) exactly.
struct PowBase {
  double x, lhi, llo;
};
template <bool F32>
CSC_DEV PowBase mbase(double x) {
  PowBase b;
  b.x = x;
  b.lhi = 0.0;
  b.llo = 0.0;
#if !(defined(CLOUDSC_HOST_LIBM_GLIBC) && !defined(__CUDA_ARCH__))
  if (!F32) plibm_log_base(x, &b.lhi, &b.llo);
#endif
  return b;
}
template <bool F32>
CSC_DEV double mpowb(const PowBase &b, double y) {
  if (F32) return (double)xpow((float)b.x, (float)y);
#if defined(CLOUDSC_HOST_LIBM_GLIBC) && !defined(__CUDA_ARCH__)
  return pow(b.x, y);
#else
  return plibm_pow_with_log(b.x, y, b.lhi, b.llo);
#endif
}
// pow with a parameter as exponent.  With GEN the host has checked that the
// exponent is none of 0.5, 1.5, 2 and 3, in double and rounded to float
// (gen_exponents_ok), so the tests for those exponents are left out: the
// same results as mpow / mpowb with fewer branches.
CSC_DEV float xpow_gen(float x, float y) {
#if defined(__CUDA_ARCH__)
  return __powf(x, y);
#else
  return powf(x, y);
#endif
}
template <bool F32, bool GEN>
CSC_DEV double mpowp(double x, double y) {
  if (!GEN) return mpow<F32>(x, y);
  if (F32) return (double)xpow_gen((float)x, (float)y);
#if defined(CLOUDSC_HOST_LIBM_GLIBC) && !defined(__CUDA_ARCH__)
  return pow(x, y);
#else
  double lhi, llo;
  plibm_log_base(x, &lhi, &llo);
  return plibm_pow_with_log_gen(x, y, lhi, llo);
#endif
}
template <bool F32, bool GEN>
CSC_DEV double mpowbp(const PowBase &b, double y) {
  if (!GEN) return mpowb<F32>(b, y);
  if (F32) return (double)xpow_gen((float)b.x, (float)y);
#if defined(CLOUDSC_HOST_LIBM_GLIBC) && !defined(__CUDA_ARCH__)
  return pow(b.x, y);
#else
  return plibm_pow_with_log_gen(b.x, y, b.lhi, b.llo);
#endif
}
CSC_DEV double xsqrt(double x) { return sqrt(x); }
CSC_DEV float xsqrt(float x) { return sqrtf(x); }

// The scalars the column body reads, in the working precision.  Filled on the
// host from cloudsc_params (and Derived) and uploaded to constant memory.
template <typename Real>
struct KParams {
  Real rg, rd, rv, retv, rtt, rlvtt, rlstt, rpi;
  Real r2es, r3les, r3ies, r4les, r4ies, r5les, r5ies, r5alvcp, r5alscp;
  Real ralvdcp, ralsdcp, rtwat, rtice, rtwat_rtice_r, rkoop1, rkoop2;
  Real ramid, ramin, rlmin, rcldiff, rcldiff_convi, rcovpmin, rprecrhmax, rpecons;
  Real rvrfactor, rtaumel, rssicefactor, rsnowlin1, rsnowlin2, rlcritsnow, rthomo;
  Real rvice, rvsnow, rxfallspeedrain, rcldtopcf, rdepliqrefrate, rdepliqrefdepth;
  Real riceinit, rdensref, rdenswat, rcl_overlapliqice, rcl_effrime;
  Real rcl_inhomogaut, rcl_inhomogacc, rcl_kkaac, rcl_kkbac, rcl_kkaau, rcl_kkbauq;
  Real rcl_dr, rcl_x1r, rcl_x2r, rcl_lam1r, rcl_lam2r;
  Real rcl_const1r, rcl_const2r, rcl_const3r, rcl_const4r, rcl_const5r, rcl_const6r;
  Real rcl_const7r, rcl_cdenom1, rcl_cdenom2, rcl_cdenom3, rcl_fzrab;
  Real rcl_x1s, rcl_lam1s, rcl_lam2s;
  Real rcl_const1s, rcl_const2s, rcl_const3s, rcl_const4s, rcl_const5s, rcl_const6s;
  Real rcl_const7s, rcl_const8s;
  Real rcl_apb1, rcl_apb2, rcl_apb3;
  Real rmfadvw, rmfadvwdd;
  // derived, loop-invariant
  Real zrdcp, zrg_r, zrldcp, zconst_pow_land, zconst_pow_sea, flt_0p4, flt_0p8;
  Real kkbauq_m1, kkbac_m1;
  // cloud budget diagnostics (cloudsc.F90:3832-4110)
  Real ralfdcp, reisthsc;
  int lcldbudc, lcldbudl, lcldbudi, lcldbudt, lcldbud_vertint, lcldbud_timeint, lbud23;
  // SPP perturbations and the cloud-inhomogeneity/FSD path (:850-939,
  // 1937-2110, 4307-4359)
  Real ra, rcloud_frac_std, spp_mu[16], spp_xmag[16];
  int lspp, lcloud_inhomog, lrad_cloud_inhomog, spp_lramidlimit1, spp_on[8], spp_mp[8];
  int ncldtop, lmfdsnow;
  // aerosol-aware ice sedimentation and ice-to-snow autoconversion
  // (LAERICESED, LAERICEAUTO; cloudsc.F90:1798-1803, 2776-2779)
  Real rnice;
  int laericesed, laericeauto;
  // Divisions by parameters: RV/RD in the working precision, and the
  // correctly rounded reciprocals of the parameter divisors, for fast_div_k.
  // rcp_force: one of those divisors is outside fast_div's window or has an
  // all-ones significand, and every column takes the IEEE rerun.
  Real rv_rd;
  double rcp_rd, rcp_rtaumel, rcp_rcl_lam1r, rcp_rdepliqrefdepth, rcp_rvrfactor;
  int rcp_force;
};

// Double-precision copy of the scalars the FP64 stages (solve, supersaturation
// check, tendencies, fluxes) need in the mixed kernel; identical to the
// KParams<double> fields of the same name.
struct KParamsD {
  double rg, retv, rtt, rtice, rtwat, rtwat_rtice_r, r2es, r3les, r3ies, r4les, r4ies;
  double r5alvcp, r5alscp, ralvdcp, ralsdcp, rkoop1, rkoop2, rssicefactor, rlmin;
  double rlvtt, rlstt, zrg_r;
};

}  // namespace cloudsc
