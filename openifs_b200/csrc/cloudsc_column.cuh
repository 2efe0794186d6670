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
// FP32-mixed (Real = float): the state and the microphysical process rates are
// single precision; the sink truncation, the 5x5 solve, CLOUD_SUPERSATCHECK
// and the tendency and flux (budget) accumulations stay in double.
#pragma once
#include "cloudsc_common.cuh"

namespace cloudsc {

template <typename T>
__device__ __forceinline__ T mn(T a, T b) { return a < b ? a : b; }
template <typename T>
__device__ __forceinline__ T mx(T a, T b) { return a > b ? a : b; }

__device__ __forceinline__ double xexp(double x) { return exp(x); }
__device__ __forceinline__ float xexp(float x) { return expf(x); }
__device__ __forceinline__ double xpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float xpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double xsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float xsqrt(float x) { return sqrtf(x); }

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
  int ncldtop, lmfdsnow;
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
