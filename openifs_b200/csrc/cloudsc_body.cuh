// Per-column CLOUDSC body (device code), shared by the GPU kernels
// (cloudsc_kernels.cu) and by the host build of the same code that the tests
// compare against the oracle (tests/hostemu).  The including file provides:
//   CSC_DEV           function qualifiers (__device__ __forceinline__ on the GPU)
//   KP<Real>()        the KParams<Real> block, c_kd the KParamsD block
//   ld(p), atomic_add(p, v), xexp/xpow/xsqrt/xabs/xsign overloads
//   CSC_LEVEL_SYNC()  optional: a barrier of all columns of a CTA at the end
//                     of every level (nothing on the host)
// See cloudsc_column.cuh for the numerical contract.
#pragma once
#include "cloudsc_column.cuh"

#ifndef CSC_LEVEL_SYNC
#define CSC_LEVEL_SYNC()
#endif

// Every division of the column code: fast_div when FAST_ (the fast pass),
// recording in divbad_ the operands outside its exact window; IEEE division
// otherwise (cdiv, cloudsc_column.cuh).
#define DIV(...) cdiv<FAST_>(__VA_ARGS__, divbad_)
// A literal divisor: its reciprocal folded at compile time (cdivk).
#define DIVK(A, B) cdivk<FAST_>(A, B, 1.0 / (B), divbad_)
// A power-of-two literal divisor: multiplication by its exact reciprocal,
// the same bits as the division for every operand.
#define DIV2(A, B) ((A) * decltype(A)(1.0 / (B)))
// A parameter divisor with its reciprocal computed on the host (KParams rcp_*).
#define DIVP(A, B, Y) cdivk<FAST_>(A, B, Y, divbad_)
// The quotient 1/B (crcp): in the fast pass the reciprocal half of fast_div,
// recording B's window.
#define RCP(B) crcp<FAST_>(B, divbad_)
// A / B for a divisor shared by several quotients, Y = RCP(B) computed once:
// the same operations as DIV(A, B) (fast_div is fast_rcp followed by
// fast_div_k's corrections), so the same bits.
#define DIVY(A, B, Y) cdivk<FAST_>(A, B, Y, divbad_)

namespace cloudsc {

// ZSOLQA(a,b) of the reference ("+" is a source of a and a sink of b).  Every
// off-diagonal rate is added to (a,b) and subtracted from (b,a), so
// ZSOLQA(b,a) == -ZSOLQA(a,b) exactly at all times: negation is exact,
// round-to-nearest is symmetric, and the sink rescaling multiplies both by the
// same factor.  Only one entry of each pair is stored:
//   diagonal LL, II, RR, SS;  pairs LI (IL = -LI), LV (VL = -LV), IR (RI = -IR),
//   IV (VI = -IV), RS (SR = -RS), RV (VR = -RV), SV (VS = -SV).
// Every sum below is the reference's sum with a + (-b) written as a - b and
// 0 - (-b) as 0 + b, which are the same IEEE operations.
struct QA {
  double LL, II, RR, SS, LI, LV, IR, IV, RS, RV, SV;
};

// Sink sum of each row JM: -(sum over JN of ZSOLQA(JM,JN)) accumulated as
// ZSINKSUM = ZSINKSUM - ZSOLQA(JM,JN) in JN order (cloudsc.F90:3459-3466).
CSC_DEV double sink_sum(int jo, const QA &q) {
  double s;
  switch (jo) {
    case L: s = 0.0 - q.LL; s = s - q.LI; s = s - q.LV; break;
    case I: s = 0.0 + q.LI; s = s - q.II; s = s - q.IR; s = s - q.IV; break;
    case R: s = 0.0 + q.IR; s = s - q.RR; s = s - q.RS; s = s - q.RV; break;
    case S: s = 0.0 + q.RS; s = s - q.SS; s = s - q.SV; break;
    default: s = 0.0 + q.LV; s = s + q.IV; s = s + q.RV; s = s + q.SV; break;
  }
  return s;
}

// Sink truncation of one species row (cloudsc.F90:3500-3535 for one JM): the
// scaling factor ZRATIO = ZMM/MAX(ZSINKSUM,ZMM), then every negative entry
// (JO,n) rescaled together with its mirror (n,JO); a negative diagonal entry
// is scaled twice, as the reference's JN loop does.  ZRATIO is exactly 1.0
// unless the sink sum exceeds ZMM, and scaling by 1.0 changes nothing, so only
// that case scales.
#define SCL2(F, A) \
  if (F) {         \
    A = A * zr;    \
    A = A * zr;    \
  }
#define SCL1(F, A) \
  if (F) A = A * zr;
template <bool FAST_>
CSC_DEV void scale_row(int jo, QA &q, const double qx[5], DivCheck &divbad_) {
  const double zepsec = 1.E-14;
  const double ss = sink_sum(jo, q);
  const double zmm = mx(qx[jo], zepsec);
  if (!(ss > zmm)) return;
  const double zr = DIV(zmm, ss);
  switch (jo) {
    case L: {
      bool fLL = q.LL < 0.0, fLI = q.LI < 0.0, fLV = q.LV < 0.0;
      SCL2(fLL, q.LL) SCL1(fLI, q.LI) SCL1(fLV, q.LV)
    } break;
    case I: {  // (I,L) = -LI < 0  <=>  LI > 0
      bool fIL = q.LI > 0.0, fII = q.II < 0.0, fIR = q.IR < 0.0, fIV = q.IV < 0.0;
      SCL1(fIL, q.LI) SCL2(fII, q.II) SCL1(fIR, q.IR) SCL1(fIV, q.IV)
    } break;
    case R: {
      bool fRI = q.IR > 0.0, fRR = q.RR < 0.0, fRS = q.RS < 0.0, fRV = q.RV < 0.0;
      SCL1(fRI, q.IR) SCL2(fRR, q.RR) SCL1(fRS, q.RS) SCL1(fRV, q.RV)
    } break;
    case S: {
      bool fSR = q.RS > 0.0, fSS = q.SS < 0.0, fSV = q.SV < 0.0;
      SCL1(fSR, q.RS) SCL2(fSS, q.SS) SCL1(fSV, q.SV)
    } break;
    default: {
      bool fVL = q.LV > 0.0, fVI = q.IV > 0.0, fVR = q.RV > 0.0, fVS = q.SV > 0.0;
      SCL1(fVL, q.LV) SCL1(fVI, q.IV) SCL1(fVR, q.RV) SCL1(fVS, q.SV)
    } break;
  }
}
#undef SCL1
#undef SCL2

// ZRATIO for every species from the current ZSOLQA (cloudsc.F90:3455-3474).
template <bool FAST_>
CSC_DEV void sink_ratios(const QA &q, const double qx[5], double r[5], DivCheck &divbad_) {
  const double zepsec = 1.E-14;
#pragma unroll
  for (int jm = 0; jm < 5; ++jm) {
    double zmax = mx(qx[jm], zepsec);
    r[jm] = DIV(zmax, mx(sink_sum(jm, q), zmax));
  }
}

// ---------------------------------------------------------------------------
// CLOUD_SUPERSATCHECK (cloud_supersatcheck.F90:111-226, KFTLIQICE=1), double.
// ---------------------------------------------------------------------------
template <bool FAST_>
CSC_DEV void supersatcheck(double pt, double pq, double pa, double pp, double &t_adj, double &q_adj,
                           double &a_adj, double &l_adj, double &i_adj, DivCheck &divbad_) {
  const KParamsD &k = c_kd;
  const double zepsec = 1.E-14;
  double zda = 0.0;
  double zt = mx(pt, 160.0);
  double za = mx(mn(pa, 1.0), 0.0);
  double zp_r = RCP(pp);
  double el = xexp(DIV(k.r3les * (zt - k.rtt), (zt - k.r4les)));
  double x = (mx(k.rtice, mn(k.rtwat, zt)) - k.rtice) * k.rtwat_rtice_r;
  double alfa = mn(1.0, x * x);
  bool delta = copysign(1.0, zt - k.rtt) > 0.0;  // FOEDELTA = 1
  // computed whether or not a term needs it: without the branch the two
  // exponentials overlap (the same bits where it is used)
  double ei = xexp(DIV(k.r3ies * (zt - k.rtt), (zt - k.r4ies)));
  double zfoeeliq = mn((k.r2es * el) * zp_r, 0.5);
  double foeew = delta ? k.r2es * el : k.r2es * ei;
  double zfoeeice = mn(foeew * zp_r, 0.5);
  double zfokoop = mn(zfoeeice * (k.rkoop1 - k.rkoop2 * zt), zfoeeliq);
  double zqsliqk = DIV(zfokoop, (1.0 - k.retv * zfokoop));
  double wsum = (alfa < 1.0) ? alfa * el + (1.0 - alfa) * ei : el;
  double zfoeemix = mn((k.r2es * wsum) * zp_r, 0.5);
  double zcor = RCP(1.0 - k.retv * zfoeemix);
  double zqsmix = zfoeemix * zcor;
  double xl = zt - k.r4les, xi = zt - k.r4ies;
  double foedem = alfa * k.r5alvcp * (RCP(xl * xl)) + (1.0 - alfa) * k.r5alscp * (RCP(xi * xi));
  double zcorqsmix = 1.0 + zqsmix * zcor * foedem;
  zqsliqk = 0.5 * (zqsliqk + zqsmix);
  double zqslim = za * zqsmix + (1.0 - za) * zqsliqk;
  double zcond = mx(pq - zqslim, 0.0);
  if (zcond > zepsec) {
    double zfaci = alfa + (1.0 - alfa) * k.rssicefactor;
    zda = (1.0 - za) * zfaci;
    double za_upd = za + zda;
    zqslim = za_upd * zqsmix + (1.0 - za_upd) * zqsliqk;
    zcond = DIV((pq - zqslim), zcorqsmix);
  }
  double foeldcpm = alfa * k.ralvdcp + (1.0 - alfa) * k.ralsdcp;
  t_adj = foeldcpm * zcond;
  q_adj = -zcond;
  a_adj = zda;
  l_adj = zcond * alfa;
  i_adj = zcond * (1.0 - alfa);
}

// ---------------------------------------------------------------------------
// Cloud budget diagnostics of one level (cloudsc.F90:3832-4110): the level's
// budget terms added to PEXTRA(JL, *, *) (INOUT, (KLON,KLEV,KFLDX) per block;
// `base` is the offset of PEXTRA(JL,1,1)).  Field pointer IS starts at 26
// with LBUD23; each section on moves it on (+1, +12, +22, +20, +13).  The
// vertical integral accumulates over the levels into the slots IK = 1..83 of
// one field.  ZPIEVAP, ZPRACS and ZPRACI are zero in this configuration
// (ISUBLICE = 0, PRACS and PRACI off); the KTYPE/KPBLTYPE == IS+1 tests are
// as written at :3925,3929.
//
// Every slot one level updates is distinct (the entry points require KLEV >=
// 84 with the vertical integral, so IK never reaches the next field), and a
// slot is updated at most once per level.  Each group of updates therefore
// loads all its old values before it stores any: the compiler cannot move a
// load above the store before it by itself (the slots lie a run-time
// multiple of NPROMA apart), and one update after another would wait a full
// memory round trip each.  The additions and their operands are the
// reference's, one rounding each, so the values are unchanged.
// ---------------------------------------------------------------------------
template <int N>
CSC_DEV void px_add(double *px, const size_t (&o)[N], const double (&v)[N]) {
  double old[N];
#pragma unroll
  for (int n = 0; n < N; ++n) old[n] = px[o[n]];
#pragma unroll
  for (int n = 0; n < N; ++n) px[o[n]] = old[n] + v[n];
}
// the same where update n happens only when c[n] holds
template <int N>
CSC_DEV void px_add_if(double *px, const size_t (&o)[N], const double (&v)[N], const bool (&c)[N]) {
  double old[N];
#pragma unroll
  for (int n = 0; n < N; ++n) old[n] = px[o[n]];
#pragma unroll
  for (int n = 0; n < N; ++n)
    if (c[n]) px[o[n]] = old[n] + v[n];
}

template <typename Real>
CSC_DEV void write_budgets(const Fields &F, const KParams<Real> &P, const double *cc, const double *bl,
                           const double *bi, size_t base, int np, int klev, int k, double dt, double zqtmst,
                           double zdp, double zrho, double pvfa, double pdyna, double pvfl, double pdynl,
                           double pvfi, double pdyni, double pdyns, double phrsw, double phrlw, double xl,
                           double xi, double psdep, double psacr, double piacr, double prainfrac, int ktype,
                           int kpbltype, int kctop, double peis) {
  double *px = F.pextra + base;
  const size_t sk = (size_t)np, sf = (size_t)np * klev;
  // offset of PEXTRA(JL, IK, IS) with 1-based IK and IS
  auto S = [&](int ik, int is) -> size_t { return (size_t)(is - 1) * sf + (size_t)(ik - 1) * sk; };
  int is = P.lbud23 ? 26 : 0;
  const double zdt = P.lcldbud_timeint ? dt : 1.0;
  const int jk = k + 1;
  if (P.lcldbud_vertint) {
    const double zdz = zdp / (zrho * double(P.rg));
    const int f = is + 1;
    {
      const size_t o[8] = {S(4, f), S(6, f), S(7, f), S(8, f), S(9, f), S(10, f), S(11, f), S(12, f)};
      const double v[8] = {cc[2] * zdz * zdt,          cc[3] * zdz * zdt, (cc[4] + cc[6]) * zdz * zdt,
                           cc[5] * zdz * zdt,          cc[7] * zdz * zdt, cc[12] * zdz * zdt,
                           pvfa * zdz * zdt,           pdyna * zdz * zdt};
      px_add(px, o, v);
    }
    {
      const size_t o[11] = {S(14 + 5, f),  S(14 + 7, f),  S(14 + 8, f),  S(14 + 9, f),  S(14 + 10, f), S(14 + 11, f),
                            S(14 + 12, f), S(14 + 13, f), S(14 + 14, f), S(14 + 15, f), S(14 + 16, f)};
      const double v[11] = {bl[2] * zdz * zdt,  bl[3] * zdz * zdt,  (bl[4] + bl[6]) * zdz * zdt,
                            bl[5] * zdz * zdt,  bl[7] * zdz * zdt,  bl[11] * zdz * zdt,
                            bl[14] * zdz * zdt, bl[15] * zdz * zdt, bl[12] * zdz * zdt,
                            bl[13] * zdz * zdt, bl[17] * zdz * zdt};
      px_add(px, o, v);
    }
    {
      const size_t o[9] = {S(14 + 17, f), S(14 + 18, f), S(14 + 19, f), S(14 + 20, f), S(14 + 21, f),
                           S(14 + 22, f), S(14 + 23, f), S(14 + 24, f), S(14 + 25, f)};
      const double v[9] = {(bl[18] + bl[19]) * zdz * zdt, bl[20] * zdz * zdt,
                           bl[21] * zdz * zdt,            0.0 * zdz * zdt * zqtmst,
                           psacr * zdz * zdt * zqtmst,    0.0 * zdz * zdt * zqtmst,
                           piacr * zdz * zdt * zqtmst,    pvfl * zdz * zdt,
                           pdynl * zdz * zdt};
      px_add(px, o, v);
    }
    px[S(60, f)] = prainfrac;
    {
      const size_t o[15] = {S(39 + 5, f),  S(39 + 7, f),  S(39 + 8, f),  S(39 + 9, f),  S(39 + 10, f),
                            S(39 + 11, f), S(39 + 12, f), S(39 + 13, f), S(39 + 14, f), S(39 + 15, f),
                            S(39 + 16, f), S(39 + 17, f), S(39 + 18, f), S(39 + 19, f), S(78, f)};
      const double v[15] = {bi[2] * zdz * zdt,           bi[3] * zdz * zdt,  (bi[4] + bi[6]) * zdz * zdt,
                            bi[5] * zdz * zdt,           bi[7] * zdz * zdt,  bi[11] * zdz * zdt,
                            (bi[12] + bi[13]) * zdz * zdt, bi[14] * zdz * zdt, bi[16] * zdz * zdt,
                            bi[17] * zdz * zdt,          psdep * zqtmst * zdz * zdt,
                            pvfi * zdz * zdt,            pdyni * zdz * zdt,  pdyns * zdz * zdt,
                            peis};
      px_add(px, o, v);
    }
    {
      const size_t o[12] = {S(70, f), S(71, f), S(72, f), S(73, f), S(74, f), S(75, f),
                            S(76, f), S(77, f), S(79, f), S(80, f), S(81, f), S(82, f)};
      const double v[12] = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
      const bool c[12] = {ktype == 0,     ktype == is + 1,     ktype == 2,     ktype == 3,
                          kpbltype == 0,  kpbltype == is + 1,  kpbltype == 2,  kpbltype == 3,
                          peis > 6.0,     peis > 8.0,          peis > 10.0,
                          ktype >= 2 && peis < double(P.reisthsc)};
      px_add_if(px, o, v, c);
    }
    if (ktype > 0) px[S(83, f)] = double(kctop);
    is = is + 1;
  }
  if (P.lcldbudc) {  // :3948-3970
    const size_t o[7] = {S(jk, is + 4), S(jk, is + 6), S(jk, is + 7), S(jk, is + 8),
                         S(jk, is + 9), S(jk, is + 11), S(jk, is + 12)};
    const double v[7] = {cc[2] * zdt, cc[3] * zdt, (cc[4] + cc[6]) * zdt, cc[5] * zdt,
                         cc[7] * zdt, pvfa * zdt,  pdyna * zdt};
    px_add(px, o, v);
    is = is + 12;
  }
  if (P.lcldbudl) {  // :3972-4007
    {
      const size_t o[9] = {S(jk, is + 5),  S(jk, is + 7),  S(jk, is + 8),  S(jk, is + 9), S(jk, is + 10),
                           S(jk, is + 11), S(jk, is + 12), S(jk, is + 13), S(jk, is + 14)};
      const double v[9] = {bl[2] * zdt,  bl[3] * zdt,  (bl[4] + bl[6]) * zdt, bl[5] * zdt, bl[7] * zdt,
                           bl[11] * zdt, bl[12] * zdt, bl[13] * zdt,          bl[14] * zdt};
      px_add(px, o, v);
    }
    {
      const size_t o[8] = {S(jk, is + 15), S(jk, is + 16), S(jk, is + 17), S(jk, is + 18),
                           S(jk, is + 19), S(jk, is + 20), S(jk, is + 21), S(jk, is + 22)};
      const double v[8] = {bl[15] * zdt, bl[17] * zdt, (bl[18] + bl[19]) * zdt, bl[20] * zdt,
                           bl[21] * zdt, pvfl * zdt,   pdynl * zdt,             xl};
      px_add(px, o, v);
    }
    is = is + 22;
  }
  if (P.lcldbudi) {  // :4009-4048
    {
      const size_t o[8] = {S(jk, is + 5), S(jk, is + 7),  S(jk, is + 8),  S(jk, is + 9),
                           S(jk, is + 10), S(jk, is + 11), S(jk, is + 12), S(jk, is + 13)};
      const double v[8] = {bi[2] * zdt, bi[3] * zdt,  (bi[4] + bi[6]) * zdt,   bi[5] * zdt,
                           bi[7] * zdt, bi[11] * zdt, (bi[12] + bi[13]) * zdt, bi[14] * zdt};
      px_add(px, o, v);
    }
    {
      const size_t o[7] = {S(jk, is + 14), S(jk, is + 15), S(jk, is + 16), S(jk, is + 17),
                           S(jk, is + 18), S(jk, is + 19), S(jk, is + 20)};
      const double v[7] = {(bi[15] + bi[16]) * zdt, psdep * zqtmst * zdt, bi[17] * zdt, pvfi * zdt,
                           0.0 * zqtmst * zdt,      pdyni * zdt,          xi};
      px_add(px, o, v);
    }
    is = is + 20;
  }
  if (P.lcldbudt) {  // :4051-4106
    const double lv = double(P.ralvdcp), ls = double(P.ralsdcp), lf = double(P.ralfdcp);
    {
      const size_t o[7] = {S(jk, is + 1), S(jk, is + 2), S(jk, is + 3), S(jk, is + 4),
                           S(jk, is + 5), S(jk, is + 6), S(jk, is + 7)};
      const double v[7] = {phrsw,
                           phrlw,
                           ((bl[1] + bl[2] + bl[9] + bl[10]) * lv - bi[11] * lv) * zdt,
                           (bi[1] + bi[2] + bi[9] + bi[10] + bi[11]) * ls * zdt,
                           bi[11] * lf * zdt,
                           (bl[7] + bl[8] + bl[5]) * lv * zdt,
                           (bi[7] + bi[8] + bi[5]) * ls * zdt};
      px_add(px, o, v);
    }
    {
      const size_t o[6] = {S(jk, is + 8),  S(jk, is + 9),  S(jk, is + 10),
                           S(jk, is + 11), S(jk, is + 12), S(jk, is + 13)};
      // X(JK, IS+12) is decremented (:4100): the subtraction is kept as such
      double old[6];
#pragma unroll
      for (int n = 0; n < 6; ++n) old[n] = px[o[n]];
      px[o[0]] = old[0] + bl[20] * lv * zdt;
      px[o[1]] = old[1] + bi[17] * ls * zdt;
      px[o[2]] = old[2] + bi[15] * lf * zdt;
      px[o[3]] = old[3] + bi[16] * lf * zdt;
      px[o[4]] = old[4] - (bl[12] + bl[13] + bl[18] + bl[19]) * lf * zdt;
      px[o[5]] = old[5] + bl[21] * lf * zdt;
    }
  }
}

// ---------------------------------------------------------------------------
// The column body.
// ---------------------------------------------------------------------------
// `active` false: the thread only keeps a CTA's per-level barrier company
// (it computes column (ib, jl), which must be valid, and stores nothing).
// BUD: the form with the cloud budget diagnostics (cloudsc.F90:3832-4110),
// FP64 only; the budget terms ZBUDCC/ZBUDL/ZBUDI of each level are collected
// where the reference stores them and written to PEXTRA at the end of the
// level.  Without BUD none of this code is compiled.
// OPT: the form with the SPP perturbations (LSPP) and the cloud-inhomogeneity
// paths (LCLOUD_INHOMOG, LRAD_CLOUD_INHOMOG -> PFSD), FP64 only
// (cloudsc.F90:850-939, 1937-2110, 2282-2348, 2781-2783, 3288-3290,
// 3819-3823, 4112-4125, 4307-4359).  Without OPT none of this code exists.
// FT: the pointer set, Fields (double arrays) or FieldsSP (float arrays of the
// single-precision interface: every load is widened to double and every store
// rounded to float, the arithmetic is the same).
// GEN: every pow whose exponent is a parameter (mpowp, mpowbp) skips the
// tests for the exponents 0.5, 1.5, 2 and 3, which the host has ruled out
// for the uploaded parameters (gen_exponents_ok); same results, fewer
// branches.
// PASS (kPassPlain, kPassFast, kPassRedo; cloudsc_column.cuh): the fast pass
// divides with fast_div, sets *bad when an operand of one of its divisions
// fell outside that division's exact window, and saves the PLUDE input of every level in
// plude_in[0..KLEV-1]; the redo pass, the column run again with IEEE division,
// reads PLUDE from plude_in.  A column whose fast pass sets *bad must be rerun
// (its outputs, stored in the same places by both passes, are then final) and
// leaves its warning count to the rerun.
// With BUD, PEXTRA is accumulated in place, so the two passes share its
// levels: the fast pass adds a level's budget terms only while no division
// has reported (everything it computed up to there is IEEE's), and records
// in *kbud the first level it left out; the redo pass adds the terms of the
// levels from *kbud on.  Every slot then receives IEEE's terms once each, in
// level order, as in one IEEE run.
template <typename Real, bool F32M, bool BUD = false, bool OPT = false, typename FT = Fields, bool GEN = false,
          int PASS = kPassPlain>
CSC_DEV void cloudsc_column(const FT &F, const Shape &sh, int ib, int jl, bool active = true, bool *bad = nullptr,
                            double *plude_in = nullptr, int *kbud = nullptr) {
  const KParams<Real> &P = KP<Real>();
  const KParamsD &PD = c_kd;
  typedef double D;
#define C(x) Real(x)
  constexpr bool FAST_ = PASS == kPassFast;
  DivCheck divbad_;
  if constexpr (FAST_) {
    if (P.rcp_force) divbad_.acc = ~0u;  // a parameter divisor fast_div_k cannot take: rerun
  }
  const int np = sh.nproma, klev = sh.klev;
  const size_t s2 = (size_t)np * klev, s2h = (size_t)np * (klev + 1);
  const size_t o2 = (size_t)ib * s2 + jl, o2h = (size_t)ib * s2h + jl, o1 = (size_t)ib * np + jl;
  const D dt = sh.ptsphy;
  const D zqtmst = 1.0 / dt;
  const Real rdt = Real(dt), rqtmst = Real(zqtmst);
  const Real zepsec = C(1.E-14);
  const D zepsecd = 1.E-14;
  const Real zepsilon = C(100.0 * 0x1p-52);  // 100*EPSILON(1._JPRB), cloudsc.F90:693
  const int ncldtop0 = P.ncldtop - 1;  // 0-based first level of the loop
  const Real zrdtgdp_f = C(1.0) / (rdt * P.rg);

  // per-column inputs
  const Real plsm = Real(ld(F.plsm + o1));
  const bool ldcum = ld(F.ldcum + o1) != 0;
  const int ktype = ld(F.ktype + o1);
  const Real peis = Real(ld(F.peis + o1));
  const D paph_surf = ld(F.paph + o2h + (size_t)klev * np);
  // reciprocals of the column's constant divisors (time step, surface
  // pressure), taken once
  const Real rrdt = RCP(rdt), rpsurf = RCP(Real(paph_surf));
  Real zadvw = C(1.0), zadvwd = C(1.0);
  if (ktype == 1 && P.rmfadvw > C(0.0)) {
    zadvw = C(1.0) - P.rmfadvw;
    zadvwd = C(1.0) - P.rmfadvw * P.rmfadvwdd;
  }
  const Real zconstpow = plsm > C(0.5) ? P.zconst_pow_land : P.zconst_pow_sea;

  // SPP: the factors EXP(MU + XMAG*PGP2DSPP(JL,MP)) of this column, one per
  // perturbation (CLOUDINHOM: two, fields MP and MP+1); grid-box length and
  // the default FSD for the inhomogeneity paths
  double sppf[9];
  double zgridlen = 0.0;
  const bool spp = OPT && P.lspp;
  if constexpr (OPT) {
#pragma unroll
    for (int n = 0; n < 9; ++n) sppf[n] = 1.0;
    if (P.lspp) {
      const double *g = F.pgp2dspp + (size_t)ib * np * F.nrftotal + jl;
#pragma unroll 1
      for (int n = 0; n < 8; ++n)
        if (P.spp_on[n]) sppf[n] = xexp(double(P.spp_mu[2 * n]) + double(P.spp_xmag[2 * n]) * ld(g + (size_t)(P.spp_mp[n] - 1) * np));
      if (P.spp_on[CLOUDSC_SPP_CLOUDINHOM])
        sppf[8] = xexp(double(P.spp_mu[2 * CLOUDSC_SPP_CLOUDINHOM + 1]) +
                       double(P.spp_xmag[2 * CLOUDSC_SPP_CLOUDINHOM + 1]) *
                           ld(g + (size_t)P.spp_mp[CLOUDSC_SPP_CLOUDINHOM] * np));
    }
    if (P.lcloud_inhomog || P.lrad_cloud_inhomog)
      zgridlen = 2 * double(P.ra) * xsqrt(double(P.rpi) * ld(F.pgaw + o1)) * 0.001;  // :1944
  }

  // state carried between levels
  D paph_k = ld(F.paph + o2h);
  Real pmfu_k = Real(ld(F.pmfu + o2)), pmfd_k = Real(ld(F.pmfd + o2));
  Real za_prev = C(0.0), qr_prev = C(0.0), qs_prev = C(0.0), t_prev = C(0.0), pap_prev = C(0.0);
  Real qxnm1_l = C(0.0), qxnm1_i = C(0.0), qxnm1_r = C(0.0), qxnm1_s = C(0.0);
  Real zanewm1 = C(0.0), zcovptot = C(0.0), zcovpmax = C(0.0), zcldtopdist = C(0.0);
  bool llrainliq = true;
  Real prainfrac = C(0.0);
  Real pfplsx_i = C(0.0), pfplsx_r = C(0.0), pfplsx_s = C(0.0);  // ZPFPLSX(JK)
  D fsqlf = 0.0, fsqif = 0.0, fcqlng = 0.0, fcqnng = 0.0, fsqltur = 0.0, fsqitur = 0.0;
  unsigned nwarn = 0;
  // first level whose budget terms the fast pass leaves to the redo pass
  int kbud_l = klev;
  if constexpr (BUD && PASS == kPassRedo) kbud_l = *kbud;

  // flux index 1 (:4231-4241)
  if (active) {
    F.pfsqlf[o2h] = 0.0; F.pfsqif[o2h] = 0.0; F.pfsqrf[o2h] = 0.0; F.pfsqsf[o2h] = 0.0;
    F.pfcqlng[o2h] = 0.0; F.pfcqnng[o2h] = 0.0; F.pfcqrng[o2h] = 0.0; F.pfcqsng[o2h] = 0.0;
    F.pfsqltur[o2h] = 0.0; F.pfsqitur[o2h] = 0.0;
  }

  // (KLON,KLEV,N) arrays: the block stride is N*KLON*KLEV, species m at +m*KLON*KLEV
  const size_t o5 = (size_t)ib * 5 * s2 + jl, o4 = (size_t)ib * 4 * s2 + jl, o2s = (size_t)ib * 2 * s2 + jl;
  for (int k = 0; k < klev; ++k) {
    const size_t ok = o2 + (size_t)k * np;
    const size_t ok5 = o5 + (size_t)k * np, ok4 = o4 + (size_t)k * np, ok2s = o2s + (size_t)k * np;
    // ---------------- loads for level k ----------------
    const D pt_k = ld(F.pt + ok), pq_k = ld(F.pq + ok), pa_k = ld(F.pa + ok);
    const D cml_t = ld(F.cml_t + ok), cml_q = ld(F.cml_q + ok), cml_a = ld(F.cml_a + ok);
    const D cl_l = ld(F.cml_cld + ok5), cl_i = ld(F.cml_cld + ok5 + s2),
            cl_r = ld(F.cml_cld + ok5 + 2 * s2), cl_s = ld(F.cml_cld + ok5 + 3 * s2);
    const D pc_l = ld(F.pclv + ok5), pc_i = ld(F.pclv + ok5 + s2), pc_r = ld(F.pclv + ok5 + 2 * s2),
            pc_s = ld(F.pclv + ok5 + 3 * s2);
    const D pap_kd = ld(F.pap + ok);
    const D paph_k1 = ld(F.paph + o2h + (size_t)(k + 1) * np);
    const D pvfl = ld(F.pvfl + ok), pvfi = ld(F.pvfi + ok);
    const D pludeli1 = ld(F.pludeli + ok4), pludeli2 = ld(F.pludeli + ok4 + s2);
    const bool last = (k == klev - 1);
    Real pmfu_k1 = C(0.0), pmfd_k1 = C(0.0), plu_k1 = C(0.0);
    if (!last) {
      pmfu_k1 = Real(ld(F.pmfu + ok + np));
      pmfd_k1 = Real(ld(F.pmfd + ok + np));
      plu_k1 = Real(ld(F.plu + ok + np));
    }
    // PLUDE is read and written in place: the fast pass keeps each level's
    // input for a rerun of the column, which reads it back from there
    D plude_k;
    if constexpr (PASS == kPassRedo) {
      plude_k = plude_in[k];
    } else {
      plude_k = F.plude[ok];
      if constexpr (PASS == kPassFast) plude_in[k] = plude_k;
    }
    const Real pap_k = Real(pap_kd);

    // ---------------- first guess (:982-1002) ----------------
    // The state is kept in double in both kernels (tendencies are small
    // differences of it); `Real` copies feed the process rates.
    const D tD = pt_k + dt * cml_t;
    D qvD = pq_k + dt * cml_q;
    D aD = pa_k + dt * cml_a;
    const D aorig = aD;
    const D q0_l = pc_l + dt * cl_l, q0_i = pc_i + dt * cl_i, q0_r = pc_r + dt * cl_r,
            q0_s = pc_s + dt * cl_s;
    D qlD = q0_l, qiD = q0_i, qrD = q0_r, qsD = q0_s;
    const Real t = Real(tD);

    // ---------------- saturation (:1087-1115) ----------------
    // (only the loop levels JK >= NCLDTOP read these)
    Real alfa = C(0.0), zfoeewm = C(0.0), zqsmix = C(0.0), zfoeew = C(0.0), zqsice = C(0.0);
    Real zfoeeliqt = C(0.0), zqsliq = C(0.0), el_e = C(0.0), ei_e = C(0.0);
    // 1/(1 - RETV FOEEW) for the mixed, ice and liquid saturation pressures:
    // the divisors of ZQSMIX/ZQSICE/ZQSLIQ and the ZCOR factors below
    Real rmix = C(0.0), rice = C(0.0), rliq = C(0.0);
    if (k >= ncldtop0) {
      Real x = (mx(P.rtice, mn(P.rtwat, t)) - P.rtice) * P.rtwat_rtice_r;
      alfa = mn(C(1.0), x * x);
      el_e = mexp<F32M>(DIV(P.r3les * (t - P.rtt), (t - P.r4les)));
      bool delta = xsign(C(1.0), t - P.rtt) > C(0.0);
      // the ice exponential whether or not a term needs it (no branch: the
      // two exponentials overlap)
      ei_e = mexp<F32M>(DIV(P.r3ies * (t - P.rtt), (t - P.r4ies)));
      Real wsum = (alfa < C(1.0)) ? alfa * el_e + (C(1.0) - alfa) * ei_e : el_e;
      const Real rpap = RCP(pap_k);
      zfoeewm = mn(DIVY((P.r2es * wsum), pap_k, rpap), C(0.5));
      zqsmix = zfoeewm;
      const Real dmix = C(1.0) - P.retv * zqsmix;
      rmix = RCP(dmix);
      zqsmix = DIVY(zqsmix, dmix, rmix);
      Real eew = delta ? P.r2es * el_e : P.r2es * ei_e;
      zfoeew = mn(DIVY(eew, pap_k, rpap), C(0.5));
      zfoeew = mn(C(0.5), zfoeew);
      const Real dice = C(1.0) - P.retv * zfoeew;
      rice = RCP(dice);
      zqsice = DIVY(zfoeew, dice, rice);
      zfoeeliqt = mn(DIVY((P.r2es * el_e), pap_k, rpap), C(0.5));
      zqsliq = zfoeeliqt;
      const Real dliq = C(1.0) - P.retv * zqsliq;
      rliq = RCP(dliq);
      zqsliq = DIVY(zqsliq, dliq, rliq);
    }

    // ---------------- tidy up (:1127-1199), double ----------------
    D loc_t = 0.0, loc_q = 0.0;
    D lneg_l = 0.0, lneg_i = 0.0, lneg_r = 0.0, lneg_s = 0.0;
    if (qlD + qiD < D(P.rlmin) || aD < D(P.ramin)) {
      D qadj;
      lneg_l = lneg_l + qlD;
      qadj = qlD * zqtmst;
      loc_q = loc_q + qadj;
      loc_t = loc_t - PD.ralvdcp * qadj;
      qvD = qvD + qlD;
      qlD = 0.0;
      lneg_i = lneg_i + qiD;
      qadj = qiD * zqtmst;
      loc_q = loc_q + qadj;
      loc_t = loc_t - PD.ralsdcp * qadj;
      qvD = qvD + qiD;
      qiD = 0.0;
      aD = 0.0;
    }
#define TIDY(QQ, LNEG, RAL)               \
  if (QQ < D(P.rlmin)) {                  \
    LNEG = LNEG + QQ;                     \
    D qadj = QQ * zqtmst;                 \
    loc_q = loc_q + qadj;                 \
    loc_t = loc_t - PD.RAL * qadj;        \
    qvD = qvD + QQ;                       \
    QQ = 0.0;                             \
  }
    TIDY(qlD, lneg_l, ralvdcp)
    TIDY(qiD, lneg_i, ralsdcp)
    TIDY(qrD, lneg_r, ralvdcp)
    TIDY(qsD, lneg_s, ralsdcp)
#undef TIDY
    aD = mx(0.0, mn(1.0, aD));
    const Real qv = Real(qvD), a = Real(aD);
    const Real ql = Real(qlD), qi = Real(qiD), qr = Real(qrD), qs = Real(qsD);
    const Real zli = ql + qi;
    Real liqfrac = C(0.0), icefrac = C(0.0);
    if (zli > P.rlmin) {
      liqfrac = DIV(ql, zli);
      icefrac = C(1.0) - liqfrac;
    }

    // FSD bookkeeping of this level (ZLFSD, ZANEWP, ZRATFSD, ZICEF, ZLIQF;
    // initial values :942-954)
    double lfsd = double(P.rcloud_frac_std), anewp = 0.0, ratfsd = 0.0, icef = 0.0, liqf = 0.0;
    D loc_a = 0.0, loc_cl = 0.0, loc_ci = 0.0, loc_cr = 0.0, loc_cs = 0.0;
    D qxn2d_l = 0.0, qxn2d_i = 0.0, qxn2d_r = 0.0, qxn2d_s = 0.0;
    Real pfplsx_i_n = C(0.0), pfplsx_r_n = C(0.0), pfplsx_s_n = C(0.0);
    Real covp_out = C(0.0);

    if (k >= ncldtop0) {
      // ================= level physics (:1228-3823) =================
      // running first-guess amounts (ZQXFG) in double: the limiters below take
      // min(rate, ZQXFG) and the clean-up removes ZQXFG exactly, so the solve's
      // residues stay at double rounding in the FP32-mixed kernel too
      D qxfg_l = qlD, qxfg_i = qiD, qxfg_r = qrD, qxfg_s = qsD;
      Real solac = C(0.0), solab = C(0.0);
      QA q;
      q.LL = q.II = q.RR = q.SS = q.LI = q.LV = q.IR = q.IV = q.RS = q.RV = q.SV = 0.0;
      Real qb_ll = C(0.0), qb_ii = C(0.0), qb_rl = C(0.0), qb_si = C(0.0), qb_sl = C(0.0);
      Real convsrce_l = C(0.0), convsrce_i = C(0.0), convsrce_r = C(0.0), convsrce_s = C(0.0);
      Real convsink_l = C(0.0), convsink_i = C(0.0);
      Real fallsrce_i = C(0.0), fallsrce_r = C(0.0), fallsrce_s = C(0.0);
      D qpretot = 0.0;
      // cloud budget terms of this level, 1-based as ZBUDCC(:,1:12),
      // ZBUDL(:,1:21), ZBUDI(:,1:17) (zero at the start of each level,
      // :1271-1273), and the process rates the budget reads
      struct Bud {
        double cc[13], l[22], i[18];
      } bd;
      Real b_rainaut = C(0.0), b_rainacc = C(0.0), b_snowaut = C(0.0), b_snowrime = C(0.0);
      Real b_psdep = C(0.0), b_psacr = C(0.0), b_piacr = C(0.0);
      if constexpr (BUD) {
#pragma unroll
        for (int n = 0; n < 13; ++n) bd.cc[n] = 0.0;
#pragma unroll
        for (int n = 0; n < 22; ++n) bd.l[n] = 0.0;
#pragma unroll
        for (int n = 0; n < 18; ++n) bd.i[n] = 0.0;
      }
      // The ZSOLQA accumulators are double in both instantiations; in the
      // FP32-mixed kernel each process rate (Real) is widened when added.
      // QADD/QSUB act on the stored entry of a pair (see struct QA); the
      // comment beside each names the reference's pair of updates.
#define QADD(E, X) q.E = q.E + double(X)
#define QSUB(E, X) q.E = q.E - double(X)

      // derived variables (:1281-1324)
      const Real zdp = Real(paph_k1 - paph_k);
      const Real zgdp = DIV(P.rg, zdp);
      const Real zrho = DIV(pap_k, (P.rd * t));
      const Real rrho = RCP(zrho);
      // (RDENSREF/ZRHO)**0.4 appears in three processes: one shared logarithm
      const PowBase b_dens = mbase<F32M>(DIVY(P.rdensref, zrho, rrho));
      // its two powers (0.4 in the rain fall speed, the binary32 0.4 in rain
      // evaporation and riming), computed here for every point so that they
      // overlap with the code around them instead of waiting inside their
      // processes' branches
      const Real fallcorr_r = mpowb<F32M>(b_dens, C(0.4));
      const Real fallcorr_f = mpowbp<F32M, GEN>(b_dens, P.flt_0p4);
      const Real zdtgdp = rdt * zgdp;
      const Real zrdtgdp = zdp * zrdtgdp_f;
      Real zcorqsliq, zcorqsice, zcorqsmix, zdqsmixdt, zevaplimmix, rcqsmix;
      {
        Real xl = t - P.r4les, xi = t - P.r4ies;
        Real zfacw = DIV(P.r5les, (xl * xl));
        Real zcor = rliq;  // 1/(1 - RETV ZFOEELIQT)
        Real zdqsliqdt = zfacw * zcor * zqsliq;
        zcorqsliq = C(1.0) + P.ralvdcp * zdqsliqdt;
        Real zfaci = DIV(P.r5ies, (xi * xi));
        zcor = rice;  // 1/(1 - RETV ZFOEEW)
        Real zdqsicedt = zfaci * zcor * zqsice;
        zcorqsice = C(1.0) + P.ralsdcp * zdqsicedt;
        Real zfac = alfa * zfacw + (C(1.0) - alfa) * zfaci;
        zcor = rmix;  // 1/(1 - RETV ZFOEEWM)
        zdqsmixdt = zfac * zcor * zqsmix;
        Real foeldcpm = alfa * P.ralvdcp + (C(1.0) - alfa) * P.ralsdcp;
        zcorqsmix = C(1.0) + foeldcpm * zdqsmixdt;
        rcqsmix = RCP(zcorqsmix);
        zevaplimmix = mx(DIVY((zqsmix - qv), zcorqsmix, rcqsmix), C(0.0));
      }
      const Real ztmpa = RCP(mx(a, C(0.01)));
      // MAX(ZEPSEC, 1 - ZA), the divisor of the clear-sky humidity and of
      // the precipitation's relative-humidity threshold
      const Real d1ma = mx(zepsec, C(1.0) - a), r1ma = RCP(d1ma);
      Real zliqcld = ql * ztmpa;
      Real zicecld = qi * ztmpa;
      const Real zlicld = zliqcld + zicecld;

      // evaporate very small amounts (:1334-1342)
      if (qlD < D(P.rlmin)) {
        q.LV = -qlD;  // ZSOLQA(V,L) = ql, ZSOLQA(L,V) = -ql
      }
      if (qiD < D(P.rlmin)) {
        q.IV = -qiD;  // ZSOLQA(V,I) = qi, ZSOLQA(I,V) = -qi
      }

      // 3.2 detrainment (:1362-1398)
      if (!last) {
        plude_k = plude_k * D(zdtgdp);
        if (ldcum && Real(plude_k) > zepsec && plu_k1 > zepsec) {
          solac = solac + DIV(Real(plude_k), plu_k1);
          convsrce_l = Real(pludeli1) * zdtgdp;
          convsrce_i = Real(pludeli2) * zdtgdp;
          QADD(LL, convsrce_l);
          QADD(II, convsrce_i);
          if constexpr (BUD) {  // :1378-1380
            bd.l[3] = convsrce_l * zqtmst;
            bd.i[3] = convsrce_i * zqtmst;
            bd.cc[3] = DIV(zqtmst * plude_k, plu_k1);
          }
        } else {
          plude_k = 0.0;
        }
        if (P.lmfdsnow) {
          convsrce_r = Real(ld(F.psnde + ok2s)) * zdtgdp;
          convsrce_s = Real(ld(F.psnde + ok2s + s2)) * zdtgdp;
          QADD(RR, convsrce_r);
          QADD(SS, convsrce_s);
        }
        if (active) F.plude[ok] = plude_k;
      }

      // 3.3 subsidence source and evaporation (:1419-1492)
      if (k > ncldtop0) {
        Real zmf = mx(C(0.0), (pmfu_k * zadvw + pmfd_k * zadvwd) * zdtgdp);
        Real zacust = zmf * zanewm1;
        Real lcust_l = zmf * qxnm1_l;
        Real lcust_i = zmf * qxnm1_i;
        convsrce_l = convsrce_l + lcust_l;
        convsrce_i = convsrce_i + lcust_i;
        Real zdtdp = DIV(P.zrdcp * C(0.5) * (t_prev + t), Real(paph_k));
        Real zwtot = mn(P.rg * (pmfu_k * zadvw + pmfd_k * zadvwd), DIVY((pap_k - pap_prev), rdt, rrdt));
        Real zdtforc = zdtdp * rdt * zwtot;
        Real zdqs = zanewm1 * zdtforc * zdqsmixdt;
        Real lfinalsum = C(0.0);
        {
          Real zlfinal = mx(C(0.0), lcust_l - zdqs);
          Real zevap = mn((lcust_l - zlfinal), zevaplimmix);
          zlfinal = lcust_l - zevap;
          lfinalsum = lfinalsum + zlfinal;
          QADD(LL, lcust_l);
          QSUB(LV, zevap);  // (V,L) += zevap, (L,V) -= zevap
          if constexpr (BUD) {  // :1459-1460
            bd.l[4] = lcust_l * zqtmst;
            bd.l[5] = -zevap * zqtmst;
          }
        }
        {
          Real zlfinal = mx(C(0.0), lcust_i - zdqs);
          Real zevap = mn((lcust_i - zlfinal), zevaplimmix);
          zlfinal = lcust_i - zevap;
          lfinalsum = lfinalsum + zlfinal;
          QADD(II, lcust_i);
          QSUB(IV, zevap);  // (V,I) += zevap, (I,V) -= zevap
          if constexpr (BUD) {  // :1475-1476
            bd.i[4] = lcust_i * zqtmst;
            bd.i[5] = -zevap * zqtmst;
          }
        }
        solac = solac + zacust;
        if constexpr (BUD) bd.cc[4] = zacust * zqtmst;  // :1484
        if (lfinalsum < zepsec) {
          solac = solac - zacust;
          if constexpr (BUD) bd.cc[5] = -zacust * zqtmst;  // :1488
        }
      }

      // subsidence sink (:1499-1514)
      if (!last) {
        Real zmfdn = mx(C(0.0), (pmfu_k1 * zadvw + pmfd_k1 * zadvwd) * zdtgdp);
        solab = solab + zmfdn;
        qb_ll = qb_ll + zmfdn;
        qb_ii = qb_ii + zmfdn;
        convsink_l = zmfdn;
        convsink_i = zmfdn;
      }

      // 3.4 erosion, ITURBEROSION=3 (:1689-1754)
      {
        Real zldifdt = P.rcldiff * rdt;
        if (spp && P.spp_on[CLOUDSC_SPP_RCLDIFF]) zldifdt = P.rcldiff * rdt * Real(sppf[CLOUDSC_SPP_RCLDIFF]);
        Real pl = Real(plude_k);
        if (ktype >= 2 && pl > zepsec && peis < C(10.0)) {
          zldifdt = C(20.0) * P.rcldiff_convi * zldifdt;
        } else if (ktype == 1 && pl > zepsec) {
          zldifdt = C(2.0) * P.rcldiff_convi * zldifdt;
        }
        if (zli > zepsec) {
          Real zqe = DIVY((qv - a * zqsmix), d1ma, r1ma);
          Real ze = mx(zqsmix - zqe, C(0.0));
          Real zleros = C(0.333) * a * (C(1.) - a) * zldifdt * ze;
          zleros = mn(zleros, zevaplimmix);
          zleros = mn(zleros, zli);
          Real zaeros = DIV(C(0.5) * zleros, zlicld);
          solac = solac - zaeros;
          QSUB(LV, liqfrac * zleros);  // (V,L) +=, (L,V) -=
          QSUB(IV, icefrac * zleros);  // (V,I) +=, (I,V) -=
          if constexpr (BUD) {  // :1749-1751
            bd.l[7] = -liqfrac * zleros * zqtmst;
            bd.i[7] = -icefrac * zleros * zqtmst;
            bd.cc[7] = -zaeros * zqtmst;
          }
        }
      }

      // 4.1 fall speeds (:1783-1844), sedimentation (:1852-1877)
      Real fs_i0 = P.rvice;
      if constexpr (OPT) {
        // LAERICESED: 0.002 ZRE_ICE**1.0 from the ice effective radius (:1798-1803)
        if (P.laericesed) fs_i0 = C(0.002) * Real(ld(F.pre_ice + ok));
      }
      const Real fs_i = (spp && P.spp_on[CLOUDSC_SPP_FALLSPEED]) ? fs_i0 * Real(sppf[CLOUDSC_SPP_FALLSPEED])
                                                                 : fs_i0;  // :1806-1808
      const Real fs_s = P.rvsnow;
      Real fs_r = C(0.0);
      {
        Real ztemp = C(0.5) * (qr + qxnm1_r);
        if (ztemp != C(0.0)) {
          Real zfallcorr = fallcorr_r;
          Real zrlambda = mpowp<F32M, GEN>(DIVP(zrho * ztemp, P.rcl_lam1r, P.rcp_rcl_lam1r), P.rcl_lam2r);
          fs_r = P.rxfallspeedrain * zfallcorr * P.rcl_const7r * mpowp<F32M, GEN>(zrlambda, P.rcl_dr);
        }
      }
      if (k > ncldtop0) {
        fallsrce_i = pfplsx_i * zdtgdp;
        QADD(II, fallsrce_i);
        if constexpr (BUD) bd.i[12] = fallsrce_i * zqtmst;  // :1865
        qxfg_i = qxfg_i + fallsrce_i;
        qpretot = qpretot + qxfg_i;
        fallsrce_r = pfplsx_r * zdtgdp;
        QADD(RR, fallsrce_r);
        qxfg_r = qxfg_r + fallsrce_r;
        qpretot = qpretot + qxfg_r;
        fallsrce_s = pfplsx_s * zdtgdp;
        QADD(SS, fallsrce_s);
        qxfg_s = qxfg_s + fallsrce_s;
        qpretot = qpretot + qxfg_s;
      }
      const Real fallsink_i = zdtgdp * zrho * fs_i;
      const Real fallsink_r = zdtgdp * zrho * fs_r;
      const Real fallsink_s = zdtgdp * zrho * fs_s;

      // 4.2 precipitation fraction (:1898-1919)
      Real zcovpclr, zraincld, zraincldm1, zsnowcld;
      if (qpretot > zepsec) {
        zcovptot = C(1.0) - (DIV((C(1.0) - zcovptot) * (C(1.0) - mx(a, za_prev)), (C(1.0) - mn(za_prev, C(1.0) - C(1.E-06)))));
        zcovptot = mx(zcovptot, P.rcovpmin);
        zcovpclr = mx(C(0.0), zcovptot - a);
        const Real rcov = RCP(zcovptot);
        zraincld = DIVY(C(0.5) * (qr + qr_prev), zcovptot, rcov);
        zraincldm1 = DIVY(C(0.5) * (qr + qxnm1_r), zcovptot, rcov);
        zsnowcld = DIVY(C(0.5) * (qs + qs_prev), zcovptot, rcov);
        zcovpmax = mx(zcovptot, zcovpmax);
      } else {
        zraincld = C(0.0);
        zraincldm1 = C(0.0);
        zsnowcld = C(0.0);
        zcovptot = C(0.0);
        zcovpclr = C(0.0);
        zcovpmax = C(0.0);
      }

      // 4.3 warm rain, IWARMRAIN=3, IRAINACC=1 (:1930-2259)
      if (zliqcld > zepsec) {
        const PowBase b_liq = mbase<F32M>(zliqcld);
        Real zeaut = P.rcl_inhomogaut, zeacc = P.rcl_inhomogacc;
        if constexpr (OPT) {
          double zcldraincorr = 0.0;
          if (P.lcloud_inhomog || P.lrad_cloud_inhomog) {  // :1937-1967
            const double zqtot = mn((qvD + qlD) * 1000.0, 30.0);
            zcldraincorr = 1.0 - 0.8 * double(a);
            const double zphip1 = .2 + .01 * zqtot + .0027 * (zqtot * zqtot) - .00008 * (zqtot * zqtot * zqtot);
            const double zphip2 = zphip1 - 0.2;
            const double zphip3 = 0.123 * xexp(-zphip1 * 0.55);
            const double zanew2 = mx(double(a), 0.1);
            const double zphic = xpow(zgridlen * zanew2, (1.0 / 3.0)) *
                                 xpow(xpow(zphip3 * zgridlen * zanew2, 1.5) + 3.0 * zphip3, -0.17);
            double zfracsdc = (zphip1 - zphip2 * zanew2) * zphic;
            if (double(a) > 0.95) zfracsdc = 0.17 * zphic;
            lfsd = 1.3 * zfracsdc;
          }
          if (P.lcloud_inhomog) {  // :2075-2098
            const double aa = double(a);
            const double fc2 = xpow(lfsd, 2.0);
            const double zea = xpow(1.0 + fc2, DIV((double(P.rcl_kkbauq) - 1.0) * double(P.rcl_kkbauq), 2.0));
            const double zphir = xpow(zgridlen * aa, (1.0 / 3.0)) * xpow(xpow(0.11 * zgridlen * aa, 1.14) + 1.0, -0.22);
            double zfracsdr = (1.1 - 0.8 * aa) * zphir;
            if (aa > 0.95) zfracsdr = 0.3 * zphir;
            const double fr2 = xpow(zfracsdr, 2.0);
            const double kb = double(P.rcl_kkbac);
            const double zec = xpow(1.0 + fc2, DIV((kb - 1.0) * kb, 2.0)) * xpow(1.0 + fr2, DIV((kb - 1.0) * kb, 2.0)) *
                               xexp(zcldraincorr * kb * kb * xsqrt(xlog(1.0 + fc2) * xlog(1.0 + fr2)));
            zeaut = Real(zea);
            zeacc = Real(zec);
          }
          if (spp && P.spp_on[CLOUDSC_SPP_CLOUDINHOM]) {  // :2106-2109
            zeaut = zeaut * Real(sppf[CLOUDSC_SPP_CLOUDINHOM]);
            zeacc = zeacc * Real(sppf[8]);
          }
        }
        Real zrainaut = zeaut * rdt * P.rcl_kkaau * mpowbp<F32M, GEN>(b_liq, P.kkbauq_m1) * zconstpow;
        qb_rl = qb_rl + zrainaut;
        Real zrainacc = C(0.0);
        if (zraincld > zepsec) {
          zrainacc = zeacc * rdt * P.rcl_kkaac * mpowbp<F32M, GEN>(b_liq, P.kkbac_m1) *
                     mpowp<F32M, GEN>(zraincld, P.rcl_kkbac);
        }
        qb_rl = qb_rl + zrainacc;
        if constexpr (BUD) {
          b_rainaut = zrainaut;
          b_rainacc = zrainacc;
        }
      }

      // 4.4 rain evaporation (:2271-2378)
      {
        Real zzrh = P.rprecrhmax + DIVY((C(1.0) - P.rprecrhmax) * zcovpmax, d1ma, r1ma);
        zzrh = mn(mx(zzrh, P.rprecrhmax), C(1.0));
        Real zxramid = P.ramid;
        if (spp && P.spp_on[CLOUDSC_SPP_RAMID]) {  // :2282-2287
          zxramid = P.ramid * Real(sppf[CLOUDSC_SPP_RAMID]);
          if (P.spp_lramidlimit1) zxramid = mn(C(1.0), zxramid);
        }
        Real zrhc = zxramid;
        Real zsigk = DIVY(pap_k, Real(paph_surf), rpsurf);
        if (zsigk > C(0.8)) {
          Real s = DIVK((zsigk - C(0.8)), 0.2);
          zrhc = zxramid + (C(1.0) - zxramid) * (s * s);
        }
        zzrh = mn(zrhc, zzrh);
        zzrh = mn(C(0.9), zzrh);
        Real zqe = mx(C(0.0), mn(qv, zqsliq));
        if (zcovpclr > zepsec && zraincldm1 > zepsec && zqe < zzrh * zqsliq) {
          Real zpreclr = zraincldm1;
          Real zfallcorr = fallcorr_f;
          Real zesatliq = P.rv_rd * (P.r2es * el_e);
          Real zlambda = mpowp<F32M, GEN>(DIV(P.rcl_lam1r, (zrho * zpreclr)), P.rcl_lam2r);
          const PowBase b_lam = mbase<F32M>(zlambda);
          Real zevap_denom = P.rcl_cdenom1 * zesatliq - P.rcl_cdenom2 * t * zesatliq +
                             P.rcl_cdenom3 * mpow<F32M>(t, C(3.0)) * pap_k;
          Real zcorr2 = DIV(mpow<F32M>(DIVK(t, 273.), C(1.5)) * C(393.), (t + C(120.)));
          Real zsubsat = mx(zzrh * zqsliq - zqe, C(0.0));
          Real zbeta = (DIV(C(0.15), zqsliq)) * (t * t) * zesatliq * P.rcl_const1r * (DIV(zcorr2, zevap_denom)) *
                       (DIV(C(0.78), (mpowbp<F32M, GEN>(b_lam, P.rcl_const4r))) +
                        DIV(P.rcl_const2r * mpow<F32M>(zrho * zfallcorr, C(0.5)), (mpow<F32M>(zcorr2, C(0.5)) * mpowbp<F32M, GEN>(b_lam, P.rcl_const3r))));
          Real zdenom = C(1.0) + zbeta * rdt * zcorqsliq;
          Real zdpevap = DIV(zcovpclr * zbeta * rdt * zsubsat, zdenom);
          if (spp && P.spp_on[CLOUDSC_SPP_RAINEVAP]) zdpevap = zdpevap * Real(sppf[CLOUDSC_SPP_RAINEVAP]);
          D zevap = mn(D(zdpevap), qxfg_r);
          QSUB(RV, zevap);  // (V,R) += zevap, (R,V) -= zevap
          if constexpr (BUD) bd.l[20] = -zevap * zqtmst;  // :2363
          qxfg_r = qxfg_r - zevap;
        }
      }

      // 4.5 ice deposition, IDEPICE=1 (:2404-2499)
      {
        if (za_prev < P.rcldtopcf && a >= P.rcldtopcf) {
          zcldtopdist = C(0.0);
        } else {
          zcldtopdist = zcldtopdist + DIV(zdp, (zrho * P.rg));
        }
        if (t < (P.rtt - C(5.)) && qxfg_l > P.rlmin) {
          Real zsupersatice = DIV((zqsliq - zqsice), zqsice);
          Real zvpice = DIVP((P.r2es * ei_e) * P.rv, P.rd, P.rcp_rd);
          Real zicenuclei = C(1000.0) * mexp<F32M>(C(12.96) * zsupersatice - C(0.639));
          Real zadd = DIV(P.rlstt * (DIV(P.rlstt, (P.rv * t)) - C(1.0)), (C(2.4E-2) * t));
          Real zbdd = DIV(P.rv * t * pap_k, (C(2.21) * zvpice));
          Real zcvds = DIV(C(7.8) * mpow<F32M>(DIVY(zicenuclei, zrho, rrho), C(0.666)) * zsupersatice, (C(8.87) * (zadd + zbdd)));
          Real zice0 = mx(zicecld, DIVY(zicenuclei * P.riceinit, zrho, rrho));
          Real zinew = mpow<F32M>(C(0.666) * zcvds * rdt + mpow<F32M>(zice0, C(0.666)), C(1.5));
          D zdepos = D(mx(P.rcl_overlapliqice * a * (zinew - zice0), C(0.0)));
          zdepos = mn(zdepos, qxfg_l);
          Real zinfactor = mn(DIVK(zicenuclei, 15000.), C(1.0));
          zdepos = zdepos * D(mn(zinfactor + (C(1.0) - zinfactor) *
                                               (P.rdepliqrefrate + DIVP(zcldtopdist, P.rdepliqrefdepth, P.rcp_rdepliqrefdepth)),
                               C(1.0)));
          QSUB(LI, zdepos);  // (I,L) += zdepos, (L,I) -= zdepos
          qxfg_i = qxfg_i + zdepos;
          qxfg_l = qxfg_l - zdepos;
          if constexpr (BUD) {  // :2495-2496
            bd.l[11] = -zdepos * zqtmst;
            bd.i[11] = zdepos * zqtmst;
          }
        }
      }

      // 4.7 snow deposition, IDEPSNOW=1 (:2698-2745)
      {
        Real zsupersatice = mx(DIV((qv - zqsmix), zqsmix), C(0.0));
        if (t < P.rtt && zsnowcld > zepsec && zsupersatice > C(0.0)) {
          Real zvpice = DIVP((P.r2es * ei_e) * P.rv, P.rd, P.rcp_rd);
          Real zaplusb = P.rcl_apb1 * zvpice - P.rcl_apb2 * zvpice * t + pap_k * P.rcl_apb3 * (t * t * t);
          Real zcorrfac = mpow<F32M>(rrho, C(0.5));
          Real zcorrfac2 = (mpow<F32M>(DIVK(t, 273.0), C(1.5))) * (DIV(C(393.0), (t + C(120.0))));
          Real zpr02 = zrho * zsnowcld * P.rcl_const1s;
          const PowBase b_pr02 = mbase<F32M>(zpr02);
          Real zterm1 = DIV(zsupersatice * (t * t) * zvpice * zcorrfac2 * P.rcl_const2s, (zrho * zaplusb));
          Real zterm2 = C(0.65) * P.rcl_const6s * mpowbp<F32M, GEN>(b_pr02, P.rcl_const4s) +
                        DIV(P.rcl_const3s * mpow<F32M>(zcorrfac, C(0.5)) * mpow<F32M>(zrho, C(0.5)) *
                            mpowbp<F32M, GEN>(b_pr02, P.rcl_const5s), mpow<F32M>(zcorrfac2, C(0.5)));
          Real zpsdep = mx(zcovptot * zterm1 * zterm2 * rdt, C(0.0));
          zpsdep = DIVY(mn(zpsdep, qv - zqsmix), zcorqsmix, rcqsmix);
          QADD(SV, zpsdep);  // (S,V) += zpsdep, (V,S) -= zpsdep
          if constexpr (BUD) b_psdep = zpsdep;
        }
      }

      // revise in-cloud condensate (:2750-2754)
      zliqcld = Real(qxfg_l) * ztmpa;
      zicecld = Real(qxfg_i) * ztmpa;

      // 4.8 ice -> snow autoconversion (:2769-2800)
      if (t <= P.rtt && zicecld > zepsec) {
        Real zzco = rdt * P.rsnowlin1 * mexp<F32M>(P.rsnowlin2 * (t - P.rtt));
        Real zlcrit = P.rlcritsnow;
        bool aer = false;
        if constexpr (OPT) {
          // LAERICEAUTO: the aerosol's critical ice amount, the rate scaled by
          // (RNICE/PNICE)**0.333 (:2776-2779)
          if (P.laericeauto) {
            zlcrit = Real(ld(F.picrit_aer + ok));
            zzco = zzco * mpow<F32M>(DIV(P.rnice, Real(ld(F.pnice + ok))), C(0.333));
            aer = true;
          }
        }
        if (!aer && spp && P.spp_on[CLOUDSC_SPP_RLCRITSNOW])
          zlcrit = P.rlcritsnow * Real(sppf[CLOUDSC_SPP_RLCRITSNOW]);
        Real r = DIV(zicecld, zlcrit);
        Real ztemp = C(-1.) * (r * r);
        Real zsnowaut = (ztemp < C(50.0)) ? zzco * (C(1.0) - mexp<F32M>(ztemp)) : zzco;
        qb_si = qb_si + zsnowaut;
        if constexpr (BUD) b_snowaut = zsnowaut;
      }

      // 4.12 melting (:2815-2862)
      {
        D zicetot = qxfg_i + qxfg_s;
        Real zmeltmax = C(0.0);
        if (zicetot > zepsec && t > P.rtt) {
          Real zsubsat = mx(zqsice - qv, C(0.0));
          Real ztdmtw0 = t - P.rtt -
                         zsubsat * (C(1329.31) + C(0.0074615) * (pap_k - C(0.85E5)) - C(40.637) * (t - C(275.0)));
          Real zcons1 = xabs(DIVP(rdt * (C(1.0) + C(0.5) * ztdmtw0), P.rtaumel, P.rcp_rtaumel));
          zmeltmax = mx(ztdmtw0 * zcons1 * P.zrldcp, C(0.0));
        }
        if (zmeltmax > zepsec && zicetot > zepsec) {
          const D rit = RCP(D(zicetot));
          D zalfa = DIVY(qxfg_i, D(zicetot), rit);
          D zmelt = mn(qxfg_i, zalfa * D(zmeltmax));
          qxfg_i = qxfg_i - zmelt;
          qxfg_r = qxfg_r + zmelt;
          QSUB(IR, zmelt);  // (R,I) += zmelt, (I,R) -= zmelt
          if constexpr (BUD) {  // :2856-2857
            bd.i[15] = -zmelt * zqtmst;
            bd.l[17] = zmelt * zqtmst;
          }
          zalfa = DIVY(qxfg_s, D(zicetot), rit);
          zmelt = mn(qxfg_s, zalfa * D(zmeltmax));
          qxfg_s = qxfg_s - zmelt;
          qxfg_r = qxfg_r + zmelt;
          QADD(RS, zmelt);  // (R,S) += zmelt, (S,R) -= zmelt
          if constexpr (BUD) bd.i[16] = -zmelt * zqtmst;  // :2858
        }
      }

      // 4.13 rain freezing (:2877-2933)
      if (qr > zepsec) {
        if (t <= P.rtt && t_prev > P.rtt) {
          Real zqpre = mx(qs + qr, zepsec);
          prainfrac = DIV(qr, zqpre);
          llrainliq = prainfrac > P.flt_0p8;
        }
        if (t < P.rtt) {
          Real zfrzmax;
          if (llrainliq) {
            Real zlambda = mpowp<F32M, GEN>(DIV(P.rcl_lam1r, (zrho * qr)), P.rcl_lam2r);
            Real ztemp = mn(P.rcl_fzrab * (t - P.rtt), C(50.));
            Real zfrz = rdt * (DIVY(P.rcl_const5r, zrho, rrho)) * (mexp<F32M>(ztemp) - C(1.)) * mpowp<F32M, GEN>(zlambda, P.rcl_const6r);
            zfrzmax = mx(zfrz, C(0.0));
          } else {
            Real zcons1 = xabs(DIVP(rdt * (C(1.0) + C(0.5) * (P.rtt - t)), P.rtaumel, P.rcp_rtaumel));
            zfrzmax = mx((P.rtt - t) * zcons1 * P.zrldcp, C(0.0));
          }
          if (zfrzmax > zepsec) {
            D zfrz = mn(qrD, D(zfrzmax));
            QSUB(RS, zfrz);  // (S,R) += zfrz, (R,S) -= zfrz
            if constexpr (BUD) bd.l[18] = -zfrz * zqtmst;  // :2927
          }
        }
      }

      // 4.14 homogeneous freezing of cloud liquid (:2948-2960)
      {
        Real zfrzmax = mx((P.rthomo - t) * P.zrldcp, C(0.0));
        if (zfrzmax > zepsec && qxfg_l > zepsec) {
          D zfrz = mn(qxfg_l, D(zfrzmax));
          QSUB(LI, zfrz);  // (I,L) += zfrz, (L,I) -= zfrz
          if constexpr (BUD) bd.l[19] = -zfrz * zqtmst;  // :2958
        }
      }

      // 4.9 riming (:2973-3017)
      if (t <= P.rtt && zliqcld > zepsec && zsnowcld > zepsec && zcovptot > C(0.01)) {
        Real zfallcorr = fallcorr_f;
        Real zsnowrime = P.rcl_effrime * zcovptot * rdt * P.rcl_const7s * zfallcorr *
                         mpowp<F32M, GEN>(zrho * zsnowcld * P.rcl_const1s, P.rcl_const8s);
        zsnowrime = mn(zsnowrime, C(1.0));
        qb_sl = qb_sl + zsnowrime;
        if constexpr (BUD) b_snowrime = zsnowrime;
      }

      // PSD slopes (:3026-3069), PSACR (:3084-3115), PIACR (:3171-3198)
      if (t <= P.rtt && prainfrac < zepsec && zraincld > zepsec) {
        Real zlamr = mpowp<F32M, GEN>(DIV(P.rcl_lam1r, (zrho * zraincld)), P.rcl_lam2r);
        Real zn0r = P.rcl_x1r * mpowp<F32M, GEN>(zlamr, P.rcl_x2r);
        Real zlamr3 = zlamr * zlamr * zlamr;
        if (zsnowcld > zepsec) {
          Real zlams = mpowp<F32M, GEN>(DIV(P.rcl_lam1s, (zrho * zsnowcld)), P.rcl_lam2s);
          Real zn0s = P.rcl_x1s;
          Real zfalldiff = mx(xabs(fs_r - fs_s), DIV2((fs_r + fs_s), C(8.)));
          Real zfac = DIV(P.rpi * P.rpi * P.rdenswat * zrho * zn0r * zn0s, (zlams * zlamr3));
          Real zrat = DIV(zlamr, zlams);
          Real zpsacr =
              DIV(zcovptot * rdt * zfac * zfalldiff * ((C(0.5) * zrat + C(2.)) * zrat + C(5.)), zlamr3);
          QSUB(RS, zpsacr);  // (S,R) += zpsacr, (R,S) -= zpsacr
          if constexpr (BUD) b_psacr = zpsacr;
        }
        if (zicecld > zepsec) {
          Real zlami = mpowp<F32M, GEN>(DIV(P.rcl_lam1s, (zrho * zicecld)), P.rcl_lam2s);
          Real zn0i = P.rcl_x1s;
          Real zfalldiff = mx(xabs(fs_r - fs_i), DIV2((fs_r + fs_i), C(8.)));
          Real zfac = DIV(P.rpi * P.rpi * P.rdenswat * C(0.1) * zrho * zn0r * zn0i, (zlami * zlamr3));
          Real zrat = DIV(zlamr, zlami);
          Real zpiacr =
              DIV(zcovptot * rdt * zfac * zfalldiff * ((C(0.5) * zrat + C(2.)) * zrat + C(5.)), zlamr3);
          QADD(IR, zpiacr);  // (I,R) += zpiacr, (R,I) -= zpiacr
          if constexpr (BUD) b_piacr = zpiacr;
        }
      }

      // 4.15 snow sublimation, ISUBLSNOW=1 (:3254-3318)
      {
        Real zzrh = P.rprecrhmax + DIVY((C(1.0) - P.rprecrhmax) * zcovpmax, d1ma, r1ma);
        zzrh = mn(mx(zzrh, P.rprecrhmax), C(1.0));
        Real zqe = DIVY((qv - a * zqsice), d1ma, r1ma);
        zqe = mx(C(0.0), mn(zqe, zqsice));
        if (zcovpclr > zepsec && qxfg_s > zepsec && zqe < zzrh * zqsice) {
          Real aa = zcovptot * zdtgdp;
          Real zpreclr = DIV(Real(qxfg_s) * zcovpclr, xsign(mx(xabs(aa), zepsilon), aa));
          Real zbeta1 = DIV(DIVP(xsqrt(DIVY(pap_k, Real(paph_surf), rpsurf)), P.rvrfactor, P.rcp_rvrfactor) * zpreclr, mx(zcovpclr, zepsec));
          Real zbeta = P.rg * P.rpecons * mpow<F32M>(zbeta1, C(0.5777));
          Real zdenom = C(1.0) + zbeta * rdt * zcorqsice;
          Real zdpr = DIV(zcovpclr * zbeta * (zqsice - zqe), zdenom) * zdp * P.zrg_r;
          Real zdpevap = zdpr * zdtgdp;
          if (spp && P.spp_on[CLOUDSC_SPP_SNOWSUBLIM]) zdpevap = zdpevap * Real(sppf[CLOUDSC_SPP_SNOWSUBLIM]);
          D zevap = mn(D(zdpevap), qxfg_s);
          QSUB(SV, zevap);  // (V,S) += zevap, (S,V) -= zevap
          if constexpr (BUD) bd.i[17] = -zevap * zqtmst;  // :3304
          zcovptot = mx(P.rcovpmin, zcovptot - mx(C(0.0), Real(DIV(D(zcovptot - a) * zevap, qxfg_s))));
          qxfg_s = qxfg_s - zevap;
        }
      }

      // evaporate small precipitation amounts (:3402-3412)
      if (qxfg_i < P.rlmin) QSUB(IV, qxfg_i);  // (V,I) +=, (I,V) -=
      if (qxfg_r < P.rlmin) QSUB(RV, qxfg_r);  // (V,R) +=, (R,V) -=
      if (qxfg_s < P.rlmin) QSUB(SV, qxfg_s);  // (V,S) +=, (S,V) -=
#undef QADD
#undef QSUB

      // 5.1 cloud cover (:3429-3438)
      D zda;
      {
        Real zanew = DIV((a + solac), (C(1.0) + solab));
        zanew = mn(zanew, C(1.0));
        if (zanew < P.ramin) zanew = C(0.0);
        zda = D(zanew) - aorig;
        zanewm1 = zanew;
      }

      // 5.2.1 sink truncation (:3455-3536), double: ratios, insertion sort
      // (IORDV, stable for ties), rows rescaled in sorted order
      const double qx[5] = {qlD, qiD, qrD, qsD, qvD};
      {
        double ratio[5];
        sink_ratios<FAST_>(q, qx, ratio, divbad_);
        double sr[5];
        int ord[5];
        sr[0] = ratio[0];
        ord[0] = 0;
#pragma unroll
        for (int jm = 1; jm < 5; ++jm) {
          const double rj = ratio[jm];
          bool done = false;
#pragma unroll
          for (int jn = jm - 1; jn >= 0; --jn) {
            if (!done) {
              if (sr[jn] <= rj) {
                sr[jn + 1] = rj;
                ord[jn + 1] = jm;
                done = true;
              } else {
                sr[jn + 1] = sr[jn];
                ord[jn + 1] = ord[jn];
              }
            }
          }
          if (!done) {
            sr[0] = rj;
            ord[0] = jm;
          }
        }
        // the order packed 3 bits per position: one copy of the row code
        unsigned code = 0;
#pragma unroll
        for (int jm = 0; jm < 5; ++jm) code |= (unsigned)ord[jm] << (3 * jm);
#pragma unroll 1
        for (int jm = 0; jm < 5; ++jm) scale_row<FAST_>((int)((code >> (3 * jm)) & 7u), q, qx, divbad_);
      }

      // 5.2.2 solve (:3546-3628), double, lower-triangular form
      double x_l, x_i, x_r, x_s, x_v;
      {
        x_l = qx[L] + (((0.0 + q.LL) + q.LI) + q.LV);
        x_i = qx[I] + ((((0.0 - q.LI) + q.II) + q.IR) + q.IV);
        x_r = qx[R] + ((((0.0 - q.IR) + q.RR) + q.RS) + q.RV);
        x_s = qx[S] + (((0.0 - q.RS) + q.SS) + q.SV);
        x_v = qx[V] + ((((0.0 - q.LV) - q.IV) - q.RV) - q.SV);
        const double d_l = ((1.0 + 0.0) + double(qb_ll) + double(qb_rl)) + double(qb_sl);
        const double d_i = ((1.0 + double(fallsink_i)) + double(qb_ii)) + double(qb_si);
        const double d_r = 1.0 + double(fallsink_r);
        const double d_s = 1.0 + double(fallsink_s);
        const double rd_l = RCP(d_l), rd_i = RCP(d_i);
        const double m_rl = DIVY((-double(qb_rl)), d_l, rd_l);
        const double m_sl = DIVY((-double(qb_sl)), d_l, rd_l);
        const double m_si = DIVY((-double(qb_si)), d_i, rd_i);
        x_r = x_r - m_rl * x_l;
        x_s = x_s - m_sl * x_l;
        x_s = x_s - m_si * x_i;
        x_s = DIV(x_s, d_s);
        x_r = DIV(x_r, d_r);
        x_i = DIVY(x_i, d_i, rd_i);
        x_l = DIVY(x_l, d_l, rd_l);
        // clip (:3633-3640)
        if (x_l < zepsecd) { x_v = x_v + x_l; x_l = 0.0; }
        if (x_i < zepsecd) { x_v = x_v + x_i; x_i = 0.0; }
        if (x_r < zepsecd) { x_v = x_v + x_r; x_r = 0.0; }
        if (x_s < zepsecd) { x_v = x_v + x_s; x_s = 0.0; }
      }
      qxnm1_l = Real(x_l);
      qxnm1_i = Real(x_i);
      qxnm1_r = Real(x_r);
      qxnm1_s = Real(x_s);
      qxn2d_l = x_l; qxn2d_i = x_i; qxn2d_r = x_r; qxn2d_s = x_s;

      // 5.3 fluxes to next level (:3658-3672)
      pfplsx_i_n = Real(double(fallsink_i) * x_i * double(zrdtgdp));
      pfplsx_r_n = Real(double(fallsink_r) * x_r * double(zrdtgdp));
      pfplsx_s_n = Real(double(fallsink_s) * x_s * double(zrdtgdp));
      if (pfplsx_s_n + pfplsx_r_n < zepsec) zcovptot = C(0.0);

      if constexpr (BUD) {  // diagnosed implicit rates (:3675-3699)
        bd.l[14] = -b_rainaut * x_l * zqtmst;
        bd.l[15] = -b_rainacc * x_l * zqtmst;
        bd.cc[6] = -convsink_l * zanewm1 * zqtmst;
        bd.l[6] = -convsink_l * x_l * zqtmst;
        bd.i[6] = -convsink_i * x_i * zqtmst;
        bd.i[13] = -fallsink_i * x_i * zqtmst;
        bd.l[21] = -b_snowrime * x_l * zqtmst;
        bd.i[14] = -b_snowaut * x_i * zqtmst;
      }

      // 6.1-6.3 tendencies (:3713-3769), double
      {
        D fq;
        fq = D(convsrce_l) + 0.0 - (0.0 + D(convsink_l)) * x_l;
        loc_t = loc_t + PD.ralvdcp * (x_l - qlD - fq) * zqtmst;
        loc_cl = 0.0 + (x_l - q0_l) * zqtmst;
        fq = D(convsrce_i) + D(fallsrce_i) - (D(fallsink_i) + D(convsink_i)) * x_i;
        loc_t = loc_t + PD.ralsdcp * (x_i - qiD - fq) * zqtmst;
        loc_ci = 0.0 + (x_i - q0_i) * zqtmst;
        fq = D(convsrce_r) + D(fallsrce_r) - (D(fallsink_r) + 0.0) * x_r;
        loc_t = loc_t + PD.ralvdcp * (x_r - qrD - fq) * zqtmst;
        loc_cr = 0.0 + (x_r - q0_r) * zqtmst;
        fq = D(convsrce_s) + D(fallsrce_s) - (D(fallsink_s) + 0.0) * x_s;
        loc_t = loc_t + PD.ralsdcp * (x_s - qsD - fq) * zqtmst;
        loc_cs = 0.0 + (x_s - q0_s) * zqtmst;
        loc_q = loc_q + (x_v - qvD) * zqtmst;
        loc_a = 0.0 + zda * zqtmst;
      }
      // 6.4 supersaturation check (:3765-3809), double
      {
        D q_upd = pq_k + dt * (loc_q + cml_q);
        D t_upd = pt_k + dt * (loc_t + cml_t);
        D a_upd = pa_k + dt * (loc_a + cml_a);
        D t_adj, q_adj, a_adj, l_adj, i_adj;
        supersatcheck<FAST_>(t_upd, q_upd, a_upd, pap_kd, t_adj, q_adj, a_adj, l_adj, i_adj, divbad_);
        loc_q = loc_q + q_adj * zqtmst;
        loc_t = loc_t + t_adj * zqtmst;
        loc_a = loc_a + a_adj * zqtmst;
        loc_cl = loc_cl + l_adj * zqtmst;
        loc_ci = loc_ci + i_adj * zqtmst;
        if constexpr (BUD) {  // :3787-3789
          bd.cc[2] = a_adj * zqtmst;
          bd.l[2] = l_adj * zqtmst;
          bd.i[2] = i_adj * zqtmst;
        }
        D zl_adj = q0_l + loc_cl * dt;
        if (zl_adj < -PD.rlmin) nwarn++;
        if (zl_adj < 0.0) {
          loc_cl = loc_cl - zl_adj * zqtmst;
          loc_q = loc_q + zl_adj * zqtmst;
          loc_t = loc_t - PD.ralvdcp * zl_adj * zqtmst;
        }
        D zi_adj = q0_i + loc_ci * dt;
        if (zi_adj < -PD.rlmin) nwarn++;
        if (zi_adj < 0.0) {
          loc_ci = loc_ci - zi_adj * zqtmst;
          loc_q = loc_q + zi_adj * zqtmst;
          loc_t = loc_t - PD.ralsdcp * zi_adj * zqtmst;
        }
      }
      covp_out = zcovptot;
      if constexpr (OPT) {
        if (P.lrad_cloud_inhomog) {
          const double pda = pa_k + zda;  // :3819-3823
          if (pda > 0.001) anewp = mx(mx(pda, double(covp_out)), 0.1);
          if (q0_l + q0_i + plude_k > double(P.rlmin)) {  // :4112-4125
            ratfsd = DIV(plude_k, (plude_k + q0_l + q0_i));
            ratfsd = mx(0.0, mn(1.0, ratfsd));
          }
          icef = x_i;
          liqf = x_l;
        }
      }
      if constexpr (BUD) {
        // inputs a section that is off does not read may be NULL
        auto opt = [&](const double *q) { return q ? ld(q + ok) : 0.0; };
        auto opti = [&](const int32_t *q) { return q ? ld(q + o1) : 0; };
        bool wr = active;
        if constexpr (FAST_) {
          if (divbad_.bad()) {
            wr = false;
            kbud_l = k < kbud_l ? k : kbud_l;
          }
        }
        if constexpr (PASS == kPassRedo) wr = wr && k >= kbud_l;
        if (wr)
          write_budgets(F, P, bd.cc, bd.l, bd.i, (size_t)ib * np * klev * F.kfldx + jl, np, klev, k, dt,
                        zqtmst, double(zdp), double(zrho), opt(F.pvfa), opt(F.pdyna), double(pvfl),
                        opt(F.pdynl), double(pvfi), opt(F.pdyni), opt(F.pdyns), opt(F.phrsw), opt(F.phrlw),
                        x_l, x_i, double(b_psdep), double(b_psacr), double(b_piacr), double(prainfrac), ktype,
                        opti(F.kpbltype), opti(F.kctop), double(peis));
      }
    }  // k >= ncldtop0

    // ice/liquid FSD of level k (:4307-4359), every level; the binary32
    // literals written as such at :4316,4321-4322 are their float values
    if constexpr (OPT) {
      if (P.lrad_cloud_inhomog) {
        const double zifsdback = 0.446585 * xpow(zgridlen, (1.0 / 3.0)) * xpow(xpow(0.308061 * zgridlen, 0.395736) + 1.0, -0.744527);
        const double zqtot = mx(mn((qvD + qiD) * 1000.0, 30.0), double(0.00001f));
        const double zrho_f = DIV(pap_kd, (double(P.rd) * tD));
        double zdelz = RCP(double(P.rg) * zrho_f) * (paph_k1 - paph_k) * 0.001;
        zdelz = mx(mn(zdelz, double(0.5f)), double(0.001f));
        const double zphi = xpow(DIV(zdelz, double(0.24f)), double(0.11f)) * xpow(DIV(zqtot, double(10.f)), double(0.03f));
        double zifsd = double(P.rcloud_frac_std);
        if (anewp > 0.95) {
          zifsd = zifsdback * zphi;
          zifsd = 1.3 * (zifsd + ratfsd * 1.5);
        } else if (anewp > 0.001 && anewp <= 0.95) {
          zifsd = zifsdback * zphi * 1.5;
          zifsd = 1.3 * (zifsd + ratfsd * 1.5);
        }
        double zfsd = double(P.rcloud_frac_std);
        if (icef > zepsecd) zfsd = zifsd;
        if (liqf > 0.0 && icef <= zepsecd) zfsd = lfsd;
        zfsd = mn(mx(0.1, zfsd), 3.575);
        if (active) F.pfsd[ok] = zfsd;
      }
    }

    // ---------------- outputs of level k ----------------
    if (active) {
      F.loc_t[ok] = loc_t;
      F.loc_q[ok] = loc_q;
      F.loc_a[ok] = loc_a;
      F.loc_cld[ok5] = loc_cl;
      F.loc_cld[ok5 + s2] = loc_ci;
      F.loc_cld[ok5 + 2 * s2] = loc_cr;
      F.loc_cld[ok5 + 3 * s2] = loc_cs;
      F.pcovptot[ok] = D(covp_out);
    }

    // precipitation fluxes at half level k (:4218-4224, 4297-4303)
    {
      const size_t oh = o2h + (size_t)k * np;
      const D fl = D(pfplsx_r) + 0.0, fn = D(pfplsx_s) + D(pfplsx_i);
      if (active) {
        F.pfplsl[oh] = fl;
        F.pfplsn[oh] = fn;
        F.pfhpsl[oh] = -PD.rlvtt * fl;
        F.pfhpsn[oh] = -PD.rlstt * fn;
      }
    }
    // DDH flux recurrences to half level k+1 (:4244-4292)
    {
      const size_t oh1 = o2h + (size_t)(k + 1) * np;
      const D zgdph_r = -PD.zrg_r * (paph_k1 - paph_k) * zqtmst;
      const D sqrf = fsqlf + (qxn2d_r - q0_r) * zgdph_r;
      const D cqrng = fcqlng + lneg_r * zgdph_r;
      const D sqsf = fsqif + (qxn2d_s - q0_s) * zgdph_r;
      const D cqsng = fcqnng + lneg_s * zgdph_r;
      fsqlf = fsqlf + (qxn2d_l - q0_l + pvfl * dt) * zgdph_r + pludeli1;
      fcqlng = fcqlng + lneg_l * zgdph_r;
      fsqltur = fsqltur + pvfl * dt * zgdph_r;
      fsqif = fsqif + (qxn2d_i - q0_i + pvfi * dt) * zgdph_r + pludeli2;
      fcqnng = fcqnng + lneg_i * zgdph_r;
      fsqitur = fsqitur + pvfi * dt * zgdph_r;
      if (active) {
        F.pfsqlf[oh1] = fsqlf;
        F.pfsqif[oh1] = fsqif;
        F.pfsqrf[oh1] = sqrf;
        F.pfsqsf[oh1] = sqsf;
        F.pfcqlng[oh1] = fcqlng;
        F.pfcqnng[oh1] = fcqnng;
        F.pfcqrng[oh1] = cqrng;
        F.pfcqsng[oh1] = cqsng;
        F.pfsqltur[oh1] = fsqltur;
        F.pfsqitur[oh1] = fsqitur;
      }
    }

    // carry to level k+1
    za_prev = a;
    qr_prev = qr;
    qs_prev = qs;
    t_prev = t;
    pap_prev = pap_k;
    paph_k = paph_k1;
    pmfu_k = pmfu_k1;
    pmfd_k = pmfd_k1;
    pfplsx_i = pfplsx_i_n;
    pfplsx_r = pfplsx_r_n;
    pfplsx_s = pfplsx_s_n;
    CSC_LEVEL_SYNC();
  }
  // precipitation fluxes at the surface half level KLEV+1
  {
    const size_t oh = o2h + (size_t)klev * np;
    const D fl = D(pfplsx_r) + 0.0, fn = D(pfplsx_s) + D(pfplsx_i);
    if (active) {
      F.pfplsl[oh] = fl;
      F.pfplsn[oh] = fn;
      F.pfhpsl[oh] = -PD.rlvtt * fl;
      F.pfhpsn[oh] = -PD.rlstt * fn;
    }
  }
  if (active) F.prainfrac_toprfz[o1] = D(prainfrac);
  if (active && nwarn && F.ncounters && !(FAST_ && divbad_.bad())) atomic_add(F.ncounters, nwarn);
  if constexpr (FAST_) *bad = active && divbad_.bad();
  if constexpr (FAST_ && BUD) *kbud = kbud_l;
#undef C
}

#undef DIV
#undef DIVK
#undef DIV2
#undef DIVP
#undef RCP
#undef DIVY

}  // namespace cloudsc
