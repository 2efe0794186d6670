// TEST INFRASTRUCTURE ONLY -- not part of the product library.
//
// The GPU kernels' per-column code (openifs_b200/csrc/cloudsc_body.cuh),
// compiled unchanged for the host with no FMA contraction.  Double precision
// uses plibm.h's exp/pow, exactly as on the GPU; compiled with
// -DHOSTEMU_GLIBC the double-precision exp/pow are glibc's instead.  The tests
// compare it with the oracle built against the same libm: a bit-for-bit match
// proves that the kernel's logic (its fused single pass, sparse 5x5 matrices,
// operation order) restates the reference exactly.
#include <cmath>
#include <cstdint>
#include <cstring>

#define CSC_DEV inline
#include "../../openifs_b200/csrc/cloudsc_column.cuh"
#include "../../openifs_b200/csrc/cloudsc_kparams.h"

namespace cloudsc {
static KParams<double> c_kpd;
static KParams<float> c_kpf;
static KParamsD c_kd;
template <typename Real>
inline const KParams<Real> &KP();
template <>
inline const KParams<double> &KP<double>() { return c_kpd; }
template <>
inline const KParams<float> &KP<float>() { return c_kpf; }
template <typename T>
inline T ld(const T *p) { return *p; }
inline void atomic_add(uint32_t *p, uint32_t v) { *p += v; }
inline double xabs(double x) { return std::fabs(x); }
inline float xabs(float x) { return std::fabs(x); }
inline double xsign(double a, double b) { return std::copysign(a, b); }
inline float xsign(float a, float b) { return std::copysign(a, b); }
}  // namespace cloudsc

#include "../../openifs_b200/csrc/cloudsc_body.cuh"

using namespace cloudsc;

// FD: the kernels' fast pass and, for a column it reported, the rerun with
// IEEE division reading PLUDE from the fast pass's copy (on the host every
// division is IEEE; the redo build reports every one, so every column runs
// twice).
template <typename Real, bool F32M, bool GEN, bool FD>
static void column(const Fields &f, const Shape &sh, int ib, int jl) {
  if (FD && sh.klev <= kMaxLevFast) {
    double plude_in[kMaxLevFast];
    bool bad = false;
    cloudsc_column<Real, F32M, false, false, Fields, GEN, kPassFast>(f, sh, ib, jl, true, &bad, plude_in);
    if (bad) cloudsc_column<Real, F32M, false, false, Fields, GEN, kPassRedo>(f, sh, ib, jl, true, nullptr, plude_in);
  } else {
    cloudsc_column<Real, F32M, false, false, Fields, GEN>(f, sh, ib, jl);
  }
}
typedef void (*ColumnFn)(const Fields &, const Shape &, int, int);
// indexed by form + 3 * GEN + 6 * FASTDIV
static const ColumnFn kColumn[12] = {
    column<double, false, false, false>, column<double, true, false, false>, column<float, true, false, false>,
    column<double, false, true, false>,  column<double, true, true, false>,  column<float, true, true, false>,
    column<double, false, false, true>,  column<double, true, false, true>,  column<float, true, false, true>,
    column<double, false, true, true>,   column<double, true, true, true>,   column<float, true, true, true>};

extern "C" int hostemu_batched(const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot,
                               double ptsphy, void **a, int precision) {
  Derived d;
#ifdef CLOUDSC_HOST_LIBM_GLIBC
  d.zconst_pow_land = std::pow(p->rcl_kk_cloud_num_land, p->rcl_kkbaun);
  d.zconst_pow_sea = std::pow(p->rcl_kk_cloud_num_sea, p->rcl_kkbaun);
#else
  d.zconst_pow_land = plibm_pow(p->rcl_kk_cloud_num_land, p->rcl_kkbaun);
  d.zconst_pow_sea = plibm_pow(p->rcl_kk_cloud_num_sea, p->rcl_kkbaun);
#endif
  d.flt_0p4 = (double)0.4f;
  d.flt_0p8 = (double)0.8f;
  fill_kparams(*p, d, c_kpd);
  fill_kparams(*p, d, c_kpf);
  fill_kparams_d(*p, c_kd);
  uint32_t nwarn = 0;
  Fields f;
  f.pt = (const double *)a[0]; f.pq = (const double *)a[1]; f.cml_t = (const double *)a[2];
  f.cml_q = (const double *)a[3]; f.cml_a = (const double *)a[4]; f.cml_cld = (const double *)a[5];
  f.loc_t = (double *)a[6]; f.loc_q = (double *)a[7]; f.loc_a = (double *)a[8]; f.loc_cld = (double *)a[9];
  f.pvfl = (const double *)a[10]; f.pvfi = (const double *)a[11]; f.pap = (const double *)a[12];
  f.paph = (const double *)a[13]; f.plsm = (const double *)a[14]; f.ldcum = (const int32_t *)a[15];
  f.ktype = (const int32_t *)a[16]; f.peis = (const double *)a[17]; f.plu = (const double *)a[18];
  f.plude = (double *)a[19]; f.pludeli = (const double *)a[20]; f.psnde = (const double *)a[21];
  f.pmfu = (const double *)a[22]; f.pmfd = (const double *)a[23]; f.pa = (const double *)a[24];
  f.pclv = (const double *)a[25]; f.pcovptot = (double *)a[26]; f.prainfrac_toprfz = (double *)a[27];
  f.pfsqlf = (double *)a[28]; f.pfsqif = (double *)a[29]; f.pfcqnng = (double *)a[30];
  f.pfcqlng = (double *)a[31]; f.pfsqrf = (double *)a[32]; f.pfsqsf = (double *)a[33];
  f.pfcqrng = (double *)a[34]; f.pfcqsng = (double *)a[35]; f.pfsqltur = (double *)a[36];
  f.pfsqitur = (double *)a[37]; f.pfplsl = (double *)a[38]; f.pfplsn = (double *)a[39];
  f.pfhpsl = (double *)a[40]; f.pfhpsn = (double *)a[41];
  f.ncounters = &nwarn;
  Shape sh = {nproma, klev, ngpblks, ngptot, 0, ptsphy};
  for (int ib = 0; ib < ngpblks; ++ib) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    for (int jl = 0; jl < icend; ++jl) {
      // precision: the form (0 FP64, 1 FP32-mixed, 2 FP32 physics), plus
      // 0x100 for the GEN column code (parameter-exponent pows untested) and
      // 0x200 for the kernels' fast pass with its rerun (column, FD)
      const int form = (precision & 0xff) > 2 ? 2 : (precision & 0xff);
      const int gen = (precision & 0x100) ? 1 : 0, fd = (precision & 0x200) ? 1 : 0;
      kColumn[form + 3 * gen + 6 * fd](f, sh, ib, jl);
    }
  }
  return (int)nwarn;
}

// CLOUD_SATADJ: the kernel's point code (satadj_point.cuh) over every point of
// the batched arrays, in the order of fields.SATADJ_FIELDS.
#include "../../openifs_b200/csrc/satadj_point.cuh"

extern "C" int hostemu_satadj_batched(const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot,
                                      double ptsphy, void **a) {
  Derived d;
  d.zconst_pow_land = d.zconst_pow_sea = 0.0;
  d.flt_0p4 = (double)0.4f;
  d.flt_0p8 = (double)0.8f;
  fill_kparams(*p, d, c_kpd);
  const double **in = (const double **)a;
  double **out = (double **)(a + 18);
  const KParams<double> &k = c_kpd;
  const double zqtmst = 1.0 / ptsphy;
  const size_t np = nproma, kl = klev;
  int nwarn = 0;
  for (int ib = 0; ib < ngpblks; ++ib) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    for (int jk = 0; jk < klev; ++jk)
      for (int jl = 0; jl < icend; ++jl) {
        const size_t i = (ib * kl + jk) * np + jl;
        if (jk < k.ncldtop - 1) {
          for (int m = 0; m < 5; ++m) out[m][i] = 0.0;
          continue;
        }
        const size_t oh = (ib * (kl + 1) + jk) * np + jl, o4 = (ib * 4 * kl + jk) * np + jl;
        satadj_point(k, ptsphy, zqtmst, in[0][i], in[1][oh], in[1][oh + np], in[1][(ib * (kl + 1) + kl) * np + jl],
                     in[2][i], in[3][i], in[4][i], in[5][i], in[6][i], in[7][i], in[8][i], in[9][i], in[10][i],
                     in[11][i], in[12][i], in[13][i], in[14][i], in[15][i], in[16][o4 + 2 * kl * np],
                     in[16][o4 + 3 * kl * np], in[17][i], out[0][i], out[1][i], out[2][i], out[3][i], out[4][i],
                     nwarn);
      }
  }
  return nwarn;
}

// SLTEND's supersaturation adjustment: the kernel's point code over every
// point, arrays in the order of fields.SLTEND_FIELDS.
extern "C" int hostemu_sltend_batched(const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot,
                                      double tsphy, void **a) {
  Derived d;
  d.zconst_pow_land = d.zconst_pow_sea = 0.0;
  d.flt_0p4 = (double)0.4f;
  d.flt_0p8 = (double)0.8f;
  fill_kparams(*p, d, c_kpd);
  const KParams<double> &k = c_kpd;
  const double **in = (const double **)a;
  double *ptent = (double *)a[8], *ptenq = (double *)a[9], *ptena = (double *)a[10], *ptencld = (double *)a[11];
  double *padja = (double *)a[12], *padjl = (double *)a[13], *padji = (double *)a[14];
  const double zrtsphy = 1.0 / tsphy;
  const size_t np = nproma, kl = klev;
  for (int ib = 0; ib < ngpblks; ++ib) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    for (int jk = k.ncldtop - 1; jk < klev; ++jk)
      for (int jl = 0; jl < icend; ++jl) {
        const size_t i = (ib * kl + jk) * np + jl, oc = (ib * 5 * kl + jk) * np + jl;
        const double zt = in[0][i] + tsphy * (in[5][i] + ptent[i]);
        const double zq = in[1][i] + tsphy * (in[6][i] + ptenq[i]);
        const double za = in[2][i] + tsphy * (in[7][i] + ptena[i]);
        double ta, qa, aa, la, ia;
        supersatcheck_kft1(k, zt, zq, za, in[3][i], ta, qa, aa, la, ia);
        ptent[i] = ptent[i] + ta * zrtsphy;
        ptenq[i] = ptenq[i] + qa * zrtsphy;
        ptena[i] = ptena[i] + aa * zrtsphy;
        ptencld[oc] = ptencld[oc] + la * zrtsphy;
        ptencld[oc + kl * np] = ptencld[oc + kl * np] + ia * zrtsphy;
        padja[i] = aa * zrtsphy;
        padjl[i] = la * zrtsphy;
        padji[i] = ia * zrtsphy;
      }
  }
  return 0;
}

// The kernels' forms 3-5 on one column: the plain column code, or (FD) the
// fast pass and, for a column it reported, the rerun, the two passes
// splitting PEXTRA's levels as the kernels do.
template <bool BUD, bool OPT, bool GEN, bool FD>
static void column_opt(const Fields &f, const Shape &sh, int ib, int jl) {
  if (FD && sh.klev <= kMaxLevFast) {
    double plude_in[kMaxLevFast];
    bool bad = false;
    int kbud = sh.klev;
    cloudsc_column<double, false, BUD, OPT, Fields, GEN, kPassFast>(f, sh, ib, jl, true, &bad, plude_in, &kbud);
    if (bad)
      cloudsc_column<double, false, BUD, OPT, Fields, GEN, kPassRedo>(f, sh, ib, jl, true, nullptr, plude_in,
                                                                      &kbud);
  } else {
    cloudsc_column<double, false, BUD, OPT, Fields, GEN>(f, sh, ib, jl);
  }
}
// indexed by (BUD && OPT ? 2 : OPT ? 1 : 0) + 3 * GEN + 6 * FD
static const ColumnFn kColumnOpt[12] = {
    column_opt<true, false, false, false>, column_opt<false, true, false, false>, column_opt<true, true, false, false>,
    column_opt<true, false, true, false>,  column_opt<false, true, true, false>,  column_opt<true, true, true, false>,
    column_opt<true, false, false, true>,  column_opt<false, true, false, true>,  column_opt<true, true, false, true>,
    column_opt<true, false, true, true>,   column_opt<false, true, true, true>,   column_opt<true, true, true, true>};

// CLOUDSC with the optional configurations (the kernel's BUD and OPT forms):
// the BATCHED_FIELDS arrays in `a`, the fields.DIAG_FIELDS arrays in `b`;
// flags 0x100 for the GEN column code, 0x200 for the fast pass with its rerun.
extern "C" int hostemu_batched_diag(const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot,
                                    double ptsphy, void **a, void **b, int kfldx, int flags) {
  Derived d;
#ifdef CLOUDSC_HOST_LIBM_GLIBC
  d.zconst_pow_land = std::pow(p->rcl_kk_cloud_num_land, p->rcl_kkbaun);
  d.zconst_pow_sea = std::pow(p->rcl_kk_cloud_num_sea, p->rcl_kkbaun);
#else
  d.zconst_pow_land = plibm_pow(p->rcl_kk_cloud_num_land, p->rcl_kkbaun);
  d.zconst_pow_sea = plibm_pow(p->rcl_kk_cloud_num_sea, p->rcl_kkbaun);
#endif
  d.flt_0p4 = (double)0.4f;
  d.flt_0p8 = (double)0.8f;
  fill_kparams(*p, d, c_kpd);
  fill_kparams(*p, d, c_kpf);
  fill_kparams_d(*p, c_kd);
  uint32_t nwarn = 0;
  Fields f{};
  const double **ad = (const double **)a;
  f.pt = ad[0]; f.pq = ad[1]; f.cml_t = ad[2]; f.cml_q = ad[3]; f.cml_a = ad[4]; f.cml_cld = ad[5];
  f.loc_t = (double *)a[6]; f.loc_q = (double *)a[7]; f.loc_a = (double *)a[8]; f.loc_cld = (double *)a[9];
  f.pvfl = ad[10]; f.pvfi = ad[11]; f.pap = ad[12]; f.paph = ad[13]; f.plsm = ad[14];
  f.ldcum = (const int32_t *)a[15]; f.ktype = (const int32_t *)a[16]; f.peis = ad[17]; f.plu = ad[18];
  f.plude = (double *)a[19]; f.pludeli = ad[20]; f.psnde = ad[21]; f.pmfu = ad[22]; f.pmfd = ad[23];
  f.pa = ad[24]; f.pclv = ad[25]; f.pcovptot = (double *)a[26]; f.prainfrac_toprfz = (double *)a[27];
  f.pfsqlf = (double *)a[28]; f.pfsqif = (double *)a[29]; f.pfcqnng = (double *)a[30];
  f.pfcqlng = (double *)a[31]; f.pfsqrf = (double *)a[32]; f.pfsqsf = (double *)a[33];
  f.pfcqrng = (double *)a[34]; f.pfcqsng = (double *)a[35]; f.pfsqltur = (double *)a[36];
  f.pfsqitur = (double *)a[37]; f.pfplsl = (double *)a[38]; f.pfplsn = (double *)a[39];
  f.pfhpsl = (double *)a[40]; f.pfhpsn = (double *)a[41];
  f.ncounters = &nwarn;
  const double **bd = (const double **)b;
  f.pvfa = bd[0]; f.pdyna = bd[1]; f.pdynl = bd[2]; f.pdyni = bd[3]; f.pdyns = bd[4];
  f.phrsw = bd[5]; f.phrlw = bd[6]; f.pgaw = bd[7]; f.kctop = (const int32_t *)b[8];
  f.kpbltype = (const int32_t *)b[9]; f.pgp2dspp = bd[10];
  f.pre_ice = bd[11]; f.picrit_aer = bd[12]; f.pnice = bd[13];
  f.pfsd = (double *)b[14];
  f.pextra = (double *)b[15];
  f.kfldx = kfldx;
  f.nrftotal = p->spp_nrftotal;
  const bool bud = p->lcldbudc || p->lcldbudl || p->lcldbudi || p->lcldbudt || p->lcldbud_vertint;
  const bool opt = p->lspp || p->lcloud_inhomog || p->lrad_cloud_inhomog || p->laericesed || p->laericeauto;
  Shape sh = {nproma, klev, ngpblks, ngptot, 0, ptsphy};
  for (int ib = 0; ib < ngpblks; ++ib) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    for (int jl = 0; jl < icend; ++jl) {
      const int form = bud && opt ? 2 : (opt ? 1 : 0);
      kColumnOpt[form + ((flags & 0x100) ? 3 : 0) + ((flags & 0x200) ? 6 : 0)](f, sh, ib, jl);
    }
  }
  return (int)nwarn;
}
