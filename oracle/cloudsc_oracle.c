/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Never linked into the product library;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Line-by-line CPU restatement of the reference's double-precision CLOUDSC:
 *   ifs-source/arpifs/phys_ec/cloudsc.F90            (SUBROUTINE CLOUDSC)
 *   ifs-source/arpifs/phys_ec/cloud_supersatcheck.F90:111-226
 *   ifs-source/arpifs/function/fcttre.func.h:37-184   (saturation functions)
 *   ifs-source/arpifs/function/fccld.func.h:26-27     (FOKOOP)
 * in the reference's default configuration (options hard-wired at
 * cloudsc.F90:727-793), plus the optional paths the switches turn on: the
 * cloud budget diagnostics (LCLDBUD*, :3832-4110), the SPP perturbations
 * (LSPP, :850-939) and the cloud-inhomogeneity/FSD paths (LCLOUD_INHOMOG,
 * LRAD_CLOUD_INHOMOG, :1937-2110, 4307-4359); the aerosol switches are off.
 * Loop order (JK outer, JL inner), local arrays and the order of every
 * floating-point operation follow the Fortran source; it is compiled with
 * -O2 -ffp-contract=off (no FMA contraction, like the reference's -no-fma
 * builds, compile_flags.cmake:535) and uses glibc exp/log/pow.
 * Precision quirks reproduced: default-REAL (binary32) literals at
 * cloudsc.F90:2320,2889,2980; the MIN(..)/ZCORQSMIX parenthesisation at :2733;
 * the PFSQRF/PFSQSF/PFCQRNG/PFCQSNG recurrences at :4251-4256.
 *
 * Parity unpinned: no CLOUDSC golden vector exists in the reference and the
 * Fortran cannot be compiled in this image; this restatement is the checker.
 * Outputs the reference leaves undefined are written as zeros here:
 * PCOVPTOT(:,1:NCLDTOP-1).  PTENDENCY_LOC_CLD(:,:,NCLV) and PFSD are not touched.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "oracle.h"

/*
 * libm: the reference's results depend on the last bit of EXP and ** (see
 * plibm.h).  The default build uses the system libm (glibc), i.e. the
 * reference as a gfortran build on Linux would run it; built with
 * -DORACLE_PLIBM it uses the portable exp/pow of plibm.h, the libm the B200
 * kernels use, so that the comparison isolates the kernels' logic.
 */
#ifdef ORACLE_PLIBM
#include "../openifs_b200/csrc/plibm.h"
#define exp(x) plibm_exp(x)
#define pow(x, y) plibm_pow(x, y)
#define log(x) plibm_log(x)
#endif

#define NCLV 5
#define NCLDQL 1
#define NCLDQI 2
#define NCLDQR 3
#define NCLDQS 4
#define NCLDQV 5

/* 1-based Fortran-order accessors */
#define A1(a, jl) (a)[(jl)-1]
/* budget terms and PEXTRA(KLON,KLEV,KFLDX), 1-based like the Fortran */
#define BCC(jl, n) zbudcc[((size_t)(n)-1) * klon + ((jl)-1)]
#define BL(jl, n) zbudl[((size_t)(n)-1) * klon + ((jl)-1)]
#define BI(jl, n) zbudi[((size_t)(n)-1) * klon + ((jl)-1)]
#define PX(jl, ik, is) pextra[(((size_t)(is)-1) * klev + ((ik)-1)) * klon + ((jl)-1)]
#define A2(a, jl, jk) (a)[((size_t)(jk)-1) * klon + ((jl)-1)]
#define A3(a, jl, jk, jm, n2) (a)[(((size_t)(jm)-1) * (n2) + ((jk)-1)) * klon + ((jl)-1)]
#define L2(a, jl, jm) (a)[((size_t)(jm)-1) * klon + ((jl)-1)]
#define L3(a, jl, jm, jn) (a)[((((size_t)(jn)-1) * NCLV + ((jm)-1)) * klon) + ((jl)-1)]

static inline double fmin_(double a, double b) { return a < b ? a : b; }
static inline double fmax_(double a, double b) { return a > b ? a : b; }

/* ---------------- fcttre.func.h / fccld.func.h ---------------- */
static inline double foedelta(const cloudsc_params *p, double t) {
  return fmax_(0.0, copysign(1.0, t - p->rtt));
}
static inline double foealfa(const cloudsc_params *p, double t) {
  double x = (fmax_(p->rtice, fmin_(p->rtwat, t)) - p->rtice) * p->rtwat_rtice_r;
  return fmin_(1.0, x * x);
}
static inline double foeewm(const cloudsc_params *p, double t) {
  return p->r2es * (foealfa(p, t) * exp(p->r3les * (t - p->rtt) / (t - p->r4les)) +
                    (1.0 - foealfa(p, t)) * exp(p->r3ies * (t - p->rtt) / (t - p->r4ies)));
}
static inline double foedem(const cloudsc_params *p, double t) {
  double xl = t - p->r4les, xi = t - p->r4ies;
  return foealfa(p, t) * p->r5alvcp * (1.0 / (xl * xl)) +
         (1.0 - foealfa(p, t)) * p->r5alscp * (1.0 / (xi * xi));
}
static inline double foeldcpm(const cloudsc_params *p, double t) {
  return foealfa(p, t) * p->ralvdcp + (1.0 - foealfa(p, t)) * p->ralsdcp;
}
static inline double foeeliq(const cloudsc_params *p, double t) {
  return p->r2es * exp(p->r3les * (t - p->rtt) / (t - p->r4les));
}
static inline double foeeice(const cloudsc_params *p, double t) {
  return p->r2es * exp(p->r3ies * (t - p->rtt) / (t - p->r4ies));
}
static inline double foeew(const cloudsc_params *p, double t) {
  double d = foedelta(p, t);
  return p->r2es * exp((p->r3les * d + p->r3ies * (1.0 - d)) * (t - p->rtt) /
                       (t - (p->r4les * d + p->r4ies * (1.0 - d))));
}
static inline double foeeliq2ice(const cloudsc_params *p, double t) {
  return exp((t - p->rtt) * (p->r3les / (t - p->r4les) - p->r3ies / (t - p->r4ies)));
}
static inline double fokoop(const cloudsc_params *p, double t) {
  return fmin_(p->rkoop1 - p->rkoop2 * t, foeeliq2ice(p, t));
}

/* ---------------- cloud_supersatcheck.F90:111-226 ---------------- */
static void supersatcheck(const cloudsc_params *p, int kidia, int kfdia, int kftliqice,
                          const double *pt, const double *pq, const double *pa, const double *pp,
                          double *pt_adj, double *pq_adj, double *pa_adj, double *pl_adj,
                          double *pi_adj) {
  const double zepsec = 1.E-14;
  for (int jl = kidia; jl <= kfdia; jl++) {
    double za_upd = 0.0, zda = 0.0;
    double zt = pt[jl - 1], zq = pq[jl - 1], za = pa[jl - 1];
    double zp_r = 1.0 / pp[jl - 1];
    zt = fmax_(zt, 160.0);
    za = fmax_(fmin_(za, 1.0), 0.0);
    /* ZRHC/ZSIGK (:128-133) are computed by the reference but never used */
    double zfoeeliq = fmin_(foeeliq(p, zt) * zp_r, 0.5);
    double zqsliq = zfoeeliq / (1.0 - p->retv * zfoeeliq);
    (void)zqsliq;
    double zfoeeice = fmin_(foeew(p, zt) * zp_r, 0.5);
    double zfokoop = fmin_(zfoeeice * (p->rkoop1 - p->rkoop2 * zt), zfoeeliq);
    double zqsliqk = zfokoop / (1.0 - p->retv * zfokoop);
    double zfoealfa = foealfa(p, zt);
    double zfoeemix = fmin_(foeewm(p, zt) * zp_r, 0.5);
    double zcor = 1.0 / (1.0 - p->retv * zfoeemix);
    double zqsmix = zfoeemix * zcor;
    double zcorqsmix = 1.0 + zqsmix * zcor * foedem(p, zt);
    zqsliqk = 0.5 * (zqsliqk + zqsmix);
    double zqslim = za * zqsmix + (1.0 - za) * zqsliqk;
    double zcond = fmax_(zq - zqslim, 0.0);
    if (zcond > zepsec) {
      double zfaci = zfoealfa + (1.0 - zfoealfa) * p->rssicefactor;
      zda = (1.0 - za) * zfaci;
      za_upd = za + zda;
      zqslim = za_upd * zqsmix + (1.0 - za_upd) * zqsliqk;
      zcond = (zq - zqslim) / zcorqsmix;
    }
    pt_adj[jl - 1] = foeldcpm(p, zt) * zcond;
    pq_adj[jl - 1] = -zcond;
    pa_adj[jl - 1] = zda;
    if (kftliqice == 1) { /* split by the mixed-phase fraction (:211-214) */
      pl_adj[jl - 1] = zcond * zfoealfa;
      pi_adj[jl - 1] = zcond * (1.0 - zfoealfa);
    } else { /* all liquid down to homogeneous freezing (:215-223) */
      int liquid = pt[jl - 1] + pt_adj[jl - 1] >= p->rthomo;
      pl_adj[jl - 1] = liquid ? zcond : 0.0;
      pi_adj[jl - 1] = liquid ? 0.0 : zcond;
    }
  }
}


/* SPP factor EXP(MU(i+1) + XMAG(i+1)*PGP2DSPP(JL, MP + off)) of perturbation
 * n (cloudsc.F90:1692,1807,2106-2107,2283,2347,2782,3289). */
static double spp_fac(const cloudsc_params *p, const double *pgp2dspp, int klon, int jl, int n, int i,
                      int off) {
  return exp(p->spp_mu[2 * n + i] + p->spp_xmag[2 * n + i] * pgp2dspp[(size_t)(p->spp_mp[n] + off - 1) * klon + (jl - 1)]);
}
#define SPP_ON(n) (p->lspp && p->spp_on[n])

int oracle_cloudsc(
    const cloudsc_params *p, int kidia, int kfdia, int klon, int klev, int lddiag,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_cld, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_cld, const double *pvfa,
    const double *pvfl, const double *pvfi, const double *pdyna, const double *pdynl,
    const double *pdyni, const double *pdynr, const double *pdyns, const double *phrsw,
    const double *phrlw, const double *pvervel, const double *pap, const double *paph,
    const double *pgeom, const double *plsm, const double *pgaw, const int32_t *ldcum,
    const int32_t *kctop, const int32_t *ktype, const int32_t *kpbltype, double *peis,
    const double *plu, double *plude, const double *pludeli, const double *psnde,
    const double *pmfu, const double *pmfd, const double *pgp2dspp, int ldslphy,
    const double *pa, const double *pclv, const double *plcrit_aer,
    const double *picrit_aer, const double *pre_ice, const double *pccn,
    const double *pnice, double *pcovptot, double *pfsd, double *prainfrac_toprfz,
    double *pfsqlf, double *pfsqif, double *pfcqnng, double *pfcqlng, double *pfsqrf,
    double *pfsqsf, double *pfcqrng, double *pfcqsng, double *pfsqltur,
    double *pfsqitur, double *pfplsl, double *pfplsn, double *pfhpsl, double *pfhpsn,
    double *pextra, int kfldx) {
  /* PLCRIT_AER and PCCN are read only by LAERLIQAUTOLSP and LAERLIQCOLL,
     whose code sits in the IWARMRAIN = 1 branch (:1985-1989, :2020-2023);
     IWARMRAIN is 3 (:727), so those two switches change nothing. */
  (void)lddiag; (void)pdynr; (void)pvervel; (void)pgeom; (void)ldslphy; (void)plcrit_aer; (void)pccn;

  if (!p || p->magic != CLOUDSC_PARAMS_MAGIC) return CLOUDSC_E_PARAMS;
  if (kidia < 1 || kfdia > klon || kidia > kfdia || klev < 2) return CLOUDSC_E_SHAPE;
  const int ncldtop = p->ncldtop;
  if (ncldtop < 2 || ncldtop > klev) return CLOUDSC_E_SHAPE;
  int nwarn = 0;

  /* cloud budget diagnostics (:3832-4110): which sections are on, and the
     PEXTRA fields they need (the reference ABORTs when KFLDX is too small,
     :3945,3970,4007,4048,4106, or KLEV < 60 with the vertical integral,
     :3851; the vertical integral writes level slots up to 83) */
  /* SPP perturbations and the cloud-inhomogeneity/FSD path (:850-939,
     1937-1971, 2075-2110, 3819-3823, 4112-4124, 4307-4359) */
  if (p->lspp) {
    for (int n = 0; n < 8; n++) {
      if (!p->spp_on[n]) continue;
      if (!pgp2dspp || p->spp_mp[n] < 1 || p->spp_mp[n] + (n == 7 ? 1 : 0) > p->spp_nrftotal)
        return CLOUDSC_E_SHAPE;
    }
  }
  const int linhom = p->lcloud_inhomog || p->lrad_cloud_inhomog;
  if (linhom && !pgaw) return CLOUDSC_E_NULL;
  /* aerosol-aware ice sedimentation and ice-to-snow autoconversion */
  if ((p->laericesed && !pre_ice) || (p->laericeauto && (!picrit_aer || !pnice))) return CLOUDSC_E_NULL;
  if (p->lrad_cloud_inhomog && !pfsd) return CLOUDSC_E_NULL;
  const int lbud = p->lcldbudc || p->lcldbudl || p->lcldbudi || p->lcldbudt || p->lcldbud_vertint;
  if (lbud) {
    int need = (p->lbud23 ? 26 : 0) + (p->lcldbud_vertint ? 1 : 0) + (p->lcldbudc ? 12 : 0) +
               (p->lcldbudl ? 22 : 0) + (p->lcldbudi ? 20 : 0) + (p->lcldbudt ? 13 : 0);
    if (!pextra || kfldx < need) return CLOUDSC_E_SHAPE;
    if (p->lcldbud_vertint && (klev < 84 || !ktype || !kpbltype || !kctop)) return CLOUDSC_E_SHAPE;
    if ((p->lcldbudc || p->lcldbud_vertint) && (!pvfa || !pdyna)) return CLOUDSC_E_NULL;
    if ((p->lcldbudl || p->lcldbud_vertint) && !pdynl) return CLOUDSC_E_NULL;
    if ((p->lcldbudi || p->lcldbud_vertint) && !pdyni) return CLOUDSC_E_NULL;
    if (p->lcldbud_vertint && !pdyns) return CLOUDSC_E_NULL;
    if (p->lcldbudt && (!phrsw || !phrlw)) return CLOUDSC_E_NULL;
  }

  /* constants (cloudsc.F90:693-848) */
  const double zepsilon = 100.0 * 0x1p-52; /* 100*EPSILON(1._JPRB) */
  const int iphase[NCLV + 1] = {0, 1, 2, 1, 2, 0};
  const int imelt[NCLV + 1] = {0, NCLDQI, NCLDQR, NCLDQS, NCLDQR, -99};
  double zvqx[NCLV + 1];
  int llfall[NCLV + 1];
  zvqx[NCLDQV] = 0.0;
  zvqx[NCLDQL] = 0.0;
  zvqx[NCLDQI] = p->rvice;
  zvqx[NCLDQR] = p->rvrain;
  zvqx[NCLDQS] = p->rvsnow;
  for (int jm = 1; jm <= NCLV; jm++) llfall[jm] = zvqx[jm] > 0.0;

  const double zqtmst = 1.0 / ptsphy;
  const double zrdcp = p->rd / p->rcpd;
  const double zepsec = 1.E-14;
  const double zrg_r = 1.0 / p->rg;
  const double zrldcp = 1.0 / (p->ralsdcp - p->ralvdcp);
  const double ztw1 = 1329.31, ztw2 = 0.0074615, ztw3 = 0.85E5, ztw4 = 40.637, ztw5 = 275.0;
  const double flt_0p4 = (double)0.4f, flt_0p8 = (double)0.8f;

  /* ---- local arrays ---- */
  size_t n1 = (size_t)klon, n2 = (size_t)klon * klev, n2h = (size_t)klon * (klev + 1);
  /* 67 (KLON) arrays, 13 (KLON,KLEV) arrays, 4 (KLON,KLEV,NCLV), 1 (KLON,KLEV+1,NCLV),
     13 (KLON,NCLV) and 3 (KLON,NCLV,NCLV); sized with margin */
  double *buf = (double *)calloc(
      n1 * 140 + n2 * 22 + n2 * NCLV * 4 + n2h * NCLV + n1 * NCLV * 16 + n1 * NCLV * NCLV * 3,
      sizeof(double));
  if (!buf) return CLOUDSC_E_TOO_LARGE;
  double *w = buf;
#define TAKE(n) (w += (n), w - (n))
  double *zadvw = TAKE(n1), *zadvwd = TAKE(n1), *zpaphd = TAKE(n1);
  double *zliqcld = TAKE(n1), *zicecld = TAKE(n1), *zlicld = TAKE(n1), *zrainaut = TAKE(n1);
  double *zrainacc = TAKE(n1), *zsnowaut = TAKE(n1), *zsnowrime = TAKE(n1), *zldefr = TAKE(n1);
  double *zacust = TAKE(n1), *zqpretot = TAKE(n1), *zlfinalsum = TAKE(n1);
  double *zsolab = TAKE(n1), *zsolac = TAKE(n1), *zicetot = TAKE(n1), *zdp = TAKE(n1);
  double *zgdp = TAKE(n1), *zrho = TAKE(n1), *zdtgdp = TAKE(n1), *zrdtgdp = TAKE(n1);
  double *zdtgdpf = TAKE(n1), *zdqsliqdt = TAKE(n1), *zdqsicedt = TAKE(n1), *zdqsmixdt = TAKE(n1);
  double *zcorqsliq = TAKE(n1), *zcorqsice = TAKE(n1), *zcorqsmix = TAKE(n1);
  double *zevaplimliq = TAKE(n1), *zevaplimice = TAKE(n1), *zevaplimmix = TAKE(n1);
  double *zmf = TAKE(n1), *zdqs = TAKE(n1), *zldifdt = TAKE(n1), *zanewm1 = TAKE(n1);
  double *zda = TAKE(n1), *zcovpclr = TAKE(n1), *zcovpmax = TAKE(n1), *zcovptot = TAKE(n1);
  double *zcldtopdist = TAKE(n1), *zraincld = TAKE(n1), *zraincldm1 = TAKE(n1);
  double *zsnowcld = TAKE(n1), *zsnowcldm1 = TAKE(n1), *zicenuclei = TAKE(n1);
  double *zmeltmax = TAKE(n1), *zfrzmax = TAKE(n1), *zlamr = TAKE(n1), *zlams = TAKE(n1);
  double *zlami = TAKE(n1), *zn0r = TAKE(n1), *zn0s = TAKE(n1), *zn0i = TAKE(n1);
  double *zpsacr = TAKE(n1), *zpiacr = TAKE(n1), *zpsdep = TAKE(n1), *zsinksum = TAKE(n1);
  double *zq_upd = TAKE(n1), *zt_upd = TAKE(n1), *za_upd = TAKE(n1);
  double *zt_adj = TAKE(n1), *zq_adj = TAKE(n1), *za_adj = TAKE(n1), *zl_adj = TAKE(n1);
  double *zi_adj = TAKE(n1);
  /* budget terms ZBUDCC(:,1:12), ZBUDL(:,1:21), ZBUDI(:,1:17), reset per level */
  double *zbudcc = TAKE(n1 * 12), *zbudl = TAKE(n1 * 21), *zbudi = TAKE(n1 * 17);
  /* FSD arrays (:581-586), initialised at :942-954 */
  double *zlfsd = TAKE(n2), *zanewp = TAKE(n2), *zratfsd = TAKE(n2), *zicef = TAKE(n2), *zliqf = TAKE(n2);
  int *llrainliq = (int *)TAKE(n1); /* n1 doubles >= n1 ints */

  double *ztp1 = TAKE(n2), *zli = TAKE(n2), *za = TAKE(n2), *zaorig = TAKE(n2);
  double *zliqfrac = TAKE(n2), *zicefrac = TAKE(n2), *zfoealfa = TAKE(n2);
  double *zfoeewm = TAKE(n2), *zfoeew = TAKE(n2), *zfoeeliqt = TAKE(n2);
  double *zqsmix = TAKE(n2), *zqsliq = TAKE(n2), *zqsice = TAKE(n2);
  double *zqx = TAKE(n2 * NCLV), *zqx0 = TAKE(n2 * NCLV), *zlneg = TAKE(n2 * NCLV);
  double *zqxn2d = TAKE(n2 * NCLV);
  double *zpfplsx = TAKE(n2h * NCLV);
  double *zqxn = TAKE(n1 * NCLV), *zqxfg = TAKE(n1 * NCLV), *zqxnm1 = TAKE(n1 * NCLV);
  double *zfluxq = TAKE(n1 * NCLV), *zfallsink = TAKE(n1 * NCLV), *zfallsrce = TAKE(n1 * NCLV);
  double *zfallspeed = TAKE(n1 * NCLV), *zconvsrce = TAKE(n1 * NCLV), *zconvsink = TAKE(n1 * NCLV);
  double *zlcust = TAKE(n1 * NCLV), *zratio = TAKE(n1 * NCLV);
  int *iorder = (int *)TAKE(n1 * NCLV);
  int *llindex3 = (int *)TAKE(n1 * NCLV);
  double *zsolqa = TAKE(n1 * NCLV * NCLV), *zsolqb = TAKE(n1 * NCLV * NCLV);
  double *zqlhs = TAKE(n1 * NCLV * NCLV);
#undef TAKE

  int jl, jk, jm, jn, jo, ik;
  for (jk = 1; jk <= klev; jk++) /* :942-954 (the zero arrays are zero from calloc) */
    for (jl = kidia; jl <= kfdia; jl++) A2(zlfsd, jl, jk) = p->rcloud_frac_std;

  /* cloudsc.F90:696-703 */
  for (jl = kidia; jl <= kfdia; jl++) {
    A1(zadvw, jl) = 1.0;
    A1(zadvwd, jl) = 1.0;
    if (A1(ktype, jl) == 1 && p->rmfadvw > 0) {
      A1(zadvw, jl) = 1.0 - p->rmfadvw;
      A1(zadvwd, jl) = 1.0 - p->rmfadvw * p->rmfadvwdd;
    }
  }

  /* 1. initial values (:963-1011) */
  for (jk = 1; jk <= klev; jk++)
    for (jl = kidia; jl <= kfdia; jl++) {
      A2(ptendency_loc_t, jl, jk) = 0.0;
      A2(ptendency_loc_q, jl, jk) = 0.0;
      A2(ptendency_loc_a, jl, jk) = 0.0;
    }
  for (jm = 1; jm <= NCLV - 1; jm++)
    for (jk = 1; jk <= klev; jk++)
      for (jl = kidia; jl <= kfdia; jl++) A3(ptendency_loc_cld, jl, jk, jm, klev) = 0.0;

  for (jk = 1; jk <= klev; jk++)
    for (jl = kidia; jl <= kfdia; jl++) {
      A2(ztp1, jl, jk) = A2(pt, jl, jk) + ptsphy * A2(ptendency_cml_t, jl, jk);
      A3(zqx, jl, jk, NCLDQV, klev) = A2(pq, jl, jk) + ptsphy * A2(ptendency_cml_q, jl, jk);
      A3(zqx0, jl, jk, NCLDQV, klev) = A2(pq, jl, jk) + ptsphy * A2(ptendency_cml_q, jl, jk);
      A2(za, jl, jk) = A2(pa, jl, jk) + ptsphy * A2(ptendency_cml_a, jl, jk);
      A2(zaorig, jl, jk) = A2(pa, jl, jk) + ptsphy * A2(ptendency_cml_a, jl, jk);
    }
  for (jm = 1; jm <= NCLV - 1; jm++)
    for (jk = 1; jk <= klev; jk++)
      for (jl = kidia; jl <= kfdia; jl++) {
        A3(zqx, jl, jk, jm, klev) =
            A3(pclv, jl, jk, jm, klev) + ptsphy * A3(ptendency_cml_cld, jl, jk, jm, klev);
        A3(zqx0, jl, jk, jm, klev) =
            A3(pclv, jl, jk, jm, klev) + ptsphy * A3(ptendency_cml_cld, jl, jk, jm, klev);
      }
  /* ZPFPLSX, ZQXN2D, ZLNEG are zero from calloc (:1007-1009) */
  for (jl = kidia; jl <= kfdia; jl++) {
    A1(prainfrac_toprfz, jl) = 0.0;
    A1(llrainliq, jl) = 1;
  }
  /* tropopause search (:1016-1027) is dead code: ZTRPAUS is never used */

  /* saturation values (:1087-1115) */
  for (jk = 1; jk <= klev; jk++)
    for (jl = kidia; jl <= kfdia; jl++) {
      double t = A2(ztp1, jl, jk), pap_ = A2(pap, jl, jk);
      A2(zfoealfa, jl, jk) = foealfa(p, t);
      A2(zfoeewm, jl, jk) = fmin_(foeewm(p, t) / pap_, 0.5);
      A2(zqsmix, jl, jk) = A2(zfoeewm, jl, jk);
      A2(zqsmix, jl, jk) = A2(zqsmix, jl, jk) / (1.0 - p->retv * A2(zqsmix, jl, jk));
      double zalfa = foedelta(p, t);
      A2(zfoeew, jl, jk) = fmin_((zalfa * foeeliq(p, t) + (1.0 - zalfa) * foeeice(p, t)) / pap_, 0.5);
      A2(zfoeew, jl, jk) = fmin_(0.5, A2(zfoeew, jl, jk));
      A2(zqsice, jl, jk) = A2(zfoeew, jl, jk) / (1.0 - p->retv * A2(zfoeew, jl, jk));
      A2(zfoeeliqt, jl, jk) = fmin_(foeeliq(p, t) / pap_, 0.5);
      A2(zqsliq, jl, jk) = A2(zfoeeliqt, jl, jk);
      A2(zqsliq, jl, jk) = A2(zqsliq, jl, jk) / (1.0 - p->retv * A2(zqsliq, jl, jk));
    }

  /* 2. tidy up (:1127-1199) */
  for (jk = 1; jk <= klev; jk++)
    for (jl = kidia; jl <= kfdia; jl++) {
      if (A3(zqx, jl, jk, NCLDQL, klev) + A3(zqx, jl, jk, NCLDQI, klev) < p->rlmin ||
          A2(za, jl, jk) < p->ramin) {
        double zqadj;
        A3(zlneg, jl, jk, NCLDQL, klev) = A3(zlneg, jl, jk, NCLDQL, klev) + A3(zqx, jl, jk, NCLDQL, klev);
        zqadj = A3(zqx, jl, jk, NCLDQL, klev) * zqtmst;
        A2(ptendency_loc_q, jl, jk) = A2(ptendency_loc_q, jl, jk) + zqadj;
        A2(ptendency_loc_t, jl, jk) = A2(ptendency_loc_t, jl, jk) - p->ralvdcp * zqadj;
        A3(zqx, jl, jk, NCLDQV, klev) = A3(zqx, jl, jk, NCLDQV, klev) + A3(zqx, jl, jk, NCLDQL, klev);
        A3(zqx, jl, jk, NCLDQL, klev) = 0.0;
        A3(zlneg, jl, jk, NCLDQI, klev) = A3(zlneg, jl, jk, NCLDQI, klev) + A3(zqx, jl, jk, NCLDQI, klev);
        zqadj = A3(zqx, jl, jk, NCLDQI, klev) * zqtmst;
        A2(ptendency_loc_q, jl, jk) = A2(ptendency_loc_q, jl, jk) + zqadj;
        A2(ptendency_loc_t, jl, jk) = A2(ptendency_loc_t, jl, jk) - p->ralsdcp * zqadj;
        A3(zqx, jl, jk, NCLDQV, klev) = A3(zqx, jl, jk, NCLDQV, klev) + A3(zqx, jl, jk, NCLDQI, klev);
        A3(zqx, jl, jk, NCLDQI, klev) = 0.0;
        A2(za, jl, jk) = 0.0;
      }
    }
  for (jm = 1; jm <= NCLV - 1; jm++)
    for (jk = 1; jk <= klev; jk++)
      for (jl = kidia; jl <= kfdia; jl++) {
        if (A3(zqx, jl, jk, jm, klev) < p->rlmin) {
          A3(zlneg, jl, jk, jm, klev) = A3(zlneg, jl, jk, jm, klev) + A3(zqx, jl, jk, jm, klev);
          double zqadj = A3(zqx, jl, jk, jm, klev) * zqtmst;
          A2(ptendency_loc_q, jl, jk) = A2(ptendency_loc_q, jl, jk) + zqadj;
          if (iphase[jm] == 1) A2(ptendency_loc_t, jl, jk) = A2(ptendency_loc_t, jl, jk) - p->ralvdcp * zqadj;
          if (iphase[jm] == 2) A2(ptendency_loc_t, jl, jk) = A2(ptendency_loc_t, jl, jk) - p->ralsdcp * zqadj;
          A3(zqx, jl, jk, NCLDQV, klev) = A3(zqx, jl, jk, NCLDQV, klev) + A3(zqx, jl, jk, jm, klev);
          A3(zqx, jl, jk, jm, klev) = 0.0;
        }
      }
  for (jk = 1; jk <= klev; jk++)
    for (jl = kidia; jl <= kfdia; jl++) {
      A2(za, jl, jk) = fmax_(0.0, fmin_(1.0, A2(za, jl, jk)));
      A2(zli, jl, jk) = A3(zqx, jl, jk, NCLDQL, klev) + A3(zqx, jl, jk, NCLDQI, klev);
      if (A2(zli, jl, jk) > p->rlmin) {
        A2(zliqfrac, jl, jk) = A3(zqx, jl, jk, NCLDQL, klev) / A2(zli, jl, jk);
        A2(zicefrac, jl, jk) = 1.0 - A2(zliqfrac, jl, jk);
      } else {
        A2(zliqfrac, jl, jk) = 0.0;
        A2(zicefrac, jl, jk) = 0.0;
      }
    }

  /* reset single-level variables (:1205-1211) -- zero from calloc */

  /* ================= level loop (:1219-4128) ================= */
  for (jk = ncldtop; jk <= klev; jk++) {
    for (jm = 1; jm <= NCLV; jm++)
      for (jl = kidia; jl <= kfdia; jl++) L2(zqxfg, jl, jm) = A3(zqx, jl, jk, jm, klev);

    for (jl = kidia; jl <= kfdia; jl++) {
      A1(zlicld, jl) = 0.0;
      A1(zrainaut, jl) = 0.0;
      A1(zrainacc, jl) = 0.0;
      A1(zsnowaut, jl) = 0.0;
      A1(zsnowrime, jl) = 0.0;
      A1(zldefr, jl) = 0.0;
      A1(zacust, jl) = 0.0;
      A1(zqpretot, jl) = 0.0;
      A1(zlfinalsum, jl) = 0.0;
      A1(zsolab, jl) = 0.0;
      A1(zsolac, jl) = 0.0;
      A1(zicetot, jl) = 0.0;
    }
    memset(zsolqb, 0, sizeof(double) * n1 * NCLV * NCLV);
    memset(zsolqa, 0, sizeof(double) * n1 * NCLV * NCLV);
    memset(zfallspeed, 0, sizeof(double) * n1 * NCLV);
    memset(zfallsrce, 0, sizeof(double) * n1 * NCLV);
    memset(zfallsink, 0, sizeof(double) * n1 * NCLV);
    memset(zconvsrce, 0, sizeof(double) * n1 * NCLV);
    memset(zconvsink, 0, sizeof(double) * n1 * NCLV);
    memset(zbudcc, 0, sizeof(double) * n1 * 12); /* :1271-1273 */
    memset(zbudl, 0, sizeof(double) * n1 * 21);
    memset(zbudi, 0, sizeof(double) * n1 * 17);

    /* derived variables (:1275-1326) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double t = A2(ztp1, jl, jk);
      A1(zdp, jl) = A2(paph, jl, jk + 1) - A2(paph, jl, jk);
      A1(zgdp, jl) = p->rg / A1(zdp, jl);
      A1(zrho, jl) = A2(pap, jl, jk) / (p->rd * t);
      A1(zdtgdp, jl) = ptsphy * A1(zgdp, jl);
      A1(zrdtgdp, jl) = A1(zdp, jl) * (1.0 / (ptsphy * p->rg));
      if (jk > 1) A1(zdtgdpf, jl) = ptsphy * p->rg / (A2(pap, jl, jk) - A2(pap, jl, jk - 1));
      double xl = t - p->r4les, xi = t - p->r4ies;
      double zfacw = p->r5les / (xl * xl);
      double zcor = 1.0 / (1.0 - p->retv * A2(zfoeeliqt, jl, jk));
      A1(zdqsliqdt, jl) = zfacw * zcor * A2(zqsliq, jl, jk);
      A1(zcorqsliq, jl) = 1.0 + p->ralvdcp * A1(zdqsliqdt, jl);
      double zfaci = p->r5ies / (xi * xi);
      zcor = 1.0 / (1.0 - p->retv * A2(zfoeew, jl, jk));
      A1(zdqsicedt, jl) = zfaci * zcor * A2(zqsice, jl, jk);
      A1(zcorqsice, jl) = 1.0 + p->ralsdcp * A1(zdqsicedt, jl);
      double zalfaw = A2(zfoealfa, jl, jk);
      double zfac = zalfaw * zfacw + (1.0 - zalfaw) * zfaci;
      zcor = 1.0 / (1.0 - p->retv * A2(zfoeewm, jl, jk));
      A1(zdqsmixdt, jl) = zfac * zcor * A2(zqsmix, jl, jk);
      A1(zcorqsmix, jl) = 1.0 + foeldcpm(p, t) * A1(zdqsmixdt, jl);
      double qv = A3(zqx, jl, jk, NCLDQV, klev);
      A1(zevaplimmix, jl) = fmax_((A2(zqsmix, jl, jk) - qv) / A1(zcorqsmix, jl), 0.0);
      A1(zevaplimliq, jl) = fmax_((A2(zqsliq, jl, jk) - qv) / A1(zcorqsliq, jl), 0.0);
      A1(zevaplimice, jl) = fmax_((A2(zqsice, jl, jk) - qv) / A1(zcorqsice, jl), 0.0);
      double ztmpa = 1.0 / fmax_(A2(za, jl, jk), 0.01);
      A1(zliqcld, jl) = A3(zqx, jl, jk, NCLDQL, klev) * ztmpa;
      A1(zicecld, jl) = A3(zqx, jl, jk, NCLDQI, klev) * ztmpa;
      A1(zlicld, jl) = A1(zliqcld, jl) + A1(zicecld, jl);
    }

    /* evaporate very small amounts (:1332-1344) */
    for (jl = kidia; jl <= kfdia; jl++) {
      if (A3(zqx, jl, jk, NCLDQL, klev) < p->rlmin) {
        L3(zsolqa, jl, NCLDQV, NCLDQL) = A3(zqx, jl, jk, NCLDQL, klev);
        L3(zsolqa, jl, NCLDQL, NCLDQV) = -A3(zqx, jl, jk, NCLDQL, klev);
      }
      if (A3(zqx, jl, jk, NCLDQI, klev) < p->rlmin) {
        L3(zsolqa, jl, NCLDQV, NCLDQI) = A3(zqx, jl, jk, NCLDQI, klev);
        L3(zsolqa, jl, NCLDQI, NCLDQV) = -A3(zqx, jl, jk, NCLDQI, klev);
      }
    }

    /* 3.2 detrainment (:1362-1398) */
    if (jk < klev && jk >= ncldtop) {
      for (jl = kidia; jl <= kfdia; jl++) {
        A2(plude, jl, jk) = A2(plude, jl, jk) * A1(zdtgdp, jl);
        if (A1(ldcum, jl) && A2(plude, jl, jk) > zepsec && A2(plu, jl, jk + 1) > zepsec) {
          A1(zsolac, jl) = A1(zsolac, jl) + A2(plude, jl, jk) / A2(plu, jl, jk + 1);
          L2(zconvsrce, jl, NCLDQL) = A3(pludeli, jl, jk, 1, klev) * A1(zdtgdp, jl);
          L2(zconvsrce, jl, NCLDQI) = A3(pludeli, jl, jk, 2, klev) * A1(zdtgdp, jl);
          L3(zsolqa, jl, NCLDQL, NCLDQL) = L3(zsolqa, jl, NCLDQL, NCLDQL) + L2(zconvsrce, jl, NCLDQL);
          L3(zsolqa, jl, NCLDQI, NCLDQI) = L3(zsolqa, jl, NCLDQI, NCLDQI) + L2(zconvsrce, jl, NCLDQI);
          BL(jl, 3) = L2(zconvsrce, jl, NCLDQL) * zqtmst; /* :1378-1380 */
          BI(jl, 3) = L2(zconvsrce, jl, NCLDQI) * zqtmst;
          BCC(jl, 3) = zqtmst * A2(plude, jl, jk) / A2(plu, jl, jk + 1);
        } else {
          A2(plude, jl, jk) = 0.0;
        }
        if (p->lmfdsnow) {
          L2(zconvsrce, jl, NCLDQR) = A3(psnde, jl, jk, 1, klev) * A1(zdtgdp, jl);
          L2(zconvsrce, jl, NCLDQS) = A3(psnde, jl, jk, 2, klev) * A1(zdtgdp, jl);
          L3(zsolqa, jl, NCLDQR, NCLDQR) = L3(zsolqa, jl, NCLDQR, NCLDQR) + L2(zconvsrce, jl, NCLDQR);
          L3(zsolqa, jl, NCLDQS, NCLDQS) = L3(zsolqa, jl, NCLDQS, NCLDQS) + L2(zconvsrce, jl, NCLDQS);
        }
      }
    }

    /* 3.3 subsidence source and evaporation (:1419-1492) */
    if (jk > ncldtop) {
      for (jl = kidia; jl <= kfdia; jl++) {
        A1(zmf, jl) = fmax_(0.0, (A2(pmfu, jl, jk) * A1(zadvw, jl) + A2(pmfd, jl, jk) * A1(zadvwd, jl)) *
                                     A1(zdtgdp, jl));
        A1(zacust, jl) = A1(zmf, jl) * A1(zanewm1, jl);
      }
      for (jl = kidia; jl <= kfdia; jl++) {
        L2(zlcust, jl, NCLDQL) = A1(zmf, jl) * L2(zqxnm1, jl, NCLDQL);
        L2(zlcust, jl, NCLDQI) = A1(zmf, jl) * L2(zqxnm1, jl, NCLDQI);
        L2(zconvsrce, jl, NCLDQL) = L2(zconvsrce, jl, NCLDQL) + L2(zlcust, jl, NCLDQL);
        L2(zconvsrce, jl, NCLDQI) = L2(zconvsrce, jl, NCLDQI) + L2(zlcust, jl, NCLDQI);
      }
      for (jl = kidia; jl <= kfdia; jl++) {
        double zdtdp = zrdcp * 0.5 * (A2(ztp1, jl, jk - 1) + A2(ztp1, jl, jk)) / A2(paph, jl, jk);
        double zwtot = fmin_(p->rg * (A2(pmfu, jl, jk) * A1(zadvw, jl) + A2(pmfd, jl, jk) * A1(zadvwd, jl)),
                             (A2(pap, jl, jk) - A2(pap, jl, jk - 1)) / ptsphy);
        double zdtforc = zdtdp * ptsphy * zwtot;
        A1(zdqs, jl) = A1(zanewm1, jl) * zdtforc * A1(zdqsmixdt, jl);
      }
      for (jl = kidia; jl <= kfdia; jl++) {
        double zlfinal = fmax_(0.0, L2(zlcust, jl, NCLDQL) - A1(zdqs, jl));
        double zevap = fmin_((L2(zlcust, jl, NCLDQL) - zlfinal), A1(zevaplimmix, jl));
        zlfinal = L2(zlcust, jl, NCLDQL) - zevap;
        A1(zlfinalsum, jl) = A1(zlfinalsum, jl) + zlfinal;
        L3(zsolqa, jl, NCLDQL, NCLDQL) = L3(zsolqa, jl, NCLDQL, NCLDQL) + L2(zlcust, jl, NCLDQL);
        L3(zsolqa, jl, NCLDQV, NCLDQL) = L3(zsolqa, jl, NCLDQV, NCLDQL) + zevap;
        L3(zsolqa, jl, NCLDQL, NCLDQV) = L3(zsolqa, jl, NCLDQL, NCLDQV) - zevap;
        BL(jl, 4) = L2(zlcust, jl, NCLDQL) * zqtmst; /* :1459-1460 */
        BL(jl, 5) = -zevap * zqtmst;
      }
      for (jl = kidia; jl <= kfdia; jl++) {
        double zlfinal = fmax_(0.0, L2(zlcust, jl, NCLDQI) - A1(zdqs, jl));
        double zevap = fmin_((L2(zlcust, jl, NCLDQI) - zlfinal), A1(zevaplimmix, jl));
        zlfinal = L2(zlcust, jl, NCLDQI) - zevap;
        A1(zlfinalsum, jl) = A1(zlfinalsum, jl) + zlfinal;
        L3(zsolqa, jl, NCLDQI, NCLDQI) = L3(zsolqa, jl, NCLDQI, NCLDQI) + L2(zlcust, jl, NCLDQI);
        L3(zsolqa, jl, NCLDQV, NCLDQI) = L3(zsolqa, jl, NCLDQV, NCLDQI) + zevap;
        L3(zsolqa, jl, NCLDQI, NCLDQV) = L3(zsolqa, jl, NCLDQI, NCLDQV) - zevap;
        BI(jl, 4) = L2(zlcust, jl, NCLDQI) * zqtmst; /* :1475-1476 */
        BI(jl, 5) = -zevap * zqtmst;
      }
      for (jl = kidia; jl <= kfdia; jl++) {
        A1(zsolac, jl) = A1(zsolac, jl) + A1(zacust, jl);
        BCC(jl, 4) = A1(zacust, jl) * zqtmst; /* :1484-1489 */
        if (A1(zlfinalsum, jl) < zepsec) {
          A1(zsolac, jl) = A1(zsolac, jl) - A1(zacust, jl);
          BCC(jl, 5) = -A1(zacust, jl) * zqtmst;
        }
      }
    }

    /* subsidence sink (:1499-1514) */
    for (jl = kidia; jl <= kfdia; jl++) {
      if (jk < klev) {
        double zmfdn = fmax_(0.0, (A2(pmfu, jl, jk + 1) * A1(zadvw, jl) + A2(pmfd, jl, jk + 1) * A1(zadvwd, jl)) *
                                      A1(zdtgdp, jl));
        A1(zsolab, jl) = A1(zsolab, jl) + zmfdn;
        L3(zsolqb, jl, NCLDQL, NCLDQL) = L3(zsolqb, jl, NCLDQL, NCLDQL) + zmfdn;
        L3(zsolqb, jl, NCLDQI, NCLDQI) = L3(zsolqb, jl, NCLDQI, NCLDQI) + zmfdn;
        L2(zconvsink, jl, NCLDQL) = zmfdn;
        L2(zconvsink, jl, NCLDQI) = zmfdn;
      }
    }

    /* 3.4 erosion, ITURBEROSION=3 (:1689-1754) */
    for (jl = kidia; jl <= kfdia; jl++) {
      A1(zldifdt, jl) = p->rcldiff * ptsphy;
      if (SPP_ON(CLOUDSC_SPP_RCLDIFF))
        A1(zldifdt, jl) = p->rcldiff * ptsphy * spp_fac(p, pgp2dspp, klon, jl, CLOUDSC_SPP_RCLDIFF, 0, 0);
      if (A1(ktype, jl) >= 2 && A2(plude, jl, jk) > zepsec && A1(peis, jl) < 10.0) {
        A1(zldifdt, jl) = 20.0 * p->rcldiff_convi * A1(zldifdt, jl);
      } else if (A1(ktype, jl) == 1 && A2(plude, jl, jk) > zepsec) {
        A1(zldifdt, jl) = 2.0 * p->rcldiff_convi * A1(zldifdt, jl);
      }
    }
    for (jl = kidia; jl <= kfdia; jl++) {
      if (A2(zli, jl, jk) > zepsec) {
        double zaa = A2(za, jl, jk);
        double zqe = (A3(zqx, jl, jk, NCLDQV, klev) - zaa * A2(zqsmix, jl, jk)) / fmax_(zepsec, 1.0 - zaa);
        double ze = fmax_(A2(zqsmix, jl, jk) - zqe, 0.0);
        double zleros = 0.333 * zaa * (1. - zaa) * A1(zldifdt, jl) * ze;
        zleros = fmin_(zleros, A1(zevaplimmix, jl));
        zleros = fmin_(zleros, A2(zli, jl, jk));
        double zaeros = 0.5 * zleros / A1(zlicld, jl);
        A1(zsolac, jl) = A1(zsolac, jl) - zaeros;
        L3(zsolqa, jl, NCLDQV, NCLDQL) = L3(zsolqa, jl, NCLDQV, NCLDQL) + A2(zliqfrac, jl, jk) * zleros;
        L3(zsolqa, jl, NCLDQL, NCLDQV) = L3(zsolqa, jl, NCLDQL, NCLDQV) - A2(zliqfrac, jl, jk) * zleros;
        L3(zsolqa, jl, NCLDQV, NCLDQI) = L3(zsolqa, jl, NCLDQV, NCLDQI) + A2(zicefrac, jl, jk) * zleros;
        L3(zsolqa, jl, NCLDQI, NCLDQV) = L3(zsolqa, jl, NCLDQI, NCLDQV) - A2(zicefrac, jl, jk) * zleros;
        BL(jl, 7) = -A2(zliqfrac, jl, jk) * zleros * zqtmst; /* :1749-1751 */
        BI(jl, 7) = -A2(zicefrac, jl, jk) * zleros * zqtmst;
        BCC(jl, 7) = -zaeros * zqtmst;
      }
    }

    /* 4.1 fall speeds (:1783-1844), IVARFALL_ICE=0, IVARFALL_RAIN=1 */
    for (jl = kidia; jl <= kfdia; jl++) {
      L2(zfallspeed, jl, NCLDQL) = zvqx[NCLDQL];
      L2(zfallspeed, jl, NCLDQI) = zvqx[NCLDQI];
      L2(zfallspeed, jl, NCLDQS) = zvqx[NCLDQS];
      double zfallcorr = pow(p->rdensref / A1(zrho, jl), 0.4);
      double ztemp = 0.5 * (A3(zqx, jl, jk, NCLDQR, klev) + L2(zqxnm1, jl, NCLDQR));
      double zrlambda = pow(A1(zrho, jl) * ztemp / p->rcl_lam1r, p->rcl_lam2r);
      L2(zfallspeed, jl, NCLDQR) =
          p->rxfallspeedrain * zfallcorr * p->rcl_const7r * pow(zrlambda, p->rcl_dr);
      if (p->laericesed) /* :1798-1803, ZRE_ICE**1.0 = ZRE_ICE */
        L2(zfallspeed, jl, NCLDQI) = 0.002 * A2(pre_ice, jl, jk);
      if (SPP_ON(CLOUDSC_SPP_FALLSPEED)) /* :1806-1808 */
        L2(zfallspeed, jl, NCLDQI) =
            L2(zfallspeed, jl, NCLDQI) * spp_fac(p, pgp2dspp, klon, jl, CLOUDSC_SPP_FALLSPEED, 0, 0);
    }
    /* sedimentation source/sink (:1852-1877) */
    for (jm = 1; jm <= NCLV; jm++) {
      if (!llfall[jm]) continue;
      for (jl = kidia; jl <= kfdia; jl++) {
        if (jk > ncldtop) {
          L2(zfallsrce, jl, jm) = A3(zpfplsx, jl, jk, jm, klev + 1) * A1(zdtgdp, jl);
          L3(zsolqa, jl, jm, jm) = L3(zsolqa, jl, jm, jm) + L2(zfallsrce, jl, jm);
          L2(zqxfg, jl, jm) = L2(zqxfg, jl, jm) + L2(zfallsrce, jl, jm);
          A1(zqpretot, jl) = A1(zqpretot, jl) + L2(zqxfg, jl, jm);
          if (jm == NCLDQI) BI(jl, 12) = L2(zfallsrce, jl, jm) * zqtmst; /* :1864-1866 */
        }
        L2(zfallsink, jl, jm) = A1(zdtgdp, jl) * A1(zrho, jl) * L2(zfallspeed, jl, jm);
      }
    }

    /* 4.2 precipitation fraction (:1898-1919) */
    for (jl = kidia; jl <= kfdia; jl++) {
      if (A1(zqpretot, jl) > zepsec) {
        A1(zcovptot, jl) = 1.0 - ((1.0 - A1(zcovptot, jl)) *
                                  (1.0 - fmax_(A2(za, jl, jk), A2(za, jl, jk - 1))) /
                                  (1.0 - fmin_(A2(za, jl, jk - 1), 1.0 - 1.E-06)));
        A1(zcovptot, jl) = fmax_(A1(zcovptot, jl), p->rcovpmin);
        A1(zcovpclr, jl) = fmax_(0.0, A1(zcovptot, jl) - A2(za, jl, jk));
        A1(zraincld, jl) = 0.5 * (A3(zqx, jl, jk, NCLDQR, klev) + A3(zqx, jl, jk - 1, NCLDQR, klev)) / A1(zcovptot, jl);
        A1(zraincldm1, jl) = 0.5 * (A3(zqx, jl, jk, NCLDQR, klev) + L2(zqxnm1, jl, NCLDQR)) / A1(zcovptot, jl);
        A1(zsnowcld, jl) = 0.5 * (A3(zqx, jl, jk, NCLDQS, klev) + A3(zqx, jl, jk - 1, NCLDQS, klev)) / A1(zcovptot, jl);
        A1(zsnowcldm1, jl) = 0.5 * (A3(zqx, jl, jk, NCLDQS, klev) + L2(zqxnm1, jl, NCLDQS)) / A1(zcovptot, jl);
        A1(zcovpmax, jl) = fmax_(A1(zcovptot, jl), A1(zcovpmax, jl));
      } else {
        A1(zraincld, jl) = 0.0;
        A1(zraincldm1, jl) = 0.0;
        A1(zsnowcld, jl) = 0.0;
        A1(zsnowcldm1, jl) = 0.0;
        A1(zcovptot, jl) = 0.0;
        A1(zcovpclr, jl) = 0.0;
        A1(zcovpmax, jl) = 0.0;
      }
    }

    /* 4.3 warm rain, IWARMRAIN=3, IRAINACC=1 (:1930-2259) */
    for (jl = kidia; jl <= kfdia; jl++) {
      if (A1(zliqcld, jl) > zepsec) {
        /* inhomogeneity (:1937-1971) */
        double zgridlen = 0.0, zcldraincorr = 0.0;
        if (linhom) {
          double zqtot = fmin_((A3(zqx, jl, jk, NCLDQV, klev) + A3(zqx, jl, jk, NCLDQL, klev)) * 1000.0, 30.0);
          zgridlen = 2 * p->ra * sqrt(p->rpi * A1(pgaw, jl)) * 0.001;
          zcldraincorr = 1.0 - 0.8 * A2(za, jl, jk);
          double zphip1 = .2 + .01 * zqtot + .0027 * (zqtot * zqtot) - .00008 * (zqtot * zqtot * zqtot);
          double zphip2 = zphip1 - 0.2;
          double zphip3 = 0.123 * exp(-zphip1 * 0.55);
          double zanew2 = fmax_(A2(za, jl, jk), 0.1);
          double zphic = pow(zgridlen * zanew2, 1.0 / 3.0) *
                         pow(pow(zphip3 * zgridlen * zanew2, 1.5) + 3.0 * zphip3, -0.17);
          double zfracsdc = (zphip1 - zphip2 * zanew2) * zphic;
          if (A2(za, jl, jk) > 0.95) zfracsdc = 0.17 * zphic;
          A2(zlfsd, jl, jk) = 1.3 * zfracsdc; /* ZR12 */
        } else {
          A2(zlfsd, jl, jk) = p->rcloud_frac_std;
        }
        double zconst, zlcrit;
        if (A1(plsm, jl) > 0.5) {
          zconst = p->rcl_kk_cloud_num_land;
          zlcrit = p->rclcrit_land;
        } else {
          zconst = p->rcl_kk_cloud_num_sea;
          zlcrit = p->rclcrit_sea;
        }
        (void)zlcrit; /* IWARMRAIN=3 reads no threshold: the RCLCRIT perturbation (:2052-2062) has no effect */
        double zeaut = p->rcl_inhomogaut, zeacc = p->rcl_inhomogacc;
        if (p->lcloud_inhomog) { /* :2075-2098 */
          double zfracsdc = A2(zlfsd, jl, jk);
          double zaa = A2(za, jl, jk);
          zeaut = pow(1.0 + pow(zfracsdc, 2.0), (p->rcl_kkbauq - 1.0) * p->rcl_kkbauq / 2.0);
          double zphir = pow(zgridlen * zaa, 1.0 / 3.0) * pow(pow(0.11 * zgridlen * zaa, 1.14) + 1.0, -0.22);
          double zfracsdr = (1.1 - 0.8 * zaa) * zphir;
          if (zaa > 0.95) zfracsdr = 0.3 * zphir;
          zeacc = pow(1.0 + pow(zfracsdc, 2.0), (p->rcl_kkbac - 1.0) * p->rcl_kkbac / 2.0) *
                  pow(1.0 + pow(zfracsdr, 2.0), (p->rcl_kkbac - 1.0) * p->rcl_kkbac / 2.0) *
                  exp(zcldraincorr * p->rcl_kkbac * p->rcl_kkbac *
                      sqrt(log(1.0 + pow(zfracsdc, 2.0)) * log(1.0 + pow(zfracsdr, 2.0))));
        }
        if (SPP_ON(CLOUDSC_SPP_CLOUDINHOM)) { /* :2106-2109 */
          zeaut = zeaut * spp_fac(p, pgp2dspp, klon, jl, CLOUDSC_SPP_CLOUDINHOM, 0, 0);
          zeacc = zeacc * spp_fac(p, pgp2dspp, klon, jl, CLOUDSC_SPP_CLOUDINHOM, 1, 1);
        }
        A1(zrainaut, jl) = zeaut * ptsphy * p->rcl_kkaau * pow(A1(zliqcld, jl), p->rcl_kkbauq - 1.0) *
                           pow(zconst, p->rcl_kkbaun);
        L3(zsolqb, jl, NCLDQR, NCLDQL) = L3(zsolqb, jl, NCLDQR, NCLDQL) + A1(zrainaut, jl);
        if (A1(zraincld, jl) > zepsec) {
          A1(zrainacc, jl) = zeacc * ptsphy * p->rcl_kkaac * pow(A1(zliqcld, jl), p->rcl_kkbac - 1.0) *
                             pow(A1(zraincld, jl), p->rcl_kkbac);
        }
        L3(zsolqb, jl, NCLDQR, NCLDQL) = L3(zsolqb, jl, NCLDQR, NCLDQL) + A1(zrainacc, jl);
      }
    }

    /* 4.4 rain evaporation (:2271-2378) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double zaa = A2(za, jl, jk);
      double zzrh = p->rprecrhmax + (1.0 - p->rprecrhmax) * A1(zcovpmax, jl) / fmax_(zepsec, 1.0 - zaa);
      zzrh = fmin_(fmax_(zzrh, p->rprecrhmax), 1.0);
      double zxramid = p->ramid;
      if (SPP_ON(CLOUDSC_SPP_RAMID)) { /* :2282-2287 */
        zxramid = p->ramid * spp_fac(p, pgp2dspp, klon, jl, CLOUDSC_SPP_RAMID, 0, 0);
        if (p->spp_lramidlimit1) zxramid = fmin_(1.0, zxramid);
      }
      double zrhc = zxramid;
      double zsigk = A2(pap, jl, jk) / A2(paph, jl, klev + 1);
      if (zsigk > 0.8) {
        double s = (zsigk - 0.8) / 0.2;
        zrhc = zxramid + (1.0 - zxramid) * (s * s);
      }
      zzrh = fmin_(zrhc, zzrh);
      zzrh = fmin_(0.9, zzrh);
      double zqsl = A2(zqsliq, jl, jk);
      double zqe = fmax_(0.0, fmin_(A3(zqx, jl, jk, NCLDQV, klev), zqsl));
      int llo1 = A1(zcovpclr, jl) > zepsec && A1(zraincldm1, jl) > zepsec && zqe < zzrh * zqsl;
      if (llo1) {
        double t = A2(ztp1, jl, jk), rho = A1(zrho, jl);
        double zpreclr = A1(zraincldm1, jl);
        double zfallcorr = pow(p->rdensref / rho, flt_0p4);
        double zesatliq = p->rv / p->rd * foeeliq(p, t);
        double zlambda = pow(p->rcl_lam1r / (rho * zpreclr), p->rcl_lam2r);
        double zevap_denom = p->rcl_cdenom1 * zesatliq - p->rcl_cdenom2 * t * zesatliq +
                             p->rcl_cdenom3 * pow(t, 3.0) * A2(pap, jl, jk);
        double zcorr2 = pow(t / 273., 1.5) * 393. / (t + 120.);
        double zsubsat = fmax_(zzrh * zqsl - zqe, 0.0);
        double zbeta = (0.15 / zqsl) * (t * t) * zesatliq * p->rcl_const1r * (zcorr2 / zevap_denom) *
                       (0.78 / (pow(zlambda, p->rcl_const4r)) +
                        p->rcl_const2r * pow(rho * zfallcorr, 0.5) /
                            (pow(zcorr2, 0.5) * pow(zlambda, p->rcl_const3r)));
        double zdenom = 1.0 + zbeta * ptsphy * A1(zcorqsliq, jl);
        double zdpevap = A1(zcovpclr, jl) * zbeta * ptsphy * zsubsat / zdenom;
        if (SPP_ON(CLOUDSC_SPP_RAINEVAP)) /* :2346-2348 */
          zdpevap = zdpevap * spp_fac(p, pgp2dspp, klon, jl, CLOUDSC_SPP_RAINEVAP, 0, 0);
        double zevap = fmin_(zdpevap, L2(zqxfg, jl, NCLDQR));
        L3(zsolqa, jl, NCLDQV, NCLDQR) = L3(zsolqa, jl, NCLDQV, NCLDQR) + zevap;
        L3(zsolqa, jl, NCLDQR, NCLDQV) = L3(zsolqa, jl, NCLDQR, NCLDQV) - zevap;
        BL(jl, 20) = -zevap * zqtmst; /* :2363 */
        L2(zqxfg, jl, NCLDQR) = L2(zqxfg, jl, NCLDQR) - zevap;
      }
    }

    /* 4.5 ice deposition, IDEPICE=1 (:2404-2499) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double zaa = A2(za, jl, jk), rho = A1(zrho, jl), t = A2(ztp1, jl, jk);
      if (A2(za, jl, jk - 1) < p->rcldtopcf && zaa >= p->rcldtopcf) {
        A1(zcldtopdist, jl) = 0.0;
      } else {
        A1(zcldtopdist, jl) = A1(zcldtopdist, jl) + A1(zdp, jl) / (rho * p->rg);
      }
      double zoverlap_liqice = p->rcl_overlapliqice;
      double zsupersatice = (A2(zqsliq, jl, jk) - A2(zqsice, jl, jk)) / A2(zqsice, jl, jk);
      if (t < (p->rtt - 5.) && L2(zqxfg, jl, NCLDQL) > p->rlmin) {
        double zvpice = foeeice(p, t) * p->rv / p->rd;
        double zvpliq = zvpice * fokoop(p, t);
        (void)zvpliq;
        A1(zicenuclei, jl) = 1000.0 * exp(12.96 * zsupersatice - 0.639);
        double zadd = p->rlstt * (p->rlstt / (p->rv * t) - 1.0) / (2.4E-2 * t);
        double zbdd = p->rv * t * A2(pap, jl, jk) / (2.21 * zvpice);
        double zcvds = 7.8 * pow(A1(zicenuclei, jl) / rho, 0.666) * zsupersatice / (8.87 * (zadd + zbdd));
        double zice0 = fmax_(A1(zicecld, jl), A1(zicenuclei, jl) * p->riceinit / rho);
        double zinew = pow(0.666 * zcvds * ptsphy + pow(zice0, 0.666), 1.5);
        double zdepos = fmax_(zoverlap_liqice * zaa * (zinew - zice0), 0.0);
        zdepos = fmin_(zdepos, L2(zqxfg, jl, NCLDQL));
        double zinfactor = fmin_(A1(zicenuclei, jl) / 15000., 1.0);
        zdepos = zdepos * fmin_(zinfactor + (1.0 - zinfactor) *
                                                (p->rdepliqrefrate + A1(zcldtopdist, jl) / p->rdepliqrefdepth),
                                1.0);
        L3(zsolqa, jl, NCLDQI, NCLDQL) = L3(zsolqa, jl, NCLDQI, NCLDQL) + zdepos;
        L3(zsolqa, jl, NCLDQL, NCLDQI) = L3(zsolqa, jl, NCLDQL, NCLDQI) - zdepos;
        L2(zqxfg, jl, NCLDQI) = L2(zqxfg, jl, NCLDQI) + zdepos;
        L2(zqxfg, jl, NCLDQL) = L2(zqxfg, jl, NCLDQL) - zdepos;
        BL(jl, 11) = -zdepos * zqtmst; /* :2495-2496 */
        BI(jl, 11) = zdepos * zqtmst;
      }
    }

    /* 4.6 ISUBLICE=0: no ice sublimation (:2613-2689) */

    /* 4.7 snow deposition, IDEPSNOW=1 (:2698-2745) */
    for (jl = kidia; jl <= kfdia; jl++) {
      A1(zpsdep, jl) = 0.0;
      double t = A2(ztp1, jl, jk), rho = A1(zrho, jl);
      double zqsm = A2(zqsmix, jl, jk), qv = A3(zqx, jl, jk, NCLDQV, klev);
      double zsupersatice = fmax_((qv - zqsm) / zqsm, 0.0);
      if (t < p->rtt && A1(zsnowcld, jl) > zepsec && zsupersatice > 0.0) {
        double zvpice = foeeice(p, t) * p->rv / p->rd;
        double ztcg = 1.0, zfacx1s = 1.0;
        double zaplusb = p->rcl_apb1 * zvpice - p->rcl_apb2 * zvpice * t + A2(pap, jl, jk) * p->rcl_apb3 * (t * t * t);
        double zcorrfac = pow(1.0 / rho, 0.5);
        double zcorrfac2 = (pow(t / 273.0, 1.5)) * (393.0 / (t + 120.0));
        double zpr02 = rho * A1(zsnowcld, jl) * p->rcl_const1s / (ztcg * zfacx1s);
        double zterm1 = zsupersatice * (t * t) * zvpice * zcorrfac2 * ztcg * p->rcl_const2s * zfacx1s / (rho * zaplusb);
        double zterm2 = 0.65 * p->rcl_const6s * pow(zpr02, p->rcl_const4s) +
                        p->rcl_const3s * pow(zcorrfac, 0.5) * pow(rho, 0.5) * pow(zpr02, p->rcl_const5s) /
                            pow(zcorrfac2, 0.5);
        A1(zpsdep, jl) = fmax_(A1(zcovptot, jl) * zterm1 * zterm2 * ptsphy, 0.0);
        A1(zpsdep, jl) = fmin_(A1(zpsdep, jl), qv - zqsm) / A1(zcorqsmix, jl);
        L3(zsolqa, jl, NCLDQS, NCLDQV) = L3(zsolqa, jl, NCLDQS, NCLDQV) + A1(zpsdep, jl);
        L3(zsolqa, jl, NCLDQV, NCLDQS) = L3(zsolqa, jl, NCLDQV, NCLDQS) - A1(zpsdep, jl);
      }
    }

    /* revise in-cloud condensate (:2750-2754) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double ztmpa = 1.0 / fmax_(A2(za, jl, jk), 0.01);
      A1(zliqcld, jl) = L2(zqxfg, jl, NCLDQL) * ztmpa;
      A1(zicecld, jl) = L2(zqxfg, jl, NCLDQI) * ztmpa;
    }

    /* 4.8 ice -> snow autoconversion (:2769-2800) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double t = A2(ztp1, jl, jk);
      if (t <= p->rtt) {
        if (A1(zicecld, jl) > zepsec) {
          double zzco = ptsphy * p->rsnowlin1 * exp(p->rsnowlin2 * (t - p->rtt));
          double zlcrit = p->rlcritsnow;
          if (p->laericeauto) { /* :2776-2779 */
            zlcrit = A2(picrit_aer, jl, jk);
            zzco = zzco * pow(p->rnice / A2(pnice, jl, jk), 0.333);
          } else if (SPP_ON(CLOUDSC_SPP_RLCRITSNOW)) /* :2781-2783 */
            zlcrit = p->rlcritsnow * spp_fac(p, pgp2dspp, klon, jl, CLOUDSC_SPP_RLCRITSNOW, 0, 0);
          double r = A1(zicecld, jl) / zlcrit;
          double ztemp = -1. * (r * r);
          if (ztemp < 50.0) {
            A1(zsnowaut, jl) = zzco * (1.0 - exp(ztemp));
          } else {
            A1(zsnowaut, jl) = zzco;
          }
          L3(zsolqb, jl, NCLDQS, NCLDQI) = L3(zsolqb, jl, NCLDQS, NCLDQI) + A1(zsnowaut, jl);
        }
      }
    }

    /* 4.12 melting (:2815-2862) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double t = A2(ztp1, jl, jk);
      A1(zicetot, jl) = L2(zqxfg, jl, NCLDQI) + L2(zqxfg, jl, NCLDQS);
      A1(zmeltmax, jl) = 0.0;
      if (A1(zicetot, jl) > zepsec && t > p->rtt) {
        double zsubsat = fmax_(A2(zqsice, jl, jk) - A3(zqx, jl, jk, NCLDQV, klev), 0.0);
        double ztdmtw0 = t - p->rtt - zsubsat * (ztw1 + ztw2 * (A2(pap, jl, jk) - ztw3) - ztw4 * (t - ztw5));
        double zcons1 = fabs(ptsphy * (1.0 + 0.5 * ztdmtw0) / p->rtaumel);
        A1(zmeltmax, jl) = fmax_(ztdmtw0 * zcons1 * zrldcp, 0.0);
      }
    }
    for (jm = 1; jm <= NCLV; jm++) {
      if (iphase[jm] != 2) continue;
      jn = imelt[jm];
      for (jl = kidia; jl <= kfdia; jl++) {
        if (A1(zmeltmax, jl) > zepsec && A1(zicetot, jl) > zepsec) {
          double zalfa = L2(zqxfg, jl, jm) / A1(zicetot, jl);
          double zmelt = fmin_(L2(zqxfg, jl, jm), zalfa * A1(zmeltmax, jl));
          L2(zqxfg, jl, jm) = L2(zqxfg, jl, jm) - zmelt;
          L2(zqxfg, jl, jn) = L2(zqxfg, jl, jn) + zmelt;
          L3(zsolqa, jl, jn, jm) = L3(zsolqa, jl, jn, jm) + zmelt;
          L3(zsolqa, jl, jm, jn) = L3(zsolqa, jl, jm, jn) - zmelt;
          if (jm == NCLDQI) BI(jl, 15) = -zmelt * zqtmst; /* :2856-2858 */
          if (jm == NCLDQI) BL(jl, 17) = zmelt * zqtmst;
          if (jm == NCLDQS) BI(jl, 16) = -zmelt * zqtmst;
        }
      }
    }

    /* 4.13 rain freezing (:2877-2933) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double t = A2(ztp1, jl, jk), qr = A3(zqx, jl, jk, NCLDQR, klev);
      if (qr > zepsec) {
        if (t <= p->rtt && A2(ztp1, jl, jk - 1) > p->rtt) {
          A1(zqpretot, jl) = fmax_(A3(zqx, jl, jk, NCLDQS, klev) + qr, zepsec);
          A1(prainfrac_toprfz, jl) = qr / A1(zqpretot, jl);
          A1(llrainliq, jl) = A1(prainfrac_toprfz, jl) > flt_0p8;
        }
        if (t < p->rtt) {
          if (A1(llrainliq, jl)) {
            double zlambda = pow(p->rcl_lam1r / (A1(zrho, jl) * qr), p->rcl_lam2r);
            double ztemp = fmin_(p->rcl_fzrab * (t - p->rtt), 50.);
            double zfrz = ptsphy * (p->rcl_const5r / A1(zrho, jl)) * (exp(ztemp) - 1.) * pow(zlambda, p->rcl_const6r);
            A1(zfrzmax, jl) = fmax_(zfrz, 0.0);
          } else {
            double zcons1 = fabs(ptsphy * (1.0 + 0.5 * (p->rtt - t)) / p->rtaumel);
            A1(zfrzmax, jl) = fmax_((p->rtt - t) * zcons1 * zrldcp, 0.0);
          }
          if (A1(zfrzmax, jl) > zepsec) {
            double zfrz = fmin_(qr, A1(zfrzmax, jl));
            L3(zsolqa, jl, NCLDQS, NCLDQR) = L3(zsolqa, jl, NCLDQS, NCLDQR) + zfrz;
            L3(zsolqa, jl, NCLDQR, NCLDQS) = L3(zsolqa, jl, NCLDQR, NCLDQS) - zfrz;
            BL(jl, 18) = -zfrz * zqtmst; /* :2927 */
          }
        }
      }
    }

    /* 4.14 homogeneous freezing of cloud liquid (:2948-2960) */
    for (jl = kidia; jl <= kfdia; jl++)
      A1(zfrzmax, jl) = fmax_((p->rthomo - A2(ztp1, jl, jk)) * zrldcp, 0.0);
    for (jl = kidia; jl <= kfdia; jl++) {
      if (A1(zfrzmax, jl) > zepsec && L2(zqxfg, jl, NCLDQL) > zepsec) {
        double zfrz = fmin_(L2(zqxfg, jl, NCLDQL), A1(zfrzmax, jl));
        L3(zsolqa, jl, NCLDQI, NCLDQL) = L3(zsolqa, jl, NCLDQI, NCLDQL) + zfrz;
        L3(zsolqa, jl, NCLDQL, NCLDQI) = L3(zsolqa, jl, NCLDQL, NCLDQI) - zfrz;
        BL(jl, 19) = -zfrz * zqtmst; /* :2958 */
      }
    }

    /* 4.9 riming (:2973-3017) */
    for (jl = kidia; jl <= kfdia; jl++) {
      if (A2(ztp1, jl, jk) <= p->rtt && A1(zliqcld, jl) > zepsec) {
        double rho = A1(zrho, jl);
        double zfallcorr = pow(p->rdensref / rho, flt_0p4);
        if (A1(zsnowcld, jl) > zepsec && A1(zcovptot, jl) > 0.01) {
          A1(zsnowrime, jl) = p->rcl_effrime * A1(zcovptot, jl) * ptsphy * p->rcl_const7s * zfallcorr *
                              pow(rho * A1(zsnowcld, jl) * p->rcl_const1s, p->rcl_const8s);
          A1(zsnowrime, jl) = fmin_(A1(zsnowrime, jl), 1.0);
          L3(zsolqb, jl, NCLDQS, NCLDQL) = L3(zsolqb, jl, NCLDQS, NCLDQL) + A1(zsnowrime, jl);
        }
      }
    }

    /* PSD slopes (:3026-3069) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double rho = A1(zrho, jl);
      if (A1(zraincld, jl) > zepsec) {
        A1(zlamr, jl) = pow(p->rcl_lam1r / (rho * A1(zraincld, jl)), p->rcl_lam2r);
        A1(zn0r, jl) = p->rcl_x1r * pow(A1(zlamr, jl), p->rcl_x2r);
      } else {
        A1(zlamr, jl) = 0.0;
        A1(zn0r, jl) = 0.0;
      }
      if (A1(zsnowcld, jl) > zepsec) {
        A1(zlams, jl) = pow(p->rcl_lam1s / (rho * A1(zsnowcld, jl)), p->rcl_lam2s);
        A1(zn0s, jl) = p->rcl_x1s;
      } else {
        A1(zlams, jl) = 0.0;
        A1(zn0s, jl) = 0.0;
      }
      if (A1(zicecld, jl) > zepsec) {
        A1(zlami, jl) = pow(p->rcl_lam1s / (rho * A1(zicecld, jl)), p->rcl_lam2s);
        A1(zn0i, jl) = p->rcl_x1s;
      } else {
        A1(zlami, jl) = 0.0;
        A1(zn0i, jl) = 0.0;
      }
    }

    /* PSACR: snow accretes rain (:3084-3115) */
    for (jl = kidia; jl <= kfdia; jl++) {
      A1(zpsacr, jl) = 0.0;
      if (A2(ztp1, jl, jk) <= p->rtt && A1(prainfrac_toprfz, jl) < zepsec && A1(zraincld, jl) > zepsec &&
          A1(zsnowcld, jl) > zepsec) {
        double fr = L2(zfallspeed, jl, NCLDQR), fs = L2(zfallspeed, jl, NCLDQS);
        double zfalldiff = fmax_(fabs(fr - fs), (fr + fs) / 8.);
        double lr = A1(zlamr, jl), ls = A1(zlams, jl);
        double zfac = p->rpi * p->rpi * p->rdenswat * 1.0 * A1(zrho, jl) * A1(zn0r, jl) * A1(zn0s, jl) /
                      (ls * (lr * lr * lr));
        double zrat = lr / ls;
        A1(zpsacr, jl) = A1(zcovptot, jl) * ptsphy * zfac * zfalldiff * ((0.5 * zrat + 2.) * zrat + 5.) /
                         (lr * lr * lr);
        L3(zsolqa, jl, NCLDQS, NCLDQR) = L3(zsolqa, jl, NCLDQS, NCLDQR) + A1(zpsacr, jl);
        L3(zsolqa, jl, NCLDQR, NCLDQS) = L3(zsolqa, jl, NCLDQR, NCLDQS) - A1(zpsacr, jl);
      }
    }
    /* PRACS off (IP_RAIN_ACCRETES_SNOW=0) */
    /* PIACR: ice accretes rain (:3171-3198) */
    for (jl = kidia; jl <= kfdia; jl++) {
      A1(zpiacr, jl) = 0.0;
      if (A2(ztp1, jl, jk) <= p->rtt && A1(prainfrac_toprfz, jl) < zepsec && A1(zraincld, jl) > zepsec &&
          A1(zicecld, jl) > zepsec) {
        double fr = L2(zfallspeed, jl, NCLDQR), fi = L2(zfallspeed, jl, NCLDQI);
        double zfalldiff = fmax_(fabs(fr - fi), (fr + fi) / 8.);
        double lr = A1(zlamr, jl), li = A1(zlami, jl);
        double zfac = p->rpi * p->rpi * p->rdenswat * 0.1 * A1(zrho, jl) * A1(zn0r, jl) * A1(zn0i, jl) /
                      (li * (lr * lr * lr));
        double zrat = lr / li;
        A1(zpiacr, jl) = A1(zcovptot, jl) * ptsphy * zfac * zfalldiff * ((0.5 * zrat + 2.) * zrat + 5.) /
                         (lr * lr * lr);
        L3(zsolqa, jl, NCLDQI, NCLDQR) = L3(zsolqa, jl, NCLDQI, NCLDQR) + A1(zpiacr, jl);
        L3(zsolqa, jl, NCLDQR, NCLDQI) = L3(zsolqa, jl, NCLDQR, NCLDQI) - A1(zpiacr, jl);
      }
    }
    /* PRACI off (IP_RAIN_ACCRETES_ICE=0) */

    /* 4.15 snow sublimation, ISUBLSNOW=1 (:3254-3318) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double zaa = A2(za, jl, jk), zqsi = A2(zqsice, jl, jk);
      double zzrh = p->rprecrhmax + (1.0 - p->rprecrhmax) * A1(zcovpmax, jl) / fmax_(zepsec, 1.0 - zaa);
      zzrh = fmin_(fmax_(zzrh, p->rprecrhmax), 1.0);
      double zqe = (A3(zqx, jl, jk, NCLDQV, klev) - zaa * zqsi) / fmax_(zepsec, 1.0 - zaa);
      zqe = fmax_(0.0, fmin_(zqe, zqsi));
      int llo1 = A1(zcovpclr, jl) > zepsec && L2(zqxfg, jl, NCLDQS) > zepsec && zqe < zzrh * zqsi;
      if (llo1) {
        double a = A1(zcovptot, jl) * A1(zdtgdp, jl);
        double zpreclr = L2(zqxfg, jl, NCLDQS) * A1(zcovpclr, jl) / copysign(fmax_(fabs(a), zepsilon), a);
        double zbeta1 = sqrt(A2(pap, jl, jk) / A2(paph, jl, klev + 1)) / p->rvrfactor * zpreclr /
                        fmax_(A1(zcovpclr, jl), zepsec);
        double zbeta = p->rg * p->rpecons * pow(zbeta1, 0.5777);
        double zdenom = 1.0 + zbeta * ptsphy * A1(zcorqsice, jl);
        double zdpr = A1(zcovpclr, jl) * zbeta * (zqsi - zqe) / zdenom * A1(zdp, jl) * zrg_r;
        double zdpevap = zdpr * A1(zdtgdp, jl);
        if (SPP_ON(CLOUDSC_SPP_SNOWSUBLIM)) /* :3288-3290 */
          zdpevap = zdpevap * spp_fac(p, pgp2dspp, klon, jl, CLOUDSC_SPP_SNOWSUBLIM, 0, 0);
        double zevap = fmin_(zdpevap, L2(zqxfg, jl, NCLDQS));
        L3(zsolqa, jl, NCLDQV, NCLDQS) = L3(zsolqa, jl, NCLDQV, NCLDQS) + zevap;
        L3(zsolqa, jl, NCLDQS, NCLDQV) = L3(zsolqa, jl, NCLDQS, NCLDQV) - zevap;
        BI(jl, 17) = -zevap * zqtmst; /* :3304 */
        A1(zcovptot, jl) = fmax_(p->rcovpmin, A1(zcovptot, jl) - fmax_(0.0, (A1(zcovptot, jl) - zaa) * zevap /
                                                                                L2(zqxfg, jl, NCLDQS)));
        L2(zqxfg, jl, NCLDQS) = L2(zqxfg, jl, NCLDQS) - zevap;
      }
    }

    /* evaporate small precipitation amounts (:3402-3412) */
    for (jm = 1; jm <= NCLV; jm++) {
      if (!llfall[jm]) continue;
      for (jl = kidia; jl <= kfdia; jl++) {
        if (L2(zqxfg, jl, jm) < p->rlmin) {
          L3(zsolqa, jl, NCLDQV, jm) = L3(zsolqa, jl, NCLDQV, jm) + L2(zqxfg, jl, jm);
          L3(zsolqa, jl, jm, NCLDQV) = L3(zsolqa, jl, jm, NCLDQV) - L2(zqxfg, jl, jm);
        }
      }
    }

    /* 5.1 cloud cover (:3429-3438) */
    for (jl = kidia; jl <= kfdia; jl++) {
      double zanew = (A2(za, jl, jk) + A1(zsolac, jl)) / (1.0 + A1(zsolab, jl));
      zanew = fmin_(zanew, 1.0);
      if (zanew < p->ramin) zanew = 0.0;
      A1(zda, jl) = zanew - A2(zaorig, jl, jk);
      A1(zanewm1, jl) = zanew;
    }

    /* 5.2.1 sink truncation (:3455-3536) */
    for (jm = 1; jm <= NCLV; jm++) {
      for (jl = kidia; jl <= kfdia; jl++) A1(zsinksum, jl) = 0.0;
      for (jn = 1; jn <= NCLV; jn++)
        for (jl = kidia; jl <= kfdia; jl++) A1(zsinksum, jl) = A1(zsinksum, jl) - L3(zsolqa, jl, jm, jn);
      for (jl = kidia; jl <= kfdia; jl++) {
        double zmax = fmax_(A3(zqx, jl, jk, jm, klev), zepsec);
        double zrat = fmax_(A1(zsinksum, jl), zmax);
        L2(zratio, jl, jm) = zmax / zrat;
      }
    }
    for (jl = kidia; jl <= kfdia; jl++) {
      int iordv[NCLV + 1];
      iordv[1] = 1;
      for (jm = 2; jm <= NCLV; jm++) {
        for (jn = jm - 1; jn >= 1; jn--) {
          if (L2(zratio, jl, iordv[jn]) <= L2(zratio, jl, jm)) break;
          iordv[jn + 1] = iordv[jn];
        }
        iordv[jn + 1] = jm;
      }
      for (jm = 1; jm <= NCLV; jm++) L2(iorder, jl, jm) = iordv[jm];
    }
    for (jm = 1; jm <= NCLV; jm++) {
      for (jl = kidia; jl <= kfdia; jl++) A1(zsinksum, jl) = 0.0;
      for (jn = 1; jn <= NCLV; jn++)
        for (jl = kidia; jl <= kfdia; jl++) {
          jo = L2(iorder, jl, jm);
          L2(llindex3, jl, jn) = L3(zsolqa, jl, jo, jn) < 0.0;
          A1(zsinksum, jl) = A1(zsinksum, jl) - L3(zsolqa, jl, jo, jn);
        }
      for (jl = kidia; jl <= kfdia; jl++) {
        jo = L2(iorder, jl, jm);
        double zmm = fmax_(A3(zqx, jl, jk, jo, klev), zepsec);
        double zrr = fmax_(A1(zsinksum, jl), zmm);
        L2(zratio, jl, 1) = zmm / zrr;
      }
      for (jl = kidia; jl <= kfdia; jl++) {
        jo = L2(iorder, jl, jm);
        double zzratio = L2(zratio, jl, 1);
        for (jn = 1; jn <= NCLV; jn++) {
          if (L2(llindex3, jl, jn)) {
            L3(zsolqa, jl, jo, jn) = L3(zsolqa, jl, jo, jn) * zzratio;
            L3(zsolqa, jl, jn, jo) = L3(zsolqa, jl, jn, jo) * zzratio;
          }
        }
      }
    }

    /* 5.2.2 LHS / RHS (:3546-3587) */
    for (jm = 1; jm <= NCLV; jm++)
      for (jn = 1; jn <= NCLV; jn++) {
        if (jn == jm) {
          for (jl = kidia; jl <= kfdia; jl++) L3(zqlhs, jl, jn, jm) = 1.0 + L2(zfallsink, jl, jm);
          for (jl = kidia; jl <= kfdia; jl++)
            for (jo = 1; jo <= NCLV; jo++) L3(zqlhs, jl, jn, jm) = L3(zqlhs, jl, jn, jm) + L3(zsolqb, jl, jo, jn);
        } else {
          for (jl = kidia; jl <= kfdia; jl++) L3(zqlhs, jl, jn, jm) = -L3(zsolqb, jl, jn, jm);
        }
      }
    for (jm = 1; jm <= NCLV; jm++)
      for (jl = kidia; jl <= kfdia; jl++) {
        double zexplicit = 0.0;
        for (jn = 1; jn <= NCLV; jn++) zexplicit = zexplicit + L3(zsolqa, jl, jm, jn);
        L2(zqxn, jl, jm) = A3(zqx, jl, jk, jm, klev) + zexplicit;
      }

    /* non-pivoting LU and substitution (:3600-3628) */
    for (jn = 1; jn <= NCLV - 1; jn++)
      for (jm = jn + 1; jm <= NCLV; jm++) {
        for (jl = kidia; jl <= kfdia; jl++) L3(zqlhs, jl, jm, jn) = L3(zqlhs, jl, jm, jn) / L3(zqlhs, jl, jn, jn);
        for (ik = jn + 1; ik <= NCLV; ik++)
          for (jl = kidia; jl <= kfdia; jl++)
            L3(zqlhs, jl, jm, ik) = L3(zqlhs, jl, jm, ik) - L3(zqlhs, jl, jm, jn) * L3(zqlhs, jl, jn, ik);
      }
    for (jn = 2; jn <= NCLV; jn++)
      for (jm = 1; jm <= jn - 1; jm++)
        for (jl = kidia; jl <= kfdia; jl++)
          L2(zqxn, jl, jn) = L2(zqxn, jl, jn) - L3(zqlhs, jl, jn, jm) * L2(zqxn, jl, jm);
    for (jl = kidia; jl <= kfdia; jl++) L2(zqxn, jl, NCLV) = L2(zqxn, jl, NCLV) / L3(zqlhs, jl, NCLV, NCLV);
    for (jn = NCLV - 1; jn >= 1; jn--) {
      for (jm = jn + 1; jm <= NCLV; jm++)
        for (jl = kidia; jl <= kfdia; jl++)
          L2(zqxn, jl, jn) = L2(zqxn, jl, jn) - L3(zqlhs, jl, jn, jm) * L2(zqxn, jl, jm);
      for (jl = kidia; jl <= kfdia; jl++) L2(zqxn, jl, jn) = L2(zqxn, jl, jn) / L3(zqlhs, jl, jn, jn);
    }

    /* clip small values (:3633-3640) */
    for (jn = 1; jn <= NCLV - 1; jn++)
      for (jl = kidia; jl <= kfdia; jl++)
        if (L2(zqxn, jl, jn) < zepsec) {
          L2(zqxn, jl, NCLDQV) = L2(zqxn, jl, NCLDQV) + L2(zqxn, jl, jn);
          L2(zqxn, jl, jn) = 0.0;
        }
    for (jm = 1; jm <= NCLV; jm++)
      for (jl = kidia; jl <= kfdia; jl++) {
        L2(zqxnm1, jl, jm) = L2(zqxn, jl, jm);
        A3(zqxn2d, jl, jk, jm, klev) = L2(zqxn, jl, jm);
      }

    /* 5.3 fluxes to next level (:3658-3672) */
    for (jm = 1; jm <= NCLV; jm++)
      for (jl = kidia; jl <= kfdia; jl++)
        A3(zpfplsx, jl, jk + 1, jm, klev + 1) = L2(zfallsink, jl, jm) * L2(zqxn, jl, jm) * A1(zrdtgdp, jl);
    for (jl = kidia; jl <= kfdia; jl++)
      A1(zqpretot, jl) = A3(zpfplsx, jl, jk + 1, NCLDQS, klev + 1) + A3(zpfplsx, jl, jk + 1, NCLDQR, klev + 1);
    for (jl = kidia; jl <= kfdia; jl++)
      if (A1(zqpretot, jl) < zepsec) A1(zcovptot, jl) = 0.0;

    /* diagnosed rates of the implicit processes (:3675-3699), IWARMRAIN=3,
       IP_SNOW_ACCRETES_RAIN=1 */
    for (jl = kidia; jl <= kfdia; jl++) {
      BL(jl, 14) = -A1(zrainaut, jl) * L2(zqxn, jl, NCLDQL) * zqtmst;
      BL(jl, 15) = -A1(zrainacc, jl) * L2(zqxn, jl, NCLDQL) * zqtmst;
      BCC(jl, 6) = -L2(zconvsink, jl, NCLDQL) * A1(zanewm1, jl) * zqtmst;
      BL(jl, 6) = -L2(zconvsink, jl, NCLDQL) * L2(zqxn, jl, NCLDQL) * zqtmst;
      BI(jl, 6) = -L2(zconvsink, jl, NCLDQI) * L2(zqxn, jl, NCLDQI) * zqtmst;
      BI(jl, 13) = -L2(zfallsink, jl, NCLDQI) * L2(zqxn, jl, NCLDQI) * zqtmst;
      BL(jl, 21) = -A1(zsnowrime, jl) * L2(zqxn, jl, NCLDQL) * zqtmst;
      BI(jl, 14) = -A1(zsnowaut, jl) * L2(zqxn, jl, NCLDQI) * zqtmst;
    }

    /* 6.1 T and condensate tendencies (:3713-3745) */
    for (jm = 1; jm <= NCLV - 1; jm++) {
      for (jl = kidia; jl <= kfdia; jl++)
        L2(zfluxq, jl, jm) = L2(zconvsrce, jl, jm) + L2(zfallsrce, jl, jm) -
                             (L2(zfallsink, jl, jm) + L2(zconvsink, jl, jm)) * L2(zqxn, jl, jm);
      if (iphase[jm] == 1)
        for (jl = kidia; jl <= kfdia; jl++)
          A2(ptendency_loc_t, jl, jk) =
              A2(ptendency_loc_t, jl, jk) +
              p->ralvdcp * (L2(zqxn, jl, jm) - A3(zqx, jl, jk, jm, klev) - L2(zfluxq, jl, jm)) * zqtmst;
      if (iphase[jm] == 2)
        for (jl = kidia; jl <= kfdia; jl++)
          A2(ptendency_loc_t, jl, jk) =
              A2(ptendency_loc_t, jl, jk) +
              p->ralsdcp * (L2(zqxn, jl, jm) - A3(zqx, jl, jk, jm, klev) - L2(zfluxq, jl, jm)) * zqtmst;
      for (jl = kidia; jl <= kfdia; jl++)
        A3(ptendency_loc_cld, jl, jk, jm, klev) =
            A3(ptendency_loc_cld, jl, jk, jm, klev) + (L2(zqxn, jl, jm) - A3(zqx0, jl, jk, jm, klev)) * zqtmst;
    }
    for (jl = kidia; jl <= kfdia; jl++) {
      A2(ptendency_loc_q, jl, jk) =
          A2(ptendency_loc_q, jl, jk) + (L2(zqxn, jl, NCLDQV) - A3(zqx, jl, jk, NCLDQV, klev)) * zqtmst;
      A2(ptendency_loc_a, jl, jk) = A2(ptendency_loc_a, jl, jk) + A1(zda, jl) * zqtmst;
      A1(zq_upd, jl) = A2(pq, jl, jk) + ptsphy * (A2(ptendency_loc_q, jl, jk) + A2(ptendency_cml_q, jl, jk));
      A1(zt_upd, jl) = A2(pt, jl, jk) + ptsphy * (A2(ptendency_loc_t, jl, jk) + A2(ptendency_cml_t, jl, jk));
      A1(za_upd, jl) = A2(pa, jl, jk) + ptsphy * (A2(ptendency_loc_a, jl, jk) + A2(ptendency_cml_a, jl, jk));
    }

    /* 6.4 supersaturation check (:3772-3809) */
    {
      double zpp[klon];
      for (jl = kidia; jl <= kfdia; jl++) zpp[jl - 1] = A2(pap, jl, jk);
      supersatcheck(p, kidia, kfdia, 1, zt_upd, zq_upd, za_upd, zpp, zt_adj, zq_adj, za_adj, zl_adj, zi_adj);
    }
    for (jl = kidia; jl <= kfdia; jl++) {
      A2(ptendency_loc_q, jl, jk) = A2(ptendency_loc_q, jl, jk) + A1(zq_adj, jl) * zqtmst;
      A2(ptendency_loc_t, jl, jk) = A2(ptendency_loc_t, jl, jk) + A1(zt_adj, jl) * zqtmst;
      A2(ptendency_loc_a, jl, jk) = A2(ptendency_loc_a, jl, jk) + A1(za_adj, jl) * zqtmst;
      A3(ptendency_loc_cld, jl, jk, NCLDQL, klev) = A3(ptendency_loc_cld, jl, jk, NCLDQL, klev) + A1(zl_adj, jl) * zqtmst;
      A3(ptendency_loc_cld, jl, jk, NCLDQI, klev) = A3(ptendency_loc_cld, jl, jk, NCLDQI, klev) + A1(zi_adj, jl) * zqtmst;
      BCC(jl, 2) = A1(za_adj, jl) * zqtmst; /* :3787-3789 */
      BL(jl, 2) = A1(zl_adj, jl) * zqtmst;
      BI(jl, 2) = A1(zi_adj, jl) * zqtmst;
      A1(zl_adj, jl) = A3(zqx0, jl, jk, NCLDQL, klev) + A3(ptendency_loc_cld, jl, jk, NCLDQL, klev) * ptsphy;
      if (A1(zl_adj, jl) < -p->rlmin) nwarn++;
      if (A1(zl_adj, jl) < 0.0) {
        A3(ptendency_loc_cld, jl, jk, NCLDQL, klev) = A3(ptendency_loc_cld, jl, jk, NCLDQL, klev) - A1(zl_adj, jl) * zqtmst;
        A2(ptendency_loc_q, jl, jk) = A2(ptendency_loc_q, jl, jk) + A1(zl_adj, jl) * zqtmst;
        A2(ptendency_loc_t, jl, jk) = A2(ptendency_loc_t, jl, jk) - p->ralvdcp * A1(zl_adj, jl) * zqtmst;
      }
      A1(zi_adj, jl) = A3(zqx0, jl, jk, NCLDQI, klev) + A3(ptendency_loc_cld, jl, jk, NCLDQI, klev) * ptsphy;
      if (A1(zi_adj, jl) < -p->rlmin) nwarn++;
      if (A1(zi_adj, jl) < 0.0) {
        A3(ptendency_loc_cld, jl, jk, NCLDQI, klev) = A3(ptendency_loc_cld, jl, jk, NCLDQI, klev) - A1(zi_adj, jl) * zqtmst;
        A2(ptendency_loc_q, jl, jk) = A2(ptendency_loc_q, jl, jk) + A1(zi_adj, jl) * zqtmst;
        A2(ptendency_loc_t, jl, jk) = A2(ptendency_loc_t, jl, jk) - p->ralsdcp * A1(zi_adj, jl) * zqtmst;
      }
    }
    for (jl = kidia; jl <= kfdia; jl++) A2(pcovptot, jl, jk) = A1(zcovptot, jl);
    /* ZANEWP (:3819-3823): cloud fraction with precipitation fraction, for the ice FSD */
    for (jl = kidia; jl <= kfdia; jl++)
      if (A2(pa, jl, jk) + A1(zda, jl) > 0.001)
        A2(zanewp, jl, jk) = fmax_(fmax_(A2(pa, jl, jk) + A1(zda, jl), A2(pcovptot, jl, jk)), 0.1);

    /* 7. cloud budget diagnostics (:3832-4110).  ZPIEVAP, ZPRACS and ZPRACI
       are zero in this configuration (ISUBLICE=0, PRACS/PRACI off). */
    if (lbud) {
      int is = p->lbud23 ? 26 : 0;
      const double zdt = p->lcldbud_timeint ? ptsphy : 1.0;
      if (p->lcldbud_vertint) {
        for (jl = kidia; jl <= kfdia; jl++) {
          const double zdz = A1(zdp, jl) / (A1(zrho, jl) * p->rg);
          int k = 0;
          PX(jl, k + 4, is + 1) = PX(jl, k + 4, is + 1) + BCC(jl, 2) * zdz * zdt;
          PX(jl, k + 6, is + 1) = PX(jl, k + 6, is + 1) + BCC(jl, 3) * zdz * zdt;
          PX(jl, k + 7, is + 1) = PX(jl, k + 7, is + 1) + (BCC(jl, 4) + BCC(jl, 6)) * zdz * zdt;
          PX(jl, k + 8, is + 1) = PX(jl, k + 8, is + 1) + BCC(jl, 5) * zdz * zdt;
          PX(jl, k + 9, is + 1) = PX(jl, k + 9, is + 1) + BCC(jl, 7) * zdz * zdt;
          PX(jl, k + 10, is + 1) = PX(jl, k + 10, is + 1) + BCC(jl, 12) * zdz * zdt;
          PX(jl, k + 11, is + 1) = PX(jl, k + 11, is + 1) + A2(pvfa, jl, jk) * zdz * zdt;
          PX(jl, k + 12, is + 1) = PX(jl, k + 12, is + 1) + A2(pdyna, jl, jk) * zdz * zdt;
          k = 14;
          PX(jl, k + 5, is + 1) = PX(jl, k + 5, is + 1) + BL(jl, 2) * zdz * zdt;
          PX(jl, k + 7, is + 1) = PX(jl, k + 7, is + 1) + BL(jl, 3) * zdz * zdt;
          PX(jl, k + 8, is + 1) = PX(jl, k + 8, is + 1) + (BL(jl, 4) + BL(jl, 6)) * zdz * zdt;
          PX(jl, k + 9, is + 1) = PX(jl, k + 9, is + 1) + BL(jl, 5) * zdz * zdt;
          PX(jl, k + 10, is + 1) = PX(jl, k + 10, is + 1) + BL(jl, 7) * zdz * zdt;
          PX(jl, k + 11, is + 1) = PX(jl, k + 11, is + 1) + BL(jl, 11) * zdz * zdt;
          PX(jl, k + 12, is + 1) = PX(jl, k + 12, is + 1) + BL(jl, 14) * zdz * zdt;
          PX(jl, k + 13, is + 1) = PX(jl, k + 13, is + 1) + BL(jl, 15) * zdz * zdt;
          PX(jl, k + 14, is + 1) = PX(jl, k + 14, is + 1) + BL(jl, 12) * zdz * zdt;
          PX(jl, k + 15, is + 1) = PX(jl, k + 15, is + 1) + BL(jl, 13) * zdz * zdt;
          PX(jl, k + 16, is + 1) = PX(jl, k + 16, is + 1) + BL(jl, 17) * zdz * zdt;
          PX(jl, k + 17, is + 1) = PX(jl, k + 17, is + 1) + (BL(jl, 18) + BL(jl, 19)) * zdz * zdt;
          PX(jl, k + 18, is + 1) = PX(jl, k + 18, is + 1) + BL(jl, 20) * zdz * zdt;
          PX(jl, k + 19, is + 1) = PX(jl, k + 19, is + 1) + BL(jl, 21) * zdz * zdt;
          PX(jl, k + 20, is + 1) = PX(jl, k + 20, is + 1) + 0.0 * zdz * zdt * zqtmst; /* ZPRACS */
          PX(jl, k + 21, is + 1) = PX(jl, k + 21, is + 1) + A1(zpsacr, jl) * zdz * zdt * zqtmst;
          PX(jl, k + 22, is + 1) = PX(jl, k + 22, is + 1) + 0.0 * zdz * zdt * zqtmst; /* ZPRACI */
          PX(jl, k + 23, is + 1) = PX(jl, k + 23, is + 1) + A1(zpiacr, jl) * zdz * zdt * zqtmst;
          PX(jl, k + 24, is + 1) = PX(jl, k + 24, is + 1) + A2(pvfl, jl, jk) * zdz * zdt;
          PX(jl, k + 25, is + 1) = PX(jl, k + 25, is + 1) + A2(pdynl, jl, jk) * zdz * zdt;
          k = 39;
          PX(jl, k + 5, is + 1) = PX(jl, k + 5, is + 1) + BI(jl, 2) * zdz * zdt;
          PX(jl, k + 7, is + 1) = PX(jl, k + 7, is + 1) + BI(jl, 3) * zdz * zdt;
          PX(jl, k + 8, is + 1) = PX(jl, k + 8, is + 1) + (BI(jl, 4) + BI(jl, 6)) * zdz * zdt;
          PX(jl, k + 9, is + 1) = PX(jl, k + 9, is + 1) + BI(jl, 5) * zdz * zdt;
          PX(jl, k + 10, is + 1) = PX(jl, k + 10, is + 1) + BI(jl, 7) * zdz * zdt;
          PX(jl, k + 11, is + 1) = PX(jl, k + 11, is + 1) + BI(jl, 11) * zdz * zdt;
          PX(jl, k + 12, is + 1) = PX(jl, k + 12, is + 1) + (BI(jl, 12) + BI(jl, 13)) * zdz * zdt;
          PX(jl, k + 13, is + 1) = PX(jl, k + 13, is + 1) + BI(jl, 14) * zdz * zdt;
          PX(jl, k + 14, is + 1) = PX(jl, k + 14, is + 1) + BI(jl, 16) * zdz * zdt;
          PX(jl, k + 15, is + 1) = PX(jl, k + 15, is + 1) + BI(jl, 17) * zdz * zdt;
          PX(jl, k + 16, is + 1) = PX(jl, k + 16, is + 1) + A1(zpsdep, jl) * zqtmst * zdz * zdt;
          PX(jl, k + 17, is + 1) = PX(jl, k + 17, is + 1) + A2(pvfi, jl, jk) * zdz * zdt;
          PX(jl, k + 18, is + 1) = PX(jl, k + 18, is + 1) + A2(pdyni, jl, jk) * zdz * zdt;
          PX(jl, k + 19, is + 1) = PX(jl, k + 19, is + 1) + A2(pdyns, jl, jk) * zdz * zdt;
          PX(jl, 60, is + 1) = A1(prainfrac_toprfz, jl);
          k = 70;
          /* KTYPE/KPBLTYPE == IS+1 as written at :3925,3929 */
          if (A1(ktype, jl) == 0) PX(jl, k, is + 1) = PX(jl, k, is + 1) + 1.0;
          if (A1(ktype, jl) == is + 1) PX(jl, k + 1, is + 1) = PX(jl, k + 1, is + 1) + 1.0;
          if (A1(ktype, jl) == 2) PX(jl, k + 2, is + 1) = PX(jl, k + 2, is + 1) + 1.0;
          if (A1(ktype, jl) == 3) PX(jl, k + 3, is + 1) = PX(jl, k + 3, is + 1) + 1.0;
          if (A1(kpbltype, jl) == 0) PX(jl, k + 4, is + 1) = PX(jl, k + 4, is + 1) + 1.0;
          if (A1(kpbltype, jl) == is + 1) PX(jl, k + 5, is + 1) = PX(jl, k + 5, is + 1) + 1.0;
          if (A1(kpbltype, jl) == 2) PX(jl, k + 6, is + 1) = PX(jl, k + 6, is + 1) + 1.0;
          if (A1(kpbltype, jl) == 3) PX(jl, k + 7, is + 1) = PX(jl, k + 7, is + 1) + 1.0;
          PX(jl, k + 8, is + 1) = PX(jl, k + 8, is + 1) + A1(peis, jl);
          if (A1(peis, jl) > 6.0) PX(jl, k + 9, is + 1) = PX(jl, k + 9, is + 1) + 1.0;
          if (A1(peis, jl) > 8.0) PX(jl, k + 10, is + 1) = PX(jl, k + 10, is + 1) + 1.0;
          if (A1(peis, jl) > 10.0) PX(jl, k + 11, is + 1) = PX(jl, k + 11, is + 1) + 1.0;
          if (A1(ktype, jl) >= 2 && A1(peis, jl) < p->reisthsc) PX(jl, k + 12, is + 1) = PX(jl, k + 12, is + 1) + 1.0;
          if (A1(ktype, jl) > 0) PX(jl, k + 13, is + 1) = (double)A1(kctop, jl);
        }
        is = is + 1;
      }
      if (p->lcldbudc) { /* :3948-3970 */
        for (jl = kidia; jl <= kfdia; jl++) {
          PX(jl, jk, is + 4) = PX(jl, jk, is + 4) + BCC(jl, 2) * zdt;
          PX(jl, jk, is + 6) = PX(jl, jk, is + 6) + BCC(jl, 3) * zdt;
          PX(jl, jk, is + 7) = PX(jl, jk, is + 7) + (BCC(jl, 4) + BCC(jl, 6)) * zdt;
          PX(jl, jk, is + 8) = PX(jl, jk, is + 8) + BCC(jl, 5) * zdt;
          PX(jl, jk, is + 9) = PX(jl, jk, is + 9) + BCC(jl, 7) * zdt;
          PX(jl, jk, is + 11) = PX(jl, jk, is + 11) + A2(pvfa, jl, jk) * zdt;
          PX(jl, jk, is + 12) = PX(jl, jk, is + 12) + A2(pdyna, jl, jk) * zdt;
        }
        is = is + 12;
      }
      if (p->lcldbudl) { /* :3972-4007 */
        for (jl = kidia; jl <= kfdia; jl++) {
          PX(jl, jk, is + 5) = PX(jl, jk, is + 5) + BL(jl, 2) * zdt;
          PX(jl, jk, is + 7) = PX(jl, jk, is + 7) + BL(jl, 3) * zdt;
          PX(jl, jk, is + 8) = PX(jl, jk, is + 8) + (BL(jl, 4) + BL(jl, 6)) * zdt;
          PX(jl, jk, is + 9) = PX(jl, jk, is + 9) + BL(jl, 5) * zdt;
          PX(jl, jk, is + 10) = PX(jl, jk, is + 10) + BL(jl, 7) * zdt;
          PX(jl, jk, is + 11) = PX(jl, jk, is + 11) + BL(jl, 11) * zdt;
          PX(jl, jk, is + 12) = PX(jl, jk, is + 12) + BL(jl, 12) * zdt;
          PX(jl, jk, is + 13) = PX(jl, jk, is + 13) + BL(jl, 13) * zdt;
          PX(jl, jk, is + 14) = PX(jl, jk, is + 14) + BL(jl, 14) * zdt;
          PX(jl, jk, is + 15) = PX(jl, jk, is + 15) + BL(jl, 15) * zdt;
          PX(jl, jk, is + 16) = PX(jl, jk, is + 16) + BL(jl, 17) * zdt;
          PX(jl, jk, is + 17) = PX(jl, jk, is + 17) + (BL(jl, 18) + BL(jl, 19)) * zdt;
          PX(jl, jk, is + 18) = PX(jl, jk, is + 18) + BL(jl, 20) * zdt;
          PX(jl, jk, is + 19) = PX(jl, jk, is + 19) + BL(jl, 21) * zdt;
          PX(jl, jk, is + 20) = PX(jl, jk, is + 20) + A2(pvfl, jl, jk) * zdt;
          PX(jl, jk, is + 21) = PX(jl, jk, is + 21) + A2(pdynl, jl, jk) * zdt;
          PX(jl, jk, is + 22) = PX(jl, jk, is + 22) + L2(zqxn, jl, NCLDQL);
        }
        is = is + 22;
      }
      if (p->lcldbudi) { /* :4009-4048 */
        for (jl = kidia; jl <= kfdia; jl++) {
          PX(jl, jk, is + 5) = PX(jl, jk, is + 5) + BI(jl, 2) * zdt;
          PX(jl, jk, is + 7) = PX(jl, jk, is + 7) + BI(jl, 3) * zdt;
          PX(jl, jk, is + 8) = PX(jl, jk, is + 8) + (BI(jl, 4) + BI(jl, 6)) * zdt;
          PX(jl, jk, is + 9) = PX(jl, jk, is + 9) + BI(jl, 5) * zdt;
          PX(jl, jk, is + 10) = PX(jl, jk, is + 10) + BI(jl, 7) * zdt;
          PX(jl, jk, is + 11) = PX(jl, jk, is + 11) + BI(jl, 11) * zdt;
          PX(jl, jk, is + 12) = PX(jl, jk, is + 12) + (BI(jl, 12) + BI(jl, 13)) * zdt;
          PX(jl, jk, is + 13) = PX(jl, jk, is + 13) + BI(jl, 14) * zdt;
          PX(jl, jk, is + 14) = PX(jl, jk, is + 14) + (BI(jl, 15) + BI(jl, 16)) * zdt;
          PX(jl, jk, is + 15) = PX(jl, jk, is + 15) + A1(zpsdep, jl) * zqtmst * zdt;
          PX(jl, jk, is + 16) = PX(jl, jk, is + 16) + BI(jl, 17) * zdt;
          PX(jl, jk, is + 17) = PX(jl, jk, is + 17) + A2(pvfi, jl, jk) * zdt;
          PX(jl, jk, is + 18) = PX(jl, jk, is + 18) + 0.0 * zqtmst * zdt; /* ZPIEVAP */
          PX(jl, jk, is + 19) = PX(jl, jk, is + 19) + A2(pdyni, jl, jk) * zdt;
          PX(jl, jk, is + 20) = PX(jl, jk, is + 20) + L2(zqxn, jl, NCLDQI);
        }
        is = is + 20;
      }
      if (p->lcldbudt) { /* :4051-4106 */
        for (jl = kidia; jl <= kfdia; jl++) {
          PX(jl, jk, is + 1) = PX(jl, jk, is + 1) + A2(phrsw, jl, jk);
          PX(jl, jk, is + 2) = PX(jl, jk, is + 2) + A2(phrlw, jl, jk);
          PX(jl, jk, is + 3) = PX(jl, jk, is + 3) +
                               ((BL(jl, 1) + BL(jl, 2) + BL(jl, 9) + BL(jl, 10)) * p->ralvdcp -
                                BI(jl, 11) * p->ralvdcp) * zdt;
          PX(jl, jk, is + 4) = PX(jl, jk, is + 4) +
                               (BI(jl, 1) + BI(jl, 2) + BI(jl, 9) + BI(jl, 10) + BI(jl, 11)) * p->ralsdcp * zdt;
          PX(jl, jk, is + 5) = PX(jl, jk, is + 5) + BI(jl, 11) * p->ralfdcp * zdt;
          PX(jl, jk, is + 6) = PX(jl, jk, is + 6) + (BL(jl, 7) + BL(jl, 8) + BL(jl, 5)) * p->ralvdcp * zdt;
          PX(jl, jk, is + 7) = PX(jl, jk, is + 7) + (BI(jl, 7) + BI(jl, 8) + BI(jl, 5)) * p->ralsdcp * zdt;
          PX(jl, jk, is + 8) = PX(jl, jk, is + 8) + BL(jl, 20) * p->ralvdcp * zdt;
          PX(jl, jk, is + 9) = PX(jl, jk, is + 9) + BI(jl, 17) * p->ralsdcp * zdt;
          PX(jl, jk, is + 10) = PX(jl, jk, is + 10) + BI(jl, 15) * p->ralfdcp * zdt;
          PX(jl, jk, is + 11) = PX(jl, jk, is + 11) + BI(jl, 16) * p->ralfdcp * zdt;
          PX(jl, jk, is + 12) = PX(jl, jk, is + 12) -
                                (BL(jl, 12) + BL(jl, 13) + BL(jl, 18) + BL(jl, 19)) * p->ralfdcp * zdt;
          PX(jl, jk, is + 13) = PX(jl, jk, is + 13) + BL(jl, 21) * p->ralfdcp * zdt;
        }
        is = is + 13;
      }
    }

    if (p->lrad_cloud_inhomog) /* :4112-4125 */
      for (jl = kidia; jl <= kfdia; jl++) {
        if (A3(zqx0, jl, jk, NCLDQL, klev) + A3(zqx0, jl, jk, NCLDQI, klev) + A2(plude, jl, jk) > p->rlmin) {
          A2(zratfsd, jl, jk) =
              A2(plude, jl, jk) / (A2(plude, jl, jk) + A3(zqx0, jl, jk, NCLDQL, klev) + A3(zqx0, jl, jk, NCLDQI, klev));
          A2(zratfsd, jl, jk) = fmax_(0.0, fmin_(1.0, A2(zratfsd, jl, jk)));
        }
        A2(zicef, jl, jk) = L2(zqxn, jl, NCLDQI);
        A2(zliqf, jl, jk) = L2(zqxn, jl, NCLDQL);
      }
  }
  /* ice FSD (:4307-4359); default-REAL (binary32) literals as written at
     :4321-4322 and the 0.00001 at :4316 */
  if (p->lrad_cloud_inhomog) {
    const double f_p5 = (double)0.5f, f_p001 = (double)0.001f, f_p24 = (double)0.24f, f_p11 = (double)0.11f;
    const double f_10 = (double)10.f, f_p03 = (double)0.03f, f_1em5 = (double)0.00001f;
    for (jk = 1; jk <= klev; jk++)
      for (jl = kidia; jl <= kfdia; jl++) {
        double zgridlen = 2 * p->ra * sqrt(p->rpi * A1(pgaw, jl)) * 0.001;
        double zifsdback = 0.446585 * pow(zgridlen, 1.0 / 3.0) * pow(pow(0.308061 * zgridlen, 0.395736) + 1.0, -0.744527);
        double zqtot = fmax_(fmin_((A3(zqx, jl, jk, NCLDQV, klev) + A3(zqx, jl, jk, NCLDQI, klev)) * 1000.0, 30.0), f_1em5);
        double zdp_ = A2(paph, jl, jk + 1) - A2(paph, jl, jk);
        double zrho_ = A2(pap, jl, jk) / (p->rd * A2(ztp1, jl, jk));
        double zdelz = 1.0 / (p->rg * zrho_) * zdp_ * 0.001;
        zdelz = fmax_(fmin_(zdelz, f_p5), f_p001);
        double zphi = pow(zdelz / f_p24, f_p11) * pow(zqtot / f_10, f_p03);
        double zifsd = p->rcloud_frac_std;
        if (A2(zanewp, jl, jk) > 0.95) {
          zifsd = zifsdback * zphi;
          zifsd = 1.3 * (zifsd + A2(zratfsd, jl, jk) * 1.5);
        } else if (A2(zanewp, jl, jk) > 0.001 && A2(zanewp, jl, jk) <= 0.95) {
          zifsd = zifsdback * zphi * 1.5;
          zifsd = 1.3 * (zifsd + A2(zratfsd, jl, jk) * 1.5);
        }
        double zfsd = p->rcloud_frac_std;
        if (A2(zicef, jl, jk) > zepsec) zfsd = zifsd;
        if (A2(zliqf, jl, jk) > 0.0 && A2(zicef, jl, jk) <= zepsec) zfsd = A2(zlfsd, jl, jk);
        zfsd = fmin_(fmax_(0.1, zfsd), 3.575);
        A2(pfsd, jl, jk) = zfsd;
      }
  }

  /* PCOVPTOT above the cloud top: left undefined by the reference, zero here */
  for (jk = 1; jk < ncldtop; jk++)
    for (jl = kidia; jl <= kfdia; jl++) A2(pcovptot, jl, jk) = 0.0;

  /* 8. fluxes (:4218-4303) */
  for (jk = 1; jk <= klev + 1; jk++)
    for (jl = kidia; jl <= kfdia; jl++) {
      A2(pfplsl, jl, jk) = A3(zpfplsx, jl, jk, NCLDQR, klev + 1) + A3(zpfplsx, jl, jk, NCLDQL, klev + 1);
      A2(pfplsn, jl, jk) = A3(zpfplsx, jl, jk, NCLDQS, klev + 1) + A3(zpfplsx, jl, jk, NCLDQI, klev + 1);
    }
  for (jl = kidia; jl <= kfdia; jl++) {
    A2(pfsqlf, jl, 1) = 0.0;
    A2(pfsqif, jl, 1) = 0.0;
    A2(pfsqrf, jl, 1) = 0.0;
    A2(pfsqsf, jl, 1) = 0.0;
    A2(pfcqlng, jl, 1) = 0.0;
    A2(pfcqnng, jl, 1) = 0.0;
    A2(pfcqrng, jl, 1) = 0.0;
    A2(pfcqsng, jl, 1) = 0.0;
    A2(pfsqltur, jl, 1) = 0.0;
    A2(pfsqitur, jl, 1) = 0.0;
  }
  for (jk = 1; jk <= klev; jk++)
    for (jl = kidia; jl <= kfdia; jl++) {
      double zgdph_r = -zrg_r * (A2(paph, jl, jk + 1) - A2(paph, jl, jk)) * zqtmst;
      A2(pfsqlf, jl, jk + 1) = A2(pfsqlf, jl, jk);
      A2(pfsqif, jl, jk + 1) = A2(pfsqif, jl, jk);
      A2(pfsqrf, jl, jk + 1) = A2(pfsqlf, jl, jk);
      A2(pfsqsf, jl, jk + 1) = A2(pfsqif, jl, jk);
      A2(pfcqlng, jl, jk + 1) = A2(pfcqlng, jl, jk);
      A2(pfcqnng, jl, jk + 1) = A2(pfcqnng, jl, jk);
      A2(pfcqrng, jl, jk + 1) = A2(pfcqlng, jl, jk);
      A2(pfcqsng, jl, jk + 1) = A2(pfcqnng, jl, jk);
      A2(pfsqltur, jl, jk + 1) = A2(pfsqltur, jl, jk);
      A2(pfsqitur, jl, jk + 1) = A2(pfsqitur, jl, jk);
      A2(pfsqlf, jl, jk + 1) =
          A2(pfsqlf, jl, jk + 1) +
          (A3(zqxn2d, jl, jk, NCLDQL, klev) - A3(zqx0, jl, jk, NCLDQL, klev) + A2(pvfl, jl, jk) * ptsphy) * zgdph_r +
          A3(pludeli, jl, jk, 1, klev);
      A2(pfcqlng, jl, jk + 1) = A2(pfcqlng, jl, jk + 1) + A3(zlneg, jl, jk, NCLDQL, klev) * zgdph_r;
      A2(pfsqltur, jl, jk + 1) = A2(pfsqltur, jl, jk + 1) + A2(pvfl, jl, jk) * ptsphy * zgdph_r;
      A2(pfsqrf, jl, jk + 1) =
          A2(pfsqrf, jl, jk + 1) + (A3(zqxn2d, jl, jk, NCLDQR, klev) - A3(zqx0, jl, jk, NCLDQR, klev)) * zgdph_r;
      A2(pfcqrng, jl, jk + 1) = A2(pfcqrng, jl, jk + 1) + A3(zlneg, jl, jk, NCLDQR, klev) * zgdph_r;
      A2(pfsqif, jl, jk + 1) =
          A2(pfsqif, jl, jk + 1) +
          (A3(zqxn2d, jl, jk, NCLDQI, klev) - A3(zqx0, jl, jk, NCLDQI, klev) + A2(pvfi, jl, jk) * ptsphy) * zgdph_r +
          A3(pludeli, jl, jk, 2, klev);
      A2(pfcqnng, jl, jk + 1) = A2(pfcqnng, jl, jk + 1) + A3(zlneg, jl, jk, NCLDQI, klev) * zgdph_r;
      A2(pfsqitur, jl, jk + 1) = A2(pfsqitur, jl, jk + 1) + A2(pvfi, jl, jk) * ptsphy * zgdph_r;
      A2(pfsqsf, jl, jk + 1) =
          A2(pfsqsf, jl, jk + 1) + (A3(zqxn2d, jl, jk, NCLDQS, klev) - A3(zqx0, jl, jk, NCLDQS, klev)) * zgdph_r;
      A2(pfcqsng, jl, jk + 1) = A2(pfcqsng, jl, jk + 1) + A3(zlneg, jl, jk, NCLDQS, klev) * zgdph_r;
    }
  for (jk = 1; jk <= klev + 1; jk++)
    for (jl = kidia; jl <= kfdia; jl++) {
      A2(pfhpsl, jl, jk) = -p->rlvtt * A2(pfplsl, jl, jk);
      A2(pfhpsn, jl, jk) = -p->rlstt * A2(pfplsn, jl, jk);
    }

  free(buf);
  return nwarn;
}

int oracle_cloudsc_batched(
    const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_cld, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_cld, const double *pvfl,
    const double *pvfi, const double *pap, const double *paph, const double *plsm,
    const int32_t *ldcum, const int32_t *ktype, const double *peis, const double *plu,
    double *plude, const double *pludeli, const double *psnde, const double *pmfu,
    const double *pmfd, const double *pa, const double *pclv, double *pcovptot,
    double *prainfrac_toprfz, double *pfsqlf, double *pfsqif, double *pfcqnng,
    double *pfcqlng, double *pfsqrf, double *pfsqsf, double *pfcqrng, double *pfcqsng,
    double *pfsqltur, double *pfsqitur, double *pfplsl, double *pfplsn, double *pfhpsl,
    double *pfhpsn, int nthreads) {
  if (nproma < 1 || ngpblks < 1 || ngptot < 1 || ngptot > nproma * ngpblks ||
      ngptot <= nproma * (ngpblks - 1))
    return CLOUDSC_E_SHAPE;
  const size_t s2 = (size_t)nproma * klev, s2h = (size_t)nproma * (klev + 1), s1 = nproma;
  int total = 0, err = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) reduction(min : err)
  for (int ib = 0; ib < ngpblks; ib++) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    double *peis_blk = (double *)(peis + ib * s1); /* read only by CLOUDSC */
    int r = oracle_cloudsc(
        p, 1, icend, nproma, klev, 0, ptsphy, pt + ib * s2, pq + ib * s2, ptendency_cml_t + ib * s2,
        ptendency_cml_q + ib * s2, ptendency_cml_a + ib * s2, ptendency_cml_cld + ib * s2 * NCLV,
        ptendency_loc_t + ib * s2, ptendency_loc_q + ib * s2, ptendency_loc_a + ib * s2,
        ptendency_loc_cld + ib * s2 * NCLV, NULL, pvfl + ib * s2, pvfi + ib * s2, NULL, NULL, NULL,
        NULL, NULL, NULL, NULL, NULL, pap + ib * s2, paph + ib * s2h, NULL, plsm + ib * s1, NULL,
        ldcum + ib * s1, NULL, ktype + ib * s1, NULL, peis_blk, plu + ib * s2, plude + ib * s2,
        pludeli + ib * s2 * 4, psnde + ib * s2 * 2, pmfu + ib * s2, pmfd + ib * s2, NULL, 0,
        pa + ib * s2, pclv + ib * s2 * NCLV, NULL, NULL, NULL, NULL, NULL, pcovptot + ib * s2, NULL,
        prainfrac_toprfz + ib * s1, pfsqlf + ib * s2h, pfsqif + ib * s2h, pfcqnng + ib * s2h,
        pfcqlng + ib * s2h, pfsqrf + ib * s2h, pfsqsf + ib * s2h, pfcqrng + ib * s2h,
        pfcqsng + ib * s2h, pfsqltur + ib * s2h, pfsqitur + ib * s2h, pfplsl + ib * s2h,
        pfplsn + ib * s2h, pfhpsl + ib * s2h, pfhpsn + ib * s2h, NULL, 0);
    if (r < 0) err = r < err ? r : err;
    else total += r;
  }
  return err < 0 ? err : total;
}

/* =========================================================================
 * CLOUD_SATADJ (ifs-source/arpifs/phys_ec/cloud_satadj.F90:13-1092), the
 * saturation adjustment CALLPAR runs before CLOUDSC (callpar.F90:1253-1279),
 * restated in its default configuration: no SPP perturbations (:313-332), the
 * budget diagnostics (:845-940) off.  Loop order and the order of every
 * floating-point operation follow the Fortran.  Quantities the reference
 * computes but never uses at this configuration (ZQSLIQ, ZCORQSLIQ,
 * ZEVAPLIMMIX, ZQSLIM, ZQSLIQ_UPD, ZQSICE_UPD, ZQSLIQK_UPD, ZRDTGDP, ZRHO,
 * ZDZ, ZLICLD) are not formed.
 * ========================================================================= */

/* QSATMIXADJ (cloud_satadj.F90:948-1017): two Newton steps of the mixed-phase
 * saturation adjustment; returns the adjusted humidity. */
static double qsatmixadj(const cloudsc_params *p, double pt, double pq, double pp) {
  double zt = pt, zq = pq;
  const double zp_r = 1.0 / pp;
  for (int ji = 1; ji <= 2; ji++) {
    double zfoeet = fmin_(foeewm(p, zt) * zp_r, 0.5);
    double zcor = 1.0 / (1.0 - p->retv * zfoeet);
    double zqsat = zfoeet * zcor;
    double zcorqs = 1.0 + zqsat * zcor * foedem(p, zt);
    double zcond = (zq - zqsat) / zcorqs;
    zt = zt + foeldcpm(p, zt) * zcond;
    zq = zq - zcond;
  }
  return zq;
}

int oracle_cloud_satadj(
    const cloudsc_params *p, int kidia, int kfdia, int klon, int klev, const int32_t *ktype,
    int lddiag, double ptsphy, const double *pap, const double *paph, const double *pt,
    const double *pq, const double *pa, const double *pl, const double *pi,
    const double *ptendency_cml_t, const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_l, const double *ptendency_cml_i, const double *phrsw,
    const double *phrlw, const double *ptendency_vdf_t, const double *ptendency_vdf_q,
    const double *pmfu, const double *pmfd, const double *pludeli, const double *pvervel,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_l, double *ptendency_loc_i) {
  (void)ktype; (void)lddiag; (void)pmfu; (void)pmfd;
  if (klon < 1 || klev < 2 || kidia < 1 || kfdia > klon || kidia > kfdia) return CLOUDSC_E_SHAPE;
  const int ncldtop = p->ncldtop;
  const double zqtmst = 1.0 / ptsphy; /* :291 */
  const double zrdcp = p->rd / p->rcpd;
  const double zepsec = 1.E-14;
  int nwarn = 0;
  const size_t nb = (size_t)klon * 19;
  double *buf = (double *)malloc(nb * sizeof(double));
  if (!buf) return CLOUDSC_E_CUDA;
  double *zt = buf, *zq = zt + klon, *za = zq + klon, *zl = za + klon, *zi = zl + klon;
  double *zdtforce = zi + klon, *zdqforce = zdtforce + klon, *zli = zdqforce + klon;
  double *zliqfrac = zli + klon, *zicefrac = zliqfrac + klon, *zrhc = zicefrac + klon;
  double *zqsliqk = zrhc + klon, *zqsmix = zqsliqk + klon, *zqsmix_upd = zqsmix + klon;
  double *zcorqsmix_upd = zqsmix_upd + klon, *zdqs = zcorqsmix_upd + klon;
  double *zt_upd = zdqs + klon, *zq_upd = zt_upd + klon, *za_upd = zq_upd + klon;
  double zt_adj[1], zq_adj[1], za_adj[1], zl_adj[1], zi_adj[1];

  for (int jk = 1; jk <= ncldtop - 1; jk++) /* :338-345 */
    for (int jl = kidia; jl <= kfdia; jl++) {
      A2(ptendency_loc_t, jl, jk) = 0.0;
      A2(ptendency_loc_q, jl, jk) = 0.0;
      A2(ptendency_loc_a, jl, jk) = 0.0;
      A2(ptendency_loc_l, jl, jk) = 0.0;
      A2(ptendency_loc_i, jl, jk) = 0.0;
    }

  for (int jk = ncldtop; jk <= klev; jk++) {
    /* updated state (:357-366) */
    for (int jl = kidia; jl <= kfdia; jl++) {
      A1(zt, jl) = A2(pt, jl, jk) + ptsphy * A2(ptendency_cml_t, jl, jk);
      A1(zq, jl) = A2(pq, jl, jk) + ptsphy * A2(ptendency_cml_q, jl, jk);
      A1(za, jl) = A2(pa, jl, jk) + ptsphy * A2(ptendency_cml_a, jl, jk);
      A1(zl, jl) = A2(pl, jl, jk) + ptsphy * A2(ptendency_cml_l, jl, jk);
      A1(zi, jl) = A2(pi, jl, jk) + ptsphy * A2(ptendency_cml_i, jl, jk);
      A1(za, jl) = fmax_(0.0, fmin_(1.0, A1(za, jl)));
    }
    /* T and q forcing of condensation/evaporation (:384-413) */
    for (int jl = kidia; jl <= kfdia; jl++) {
      double zdp = A2(paph, jl, jk + 1) - A2(paph, jl, jk);
      double zgdp = p->rg / zdp;
      double zdtgdp = ptsphy * zgdp;
      double zdtdp = zrdcp * A2(pt, jl, jk) / A2(pap, jl, jk);
      double zdpmxdt = zdp * zqtmst;
      double zwtot = A2(pvervel, jl, jk);
      zwtot = fmin_(zdpmxdt, fmax_(-zdpmxdt, zwtot));
      double zzzdt = A2(phrsw, jl, jk) + A2(phrlw, jl, jk);
      double zdtdiab = fmin_(zdpmxdt * zdtdp, fmax_(-zdpmxdt * zdtdp, zzzdt)) * ptsphy;
      A1(zdtforce, jl) = zdtdp * zwtot * ptsphy + zdtdiab + A3(pludeli, jl, jk, 4, klev) * zdtgdp +
                         A2(ptendency_vdf_t, jl, jk) * ptsphy;
      A1(zdqforce, jl) = A3(pludeli, jl, jk, 3, klev) * zdtgdp + A2(ptendency_vdf_q, jl, jk) * ptsphy;
    }
    /* saturation of the start-of-step and of the updated state (:435-552) */
    for (int jl = kidia; jl <= kfdia; jl++) {
      const double t0 = A2(pt, jl, jk), pp = A2(pap, jl, jk);
      double zp_r = 1.0 / pp;
      A1(zli, jl) = A1(zl, jl) + A1(zi, jl);
      if (A1(zli, jl) > p->rlmin) {
        A1(zliqfrac, jl) = A1(zl, jl) / A1(zli, jl);
        A1(zicefrac, jl) = 1.0 - A1(zliqfrac, jl);
      } else {
        A1(zliqfrac, jl) = 0.0;
        A1(zicefrac, jl) = 0.0;
      }
      A1(zrhc, jl) = p->ramid;
      double zsigk = pp / A2(paph, jl, klev + 1);
      if (zsigk > 0.8) {
        double x = (zsigk - 0.8) / 0.2;
        A1(zrhc, jl) = p->ramid + (1.0 - p->ramid) * (x * x);
      }
      double zfoeeliq = fmin_(foeeliq(p, t0) * zp_r, 0.5);
      double zfoeeice = fmin_(foeew(p, t0) * zp_r, 0.5);
      double zfokoop = fmin_(zfoeeice * (p->rkoop1 - p->rkoop2 * t0), zfoeeliq);
      A1(zqsliqk, jl) = zfokoop / (1.0 - p->retv * zfokoop);
      double zfoeemix = fmin_(foeewm(p, t0) * zp_r, 0.5);
      double zcor = 1.0 / (1.0 - p->retv * zfoeemix);
      A1(zqsmix, jl) = zfoeemix * zcor;
      A1(zqsliqk, jl) = 0.5 * (A1(zqsliqk, jl) + A1(zqsmix, jl));
      /* updated state */
      const double tu = A1(zt, jl);
      zfoeemix = fmin_(foeewm(p, tu) * zp_r, 0.5);
      zcor = 1.0 / (1.0 - p->retv * zfoeemix);
      A1(zqsmix_upd, jl) = zfoeemix * zcor;
      A1(zcorqsmix_upd, jl) = 1.0 + A1(zqsmix_upd, jl) * zcor * foedem(p, tu);
    }
    /* condensation/evaporation from dqsat/dt (:574-593) */
    for (int jl = kidia; jl <= kfdia; jl++) {
      double zttmp = A2(pt, jl, jk) + A1(zdtforce, jl);
      zttmp = fmax_(zttmp, 160.0);
      double zqtmp = A1(zqsmix, jl) + A1(zdqforce, jl);
      double zqsatnew = qsatmixadj(p, zttmp, zqtmp, A2(pap, jl, jk));
      A1(zdqs, jl) = zqsatnew - zqtmp;
    }
    for (int jl = kidia; jl <= kfdia; jl++) {
      const double pa0 = A2(pa, jl, jk), pq0 = A2(pq, jl, jk), t0 = A2(pt, jl, jk);
      const double dqs = A1(zdqs, jl), qsliqk = A1(zqsliqk, jl);
      /* clear-air condensation, new cloud (:602-655) */
      double env_l = 0.0, env_i = 0.0, zacond = 0.0;
      if (dqs <= -p->rlmin && pa0 < 1.0 - zepsec) {
        double zqe = (pq0 - pa0 * A1(zqsmix, jl)) / fmax_(zepsec, 1.0 - pa0);
        zqe = fmax_(0.0, zqe);
        if (zqe >= A1(zrhc, jl) * qsliqk && zqe < qsliqk) {
          zacond = -(1.0 - pa0) * dqs / fmax_(2.0 * (qsliqk - zqe), zepsec);
          zacond = fmin_(zacond, 1.0 - pa0);
          double zlcond_env = -dqs * 0.5 * zacond;
          double zzdl = 2.0 * (qsliqk - zqe) / fmax_(zepsec, 1.0 - pa0);
          if (dqs < -zzdl) {
            double zlcondlim = (pa0 - 1.0) * dqs - qsliqk + pq0;
            zlcond_env = fmin_(zlcond_env, zlcondlim);
          }
          zlcond_env = fmax_(zlcond_env, 0.0);
          if (zlcond_env < p->rlmin || (1.0 - pa0) < zepsec) {
            zlcond_env = 0.0;
            zacond = 0.0;
          }
          if (zlcond_env == 0.0) zacond = 0.0;
          if (t0 > p->rthomo) env_l = zlcond_env;
          else env_i = zlcond_env;
        }
      }
      /* condensation in the cloudy part (:662-695) */
      double cld_l = 0.0, cld_i = 0.0;
      if (pa0 > zepsec && dqs <= -p->rlmin) {
        double zlcond_cld = fmax_(-dqs, 0.0);
        double zcdmax = fmax_((A1(zq, jl) - A1(zqsmix_upd, jl)) / A1(zcorqsmix_upd, jl), 0.0);
        zlcond_cld = fmin_(zlcond_cld, zcdmax);
        zlcond_cld = pa0 * zlcond_cld;
        if (zlcond_cld < p->rlmin) zlcond_cld = 0.0;
        if (t0 > p->rthomo) cld_l = zlcond_cld;
        else cld_i = zlcond_cld;
      }
      /* evaporation of the cloudy part (:703-723) */
      double ev_l = 0.0, ev_i = 0.0, zaevap = 0.0;
      if (dqs > 0.0 && A1(zli, jl) > 0.0) {
        double zlevap_cld = fmin_(pa0 * dqs, A1(zli, jl));
        ev_l = A1(zliqfrac, jl) * zlevap_cld;
        ev_i = A1(zicefrac, jl) * zlevap_cld;
      }
      /* state for the supersaturation check (:738-757) */
      A1(zt_upd, jl) = A1(zt, jl) + p->ralvdcp * (cld_l + env_l - ev_l) + p->ralsdcp * (cld_i + env_i - ev_i);
      A1(zq_upd, jl) = A1(zq, jl) + (ev_l - cld_l - env_l) + (ev_i - cld_i - env_i);
      double zanew = A1(za, jl) + zacond - zaevap;
      zanew = fmin_(zanew, 1.0);
      if (zanew < p->ramin) zanew = 0.0;
      A1(za_upd, jl) = zanew;
      /* supersaturation check (:767-793), IFTLIQICE = 2 */
      double pp = A2(pap, jl, jk);
      supersatcheck(p, 1, 1, 2, &A1(zt_upd, jl), &A1(zq_upd, jl), &A1(za_upd, jl), &pp, zt_adj, zq_adj,
                    za_adj, zl_adj, zi_adj);
      double supl, supi;
      if (A1(zt_upd, jl) > p->rthomo) {
        supl = zl_adj[0] + zi_adj[0];
        supi = 0.0;
      } else {
        supl = 0.0;
        supi = zl_adj[0] + zi_adj[0];
      }
      double zsupsata = za_adj[0];
      /* tendencies (:801-822) */
      double tt = p->ralvdcp * (cld_l + env_l + supl - ev_l) * zqtmst +
                  p->ralsdcp * (cld_i + env_i + supi - ev_i) * zqtmst;
      double tq = (ev_l - cld_l - env_l - supl + ev_i - cld_i - env_i - supi) * zqtmst;
      zanew = A1(za, jl) + zacond - zaevap + zsupsata;
      zanew = fmin_(zanew, 1.0);
      if (zanew < p->ramin) zanew = 0.0;
      double ta = (zanew - A1(za, jl)) * zqtmst;
      double tl = (cld_l + env_l + supl - ev_l) * zqtmst;
      double ti = (cld_i + env_i + supi - ev_i) * zqtmst;
      /* negative clean-up (:824-843) */
      double ladj = A1(zl, jl) + tl * ptsphy;
      if (ladj < -p->rlmin) nwarn++;
      if (ladj < 0.0) {
        tl = tl - ladj;
        tq = tq + ladj;
        tt = tt - p->ralvdcp * ladj;
      }
      double iadj = A1(zi, jl) + ti * ptsphy;
      if (iadj < -p->rlmin) nwarn++;
      if (iadj < 0.0) {
        ti = ti - iadj;
        tq = tq + iadj;
        tt = tt - p->ralsdcp * iadj;
      }
      A2(ptendency_loc_t, jl, jk) = tt;
      A2(ptendency_loc_q, jl, jk) = tq;
      A2(ptendency_loc_a, jl, jk) = ta;
      A2(ptendency_loc_l, jl, jk) = tl;
      A2(ptendency_loc_i, jl, jk) = ti;
    }
  }
  free(buf);
  return nwarn;
}

int oracle_cloud_satadj_batched(
    const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot, double ptsphy,
    const double *pap, const double *paph, const double *pt, const double *pq, const double *pa,
    const double *pl, const double *pi, const double *ptendency_cml_t, const double *ptendency_cml_q,
    const double *ptendency_cml_a, const double *ptendency_cml_l, const double *ptendency_cml_i,
    const double *phrsw, const double *phrlw, const double *ptendency_vdf_t,
    const double *ptendency_vdf_q, const double *pludeli, const double *pvervel,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_l, double *ptendency_loc_i, int nthreads) {
  if (nproma < 1 || ngpblks < 1 || ngptot < 1 || ngptot > nproma * ngpblks ||
      ngptot <= nproma * (ngpblks - 1))
    return CLOUDSC_E_SHAPE;
  const size_t s2 = (size_t)nproma * klev, s2h = (size_t)nproma * (klev + 1);
  int total = 0, err = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) reduction(min : err)
  for (int ib = 0; ib < ngpblks; ib++) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    const size_t o = ib * s2;
    int r = oracle_cloud_satadj(
        p, 1, icend, nproma, klev, NULL, 0, ptsphy, pap + o, paph + ib * s2h, pt + o, pq + o, pa + o,
        pl + o, pi + o, ptendency_cml_t + o, ptendency_cml_q + o, ptendency_cml_a + o,
        ptendency_cml_l + o, ptendency_cml_i + o, phrsw + o, phrlw + o, ptendency_vdf_t + o,
        ptendency_vdf_q + o, NULL, NULL, pludeli + o * 4, pvervel + o, ptendency_loc_t + o,
        ptendency_loc_q + o, ptendency_loc_a + o, ptendency_loc_l + o, ptendency_loc_i + o);
    if (r < 0) err = r < err ? r : err;
    else total += r;
  }
  return err < 0 ? err : total;
}

/* =========================================================================
 * The supersaturation adjustment of SLTEND (ifs-source/arpifs/phys_ec/
 * sltend.F90:380-410): the state updated by the cumulative and the new
 * physics tendencies is checked with CLOUD_SUPERSATCHECK (KFTLIQICE = 1) on
 * levels NCLDTOP..KLEV and the adjustments are added to the tendencies.
 * PTENCLD is (KLON,KLEV,NCLV); its liquid and ice species are updated.  The
 * diagnostics ZADJA/ZADJL/ZADJI (:406-408) go to padja/padjl/padji (may be
 * NULL).  Levels above NCLDTOP are not touched.  SLTEND passes the section
 * PRSF1(KIDIA:KFDIA,JK) to the KLON-sized dummy PP of CLOUD_SUPERSATCHECK,
 * which then reads PP(JL) for JL = KIDIA..KFDIA; with KIDIA = 1 (the whole
 * block, as EC_PHYS_DRV calls it) that is PRSF1(JL,JK), which is what this
 * restatement reads for any KIDIA.
 * ========================================================================= */
int oracle_sltend_supersat(
    const cloudsc_params *p, int kidia, int kfdia, int klon, int klev, double tsphy, const double *pt,
    const double *pq, const double *pa, const double *prsf1, const double *prs1, const double *pcent,
    const double *pcenq, const double *pcena, double *ptent, double *ptenq, double *ptena, double *ptencld,
    double *padja, double *padjl, double *padji) {
  if (klon < 1 || klev < 2 || kidia < 1 || kfdia > klon || kidia > kfdia) return CLOUDSC_E_SHAPE;
  const double zrtsphy = 1.0 / tsphy; /* :271 */
  double *buf = (double *)malloc((size_t)klon * 9 * sizeof(double));
  if (!buf) return CLOUDSC_E_CUDA;
  double *zt = buf, *zq = zt + klon, *za = zq + klon, *ta = za + klon, *qa = ta + klon, *aa = qa + klon;
  double *la = aa + klon, *ia = la + klon, *pp = ia + klon;
  for (int jk = p->ncldtop; jk <= klev; jk++) {
    for (int jl = kidia; jl <= kfdia; jl++) {
      A1(zt, jl) = A2(pt, jl, jk) + tsphy * (A2(pcent, jl, jk) + A2(ptent, jl, jk));
      A1(zq, jl) = A2(pq, jl, jk) + tsphy * (A2(pcenq, jl, jk) + A2(ptenq, jl, jk));
      A1(za, jl) = A2(pa, jl, jk) + tsphy * (A2(pcena, jl, jk) + A2(ptena, jl, jk));
      A1(pp, jl) = A2(prsf1, jl, jk);
    }
    supersatcheck(p, kidia, kfdia, 1, zt, zq, za, pp, ta, qa, aa, la, ia);
    for (int jl = kidia; jl <= kfdia; jl++) {
      A2(ptent, jl, jk) = A2(ptent, jl, jk) + A1(ta, jl) * zrtsphy;
      A2(ptenq, jl, jk) = A2(ptenq, jl, jk) + A1(qa, jl) * zrtsphy;
      A2(ptena, jl, jk) = A2(ptena, jl, jk) + A1(aa, jl) * zrtsphy;
      A3(ptencld, jl, jk, NCLDQL, klev) = A3(ptencld, jl, jk, NCLDQL, klev) + A1(la, jl) * zrtsphy;
      A3(ptencld, jl, jk, NCLDQI, klev) = A3(ptencld, jl, jk, NCLDQI, klev) + A1(ia, jl) * zrtsphy;
      if (padja) A2(padja, jl, jk) = A1(aa, jl) * zrtsphy;
      if (padjl) A2(padjl, jl, jk) = A1(la, jl) * zrtsphy;
      if (padji) A2(padji, jl, jk) = A1(ia, jl) * zrtsphy;
    }
  }
  (void)prs1; /* PSURF feeds only ZRHC, which CLOUD_SUPERSATCHECK never uses */
  free(buf);
  return 0;
}

int oracle_sltend_supersat_batched(
    const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot, double tsphy, const double *pt,
    const double *pq, const double *pa, const double *prsf1, const double *prs1, const double *pcent,
    const double *pcenq, const double *pcena, double *ptent, double *ptenq, double *ptena, double *ptencld,
    double *padja, double *padjl, double *padji, int nthreads) {
  if (nproma < 1 || ngpblks < 1 || ngptot < 1 || ngptot > nproma * ngpblks ||
      ngptot <= nproma * (ngpblks - 1))
    return CLOUDSC_E_SHAPE;
  const size_t s2 = (size_t)nproma * klev, s2h = (size_t)nproma * (klev + 1);
  int err = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(min : err)
  for (int ib = 0; ib < ngpblks; ib++) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    const size_t o = ib * s2;
    int r = oracle_sltend_supersat(p, 1, icend, nproma, klev, tsphy, pt + o, pq + o, pa + o, prsf1 + o,
                                   prs1 + ib * s2h, pcent + o, pcenq + o, pcena + o, ptent + o, ptenq + o,
                                   ptena + o, ptencld + o * NCLV, padja ? padja + o : NULL,
                                   padjl ? padjl + o : NULL, padji ? padji + o : NULL);
    if (r < 0) err = r < err ? r : err;
  }
  return err;
}

/* The block loop of oracle_cloudsc_batched with the arrays the optional
 * configurations read or write (PVFA, PDYNA/L/I/S, PHRSW, PHRLW, PGAW, KCTOP,
 * KPBLTYPE, PGP2DSPP (NPROMA, NRFTOTAL, NGPBLKS), PRE_ICE, PICRIT_AER, PNICE
 * (NPROMA, KLEV, NGPBLKS), PFSD, PEXTRA (NPROMA, KLEV, KFLDX, NGPBLKS),
 * INOUT). */
int oracle_cloudsc_batched_diag(
    const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_cld, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_cld, const double *pvfl,
    const double *pvfi, const double *pap, const double *paph, const double *plsm,
    const int32_t *ldcum, const int32_t *ktype, const double *peis, const double *plu,
    double *plude, const double *pludeli, const double *psnde, const double *pmfu,
    const double *pmfd, const double *pa, const double *pclv, double *pcovptot,
    double *prainfrac_toprfz, double *pfsqlf, double *pfsqif, double *pfcqnng,
    double *pfcqlng, double *pfsqrf, double *pfsqsf, double *pfcqrng, double *pfcqsng,
    double *pfsqltur, double *pfsqitur, double *pfplsl, double *pfplsn, double *pfhpsl,
    double *pfhpsn, const double *pvfa, const double *pdyna, const double *pdynl,
    const double *pdyni, const double *pdyns, const double *phrsw, const double *phrlw,
    const double *pgaw, const int32_t *kctop, const int32_t *kpbltype, const double *pgp2dspp,
    const double *pre_ice, const double *picrit_aer, const double *pnice,
    double *pfsd, double *pextra, int kfldx, int nthreads) {
  if (nproma < 1 || ngpblks < 1 || ngptot < 1 || ngptot > nproma * ngpblks ||
      ngptot <= nproma * (ngpblks - 1))
    return CLOUDSC_E_SHAPE;
  const size_t s2 = (size_t)nproma * klev, s2h = (size_t)nproma * (klev + 1), s1 = nproma;
  const size_t sx = s2 * (size_t)(kfldx > 0 ? kfldx : 0);
  int total = 0, err = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) reduction(min : err)
  for (int ib = 0; ib < ngpblks; ib++) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    const size_t o = ib * s2, o1 = ib * s1;
    int r = oracle_cloudsc(
        p, 1, icend, nproma, klev, 0, ptsphy, pt + o, pq + o, ptendency_cml_t + o, ptendency_cml_q + o,
        ptendency_cml_a + o, ptendency_cml_cld + o * NCLV, ptendency_loc_t + o, ptendency_loc_q + o,
        ptendency_loc_a + o, ptendency_loc_cld + o * NCLV, pvfa ? pvfa + o : NULL, pvfl + o, pvfi + o,
        pdyna ? pdyna + o : NULL, pdynl ? pdynl + o : NULL, pdyni ? pdyni + o : NULL, NULL,
        pdyns ? pdyns + o : NULL, phrsw ? phrsw + o : NULL, phrlw ? phrlw + o : NULL, NULL, pap + o,
        paph + ib * s2h, NULL, plsm + o1, pgaw ? pgaw + o1 : NULL, ldcum + o1, kctop ? kctop + o1 : NULL, ktype + o1,
        kpbltype ? kpbltype + o1 : NULL, (double *)(peis + o1), plu + o, plude + o, pludeli + o * 4,
        psnde + o * 2, pmfu + o, pmfd + o,
        pgp2dspp ? pgp2dspp + o1 * (size_t)(p->spp_nrftotal > 0 ? p->spp_nrftotal : 0) : NULL, 0, pa + o,
        pclv + o * NCLV, NULL, picrit_aer ? picrit_aer + o : NULL, pre_ice ? pre_ice + o : NULL, NULL,
        pnice ? pnice + o : NULL, pcovptot + o, pfsd ? pfsd + o : NULL, prainfrac_toprfz + o1, pfsqlf + ib * s2h, pfsqif + ib * s2h,
        pfcqnng + ib * s2h, pfcqlng + ib * s2h, pfsqrf + ib * s2h, pfsqsf + ib * s2h, pfcqrng + ib * s2h,
        pfcqsng + ib * s2h, pfsqltur + ib * s2h, pfsqitur + ib * s2h, pfplsl + ib * s2h,
        pfplsn + ib * s2h, pfhpsl + ib * s2h, pfhpsn + ib * s2h, pextra ? pextra + ib * sx : NULL, kfldx);
    if (r < 0) err = r < err ? r : err;
    else total += r;
  }
  return err < 0 ? err : total;
}

/* STATE_INCREMENT (state_increment.F90:9-105) for one block: each field the
 * state carries is incremented over columns KIDIA..KFDIA of every level by
 * its increment when that is present (PA_X != NULL) and, for Q, O3, A, TKE
 * and the condensate species, when the state's KEYMASK switch is on
 * (CLOUDSC_KEY_* bits in st->keymask).  CLD is (KLON, KLEV, st->nclv); the
 * condensate increments are (KLON, KLEV) arrays, or species slices of one
 * (KLON, KLEV, inc->nclv_pa) array.  Same order of fields as the reference. */
int oracle_state_increment(int kidia, int kfdia, int klon, int klev, const cloudsc_state *st,
                           const cloudsc_increments *inc) {
  const size_t s2 = (size_t)klon * klev;
#define INC2(DST, SRC)                                   \
  for (int jk = 0; jk < klev; jk++)                      \
    for (int jl = kidia - 1; jl < kfdia; jl++) {         \
      size_t o = (size_t)jk * klon + jl;                 \
      (DST)[o] = (DST)[o] + (SRC)[o];                    \
    }
  const uint32_t km = st->keymask;
  if (inc->pa_u) { if (!st->u) return CLOUDSC_E_NULL; INC2(st->u, inc->pa_u) }
  if (inc->pa_v) { if (!st->v) return CLOUDSC_E_NULL; INC2(st->v, inc->pa_v) }
  if (inc->pa_t) { if (!st->t) return CLOUDSC_E_NULL; INC2(st->t, inc->pa_t) }
  if (inc->pa_q && (km & CLOUDSC_KEY_Q)) { if (!st->q) return CLOUDSC_E_NULL; INC2(st->q, inc->pa_q) }
  if (inc->pa_o3 && (km & CLOUDSC_KEY_O3)) { if (!st->o3) return CLOUDSC_E_NULL; INC2(st->o3, inc->pa_o3) }
  if (inc->pa_a && (km & CLOUDSC_KEY_A)) { if (!st->a) return CLOUDSC_E_NULL; INC2(st->a, inc->pa_a) }
  if (inc->pa_tke && (km & CLOUDSC_KEY_TKE)) { if (!st->tke) return CLOUDSC_E_NULL; INC2(st->tke, inc->pa_tke) }
  const double *pcld[4] = {inc->pa_ql, inc->pa_qi, inc->pa_qr, inc->pa_qs};
  const uint32_t kcld[4] = {CLOUDSC_KEY_QL, CLOUDSC_KEY_QI, CLOUDSC_KEY_QR, CLOUDSC_KEY_QS};
  for (int m = 0; m < 4; m++) {
    if (!pcld[m] || !(km & kcld[m])) continue;
    if (!st->cld) return CLOUDSC_E_NULL;
    double *dst = st->cld + (size_t)m * s2; /* CLD(:,:,NCLDQL+m) */
    INC2(dst, pcld[m])
  }
#undef INC2
  return 0;
}

/* STATE_INCREMENT over NPROMA blocks stored (NPROMA, ..., NGPBLKS); columns
 * KIDIA..ICEND of each block, ICEND = MIN(NPROMA, NGPTOT - (block-1)*NPROMA). */
int oracle_state_increment_batched(int nproma, int klev, int ngpblks, int ngptot, int kidia,
                                   const cloudsc_state *st, const cloudsc_increments *inc) {
  if (nproma < 1 || ngpblks < 1 || ngptot < 1 || ngptot > nproma * ngpblks ||
      ngptot <= nproma * (ngpblks - 1) || kidia < 1 || kidia > nproma)
    return CLOUDSC_E_SHAPE;
  const size_t s2 = (size_t)nproma * klev;
  const size_t cs = (size_t)(st->nclv > 0 ? st->nclv : 0) * s2;
  const size_t ps = inc->nclv_pa > 0 ? (size_t)inc->nclv_pa * s2 : s2;
  int err = 0;
  for (int ib = 0; ib < ngpblks; ib++) {
    int icend = ngptot - ib * nproma;
    if (icend > nproma) icend = nproma;
    if (kidia > icend) continue;
    cloudsc_state sb = *st;
    cloudsc_increments ib_inc = *inc;
#define OFF(P, STRIDE) ((P) ? (P) + ib * (STRIDE) : NULL)
    sb.u = OFF(st->u, s2); sb.v = OFF(st->v, s2); sb.t = OFF(st->t, s2); sb.o3 = OFF(st->o3, s2);
    sb.q = OFF(st->q, s2); sb.a = OFF(st->a, s2); sb.tke = OFF(st->tke, s2); sb.cld = OFF(st->cld, cs);
    ib_inc.pa_u = OFF(inc->pa_u, s2); ib_inc.pa_v = OFF(inc->pa_v, s2); ib_inc.pa_t = OFF(inc->pa_t, s2);
    ib_inc.pa_o3 = OFF(inc->pa_o3, s2); ib_inc.pa_q = OFF(inc->pa_q, s2); ib_inc.pa_a = OFF(inc->pa_a, s2);
    ib_inc.pa_tke = OFF(inc->pa_tke, s2);
    ib_inc.pa_ql = OFF(inc->pa_ql, ps); ib_inc.pa_qi = OFF(inc->pa_qi, ps);
    ib_inc.pa_qr = OFF(inc->pa_qr, ps); ib_inc.pa_qs = OFF(inc->pa_qs, ps);
#undef OFF
    int r = oracle_state_increment(kidia, icend, nproma, klev, &sb, &ib_inc);
    if (r < 0) err = r;
  }
  return err;
}
