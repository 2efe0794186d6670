/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Never linked into the product library.
 *
 * CPU restatement of the constant set-up that feeds CLOUDSC, written from the
 * reference sources:
 *   YOMCST   ifs-source/arpifs/module/yomcst.F90:508-629   (physical constants)
 *   SUPHEC   ifs-source/arpifs/phys_ec/suphec.F90:231-254  (YOETHF saturation constants)
 *   SUCLDP   ifs-source/arpifs/phys_ec/sucldp.F90:243-530,631-655 (TECLDP defaults)
 *   FCGENERALIZED_GAMMA ifs-source/arpifs/utility/fcgeneralized_gamma.F90:69-126
 *   SU0PHY   ifs-source/arpifs/setup/su0phy.F90:1336,1343 (RCLDTOPP, LRAD_CLOUD_INHOMOG)
 *   SUCUMF   ifs-source/arpifs/phys_ec/sucumf.F90:203,228  (LMFDSNOW, RMFADVW)
 *   SUECRAD  ifs-source/arpifs/phys_radi/suecrad.F90:745      (RCLOUD_FRAC_STD)
 *   SUDYNCORE ifs-source/arpifs/setup/sudyncore.F90:86-90   (RPLRG = RPLDARE = 1)
 * Built with -O2 -ffp-contract=off so every expression is evaluated in the
 * reference's order with one rounding per operation.
 *
 * Parity note: the reference's constant set-up cannot be compiled here (no
 * Fortran compiler), so these values are pinned by hand-derived unit tests of
 * the formulas, not by reference output ("parity unpinned").
 */
#include <math.h>
#include <string.h>
#include "oracle.h"

/*
 * fcgeneralized_gamma.F90:69-126.  The literals ZSTP, ZCOEF(1:6) and ZSERCST
 * are default-REAL (binary32) constants assigned to REAL(KIND=JPRB) variables,
 * so their values are the float roundings widened to double (ZSERCST becomes
 * exactly 1.0).  Only PX > 0 occurs in SUCLDP; the reflection branch is then
 * multiplied by zero and contributes nothing.
 */
double oracle_fcgeneralized_gamma(double px) {
  const double zstp = (double)2.5066282746310005f;
  const double zcoef[6] = {(double)76.18009172947146f, (double)-86.50532032941677f,
                           (double)24.01409824083091f, (double)-1.231739572450155f,
                           (double)0.1208650973866179E-2f, (double)-0.5395239384953E-5f};
  const double zsercst = (double)1.000000000190015f;
  double sgn = (px >= 0.0) ? 1.0 : 0.0; /* MAX(SIGN(1,PX),0) */
  double zx = (1.0 - px) * (1.0 - sgn) + px * sgn;
  double zy = zx;
  double zttmmp = zx + 5.5;
  double ztmp = (zx + 0.5) * log(zttmmp) - zttmmp;
  double zser = zsercst + zcoef[0] / (1. + zy) + zcoef[1] / (2. + zy) + zcoef[2] / (3. + zy) +
                zcoef[3] / (4. + zy) + zcoef[4] / (5. + zy) + zcoef[5] / (6. + zy);
  double zgamma = exp(ztmp + log(zstp * zser / zx));
  double rpi = 2.0 * asin(1.0);
  return zgamma * sgn + (rpi / sin(rpi * px) / zgamma) * (1.0 - sgn);
}

int oracle_params_default(double tsphy, int ncldtop, cloudsc_params *p) {
  memset(p, 0, sizeof(*p));
  p->magic = CLOUDSC_PARAMS_MAGIC;
  p->version = 1;

  /* ---- YOMCST (yomcst.F90:508-629), non-aqua-planet defaults ---- */
  const double rplrg = 1.0, rpldare = 1.0, rplradi = 1.0;
  double rpi = 2.0 * asin(1.0);
  double rkbol = 1.380658E-23, rnavo = 6.0221367E+23;
  double r = rnavo * rkbol;
  double rmd = 28.9644, rmv = 18.0153;
  p->rpi = rpi;
  p->ra = 6371229. * rplradi;
  p->rg = 9.80665;
  p->rd = 1000. * r / rmd;
  p->rv = 1000. * r / rmv;
  p->rcpd = 3.5 * p->rd;
  p->retv = p->rv / p->rd - 1.0;
  p->rtt = 273.16;
  p->rlvtt = 2.5008E+6;
  p->rlstt = 2.8345E+6;
  p->rlmlt = p->rlstt - p->rlvtt;

  /* ---- YOETHF (suphec.F90:231-254) ---- */
  p->r2es = 611.21 * p->rd / p->rv;
  p->r3les = 17.502;
  p->r3ies = 22.587;
  p->r4les = 32.19;
  p->r4ies = -0.7;
  p->r5les = p->r3les * (p->rtt - p->r4les);
  p->r5ies = p->r3ies * (p->rtt - p->r4ies);
  p->r5alvcp = p->r5les * p->rlvtt / p->rcpd;
  p->r5alscp = p->r5ies * p->rlstt / p->rcpd;
  p->ralvdcp = p->rlvtt / p->rcpd;
  p->ralsdcp = p->rlstt / p->rcpd;
  p->ralfdcp = p->rlmlt / p->rcpd;
  p->rtwat = p->rtt;
  p->rtice = p->rtt - 23.;
  p->rticecu = p->rtt - 23.;
  p->rtwat_rtice_r = 1.0 / (p->rtwat - p->rtice);
  p->rtwat_rticecu_r = 1.0 / (p->rtwat - p->rticecu);
  p->rkoop1 = 2.583;
  p->rkoop2 = 0.48116E-2;

  /* ---- SUCLDP (sucldp.F90:243-530) ---- */
  p->ramid = 0.8;
  p->rprc1 = 100.;
  p->ramin = 1.E-8;
  p->rlmin = 1.E-8;
  p->rcldiff = 6.0E-6 * rplrg * rpldare;
  p->rcldiff_convi = 10.0;
  p->rclcrit_sea = 2.5E-4;
  p->rclcrit_land = 5.5E-4;
  p->rkconv = rplrg * rpldare / 6000.;
  p->rcl_inhomogaut = 1.5;
  p->rcl_inhomogacc = 3.0;
  p->rsnowlin1 = rplrg * rpldare / 1000.;
  p->rsnowlin2 = 0.030;
  p->rlcritsnow = 2.0E-5;
  double zplrg = rpldare * sqrt(rplrg);
  p->rvice = 0.13 * zplrg;
  p->rvrain = 4.0 * zplrg;
  p->rvsnow = 1.0 * zplrg;
  p->rxfallspeedrain = 1.0;
  p->rxfallspeedice = 1.0;
  p->ricehi1 = 1.0 / 30000.;
  p->ricehi2 = 1.0 / 233.;
  p->rnice = 0.027;
  p->rccn = 125.0;
  p->rcldtopcf = 0.01;
  p->rdepliqrefrate = 0.5;
  p->rdepliqrefdepth = 500.0 / rplrg;
  p->rcl_overlapliqice = 0.65;
  p->rcl_effrime = 1.0;
  p->riceinit = 1.E-12;
  p->rthomo = p->rtt - 38.0;
  p->rprecrhmax = 0.7;
  p->rpecons = 5.44E-4 * rplrg * rpldare / p->rg;
  p->rvrfactor = 5.09E-3 * zplrg;
  p->rcovpmin = 0.1;
  p->rtaumel = 2.0 * 3.6E3 / (rplrg * rpldare);
  p->rkooptau = 3.0 * 3.6E3 / (rplrg * rpldare);
  p->rdenswat = 1000.0;
  p->rdensref = 1.0;

  /* rain */
  double rcl_cr = 386.8 * zplrg;
  p->rcl_dr = 0.67;
  double rcl_ar = p->rdenswat * rpi / 6.;
  double rcl_br = 3.0;
  p->rcl_x1r = 0.22;
  p->rcl_x2r = 2.20;
  double rcl_x4r = 0.0;
  p->rcl_lam1r = rcl_ar * p->rcl_x1r * oracle_fcgeneralized_gamma(rcl_br + 1. + rcl_x4r);
  p->rcl_lam2r = 1.0 / (rcl_br + 1. + rcl_x4r - p->rcl_x2r);
  p->rcl_cdenom1 = 5.57E11;
  p->rcl_cdenom2 = 1.03E8;
  p->rcl_cdenom3 = 2.04E2;
  p->rcl_ka273 = 2.4E-2;
  double rcl_schmidt = 0.6, rcl_dynvisc = 1.717E-5;
  double zgamma1r = oracle_fcgeneralized_gamma((p->rcl_dr + 5.) / 2.);
  double zgamma3r = oracle_fcgeneralized_gamma(rcl_br + 1.0 + rcl_x4r);
  double zgamma4r = oracle_fcgeneralized_gamma(p->rcl_dr + rcl_br + 1.0 + rcl_x4r);
  double zgamma5r = oracle_fcgeneralized_gamma(3.0 + p->rcl_dr + rcl_x4r);
  double zgamma6r = oracle_fcgeneralized_gamma(4.0 + rcl_br + rcl_x4r);
  p->rcl_const1r = 2. * rpi * p->rcl_x1r * rplrg * rpldare;
  p->rcl_const2r = 0.31 * pow(rcl_schmidt, 0.3333) * zgamma1r * pow(rcl_cr / rcl_dynvisc, 0.5);
  p->rcl_const3r = (p->rcl_dr + 5.) / 2. - p->rcl_x2r;
  p->rcl_const4r = 2. - p->rcl_x2r;
  p->rcl_const7r = rcl_cr * zgamma4r / zgamma3r;
  p->rcl_const8r = 0.0; /* associated in cloudsc.F90:637 but never set by SUCLDP nor read */
  p->rcl_const9r = rpi * 0.25 * p->rcl_x1r * rcl_cr * zgamma5r;
  p->rcl_const10r = 3.0 + p->rcl_dr - p->rcl_x2r;
  p->rcl_eff_racw = 0.7;
  p->rcl_kkaac = 67.;
  p->rcl_kkbac = 1.15;
  p->rcl_kkaau = 1350.;
  p->rcl_kkbauq = 2.47;
  p->rcl_kkbaun = -1.79;
  p->rcl_kk_cloud_num_sea = 50.;
  p->rcl_kk_cloud_num_land = 300.;
  p->lcloud_inhomog = 0;
  p->rcl_fzrab = -0.66;
  double rcl_fzrbb = 2.E2;
  p->rcl_const5r = rpi / (6.) * rcl_fzrbb * rcl_ar * p->rcl_x1r * zgamma6r;
  p->rcl_const6r = -1. * (4. + rcl_br + rcl_x4r - p->rcl_x2r);

  /* ice (Morrison and Gettelman values override RCL_CI/RCL_DI, sucldp.F90:456-457) */
  double rcl_ai = 0.069, rcl_bi = 2.0, rcl_ci = 100., rcl_di = 1.0;
  double rcl_x1i = 2.0E6, rcl_x2i = 0.0, rcl_x4i = 0.0;
  double zgamma1i = oracle_fcgeneralized_gamma(rcl_bi + 1.0 + rcl_x4i);
  double zgamma2i = oracle_fcgeneralized_gamma(rcl_x4i + 2.0);
  double zgamma3i = oracle_fcgeneralized_gamma((rcl_di + 5.0 + 2.0 * rcl_x4i) / 2.0);
  double zgamma4i = oracle_fcgeneralized_gamma(rcl_di + rcl_bi + 1.0 + rcl_x4i);
  p->rcl_const1i = 1.0 / (rcl_ai * rcl_x1i * zgamma1i);
  p->rcl_const2i = 1.0 * rpi * rcl_x1i;
  p->rcl_const3i = 0.44 * pow(0.6, 1.0 / 3.0) * pow(rcl_ci, 0.5) * zgamma3i / pow(1.717E-5, 0.5);
  p->rcl_const4i = (2.0 + rcl_x4i - rcl_x2i) / (rcl_bi + 1.0 + rcl_x4i - rcl_x2i);
  p->rcl_const5i = (5.0 + rcl_di + 2.0 * rcl_x4i - 2.0 * rcl_x2i) / (2.0 * (rcl_bi + 1. + rcl_x4i - rcl_x2i));
  p->rcl_const6i = zgamma2i;
  p->rcl_const7i = rcl_ci * zgamma4i / zgamma1i;
  p->rcl_apb1 = 7.14E11;
  p->rcl_apb2 = 1.16E8;
  p->rcl_apb3 = 2.416E2;

  /* snow */
  double rcl_as = 0.069, rcl_bs = 2.0, rcl_cs = 16.8 * zplrg, rcl_ds = 0.527;
  double rcl_x2s = 0.0, rcl_x4s = 0.0;
  p->rcl_x1s = 2.0E6;
  double zgamma1s = oracle_fcgeneralized_gamma(rcl_bs + 1.0 + rcl_x4s);
  double zgamma2s = oracle_fcgeneralized_gamma(3.0 + rcl_ds + rcl_x4s);
  double zgamma3s = oracle_fcgeneralized_gamma((rcl_ds + 5.0 + 2.0 * rcl_x4s) / 2.0);
  double zgamma4s = oracle_fcgeneralized_gamma(rcl_x4s + 2.0);
  p->rcl_lam1s = rcl_as * p->rcl_x1s * oracle_fcgeneralized_gamma(rcl_bs + 1.0 + rcl_x4s);
  p->rcl_lam2s = 1.0 / (rcl_bs + 1. + rcl_x4s - rcl_x2s);
  p->rcl_const1s = 1.0 / (rcl_as * p->rcl_x1s * zgamma1s);
  p->rcl_const2s = 1.0 * rpi * p->rcl_x1s;
  p->rcl_const3s = 0.44 * pow(0.6, 1.0 / 3.0) * pow(rcl_cs, 0.5) * zgamma3s / pow(1.717E-5, 0.5);
  p->rcl_const4s = (2.0 + rcl_x4s - rcl_x2s) / (rcl_bs + 1.0 + rcl_x4s - rcl_x2s);
  p->rcl_const5s = (5.0 + rcl_ds + 2.0 * rcl_x4s - 2.0 * rcl_x2s) / (2.0 * (rcl_bs + 1. + rcl_x4s - rcl_x2s));
  p->rcl_const6s = zgamma4s;
  p->rcl_const7s = rpi * 0.25 * p->rcl_x1s * rcl_cs * zgamma2s;
  p->rcl_const8s = (3.0 + rcl_ds + rcl_x4s - rcl_x2s) / (rcl_bs + 1.0 + rcl_x4s - rcl_x2s);

  /* switches (sucldp.F90:566-595, 696-701; NAERCLD=0) */
  p->ncldtop = ncldtop;
  p->lcldbudc = p->lcldbudl = p->lcldbudi = p->lcldbudt = p->lcldbud_vertint = 0;
  p->lcldbud_timeint = 1;
  p->lcldbudget = 0; /* NCLDDIAG=0 */
  p->lscmec = 0;
  p->laericeauto = p->laericesed = p->laerliqautolsp = p->laerliqcoll = 0;

  /* RSSICEFACTOR (sucldp.F90:655) */
  p->rssicefactor = fmin(tsphy / p->rkooptau, 1.0);

  /* TECUMF (sucumf.F90:203,228-229), TERAD, TEPHY, TVDF, TSPP_CONFIG */
  p->lmfdsnow = 1;
  p->rmfadvw = 0.0;
  p->rmfadvwdd = 0.0;
  p->rcloud_frac_std = 1.0;
  p->lrad_cloud_inhomog = 0;
  p->lbud23 = 0;
  p->reisthsc = 0.0; /* REISTHSC: read only by the budget path (cloudsc.F90:3937), which is off */
  p->lspp = 0;
  return 0;
}
