// Host-side conversion of cloudsc_params into the kernels' constant blocks.
#pragma once
#include <cstdint>
#include <cstring>
#include "cloudsc_column.cuh"

namespace cloudsc {

template <typename Real>
inline void fill_kparams(const cloudsc_params &p, const Derived &d, KParams<Real> &k) {
#define F_(n) k.n = Real(p.n)
  F_(rg); F_(rd); F_(rv); F_(retv); F_(rtt); F_(rlvtt); F_(rlstt); F_(rpi);
  F_(r2es); F_(r3les); F_(r3ies); F_(r4les); F_(r4ies); F_(r5les); F_(r5ies); F_(r5alvcp); F_(r5alscp);
  F_(ralvdcp); F_(ralsdcp); F_(rtwat); F_(rtice); F_(rtwat_rtice_r); F_(rkoop1); F_(rkoop2);
  F_(ramid); F_(ramin); F_(rlmin); F_(rcldiff); F_(rcldiff_convi); F_(rcovpmin); F_(rprecrhmax); F_(rpecons);
  F_(rvrfactor); F_(rtaumel); F_(rssicefactor); F_(rsnowlin1); F_(rsnowlin2); F_(rlcritsnow); F_(rthomo);
  F_(rvice); F_(rvsnow); F_(rxfallspeedrain); F_(rcldtopcf); F_(rdepliqrefrate); F_(rdepliqrefdepth);
  F_(riceinit); F_(rdensref); F_(rdenswat); F_(rcl_overlapliqice); F_(rcl_effrime);
  F_(rcl_inhomogaut); F_(rcl_inhomogacc); F_(rcl_kkaac); F_(rcl_kkbac); F_(rcl_kkaau); F_(rcl_kkbauq);
  F_(rcl_dr); F_(rcl_x1r); F_(rcl_x2r); F_(rcl_lam1r); F_(rcl_lam2r);
  F_(rcl_const1r); F_(rcl_const2r); F_(rcl_const3r); F_(rcl_const4r); F_(rcl_const5r); F_(rcl_const6r);
  F_(rcl_const7r); F_(rcl_cdenom1); F_(rcl_cdenom2); F_(rcl_cdenom3); F_(rcl_fzrab);
  F_(rcl_x1s); F_(rcl_lam1s); F_(rcl_lam2s);
  F_(rcl_const1s); F_(rcl_const2s); F_(rcl_const3s); F_(rcl_const4s); F_(rcl_const5s); F_(rcl_const6s);
  F_(rcl_const7s); F_(rcl_const8s);
  F_(rcl_apb1); F_(rcl_apb2); F_(rcl_apb3);
  F_(rmfadvw); F_(rmfadvwdd);
#undef F_
  k.zrdcp = Real(p.rd / p.rcpd);
  k.zrg_r = Real(1.0 / p.rg);
  k.zrldcp = Real(1.0 / (p.ralsdcp - p.ralvdcp));
  k.zconst_pow_land = Real(d.zconst_pow_land);
  k.zconst_pow_sea = Real(d.zconst_pow_sea);
  k.flt_0p4 = Real(d.flt_0p4);
  k.flt_0p8 = Real(d.flt_0p8);
  k.kkbauq_m1 = Real(p.rcl_kkbauq - 1.0);
  k.kkbac_m1 = Real(p.rcl_kkbac - 1.0);
  k.ralfdcp = Real(p.ralfdcp);
  k.reisthsc = Real(p.reisthsc);
  k.lcldbudc = p.lcldbudc;
  k.lcldbudl = p.lcldbudl;
  k.lcldbudi = p.lcldbudi;
  k.lcldbudt = p.lcldbudt;
  k.lcldbud_vertint = p.lcldbud_vertint;
  k.lcldbud_timeint = p.lcldbud_timeint;
  k.lbud23 = p.lbud23;
  k.ra = Real(p.ra);
  k.rcloud_frac_std = Real(p.rcloud_frac_std);
  for (int i = 0; i < 16; ++i) {
    k.spp_mu[i] = Real(p.spp_mu[i]);
    k.spp_xmag[i] = Real(p.spp_xmag[i]);
  }
  k.lspp = p.lspp;
  k.lcloud_inhomog = p.lcloud_inhomog;
  k.lrad_cloud_inhomog = p.lrad_cloud_inhomog;
  k.spp_lramidlimit1 = p.spp_lramidlimit1;
  for (int i = 0; i < 8; ++i) {
    k.spp_on[i] = p.spp_on[i];
    k.spp_mp[i] = p.spp_mp[i];
  }
  k.ncldtop = p.ncldtop;
  k.lmfdsnow = p.lmfdsnow;
  k.rnice = Real(p.rnice);
  k.laericesed = p.laericesed;
  k.laericeauto = p.laericeauto;
  // RV/RD with the division the kernels would perform (IEEE, in Real)
  k.rv_rd = Real(p.rv) / Real(p.rd);
  // 1/b correctly rounded (IEEE on the host) for each parameter divisor;
  // usable by fast_div_k only inside its window and without an all-ones
  // significand (the conditions of fast_div)
  bool ok = true;
  auto rcp = [&ok](double b) {
    uint64_t u;
    std::memcpy(&u, &b, 8);
    const unsigned e = (unsigned)((u >> 52) & 0x7ff);
    const bool ones = (u & ((1ull << 52) - 1)) == ((1ull << 52) - 1);
    ok = ok && e >= 767u && e <= 1278u && !ones;
    return 1.0 / b;
  };
  k.rcp_rd = rcp(p.rd);
  k.rcp_rtaumel = rcp(p.rtaumel);
  k.rcp_rcl_lam1r = rcp(p.rcl_lam1r);
  k.rcp_rdepliqrefdepth = rcp(p.rdepliqrefdepth);
  k.rcp_rvrfactor = rcp(p.rvrfactor);
  k.rcp_force = ok ? 0 : 1;
}


// The kernels' pows whose exponent is a parameter (mpowp / mpowbp in
// cloudsc_body.cuh) may skip their tests for the exponents 0.5, 1.5, 2 and 3
// (the GEN kernels) when none of these parameters is such an exponent, in
// double or rounded to float.  This list names every exponent those call
// sites use.
inline bool gen_exponents_ok(const KParams<double> &k) {
  const double ex[] = {k.flt_0p4,     k.kkbac_m1,    k.kkbauq_m1,   k.rcl_const3r, k.rcl_const4r,
                       k.rcl_const4s, k.rcl_const5s, k.rcl_const6r, k.rcl_const8s, k.rcl_dr,
                       k.rcl_kkbac,   k.rcl_lam2r,   k.rcl_lam2s,   k.rcl_x2r};
  for (double y : ex) {
    const float yf = (float)y;
    if (y == 0.5 || y == 1.5 || y == 2.0 || y == 3.0) return false;
    if (yf == 0.5f || yf == 1.5f || yf == 2.0f || yf == 3.0f) return false;
  }
  return true;
}

inline void fill_kparams_d(const cloudsc_params &p, KParamsD &dd) {
  dd.rg = p.rg; dd.retv = p.retv; dd.rtt = p.rtt; dd.rtice = p.rtice; dd.rtwat = p.rtwat;
  dd.rtwat_rtice_r = p.rtwat_rtice_r; dd.r2es = p.r2es; dd.r3les = p.r3les; dd.r3ies = p.r3ies;
  dd.r4les = p.r4les; dd.r4ies = p.r4ies; dd.r5alvcp = p.r5alvcp; dd.r5alscp = p.r5alscp;
  dd.ralvdcp = p.ralvdcp; dd.ralsdcp = p.ralsdcp; dd.rkoop1 = p.rkoop1; dd.rkoop2 = p.rkoop2;
  dd.rssicefactor = p.rssicefactor; dd.rlmin = p.rlmin; dd.rlvtt = p.rlvtt; dd.rlstt = p.rlstt;
  dd.zrg_r = 1.0 / p.rg;
}

}  // namespace cloudsc
