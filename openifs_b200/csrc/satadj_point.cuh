// CLOUD_SATADJ for one (column, level) point, double precision (device code).
//
// Restates ifs-source/arpifs/phys_ec/cloud_satadj.F90:353-843 (the level loop
// body) with QSATMIXADJ (:948-1017) and CLOUD_SUPERSATCHECK
// (cloud_supersatcheck.F90:111-223, KFTLIQICE = 2) in the default
// configuration: no SPP perturbations, budget diagnostics off.  The scheme has
// no vertical dependence (PAPH(KLEV+1) is the only other level it reads), so
// every point is independent and one GPU thread computes one point.
//
// Parity: every floating-point operation is the reference's, in its order
// (compiled with --fmad=false); the saturation functions of fcttre.func.h
// share their two exponentials per temperature as in cloudsc_body.cuh:
// FOEEW(T) is FOEELIQ(T) or the ice form exactly (FOEDELTA is 0 or 1), and
// FOEEWM's ice term is skipped where FOEALFA = 1, where it adds exactly 0.
// Quantities the reference forms but never uses at this configuration
// (ZQSLIQ, ZCORQSLIQ, ZEVAPLIMMIX, ZQSLIM, the _UPD liquid/ice/Koop values,
// ZRDTGDP, ZRHO, ZDZ, in-cloud condensate) are not computed.
#pragma once

namespace cloudsc {

// Saturation pieces of fcttre.func.h at one temperature (both exponentials
// evaluated once).
struct Sat {
  double el, ei, alfa;
  bool delta;
};
CSC_DEV Sat sat_at(const KParams<double> &k, double t) {
  Sat s;
  s.el = xexp(k.r3les * (t - k.rtt) / (t - k.r4les));
  const double x = (mx(k.rtice, mn(k.rtwat, t)) - k.rtice) * k.rtwat_rtice_r;
  s.alfa = mn(1.0, x * x);
  s.delta = copysign(1.0, t - k.rtt) > 0.0;
  s.ei = 0.0;
  if (!s.delta || s.alfa < 1.0) s.ei = xexp(k.r3ies * (t - k.rtt) / (t - k.r4ies));
  return s;
}
CSC_DEV double sat_foeewm(const KParams<double> &k, const Sat &s) {
  const double w = (s.alfa < 1.0) ? s.alfa * s.el + (1.0 - s.alfa) * s.ei : s.el;
  return k.r2es * w;
}
CSC_DEV double sat_foedem(const KParams<double> &k, const Sat &s, double t) {
  const double xl = t - k.r4les, xi = t - k.r4ies;
  return s.alfa * k.r5alvcp * (1.0 / (xl * xl)) + (1.0 - s.alfa) * k.r5alscp * (1.0 / (xi * xi));
}
CSC_DEV double sat_foeldcpm(const KParams<double> &k, const Sat &s) {
  return s.alfa * k.ralvdcp + (1.0 - s.alfa) * k.ralsdcp;
}

// QSATMIXADJ (cloud_satadj.F90:948-1017): two Newton steps towards the
// mixed-phase saturation; returns the adjusted humidity.
CSC_DEV double qsatmixadj(const KParams<double> &k, double pt, double pq, double pp) {
  double zt = pt, zq = pq;
  const double zp_r = 1.0 / pp;
#pragma unroll 1
  for (int ji = 0; ji < 2; ++ji) {
    const Sat s = sat_at(k, zt);
    const double zfoeet = mn(sat_foeewm(k, s) * zp_r, 0.5);
    const double zcor = 1.0 / (1.0 - k.retv * zfoeet);
    const double zqsat = zfoeet * zcor;
    const double zcorqs = 1.0 + zqsat * zcor * sat_foedem(k, s, zt);
    const double zcond = (zq - zqsat) / zcorqs;
    zt = zt + sat_foeldcpm(k, s) * zcond;
    zq = zq - zcond;
  }
  return zq;
}

// CLOUD_SUPERSATCHECK with KFTLIQICE = 2 (cloud_supersatcheck.F90:111-223):
// the condensate ZCOND = PL_ADJ + PI_ADJ and the cloud increase ZDA.  The
// caller only needs their sum, which is ZCOND + 0 in either phase branch.
CSC_DEV void supersat_cond(const KParams<double> &k, double pt, double pq, double pa, double pp,
                           double &cond, double &da) {
  const double zepsec = 1.E-14;
  double zda = 0.0;
  const double zt = mx(pt, 160.0);
  const double za = mx(mn(pa, 1.0), 0.0);
  const double zp_r = 1.0 / pp;
  const Sat s = sat_at(k, zt);
  const double zfoeeliq = mn((k.r2es * s.el) * zp_r, 0.5);
  const double foeew = s.delta ? k.r2es * s.el : k.r2es * s.ei;
  const double zfoeeice = mn(foeew * zp_r, 0.5);
  const double zfokoop = mn(zfoeeice * (k.rkoop1 - k.rkoop2 * zt), zfoeeliq);
  double zqsliqk = zfokoop / (1.0 - k.retv * zfokoop);
  const double zfoeemix = mn(sat_foeewm(k, s) * zp_r, 0.5);
  const double zcor = 1.0 / (1.0 - k.retv * zfoeemix);
  const double zqsmix = zfoeemix * zcor;
  const double zcorqsmix = 1.0 + zqsmix * zcor * sat_foedem(k, s, zt);
  zqsliqk = 0.5 * (zqsliqk + zqsmix);
  double zqslim = za * zqsmix + (1.0 - za) * zqsliqk;
  double zcond = mx(pq - zqslim, 0.0);
  if (zcond > zepsec) {
    const double zfaci = s.alfa + (1.0 - s.alfa) * k.rssicefactor;
    zda = (1.0 - za) * zfaci;
    const double za_upd = za + zda;
    zqslim = za_upd * zqsmix + (1.0 - za_upd) * zqsliqk;
    zcond = (pq - zqslim) / zcorqsmix;
  }
  const bool liquid = pt + sat_foeldcpm(k, s) * zcond >= k.rthomo;
  cond = (liquid ? zcond : 0.0) + (liquid ? 0.0 : zcond);
  da = zda;
}

// CLOUD_SUPERSATCHECK with KFTLIQICE = 1 (cloud_supersatcheck.F90:111-223):
// all five adjustments, liquid and ice split by the mixed-phase fraction.
CSC_DEV void supersatcheck_kft1(const KParams<double> &k, double pt, double pq, double pa, double pp,
                                double &t_adj, double &q_adj, double &a_adj, double &l_adj, double &i_adj) {
  const double zepsec = 1.E-14;
  double zda = 0.0;
  const double zt = mx(pt, 160.0);
  const double za = mx(mn(pa, 1.0), 0.0);
  const double zp_r = 1.0 / pp;
  const Sat s = sat_at(k, zt);
  const double zfoeeliq = mn((k.r2es * s.el) * zp_r, 0.5);
  const double foeew = s.delta ? k.r2es * s.el : k.r2es * s.ei;
  const double zfoeeice = mn(foeew * zp_r, 0.5);
  const double zfokoop = mn(zfoeeice * (k.rkoop1 - k.rkoop2 * zt), zfoeeliq);
  double zqsliqk = zfokoop / (1.0 - k.retv * zfokoop);
  const double zfoeemix = mn(sat_foeewm(k, s) * zp_r, 0.5);
  const double zcor = 1.0 / (1.0 - k.retv * zfoeemix);
  const double zqsmix = zfoeemix * zcor;
  const double zcorqsmix = 1.0 + zqsmix * zcor * sat_foedem(k, s, zt);
  zqsliqk = 0.5 * (zqsliqk + zqsmix);
  double zqslim = za * zqsmix + (1.0 - za) * zqsliqk;
  double zcond = mx(pq - zqslim, 0.0);
  if (zcond > zepsec) {
    const double zfaci = s.alfa + (1.0 - s.alfa) * k.rssicefactor;
    zda = (1.0 - za) * zfaci;
    const double za_upd = za + zda;
    zqslim = za_upd * zqsmix + (1.0 - za_upd) * zqsliqk;
    zcond = (pq - zqslim) / zcorqsmix;
  }
  t_adj = sat_foeldcpm(k, s) * zcond;
  q_adj = -zcond;
  a_adj = zda;
  l_adj = zcond * s.alfa;
  i_adj = zcond * (1.0 - s.alfa);
}

// The five CLOUD_SATADJ tendencies of one point at level jk >= NCLDTOP
// (arguments are that point's inputs; psurf = PAPH(KLEV+1)).  nwarn is
// incremented for each negative-condensate warning the reference prints
// (:828, :836).
CSC_DEV void satadj_point(const KParams<double> &k, double dt, double zqtmst, double pap, double paph_k,
                          double paph_k1, double psurf, double pt, double pq, double pa, double pl,
                          double pi, double cml_t, double cml_q, double cml_a, double cml_l,
                          double cml_i, double phrsw, double phrlw, double vdf_t, double vdf_q,
                          double pludeli3, double pludeli4, double pvervel, double &loc_t,
                          double &loc_q, double &loc_a, double &loc_l, double &loc_i, int &nwarn) {
  const double zepsec = 1.E-14;
  // updated state (:357-366)
  const double zt = pt + dt * cml_t;
  const double zq = pq + dt * cml_q;
  double za = pa + dt * cml_a;
  const double zl = pl + dt * cml_l;
  const double zi = pi + dt * cml_i;
  za = mx(0.0, mn(1.0, za));
  // T and q forcing (:384-413)
  const double zdp = paph_k1 - paph_k;
  const double zgdp = k.rg / zdp;
  const double zdtgdp = dt * zgdp;
  const double zdtdp = k.zrdcp * pt / pap;
  const double zdpmxdt = zdp * zqtmst;
  const double zwtot = mn(zdpmxdt, mx(-zdpmxdt, pvervel));
  const double zzzdt = phrsw + phrlw;
  const double zdtdiab = mn(zdpmxdt * zdtdp, mx(-zdpmxdt * zdtdp, zzzdt)) * dt;
  const double zdtforce = zdtdp * zwtot * dt + zdtdiab + pludeli4 * zdtgdp + vdf_t * dt;
  const double zdqforce = pludeli3 * zdtgdp + vdf_q * dt;
  // liquid/ice fractions, critical RH (:435-469)
  const double zli = zl + zi;
  double zliqfrac = 0.0, zicefrac = 0.0;
  if (zli > k.rlmin) {
    zliqfrac = zl / zli;
    zicefrac = 1.0 - zliqfrac;
  }
  double zrhc = k.ramid;
  const double zsigk = pap / psurf;
  if (zsigk > 0.8) {
    const double x = (zsigk - 0.8) / 0.2;
    zrhc = k.ramid + (1.0 - k.ramid) * (x * x);
  }
  // saturation of the start-of-step state (:474-501)
  const double zp_r = 1.0 / pap;
  const Sat s0 = sat_at(k, pt);
  const double zfoeeliq = mn((k.r2es * s0.el) * zp_r, 0.5);
  const double zfoeeice = mn((s0.delta ? k.r2es * s0.el : k.r2es * s0.ei) * zp_r, 0.5);
  const double zfokoop = mn(zfoeeice * (k.rkoop1 - k.rkoop2 * pt), zfoeeliq);
  double zqsliqk = zfokoop / (1.0 - k.retv * zfokoop);
  double zfoeemix = mn(sat_foeewm(k, s0) * zp_r, 0.5);
  double zcor = 1.0 / (1.0 - k.retv * zfoeemix);
  const double zqsmix = zfoeemix * zcor;
  zqsliqk = 0.5 * (zqsliqk + zqsmix);
  // saturation of the updated state (:507-542): ZQSMIX_UPD, ZCORQSMIX_UPD
  const Sat s1 = sat_at(k, zt);
  zfoeemix = mn(sat_foeewm(k, s1) * zp_r, 0.5);
  zcor = 1.0 / (1.0 - k.retv * zfoeemix);
  const double zqsmix_upd = zfoeemix * zcor;
  const double zcorqsmix_upd = 1.0 + zqsmix_upd * zcor * sat_foedem(k, s1, zt);
  // condensation/evaporation from dqsat/dt (:574-593)
  const double zttmp = mx(pt + zdtforce, 160.0);
  const double zqtmp = zqsmix + zdqforce;
  const double zdqs = qsatmixadj(k, zttmp, zqtmp, pap) - zqtmp;
  // clear-air condensation, new cloud (:602-655)
  double env_l = 0.0, env_i = 0.0, zacond = 0.0;
  if (zdqs <= -k.rlmin && pa < 1.0 - zepsec) {
    double zqe = (pq - pa * zqsmix) / mx(zepsec, 1.0 - pa);
    zqe = mx(0.0, zqe);
    if (zqe >= zrhc * zqsliqk && zqe < zqsliqk) {
      zacond = -(1.0 - pa) * zdqs / mx(2.0 * (zqsliqk - zqe), zepsec);
      zacond = mn(zacond, 1.0 - pa);
      double zlcond_env = -zdqs * 0.5 * zacond;
      const double zzdl = 2.0 * (zqsliqk - zqe) / mx(zepsec, 1.0 - pa);
      if (zdqs < -zzdl) {
        const double zlcondlim = (pa - 1.0) * zdqs - zqsliqk + pq;
        zlcond_env = mn(zlcond_env, zlcondlim);
      }
      zlcond_env = mx(zlcond_env, 0.0);
      if (zlcond_env < k.rlmin || (1.0 - pa) < zepsec) {
        zlcond_env = 0.0;
        zacond = 0.0;
      }
      if (zlcond_env == 0.0) zacond = 0.0;
      if (pt > k.rthomo) env_l = zlcond_env;
      else env_i = zlcond_env;
    }
  }
  // condensation in the cloudy part (:662-695)
  double cld_l = 0.0, cld_i = 0.0;
  if (pa > zepsec && zdqs <= -k.rlmin) {
    double zlcond_cld = mx(-zdqs, 0.0);
    const double zcdmax = mx((zq - zqsmix_upd) / zcorqsmix_upd, 0.0);
    zlcond_cld = mn(zlcond_cld, zcdmax);
    zlcond_cld = pa * zlcond_cld;
    if (zlcond_cld < k.rlmin) zlcond_cld = 0.0;
    if (pt > k.rthomo) cld_l = zlcond_cld;
    else cld_i = zlcond_cld;
  }
  // evaporation of the cloudy part (:703-723); ZAEVAP is 0
  double ev_l = 0.0, ev_i = 0.0;
  const double zaevap = 0.0;
  if (zdqs > 0.0 && zli > 0.0) {
    const double zlevap_cld = mn(pa * zdqs, zli);
    ev_l = zliqfrac * zlevap_cld;
    ev_i = zicefrac * zlevap_cld;
  }
  // state for the supersaturation check (:738-757)
  const double zt_upd = zt + k.ralvdcp * (cld_l + env_l - ev_l) + k.ralsdcp * (cld_i + env_i - ev_i);
  const double zq_upd = zq + (ev_l - cld_l - env_l) + (ev_i - cld_i - env_i);
  double zanew = za + zacond - zaevap;
  zanew = mn(zanew, 1.0);
  if (zanew < k.ramin) zanew = 0.0;
  // supersaturation check (:767-793)
  double zcond, zsupsata;
  supersat_cond(k, zt_upd, zq_upd, zanew, pap, zcond, zsupsata);
  double supl, supi;
  if (zt_upd > k.rthomo) {
    supl = zcond;
    supi = 0.0;
  } else {
    supl = 0.0;
    supi = zcond;
  }
  // tendencies (:801-822)
  double tt = k.ralvdcp * (cld_l + env_l + supl - ev_l) * zqtmst + k.ralsdcp * (cld_i + env_i + supi - ev_i) * zqtmst;
  double tq = (ev_l - cld_l - env_l - supl + ev_i - cld_i - env_i - supi) * zqtmst;
  zanew = za + zacond - zaevap + zsupsata;
  zanew = mn(zanew, 1.0);
  if (zanew < k.ramin) zanew = 0.0;
  const double ta = (zanew - za) * zqtmst;
  double tl = (cld_l + env_l + supl - ev_l) * zqtmst;
  double ti = (cld_i + env_i + supi - ev_i) * zqtmst;
  // negative clean-up (:824-843)
  const double ladj = zl + tl * dt;
  if (ladj < -k.rlmin) ++nwarn;
  if (ladj < 0.0) {
    tl = tl - ladj;
    tq = tq + ladj;
    tt = tt - k.ralvdcp * ladj;
  }
  const double iadj = zi + ti * dt;
  if (iadj < -k.rlmin) ++nwarn;
  if (iadj < 0.0) {
    ti = ti - iadj;
    tq = tq + iadj;
    tt = tt - k.ralsdcp * iadj;
  }
  loc_t = tt;
  loc_q = tq;
  loc_a = ta;
  loc_l = tl;
  loc_i = ti;
}

}  // namespace cloudsc
