"""Seeded synthetic CLOUDSC input state on the L137 grid.

No public dataset is involved: the reference's own test data (ICMGG* initial
conditions) is fetched from ECMWF servers and is not available, so the inputs
are drawn from a seeded generator with the shapes and value ranges below.
Each NPROMA block has its own random stream, ``default_rng([seed, ib])``, so
any subset of blocks can be regenerated bit-identically (the parity tests
rebuild a sample of the blocks of the full-size bench input).

Per column (all choices are this generator's, documented here):

* pressure: PAPH = A + B * p_s on the operational L137 hybrid half levels
  (data/l137_ab.txt, copied from ifs-test/tests/scm/common/namelists:90-366;
  coarser test grids take a subset of them, hybrid_ab), p_s ~ U(98, 103)
  kPa, PAP = (PAPH_k + PAPH_k+1)/2;
* temperature: T_s ~ U(280, 300) K, constant-lapse-rate profile
  T = T_s (p/p_s)^(R_d G/g) with G = 6.5 K/km, floored at a 216.65 K
  tropopause, plus N(0, 1.5 K) noise;
* humidity: q = RH * qsat(T, p), RH ~ U(0.2, 1.05), qsat from the scheme's
  own mixed-phase FOEEWM (fcttre.func.h:90-92); above 100 hPa q is capped at
  3 ppm (times U(0.8, 1.2));
* condensates (liquid, ice, rain, snow): each present with probability
  0.5 / 0.5 / 0.35 / 0.35, lognormal with median 1e-5 kg/kg and sigma_ln 1.5,
  capped at 5e-3; ice and snow are zero where T > 273 K, liquid is zero where
  T < 235 K; all condensates are zero above the cloud-top level NCLDTOP;
* cloud fraction: U(0, 1) where liquid or ice is present, else 0;
* cumulative tendencies: T ~ N(0, 1e-4 K/s); q, a and the condensates
  ~ N(0, 1e-5 /s) times the field's own value (a: times 1); PVFL and PVFI
  ~ N(0, 1e-5 /s) times the liquid and ice amounts;
* convection: LDCUM on 30 % of columns, KTYPE 1/2/3 with probability
  0.5/0.3/0.2; cloud base p_s - U(5, 15) kPa, top U(15, 30) kPa (deep),
  base - U(10, 25) kPa (shallow) or U(40, 60) kPa (mid-level); PMFU a sine
  profile of amplitude U(0.01, 0.1) kg m-2 s-1 between base and top, PMFD
  -0.3 times a sine profile below mid-cloud; PLU ~ U(1e-4, 2e-3) kg/kg in the
  updraught; PLUDE = (0.2 in the top 30 % of the cloud, else 0.05) * PMFU * PLU;
  PLUDELI(1:2) split PLUDE by the mixed-phase fraction, PSNDE(1:2) is 0.1 PLUDE
  split the same way; all zero (and KTYPE = 0) elsewhere;
* PLSM in {0, 1} with equal probability, PEIS ~ U(0, 15) K.
"""
import os

import numpy as np

from .fields import BATCHED_FIELDS, INPUT_NAMES, alloc, batched_shape, DTYPE

KLEV_L137 = 137
_AB = None


def l137_ab():
    """Half-level A (Pa) and B coefficients of the L137 grid, k = 0..137."""
    global _AB
    if _AB is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "l137_ab.txt")
        rows = [ln.split() for ln in open(path) if ln.strip() and not ln.startswith("#")]
        a = np.array([float(r[1]) for r in rows])
        b = np.array([float(r[2]) for r in rows])
        _AB = (a, b)
    return _AB


def hybrid_ab(klev=KLEV_L137):
    """Half-level A (Pa) and B of a KLEV-level hybrid grid: the L137 grid
    itself; for 2 <= KLEV < 137 the L137 half levels at the KLEV + 1
    indices round(i * 137 / KLEV), i = 0..KLEV (model top and surface kept);
    for 137 < KLEV <= 1000 A and B interpolated linearly in the L137 half-level
    index at i * 137 / KLEV.  The coarser grids stand in for the operational
    L60/L91 tables, which the reference tree does not carry; they and the
    finer ones exercise the scheme at other vertical resolutions."""
    a, b = l137_ab()
    if klev == KLEV_L137:
        return a, b
    if not 2 <= klev <= 1000:
        raise ValueError("the generator builds grids of 2..1000 levels")
    if klev < KLEV_L137:
        idx = np.round(np.arange(klev + 1) * KLEV_L137 / klev).astype(int)
        return a[idx], b[idx]
    x = np.arange(klev + 1) * KLEV_L137 / klev
    i = np.minimum(np.floor(x).astype(int), KLEV_L137 - 1)
    w = x - i
    return a[i] * (1.0 - w) + a[i + 1] * w, b[i] * (1.0 - w) + b[i + 1] * w


def standard_full_level_pressure(p_surf=101325.0, klev=KLEV_L137):
    a, b = hybrid_ab(klev)
    ph = a + b * p_surf
    return 0.5 * (ph[:-1] + ph[1:])


def ncldtop_for(klev=KLEV_L137, rcldtopp=100.0):
    """NCLDTOP of sucldp.F90:631-634 for the standard atmosphere on the
    KLEV-level grid of hybrid_ab."""
    stpre = standard_full_level_pressure(klev=klev)
    nc = 2
    for jlev in range(len(stpre), 1, -1):
        if stpre[jlev - 1] > rcldtopp:
            nc = jlev
    return nc


def ncldtop_l137(rcldtopp=100.0):
    """NCLDTOP of sucldp.F90:631-634 for the L137 standard atmosphere."""
    return ncldtop_for(KLEV_L137, rcldtopp)


def _qsat_mix(t, p, c):
    """Mixed-phase saturation specific humidity (FOEEWM / p, fcttre.func.h:83-92)."""
    x = (np.maximum(c["rtice"], np.minimum(c["rtwat"], t)) - c["rtice"]) * c["rtwat_rtice_r"]
    alfa = np.minimum(1.0, x * x)
    ew = c["r2es"] * (alfa * np.exp(c["r3les"] * (t - c["rtt"]) / (t - c["r4les"])) +
                      (1.0 - alfa) * np.exp(c["r3ies"] * (t - c["rtt"]) / (t - c["r4ies"])))
    qs = np.minimum(ew / p, 0.5)
    return qs / (1.0 - c["retv"] * qs), alfa


def _block(rng, nproma, klev, ncldtop, c):
    a_h, b_h = hybrid_ab(klev)
    np_ = nproma
    ps = rng.uniform(98000.0, 103000.0, np_)
    paph = a_h[:, None] + b_h[:, None] * ps[None, :]                  # (klev+1, np)
    pap = 0.5 * (paph[:-1] + paph[1:])                                 # (klev, np)

    ts = rng.uniform(280.0, 300.0, np_)
    expo = c["rd"] * 0.0065 / c["rg"]
    t = np.maximum(ts[None, :] * (pap / ps[None, :]) ** expo, 216.65)
    t = t + rng.normal(0.0, 1.5, (klev, np_))

    qsat, alfa = _qsat_mix(t, pap, c)
    q = rng.uniform(0.2, 1.05, (klev, np_)) * qsat
    # stratosphere (p < 100 hPa): a few ppm, as observed, instead of the
    # pressure-inflated saturation value
    q = np.where(pap < 10000.0, np.minimum(q, 3e-6 * rng.uniform(0.8, 1.2, (klev, np_))), q)

    def lognorm(shape):
        return np.minimum(np.exp(np.log(1e-5) + 1.5 * rng.normal(size=shape)), 5e-3)

    shp = (klev, np_)
    above_top = (np.arange(klev) < ncldtop - 1)[:, None]
    warm = t > 273.0
    ql = np.where((rng.random(shp) < 0.5) & (t >= 235.0), lognorm(shp), 0.0)
    qi = np.where((rng.random(shp) < 0.5) & ~warm, lognorm(shp), 0.0)
    qr = np.where(rng.random(shp) < 0.35, lognorm(shp), 0.0)
    qs = np.where((rng.random(shp) < 0.35) & ~warm, lognorm(shp), 0.0)
    ql, qi, qr, qs = (np.where(above_top, 0.0, x) for x in (ql, qi, qr, qs))
    cloudy = (ql > 0) | (qi > 0)
    a = np.where(cloudy, rng.random(shp), 0.0)

    out = {}
    out["pt"] = t
    out["pq"] = q
    out["tendency_cml_t"] = rng.normal(0.0, 1e-4, shp)
    out["tendency_cml_q"] = q * rng.normal(0.0, 1e-5, shp)
    out["tendency_cml_a"] = rng.normal(0.0, 1e-5, shp)
    cld = np.zeros((5, klev, np_))
    for m, x in enumerate((ql, qi, qr, qs)):
        cld[m] = x * rng.normal(0.0, 1e-5, shp)
    out["tendency_cml_cld"] = cld
    out["pvfl"] = ql * rng.normal(0.0, 1e-5, shp)
    out["pvfi"] = qi * rng.normal(0.0, 1e-5, shp)
    out["pap"] = pap
    out["paph"] = paph
    out["plsm"] = (rng.random(np_) < 0.5).astype(np.float64)
    out["peis"] = rng.uniform(0.0, 15.0, np_)

    # convection
    ldcum = rng.random(np_) < 0.3
    ktype = np.where(ldcum, rng.choice(np.array([1, 2, 3]), size=np_, p=[0.5, 0.3, 0.2]), 0)
    pbase = ps - rng.uniform(5000.0, 15000.0, np_)
    ptop = np.where(ktype == 1, rng.uniform(15000.0, 30000.0, np_),
                    np.where(ktype == 2, pbase - rng.uniform(10000.0, 25000.0, np_),
                             rng.uniform(40000.0, 60000.0, np_)))
    m0 = rng.uniform(0.01, 0.1, np_)
    inside = (pap > ptop[None, :]) & (pap < pbase[None, :]) & ldcum[None, :]
    frac = (pap - ptop[None, :]) / (pbase - ptop)[None, :]
    pmfu = np.where(inside, m0[None, :] * np.sin(np.pi * frac), 0.0)
    pmid = 0.5 * (ptop + pbase)
    down = (pap > pmid[None, :]) & (pap < ps[None, :]) & ldcum[None, :]
    fd = (pap - pmid[None, :]) / (ps - pmid)[None, :]
    pmfd = np.where(down, -0.3 * m0[None, :] * np.sin(np.pi * fd), 0.0)
    plu = np.where(inside, rng.uniform(1e-4, 2e-3, shp), 0.0)
    detr = np.where(frac < 0.3, 0.2, 0.05)
    plude = np.where(inside, detr * pmfu * plu, 0.0)
    pludeli = np.zeros((4, klev, np_))
    pludeli[0] = plude * alfa
    pludeli[1] = plude * (1.0 - alfa)
    psnde = np.zeros((2, klev, np_))
    psnde[0] = 0.1 * plude * alfa
    psnde[1] = 0.1 * plude * (1.0 - alfa)
    out["ldcum"] = ldcum.astype(np.int32)
    out["ktype"] = ktype.astype(np.int32)
    out["plu"] = plu
    out["plude"] = plude
    out["pludeli"] = pludeli
    out["psnde"] = psnde
    out["pmfu"] = pmfu
    out["pmfd"] = pmfd
    out["pa"] = a
    pclv = np.zeros((5, klev, np_))
    pclv[0], pclv[1], pclv[2], pclv[3] = ql, qi, qr, qs
    out["pclv"] = pclv
    return out


def generate_satadj(ngpblks, nproma, params, klev=KLEV_L137, seed=1, blocks=None):
    """Inputs (and zeroed outputs) of a batched CLOUD_SATADJ call, in the
    layout of fields.SATADJ_FIELDS.

    The state (T, q, cloud fraction, liquid, ice), pressures and cumulative
    tendencies are those of ``generate`` for the same seed; the fields only
    CLOUD_SATADJ reads come from a second stream per block,
    ``default_rng([seed, ib, 7])``:

    * PVERVEL (omega) ~ N(0, 0.3 Pa/s);
    * PHRSW ~ U(0, 2e-5 K/s), PHRLW ~ N(-2e-5, 1e-5 K/s);
    * PTENDENCY_VDF_T ~ N(0, 1e-4 K/s), PTENDENCY_VDF_Q ~ q N(0, 1e-5 /s);
    * PLUDELI(3) (detrained vapour) = U(0, 1) PLUDE and PLUDELI(4) (detrained
      enthalpy, K kg m-2 s-1) = 2500 PLUDE N(0, 1) on the convective levels
      of ``generate``, zero elsewhere.
    """
    base = generate(ngpblks, nproma, params, klev=klev, seed=seed, blocks=blocks)
    return satadj_from(base, nproma, klev=klev, seed=seed,
                       blocks=list(range(ngpblks)) if blocks is None else list(blocks))


def satadj_from(base, nproma, klev=KLEV_L137, seed=1, blocks=None):
    """The CLOUD_SATADJ inputs of ``generate_satadj`` built from an existing
    ``generate`` result ``base`` (same seed; ``blocks`` = the block indices
    ``base`` holds, default all)."""
    from .fields import satadj_alloc
    nb = base["pt"].shape[0]
    ids = list(range(nb)) if blocks is None else list(blocks)
    out = satadj_alloc(len(ids), nproma, klev)
    for n in ("pap", "paph", "pt", "pq", "pa", "tendency_cml_t", "tendency_cml_q", "tendency_cml_a"):
        out[n][:] = base[n]
    out["pl"][:] = base["pclv"][:, 0]
    out["pi"][:] = base["pclv"][:, 1]
    out["tendency_cml_l"][:] = base["tendency_cml_cld"][:, 0]
    out["tendency_cml_i"][:] = base["tendency_cml_cld"][:, 1]
    out["pludeli"][:, :2] = base["pludeli"][:, :2]
    for j, ib in enumerate(ids):
        rng = np.random.default_rng([int(seed), int(ib), 7])
        shp = (klev, nproma)
        out["pvervel"][j] = rng.normal(0.0, 0.3, shp)
        out["phrsw"][j] = rng.uniform(0.0, 2e-5, shp)
        out["phrlw"][j] = rng.normal(-2e-5, 1e-5, shp)
        out["tendency_vdf_t"][j] = rng.normal(0.0, 1e-4, shp)
        out["tendency_vdf_q"][j] = base["pq"][j] * rng.normal(0.0, 1e-5, shp)
        plude = base["plude"][j]
        out["pludeli"][j, 2] = rng.uniform(0.0, 1.0, shp) * plude
        out["pludeli"][j, 3] = 2500.0 * plude * rng.normal(0.0, 1.0, shp)
    return out


def generate_sltend(ngpblks, nproma, params, klev=KLEV_L137, seed=1, blocks=None):
    """Inputs of SLTEND's supersaturation adjustment in the layout of
    fields.SLTEND_FIELDS: the state, pressures and cumulative tendencies
    (PCENT/Q/A = the CML tendencies) of ``generate`` for the same seed, and
    new physics tendencies from ``default_rng([seed, ib, 11])``: PTENT ~ N(0,
    1e-4 K/s), PTENQ ~ q N(0, 2e-5 /s), PTENA ~ N(0, 1e-5 /s), PTENCLD ~ the
    species' amount times N(0, 1e-5 /s)."""
    base = generate(ngpblks, nproma, params, klev=klev, seed=seed, blocks=blocks)
    return sltend_from(base, nproma, klev=klev, seed=seed,
                       blocks=list(range(ngpblks)) if blocks is None else list(blocks))


def sltend_from(base, nproma, klev=KLEV_L137, seed=1, blocks=None):
    """The inputs of ``generate_sltend`` built from an existing ``generate``
    result ``base`` (same seed; ``blocks`` = the block indices it holds)."""
    from .fields import sltend_alloc
    nb = base["pt"].shape[0]
    ids = list(range(nb)) if blocks is None else list(blocks)
    out = sltend_alloc(len(ids), nproma, klev)
    out["pt"][:] = base["pt"]
    out["pq"][:] = base["pq"]
    out["pa"][:] = base["pa"]
    out["prsf1"][:] = base["pap"]
    out["prs1"][:] = base["paph"]
    out["pcent"][:] = base["tendency_cml_t"]
    out["pcenq"][:] = base["tendency_cml_q"]
    out["pcena"][:] = base["tendency_cml_a"]
    for j, ib in enumerate(ids):
        rng = np.random.default_rng([int(seed), int(ib), 11])
        shp = (klev, nproma)
        out["ptent"][j] = rng.normal(0.0, 1e-4, shp)
        out["ptenq"][j] = base["pq"][j] * rng.normal(0.0, 2e-5, shp)
        out["ptena"][j] = rng.normal(0.0, 1e-5, shp)
        for m in range(4):
            out["ptencld"][j, m] = base["pclv"][j, m] * rng.normal(0.0, 1e-5, shp)
    return out


def generate_diag(base, nproma, kfldx, klev=KLEV_L137, seed=1, blocks=None, nrftotal=10):
    """The inputs only the cloud budget diagnostics read (fields.DIAG_FIELDS)
    for the blocks of an existing ``generate`` result ``base``, from
    ``default_rng([seed, ib, 13])``: PVFA ~ N(0, 1e-5 /s); PDYNA ~ N(0, 1e-5
    /s); PDYNL/I/S ~ the species' amount times N(0, 1e-5 /s); PHRSW ~ U(0,
    2e-5 K/s), PHRLW ~ N(-2e-5, 1e-5 K/s); KCTOP a level index 1..KLEV on the
    convective columns, 0 elsewhere; KPBLTYPE in 0..3; PEXTRA ~ N(0, 1) (it is
    INOUT: the diagnostics add to it); PGAW ~ U(1e-7, 3e-6) (grid boxes of
    about 7-40 km); PGP2DSPP ~ N(0, 1) on ``nrftotal`` fields; PRE_ICE ~
    U(20, 120) um (ice effective radius: 0.04-0.24 m/s fall speed, around the
    default RVICE = 0.13); PICRIT_AER ~ U(1e-5, 1e-4) kg/kg (around RLCRITSNOW
    = 3e-5); PNICE ~ RNICE exp(N(0, 1)) (around RNICE = 0.027); PFSD zero (an
    output)."""
    nb = base["pt"].shape[0]
    ids = list(range(nb)) if blocks is None else list(blocks)
    shp2 = (nb, klev, nproma)
    out = {n: np.zeros(shp2) for n in ("pvfa", "pdyna", "pdynl", "pdyni", "pdyns", "phrsw", "phrlw")}
    out["kctop"] = np.zeros((nb, nproma), np.int32)
    out["kpbltype"] = np.zeros((nb, nproma), np.int32)
    out["pextra"] = np.zeros((nb, kfldx, klev, nproma))
    out["pgaw"] = np.zeros((nb, nproma))
    out["pgp2dspp"] = np.zeros((nb, nrftotal, nproma))
    out["pre_ice"] = np.zeros(shp2)
    out["picrit_aer"] = np.zeros(shp2)
    out["pnice"] = np.zeros(shp2)
    out["pfsd"] = np.zeros(shp2)
    for j, ib in enumerate(ids):
        rng = np.random.default_rng([int(seed), int(ib), 13])
        shp = (klev, nproma)
        out["pvfa"][j] = rng.normal(0.0, 1e-5, shp)
        out["pdyna"][j] = rng.normal(0.0, 1e-5, shp)
        out["pdynl"][j] = base["pclv"][j, 0] * rng.normal(0.0, 1e-5, shp)
        out["pdyni"][j] = base["pclv"][j, 1] * rng.normal(0.0, 1e-5, shp)
        out["pdyns"][j] = base["pclv"][j, 3] * rng.normal(0.0, 1e-5, shp)
        out["phrsw"][j] = rng.uniform(0.0, 2e-5, shp)
        out["phrlw"][j] = rng.normal(-2e-5, 1e-5, shp)
        conv = base["ktype"][j] > 0
        out["kctop"][j] = np.where(conv, rng.integers(1, klev + 1, nproma), 0).astype(np.int32)
        out["kpbltype"][j] = rng.integers(0, 4, nproma).astype(np.int32)
        out["pextra"][j] = rng.normal(0.0, 1.0, (kfldx, klev, nproma))
        out["pgaw"][j] = rng.uniform(1e-7, 3e-6, nproma)
        out["pgp2dspp"][j] = rng.normal(0.0, 1.0, (nrftotal, nproma))
        ra = np.random.default_rng([int(seed), int(ib), 17])  # the aerosol inputs' own stream
        out["pre_ice"][j] = ra.uniform(20.0, 120.0, shp)
        out["picrit_aer"][j] = ra.uniform(1e-5, 1e-4, shp)
        out["pnice"][j] = 0.027 * np.exp(ra.normal(0.0, 1.0, shp))
    return out


def constants_from(params):
    keys = ["rtice", "rtwat", "rtwat_rtice_r", "r2es", "r3les", "r3ies", "r4les", "r4ies", "rtt",
            "retv", "rd", "rg"]
    return {k: float(getattr(params, k)) for k in keys}


def generate(ngpblks, nproma, params, klev=KLEV_L137, seed=1, ngptot=None, blocks=None,
             alloc_fn=None):
    """Inputs (and zeroed outputs) of a batched call.

    Returns a dict name -> array in the (NGPBLKS, ..., NPROMA) layout of
    fields.BATCHED_FIELDS.  ``blocks`` selects which block indices to generate
    (default all ``range(ngpblks)``); the result then holds only those blocks,
    in that order, each identical to the same block of the full set.
    Columns beyond ``ngptot`` in the last block are generated too (they are
    padding the kernel does not touch).
    """
    c = constants_from(params)
    ncldtop = int(params.ncldtop)
    ids = list(range(ngpblks)) if blocks is None else list(blocks)
    arrs = alloc(len(ids), nproma, klev, alloc_fn=alloc_fn)
    for j, ib in enumerate(ids):
        rng = np.random.default_rng([int(seed), int(ib)])
        blk = _block(rng, nproma, klev, ncldtop, c)
        for n, v in blk.items():
            arrs[n][j] = v
    return arrs
