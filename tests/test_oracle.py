"""Self-consistency of the oracle: column water conservation (the intent of
the reference's LCLDBUDGET diagnostic, cloudsc.F90:1032-1082,4146-4212),
finite outputs, and the outputs the reference defines as simple functions of
others (PFHPSL = -RLVTT*PFPLSL, cloudsc.F90:4297-4303)."""
import numpy as np
import pytest

from openifs_b200 import inputs
from tests import util


@pytest.fixture(scope="module")
def run(built):
    p, po = util.params()
    arrs = inputs.generate(40, 32, p, seed=9)
    ref, _ = util.run_oracle(po, arrs, 32, 40, 1280, libm="glibc")
    return p, arrs, ref


def test_finite(run):
    _, _, ref = run
    for n in util.COMPARED:
        assert np.isfinite(util.defined(n, ref[n])).all(), n


def test_column_water_budget_closes(run):
    """Sum over levels of dp/g * dt * (dq + d(l+i+r+s)) equals the convective
    detrainment sources minus the surface precipitation, to rounding."""
    p, arrs, ref = run
    g, dt = p.rg, util.PTSPHY
    nc = int(p.ncldtop)
    dp = np.diff(arrs["paph"], axis=1)                               # (nb, klev, np)
    tend = ref["tendency_loc_q"] + ref["tendency_loc_cld"][:, :4].sum(axis=1)
    lhs = (dp / g * dt * tend).sum(axis=1)
    lev = np.arange(util.KLEV)
    loop = ((lev >= nc - 1) & (lev < util.KLEV - 1))[None, :, None]
    active = loop & (ref["plude"] != 0.0)                             # detrainment applied
    src_li = (arrs["pludeli"][:, 0] + arrs["pludeli"][:, 1]) * active
    src_rs = (arrs["psnde"][:, 0] + arrs["psnde"][:, 1]) * loop
    rhs = dt * (src_li + src_rs).sum(axis=1) - dt * (ref["pfplsl"][:, -1] + ref["pfplsn"][:, -1])
    scale = (np.abs(dp / g * dt * tend)).sum(axis=1) + np.abs(rhs) + 1e-30
    rel = np.abs(lhs - rhs) / scale
    assert np.median(rel) < 1e-14
    # The reference itself leaks a little: the post-solve clip (ZQXN < ZEPSEC
    # -> vapour, cloudsc.F90:3633-3640) runs before the sedimentation flux
    # ZPFPLSX(JK+1) = ZFALLSINK*ZQXN is formed (:3658-3662), so when a falling
    # species' solution drops below ZEPSEC = 1e-14 the part of it the implicit
    # solve sent downwards (ZFALLSINK * ZQXN < ~100 * 1e-14 kg/kg) is lost.
    # That bounds the column residual by ~1e-12 kg/kg * dp/g per level.
    assert np.max(np.abs(lhs - rhs)) < 1e-9


def test_enthalpy_flux_definition(run):
    p, _, ref = run
    assert np.array_equal(ref["pfhpsl"], -p.rlvtt * ref["pfplsl"])
    assert np.array_equal(ref["pfhpsn"], -p.rlstt * ref["pfplsn"])


def test_flux_quirk_reproduced(run):
    """PFSQRF(JK+1) starts from PFSQLF(JK), not PFSQRF(JK) (cloudsc.F90:4251):
    PFSQRF(k+1) - PFSQLF(k) = (ZQXN-ZQX0)(rain) * (-dp/(g dt)), and the rain
    increment is LOC_CLD(rain)*dt."""
    p, arrs, ref = run
    assert np.all(ref["pfsqrf"][:, 0] == 0.0)
    dp = np.diff(arrs["paph"], axis=1)
    incr = -ref["tendency_loc_cld"][:, 2] * dp / p.rg
    quirk = ref["pfsqrf"][:, 1:] - ref["pfsqlf"][:, :-1]
    plain = ref["pfsqrf"][:, 1:] - ref["pfsqrf"][:, :-1]
    scale = np.abs(ref["pfsqlf"]).max() + np.abs(incr).max()
    assert np.abs(quirk - incr).max() < 1e-12 * scale
    assert np.abs(plain - incr).max() > 1e-6 * scale


def test_clear_sky_has_no_precipitation(built):
    p, po = util.params()
    arrs = util.apply_case(inputs.generate(4, 32, p, seed=3), "clear")
    arrs["psnde"][:] = 0.0
    arrs["pludeli"][:] = 0.0
    arrs["ldcum"][:] = 0
    ref, _ = util.run_oracle(po, arrs, 32, 4, 128)
    assert np.all(ref["pfplsl"] == 0.0) and np.all(ref["pfplsn"] == 0.0)


def test_column_enthalpy_budget_closes(run):
    """Liquid-water enthalpy: sum over levels of dp/g (LOC_T - RALVDCP (LOC_L +
    LOC_R) - RALSDCP (LOC_I + LOC_S)) equals RALVDCP (P_rain - S_l - S_r) +
    RALSDCP (P_snow - S_i - S_s) (surface precipitation P, detrainment
    sources S): every phase change heats exactly by its latent heat and
    every transport of condensate is heat-free.  This is the second budget
    the surrogate's guard enforces (openifs_b200/csrc/surrogate_kernels.cu)."""
    p, arrs, ref = run
    g = p.rg
    nc = int(p.ncldtop)
    dp = np.diff(arrs["paph"], axis=1)
    L = ref["tendency_loc_cld"]
    lev = np.arange(util.KLEV)
    loop = ((lev >= nc - 1) & (lev < util.KLEV - 1))[None, :, None]
    active = loop & (ref["plude"] != 0.0)
    sl = (arrs["pludeli"][:, 0] * active).sum(1)
    si = (arrs["pludeli"][:, 1] * active).sum(1)
    sr = (arrs["psnde"][:, 0] * loop).sum(1)
    ss = (arrs["psnde"][:, 1] * loop).sum(1)
    lhs = (dp / g * (ref["tendency_loc_t"] - p.ralvdcp * (L[:, 0] + L[:, 2])
                     - p.ralsdcp * (L[:, 1] + L[:, 3]))).sum(axis=1)
    rhs = p.ralvdcp * (ref["pfplsl"][:, -1] - sl - sr) + p.ralsdcp * (ref["pfplsn"][:, -1] - si - ss)
    scale = (np.abs(dp / g * ref["tendency_loc_t"])).sum(axis=1) + np.abs(rhs)
    rel = np.abs(lhs - rhs) / scale
    assert np.median(rel) < 1e-14 and rel.max() < 1e-11, (np.median(rel), rel.max())


def test_satadj_conserves_water_and_enthalpy():
    """CLOUD_SATADJ only moves water between vapour and condensate: at every
    point dq + dl + di = 0 and dT = (Lv/cp) dl + (Ls/cp) di up to rounding,
    and levels above NCLDTOP are untouched (cloud_satadj.F90:338-345, 801-843)."""
    import numpy as np
    from openifs_b200 import fields, inputs
    from tests import util
    p, po = util.params()
    a = inputs.generate_satadj(16, 32, po, seed=17)
    out, _ = util.run_oracle_satadj(po, a, 32, 16, 16 * 32, libm="glibc")
    q, l, i, t = (out[f"tendency_loc_{s}"] for s in "qlit")
    scale_q = np.abs(q).max()
    assert scale_q > 0
    assert np.abs(q + l + i).max() <= 1e-12 * scale_q
    h = t - po.ralvdcp * l - po.ralsdcp * i
    assert np.abs(h).max() <= 1e-12 * np.abs(t).max()
    top = po.ncldtop - 1
    for n in fields.SATADJ_OUTPUTS:
        assert np.all(out[n][:, :top] == 0.0), n
    # condensation, evaporation and cloud-cover changes all occur
    assert (l > 0).any() and (l < 0).any() and (out["tendency_loc_a"] != 0).any()


def test_sltend_supersat_conserves():
    """SLTEND's supersaturation adjustment moves water from vapour to
    condensate only: dq + dl + di = 0 and dT = (Lv/cp) dl + (Ls/cp) di per
    point, up to rounding; levels above NCLDTOP are untouched."""
    import numpy as np
    from openifs_b200 import inputs
    from tests import util
    p, po = util.params()
    a = inputs.generate_sltend(16, 32, po, seed=23)
    out = util.run_oracle_sltend(po, a, 32, 16, 16 * 32, libm="glibc")
    dt, dq = out["ptent"] - a["ptent"], out["ptenq"] - a["ptenq"]
    dl = out["ptencld"][:, 0] - a["ptencld"][:, 0]
    di = out["ptencld"][:, 1] - a["ptencld"][:, 1]
    assert (dq != 0).any()
    assert np.abs(dq + dl + di).max() <= 1e-9 * np.abs(dq).max()
    assert np.abs(dt - po.ralvdcp * dl - po.ralsdcp * di).max() <= 1e-9 * np.abs(dt).max()
    top = po.ncldtop - 1
    assert np.array_equal(out["ptent"][:, :top], a["ptent"][:, :top])
    assert np.array_equal(out["ptencld"][:, 2:], a["ptencld"][:, 2:])
