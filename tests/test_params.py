"""Constant set-up: the product's restatement (cloudsc_b200_params_default)
and the oracle's (oracle_params.c) agree bit for bit, and both reproduce
hand-derived values of the SUCLDP / SUPHEC / YOMCST formulas."""
import math

import numpy as np
import pytest

from openifs_b200 import cloudsc, inputs
from oracle import oracle
from tests import util


@pytest.fixture(scope="module")
def pp(built):
    nc = inputs.ncldtop_l137()
    return cloudsc.default_params(3600.0, nc), oracle.params_default(3600.0, nc)


def test_product_and_oracle_params_identical(pp):
    p, po = pp
    assert p.tobytes() == po.tobytes()


def test_physical_constants(pp):
    p, _ = pp
    r = 6.0221367e23 * 1.380658e-23
    assert p.rd == 1000.0 * r / 28.9644                       # yomcst.F90 RD
    assert p.rv == 1000.0 * r / 18.0153
    assert p.rcpd == 3.5 * p.rd
    assert p.retv == p.rv / p.rd - 1.0
    assert p.rtt == 273.16 and p.rg == 9.80665
    assert p.r2es == 611.21 * p.rd / p.rv                     # suphec.F90:233
    assert p.r5les == 17.502 * (273.16 - 32.19)
    assert p.rtwat_rtice_r == 1.0 / (p.rtwat - p.rtice)
    assert abs(p.ralvdcp - 2.5008e6 / p.rcpd) == 0.0


def test_sucldp_defaults(pp):
    p, _ = pp
    assert p.ramid == 0.8 and p.rlmin == 1e-8 and p.ramin == 1e-8
    assert p.rkooptau == 10800.0 and p.rssicefactor == 3600.0 / 10800.0  # sucldp.F90:655
    assert p.rthomo == 273.16 - 38.0
    assert p.rvrain == 4.0 and p.rvsnow == 1.0 and p.rvice == 0.13
    assert p.rcl_lam2r == 1.0 / (3.0 + 1.0 + 0.0 - 2.2)
    assert p.rcl_const4s == 2.0 / 3.0
    assert p.rcl_const8s == (3.0 + 0.527) / 3.0


def test_gamma_uses_binary32_coefficients(built):
    """FCGENERALIZED_GAMMA's Lanczos coefficients are default-REAL literals
    (fcgeneralized_gamma.F90:69-72): Gamma(4) is then 6 only to ~1e-7."""
    g4 = oracle.gamma(4.0)
    assert abs(g4 - 6.0) < 1e-6
    assert g4 != 6.0
    # with the double-precision coefficients the same formula is exact to 1e-14
    coef = [76.18009172947146, -86.50532032941677, 24.01409824083091, -1.231739572450155,
            0.1208650973866179e-2, -0.5395239384953e-5]
    x = 4.0
    ser = 1.000000000190015 + sum(c / (j + 1 + x) for j, c in enumerate(coef))
    g4d = math.exp((x + 0.5) * math.log(x + 5.5) - (x + 5.5) + math.log(2.5066282746310005 * ser / x))
    assert abs(g4d - 6.0) < 1e-12
    assert abs(g4 - g4d) > 1e-10


def test_gamma_derived_constants(pp):
    p, _ = pp
    g = oracle.gamma
    assert p.rcl_lam1r == 1000.0 * (2.0 * math.asin(1.0)) / 6.0 * 0.22 * g(4.0)
    assert p.rcl_const6s == g(2.0)
    assert p.rcl_const7r == 386.8 * g(0.67 + 3.0 + 1.0) / g(4.0)


def test_ncldtop_l137():
    """sucldp.F90:631-634 with RCLDTOPP = 100 Pa on the L137 standard atmosphere."""
    nc = inputs.ncldtop_l137()
    stpre = inputs.standard_full_level_pressure()
    assert stpre[nc - 1] > 100.0 and stpre[nc - 2] <= 100.0
    import numpy as np
    from openifs_b200 import cloudsc as c
    lib = c.lib()
    assert lib.cloudsc_b200_ncldtop(137, np.ascontiguousarray(stpre).ctypes.data, 100.0) == nc


def test_aerosol_switches_accepted(pp, built):
    """Every CLOUDSC switch is accepted, the four aerosol switches (NAERCLD >
    0) included.  LAERLIQAUTOLSP and LAERLIQCOLL act only in the IWARMRAIN = 1
    branch (cloudsc.F90:1985-1989, 2020-2023) and IWARMRAIN is fixed at 3
    (:727): with them on, the oracle's outputs are the default's bit for bit,
    PLCRIT_AER and PCCN unread."""
    p, po = pp
    for name in ("laericeauto", "laericesed", "laerliqautolsp", "laerliqcoll"):
        q = util.with_flags(p, {name: 1})
        try:
            cloudsc.setup(q)
        except cloudsc.CloudscError as e:  # without a GPU the upload fails (-4) after the checks
            assert e.code == -4, (name, e.code)
    arrs = inputs.generate(3, 32, p, seed=8)
    ref, nw = util.run_oracle(po, arrs, 32, 3, 90)
    qo = util.with_flags(po, {"laerliqautolsp": 1, "laerliqcoll": 1})
    got, nw2 = util.run_oracle(qo, arrs, 32, 3, 90)
    for n in util.COMPARED:
        assert np.array_equal(util.defined(n, got[n]), util.defined(n, ref[n])), n
    assert nw == nw2
