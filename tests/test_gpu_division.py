"""The column kernels' branch-free division (fast_div in cloudsc_column.cuh)
against IEEE division, and the column rerun that keeps the kernels' results
those of IEEE division where it reports an operand (GPU tests).

The division returns a quotient from a Newton-refined reciprocal (corrected
for divisors whose significand is all ones), corrected twice with its
residual, with the dividend's sign put back at the end.  Inside its window
(2^-256 <= |b| < 2^256, and a = 0 or 2^-256 <= |a| < 2^256) it must equal
IEEE a / b bit for bit, zeros included; every operand outside it must be
reported (bad = 1), because the kernels then run the column again with IEEE
division.  The reference quotients are numpy's, IEEE double division on the
host."""
import numpy as np
import pytest

from openifs_b200 import cloudsc, inputs
from tests import util

pytestmark = pytest.mark.gpu


def _gpu_div(a, b):
    import torch
    ta = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    tb = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).cuda()
    q, bad = cloudsc.division_check(ta, tb)
    torch.cuda.synchronize()
    return q.cpu().numpy(), bad.cpu().numpy()


def _bits(x):
    return np.ascontiguousarray(x, dtype=np.float64).view(np.int64)


def _biased_exponent(x):
    return (_bits(x) >> 52) & 0x7FF


def _all_ones(b):
    """Divisors whose significand is 1.11...1 (binary)."""
    return (_bits(b) & ((1 << 52) - 1)) == (1 << 52) - 1


def _in_window(x):
    e = _biased_exponent(x)
    return (e >= 767) & (e <= 1278)


def _in_domain(a, b):
    """Where the division must not report: 2^-256 <= |b| < 2^256, and a zero
    or 2^-256 <= |a| < 2^256."""
    return ((a == 0) | _in_window(a)) & _in_window(b)


def _check(a, b):
    """Every quotient not reported equals IEEE a / b bit for bit, and the
    division reports exactly the operands outside its window."""
    with np.errstate(all="ignore"):
        ref = a / b
    q, bad = _gpu_div(a, b)
    good = bad == 0
    same = _bits(q) == _bits(ref)
    assert same[good].all(), (a[good & ~same][:4], b[good & ~same][:4])
    dom = _in_domain(a, b)
    assert (good == dom).all(), (a[good != dom][:4], b[good != dom][:4])
    return good


@pytest.mark.parametrize("emax", [300, 1000])
def test_random_operands(cuda, emax):
    """4M pairs, significands uniform, exponents uniform in [-emax, emax],
    both signs: with 300 about three quarters inside the window, with 1000
    about a twentieth (the rest reported)."""
    rng = np.random.default_rng(11 + emax)
    n = 4_000_000
    a = rng.uniform(1, 2, n) * np.ldexp(1.0, rng.integers(-emax, emax + 1, n)) * rng.choice([-1.0, 1.0], n)
    b = rng.uniform(1, 2, n) * np.ldexp(1.0, rng.integers(-emax, emax + 1, n)) * rng.choice([-1.0, 1.0], n)
    good = _check(a, b)
    assert good.mean() > (0.6 if emax == 300 else 0.04), good.mean()


def _near(x, rng, k=4):
    """x moved by a random number of ulps in [-k, k]."""
    steps = rng.integers(-k, k + 1, x.size)
    return (_bits(x) + steps).view(np.float64)


def test_hard_operands(cuda):
    """Divisors and dividends with significands of all ones and all zeros
    and a few ulps from them (where the Newton step ends on a tie or one ulp
    off, or the quotient sits next to a rounding tie), quotients within a
    fraction of an ulp of a tie, exact quotients and their neighbours, and
    lognormal values spanning the range of the physics' operands; both
    signs, all inside the window."""
    rng = np.random.default_rng(12)
    n = 1_000_000
    ones = np.nextafter(2.0, 0.0)  # 1.11...1 (binary)
    e = rng.integers(-200, 201, n)
    e2 = rng.integers(-200, 201, n)
    u = rng.uniform(1, 2, n) * np.ldexp(1.0, e2)
    sgn = rng.choice([-1.0, 1.0], n)
    sets = {
        "ones_b": (u, ones * np.ldexp(1.0, e) * sgn),
        "pow2_over_ones": (np.ldexp(1.0, e2) * sgn, ones * np.ldexp(1.0, e)),
        "ones_over_ones": (ones * np.ldexp(1.0, e2), ones * np.ldexp(1.0, e) * sgn),
        "one_minus_ulp": (u * sgn, np.nextafter(1.0, 0.0) * np.ldexp(1.0, e)),
        "near_ones_b": (u, _near(ones * np.ldexp(1.0, e), rng) * sgn),
        "pow2_over_near_ones": (_near(np.ldexp(1.0, e2), rng), _near(ones * np.ldexp(1.0, e), rng)),
        "near_pow2_b": (u * sgn, _near(np.ldexp(1.0, e), rng)),
        "ones_a": (ones * np.ldexp(1.0, e), u * sgn),
        "near_ones_over_near_pow2": (_near(ones * np.ldexp(1.0, e2), rng), _near(np.ldexp(1.0, e), rng)),
    }
    # quotients next to a tie: a = RN(m * b) with m = q0 + ulp(q0)/2 (a
    # midpoint), computed in 80-bit extended precision
    q0 = rng.uniform(1, 2, n)
    b = rng.uniform(1, 2, n) * np.ldexp(1.0, rng.integers(-200, 201, n))
    m = q0.astype(np.longdouble) + np.longdouble(2.0) ** -53
    sets["near_ties"] = ((m * b.astype(np.longdouble)).astype(np.float64), b)
    # exact quotients (26-bit significands multiply exactly) and a few ulps off
    qs = np.round(rng.uniform(1, 2, n) * 2 ** 25) / 2 ** 25
    bs = np.round(rng.uniform(1, 2, n) * 2 ** 25) / 2 ** 25 * np.ldexp(1.0, e)
    sets["exact"] = (qs * bs, bs)
    sets["near_exact"] = (_near(qs * bs, rng, 2), bs)
    # lognormal magnitudes, both signs
    a = np.exp(rng.normal(0, 12, n)) * sgn
    b = np.exp(rng.normal(0, 12, n)) * rng.choice([-1.0, 1.0], n)
    sets["lognormal"] = (a, b)
    for name, (a, b) in sets.items():
        good = _check(a, b)
        assert good.mean() > 0.99, (name, good.mean())


def test_reciprocal(cuda):
    """The reciprocal the kernels take for 1/b and for a divisor shared by
    several quotients (fast_rcp, the first half of fast_div): equal to IEEE
    1 / b bit for bit inside the window 2^-256 <= |b| < 2^256 and reported
    outside it.  Random significands over exponents of +-1000, all-ones and
    power-of-two significands and a few ulps from them, lognormal values, and
    every special value."""
    import torch
    rng = np.random.default_rng(13)
    n = 2_000_000
    ones = np.nextafter(2.0, 0.0)
    e = rng.integers(-300, 301, n)
    sgn = rng.choice([-1.0, 1.0], n)
    b = np.concatenate([
        rng.uniform(1, 2, n) * np.ldexp(1.0, rng.integers(-1000, 1001, n)) * sgn,
        ones * np.ldexp(1.0, e) * sgn,
        _near(ones * np.ldexp(1.0, e), rng) * sgn,
        np.ldexp(1.0, e) * sgn,
        _near(np.ldexp(1.0, e), rng) * sgn,
        np.nextafter(1.0, 0.0) * np.ldexp(1.0, e),
        np.exp(rng.normal(0, 12, n)) * sgn,
        np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, -1e-310, 2.0 ** -256, 2.0 ** 256,
                  np.nextafter(2.0 ** -256, 0.0), np.nextafter(2.0 ** 256, 0.0)]),
    ])
    tb = torch.from_numpy(b).cuda()
    y, bad = cloudsc.reciprocal_check(tb)
    torch.cuda.synchronize()
    y, bad = y.cpu().numpy(), bad.cpu().numpy()
    with np.errstate(all="ignore"):
        ref = 1.0 / b
    good = bad == 0
    assert (good == _in_window(b)).all(), b[good != _in_window(b)][:4]
    same = _bits(y) == _bits(ref)
    assert same[good].all(), b[good & ~same][:4]
    assert good.mean() > 0.75  # a quarter of the first set and 15 % of the next five lie outside
    yz, badz = cloudsc.reciprocal_check(torch.empty(0, dtype=torch.float64, device="cuda"))
    assert yz.numel() == 0 and badz.numel() == 0
    with pytest.raises(cloudsc.CloudscError):
        cloudsc.reciprocal_check(torch.ones(3, device="cuda"))


def test_zero_dividend_keeps_the_sign(cuda):
    """+-0 / b is the zero of sign(a) xor sign(b) for every divisor inside
    the window, all-ones significands included, without a report; divisors
    outside it (zero, subnormal, huge, infinite, NaN) are reported."""
    bs = np.array([1.0, -1.0, 3.5e-70, -2.0e70, np.nextafter(1.0, 0.0), -np.nextafter(2.0, 0.0) * 2.0 ** 100])
    a = np.concatenate([np.zeros(len(bs)), -np.zeros(len(bs))])
    b = np.concatenate([bs, bs])
    q, bad = _gpu_div(a, b)
    assert (bad == 0).all()
    assert (_bits(q) == _bits(a / b)).all()
    out = np.array([0.0, np.nan, 5e-320, 3.5e-300, np.ldexp(1.0, 1023), np.inf, -np.inf])
    q, bad = _gpu_div(np.zeros(len(out)), out)
    assert (bad == 1).all(), bad


def test_special_operands_reported(cuda):
    """Nonzero dividends with a zero, subnormal, infinite or NaN divisor, and
    infinite, NaN, subnormal, tiny or huge dividends: every one is
    reported."""
    spec_b = [0.0, -0.0, 5e-320, -4e-310, np.inf, -np.inf, np.nan, 1e-100, -1e100]
    a = np.array([1.5] * len(spec_b) + [np.inf, -np.inf, np.nan, 5e-320, -1e-310, 1e-80, -1e80])
    b = np.array(spec_b + [2.0, 3.0, 1.0, 1.0, 7.0, 3.0, 3.0])
    q, bad = _gpu_div(a, b)
    assert (bad == 1).all(), bad


def test_empty_and_errors(cuda):
    import torch
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    q, bad = cloudsc.division_check(e, e)
    assert q.numel() == 0 and bad.numel() == 0
    with pytest.raises(cloudsc.CloudscError):
        cloudsc.division_check(torch.ones(3, device="cuda"), torch.ones(3, device="cuda"))


def _pow2_below_pressure(arrs, cols):
    """In each given column of block 2, at every level whose layer holds a
    power of two between 2^10 and 2^16 Pa, the full-level pressure is set to
    the largest double below that power (significand all ones): a pressure
    within the layer that divides the saturation vapour pressure in every
    level's saturation humidity.  Returns the number of levels changed."""
    n = 0
    for jl in cols:
        for m in range(10, 17):
            x = 2.0 ** m
            paph = arrs["paph"][2, :, jl]
            ks = np.nonzero((paph[:-1] < x) & (paph[1:] > x))[0]
            for k in ks:
                arrs["pap"][2, k, jl] = np.nextafter(x, 0.0)
                n += 1
    return n


def test_kernel_all_ones_divisors(cuda):
    """Divisors with all-ones significands in the physics (pressures just
    below a power of two in three columns): the corrected reciprocal keeps
    the FP64 kernel's outputs equal to the oracle's bit for bit."""
    p, po = util.params()
    nproma, nblk = 32, 4
    arrs = inputs.generate(nblk, nproma, p, seed=21)
    assert _pow2_below_pressure(arrs, (3, 17, 30)) >= 15
    ngptot = nproma * nblk
    ref, nw = util.run_oracle(po, arrs, nproma, nblk, ngptot)
    gpu, nwg = util.run_gpu(p, arrs, nproma, nblk, ngptot)
    for n in util.COMPARED:
        assert np.array_equal(util.defined(n, gpu[n]), util.defined(n, ref[n])), n
    assert nwg == nw


@pytest.mark.parametrize("nproma,nblk,cut", [(32, 20, 0), (37, 9, 11)])
def test_kernel_reruns_columns_with_reported_divisions(cuda, nproma, nblk, cut):
    """RTAUMEL = 1e80, the melting time scale and a divisor in the melting
    branch, is outside the fast division's window: every column that melts
    reports it and is run again with IEEE division (reading PLUDE from the
    fast pass's copy, the array itself being already overwritten).  The FP64
    kernel's outputs, PLUDE included, equal the oracle's bit for bit, with a
    ragged last block; the warning count is counted once."""
    p, po = util.params()
    p = util.with_flags(p, {"rtaumel": 1e80})
    po = util.with_flags(po, {"rtaumel": 1e80})
    arrs = inputs.generate(nblk, nproma, p, seed=21)
    ngptot = nproma * nblk - cut
    ref, nw = util.run_oracle(po, arrs, nproma, nblk, ngptot)
    gpu, nwg = util.run_gpu(p, arrs, nproma, nblk, ngptot)
    for n in util.COMPARED:
        a = util.defined(n, util._valid_cols(gpu[n], ngptot, nproma))
        b = util.defined(n, util._valid_cols(ref[n], ngptot, nproma))
        assert np.array_equal(a, b), n
        assert np.isfinite(b).all(), n
    assert nwg == nw


@pytest.mark.parametrize("name,value", [("rtaumel", float(np.nextafter(8192.0, 0.0))),
                                        ("rd", float(np.nextafter(256.0, 0.0))),
                                        ("rdepliqrefdepth", float(np.nextafter(512.0, 0.0)))])
def test_kernel_parameter_divisor_outside_fast_path(cuda, name, value):
    """The kernels divide by five parameters with reciprocals computed on the
    host.  A parameter they cannot take that way (here an all-ones
    significand, near the parameter's physical value) makes every column take
    the IEEE rerun: the FP64 kernel still equals the oracle bit for bit."""
    p, po = util.params()
    p = util.with_flags(p, {name: value})
    po = util.with_flags(po, {name: value})
    nproma, nblk = 32, 6
    arrs = inputs.generate(nblk, nproma, p, seed=29)
    ngptot = nproma * nblk - 5
    ref, nw = util.run_oracle(po, arrs, nproma, nblk, ngptot)
    gpu, nwg = util.run_gpu(p, arrs, nproma, nblk, ngptot)
    for n in util.COMPARED:
        a = util.defined(n, util._valid_cols(gpu[n], ngptot, nproma))
        b = util.defined(n, util._valid_cols(ref[n], ngptot, nproma))
        assert np.array_equal(a, b), n
        assert np.isfinite(b).all(), n
    assert nwg == nw
