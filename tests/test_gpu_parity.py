"""B200 kernels vs the CPU oracle on identical seeded inputs (GPU tests).

Strict parity (FP64 kernel vs the oracle built with the kernels' libm,
plibm.h): max relative error <= 1e-12 on every defined output -- in practice
the outputs are bit-identical.  Relative error: |gpu - ref| /
max(|ref|, 1e-6 * max|ref over the field|) (tests/util.py).

Cross-libm (FP64 kernel vs the oracle linked against glibc, i.e. the
reference as a gfortran/Linux build runs it): CLOUDSC's sort and MIN()
limiters make its outputs sensitive to the last bit of EXP/**, so where glibc
rounds a call differently some columns take another branch.  The bounds
asserted are the measured ones of tests/test_cross_libm.py: the largest
relative error and the number of branch-flip columns (any element beyond
1e-12), on 3,200 columns and on every 8th block of the 262,144-column launch.
"""
import numpy as np
import pytest

from openifs_b200 import cloudsc, inputs
from tests import util

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _check(p, po, arrs, nproma, ngpblks, ngptot, tol=TOL):
    ref, nw_ref = util.run_oracle(po, arrs, nproma, ngpblks, ngptot, libm="plibm")
    gpu, nw_gpu = util.run_gpu(p, arrs, nproma, ngpblks, ngptot)
    rep, colmax = util.compare(gpu, ref, ngptot=ngptot, nproma=nproma)
    bad = {k: v for k, v in rep.items() if not v <= tol}
    nflip = int((colmax > tol).sum())
    assert not bad, f"fields above {tol}: {bad}; columns above: {nflip}"
    assert nw_gpu == nw_ref
    return rep, gpu, ref


def test_config1_3200_columns(cuda):
    """Config 1 of the metric: 100 NPROMA blocks of 32, L137, PTSPHY 3600 s."""
    p, po = util.params()
    arrs = inputs.generate(100, 32, p, seed=1)
    rep, gpu, ref = _check(p, po, arrs, 32, 100, 3200)
    exact = sum(int(np.array_equal(util.defined(n, gpu[n]), util.defined(n, ref[n]))) for n in rep)
    print(f"bit-identical fields: {exact}/{len(rep)}")


def test_cross_libm_config1(cuda):
    """GPU vs the glibc oracle on 3,200 columns: max error and flip count."""
    from tests import test_cross_libm as X
    p, po = util.params()
    arrs = inputs.generate(100, 32, p, seed=1)
    gpu, nw = util.run_gpu(p, arrs, 32, 100, 3200)
    ref_g, nw_g = util.run_oracle(po, arrs, 32, 100, 3200, libm="glibc")
    worst, flips, ncol = X.spread(gpu, ref_g)
    print(f"GPU vs glibc oracle, 3,200 columns: max {worst:.3e}, flip columns {flips} of {ncol}")
    assert worst <= X.CONFIG1_MAX and flips <= X.CONFIG1_FLIPS, (worst, flips)
    assert nw == nw_g


def test_cross_libm_config2_sample(cuda):
    """The whole 262,144-column launch on the GPU; every 8th block against
    the glibc oracle: max error and flip count."""
    import torch
    from tests import test_cross_libm as X
    p, po, full, sub = X.config2_sample()
    cloudsc.setup(p)
    dev = {k: torch.from_numpy(v).to("cuda:0") for k, v in full.items()}
    cloudsc.cloudsc_batched(p, dev, 128, util.KLEV, 2048, 2048 * 128, util.PTSPHY)
    torch.cuda.synchronize()
    idx = torch.tensor(X.SAMPLE_BLOCKS, device="cuda:0")
    gsub = {k: v.index_select(0, idx).cpu().numpy() for k, v in dev.items()}
    del dev
    n = len(X.SAMPLE_BLOCKS)
    ref_g, _ = util.run_oracle(po, sub, 128, n, 128 * n, libm="glibc")
    worst, flips, ncol = X.spread(gsub, ref_g)
    print(f"GPU vs glibc oracle, {ncol} sampled columns: max {worst:.3e}, flip columns {flips}")
    assert worst <= X.SAMPLE_MAX and flips <= X.SAMPLE_FLIPS, (worst, flips)


@pytest.mark.parametrize("klev", [60, 91])
def test_other_vertical_grids(cuda, klev):
    """60 and 91 levels (NCLDTOP from their own standard atmosphere), odd
    NPROMA, ragged last block: bit-exact against the oracle."""
    p, po = util.params(inputs.ncldtop_for(klev))
    nproma, nblk = 48, 9
    ngptot = nproma * nblk - 11
    arrs = inputs.generate(nblk, nproma, p, klev=klev, seed=29)
    ref, nw_ref = util.run_oracle(po, arrs, nproma, nblk, ngptot, klev=klev)
    gpu, nw_gpu = util.run_gpu(p, arrs, nproma, nblk, ngptot, klev=klev)
    for n in util.COMPARED:
        a = util.defined(n, util._valid_cols(gpu[n], ngptot, nproma))
        b = util.defined(n, util._valid_cols(ref[n], ngptot, nproma))
        assert np.array_equal(a, b), (klev, n)
    assert nw_gpu == nw_ref


def test_more_levels_than_the_fast_pass_keeps(cuda):
    """300 levels, above the 256 whose PLUDE inputs the fast pass keeps: the
    plain (448, 1) kernels run (at most 448 columns per CTA, whatever the
    schedule says).  FP64 bit-exact against the oracle with a ragged last
    block; the FP32-mixed form runs and stays close to it."""
    klev = 300
    p, po = util.params(inputs.ncldtop_for(klev))
    nproma, nblk = 32, 5
    ngptot = nproma * nblk - 7
    arrs = inputs.generate(nblk, nproma, p, klev=klev, seed=31)
    ref, nw_ref = util.run_oracle(po, arrs, nproma, nblk, ngptot, klev=klev)
    before = cloudsc.get_schedule(cloudsc.FP64)
    try:
        cloudsc.set_schedule(cloudsc.FP64, 0, 640, 0)  # clamped to 448 beyond the fast pass's levels
        gpu, nw_gpu = util.run_gpu(p, arrs, nproma, nblk, ngptot, klev=klev)
    finally:
        cloudsc.set_schedule(cloudsc.FP64, *before)
    for n in util.COMPARED:
        a = util.defined(n, util._valid_cols(gpu[n], ngptot, nproma))
        b = util.defined(n, util._valid_cols(ref[n], ngptot, nproma))
        assert np.array_equal(a, b), n
    assert nw_gpu == nw_ref
    mixed, _ = util.run_gpu(p, arrs, nproma, nblk, ngptot, precision=cloudsc.MIXED, klev=klev)
    t, tm = ref["tendency_loc_t"], mixed["tendency_loc_t"]
    assert np.isfinite(tm).all()
    assert np.sqrt(np.mean((tm - t) ** 2)) <= 1e-3 * np.sqrt(np.mean(t ** 2))


def test_partial_last_block_and_odd_nproma(cuda):
    """NPROMA not a multiple of 32 and NGPTOT ending inside the last block."""
    p, po = util.params()
    arrs = inputs.generate(5, 37, p, seed=7)
    _check(p, po, arrs, 37, 5, 4 * 37 + 11)


def test_single_column(cuda):
    p, po = util.params()
    arrs = inputs.generate(3, 1, p, seed=11)
    _check(p, po, arrs, 1, 3, 3)


@pytest.mark.parametrize("case", util.EDGE_CASES)
def test_edge_columns(cuda, case):
    """Edge-case columns the reference's branches single out."""
    p, po = util.params()
    arrs = inputs.generate(4, 64, p, seed=23)
    util.apply_case(arrs, case)
    _check(p, po, arrs, 64, 4, 256)


@pytest.mark.parametrize("threads", [32, 96, 128, 448])
def test_launch_shapes(cuda, threads):
    """CTA shapes that split, match and span NPROMA blocks (tiles cross block
    boundaries), with a persistent grid, give identical results."""
    p, po = util.params()
    arrs = inputs.generate(6, 128, p, seed=31)
    try:
        cloudsc.set_launch(cloudsc.FP64, threads, 1)
        _check(p, po, arrs, 128, 6, 6 * 128 - 3)
    finally:
        cloudsc.set_launch(cloudsc.FP64, 448, 0)


def test_config2_sampled_blocks(cuda):
    """Config 2 of the metric (NPROMA 128, 2048 blocks, seed 2): the whole
    262,144-column launch runs on the GPU and a sample of its blocks is
    checked against the oracle; size-independent property on all of it:
    finite outputs."""
    import torch
    p, po = util.params()
    nproma, nblk = 128, 2048
    full = inputs.generate(nblk, nproma, p, seed=2)
    cloudsc.setup(p)
    dev = {k: torch.from_numpy(v).to("cuda:0") for k, v in full.items()}
    cloudsc.cloudsc_batched(p, dev, nproma, util.KLEV, nblk, nproma * nblk, util.PTSPHY)
    torch.cuda.synchronize()
    for k, v in dev.items():
        assert bool(torch.isfinite(v.double()).all()), k
    sample = [0, 1, 517, 1024, 2046, 2047]
    idx = torch.tensor(sample, device="cuda:0")
    gsub = {k: v.index_select(0, idx).cpu().numpy() for k, v in dev.items()}
    del dev
    sub = {k: np.ascontiguousarray(v[sample]) for k, v in full.items()}
    ref, _ = util.run_oracle(po, sub, nproma, len(sample), nproma * len(sample), libm="plibm")
    rep, _ = util.compare(gsub, ref)
    bad = {k: v for k, v in rep.items() if not v <= TOL}
    assert not bad, bad


def _poison_unread(a, ax):
    sl = (slice(None),) * ax
    a["tendency_cml_cld"][sl + (4,)] = np.nan
    a["pclv"][sl + (4,)] = np.nan
    a["pludeli"][sl + (slice(2, 4),)] = np.nan


def test_host_pointer_paths(cuda):
    """cloudsc_b200_batched_host (pipelined chunks, partial last chunk and
    block) and the per-block drop-in cloudsc_b200_block give the same results
    as the oracle; the block entry leaves columns outside KIDIA..KFDIA alone.
    The input rows the scheme never reads (the vapour species of
    PTENDENCY_CML_CLD and PCLV, PLUDELI's third and fourth components) are
    NaN on the host: they are not copied to the device."""
    p, po = util.params()
    nproma, nblk, ngptot = 64, 7, 7 * 64 - 9
    arrs = inputs.generate(nblk, nproma, p, seed=41)
    ref, _ = util.run_oracle(po, arrs, nproma, nblk, ngptot, libm="plibm")
    cloudsc.setup(p)
    host = {k: v.copy() for k, v in arrs.items()}
    for n in util.fields.OUTPUT_NAMES:
        if n != "plude":
            host[n][:] = 7.0  # sentinel: untouched padding must survive
    _poison_unread(host, 1)
    cloudsc.cloudsc_batched_host(p, host, nproma, util.KLEV, nblk, ngptot, util.PTSPHY,
                                 chunk_blocks=3)
    rep, _ = util.compare(host, ref, ngptot=ngptot, nproma=nproma)
    assert max(rep.values()) <= TOL, rep
    last = ngptot - (nblk - 1) * nproma
    assert np.all(host["tendency_loc_t"][-1, :, last:] == 7.0)
    # PTENDENCY_LOC_CLD(:,:,NCLV) is never written
    assert np.all(host["tendency_loc_cld"][:, 4] == 7.0)

    # per-block drop-in on block 2, columns 5..40 only (copies: PLUDE is INOUT)
    ib, kidia, kfdia = 2, 5, 40
    one = {k: v[ib:ib + 1].copy() for k, v in arrs.items()}
    blk = {k: v[ib].copy() for k, v in arrs.items()}
    for n in util.fields.OUTPUT_NAMES:
        if n != "plude":
            blk[n][:] = 7.0
    _poison_unread(blk, 0)
    cloudsc.cloudsc_block(p, kidia, kfdia, nproma, util.KLEV, util.PTSPHY, blk)
    # oracle over the whole block; columns are independent, so compare the range
    ref1, _ = util.run_oracle(po, one, nproma, 1, nproma, libm="plibm")
    cols = slice(kidia - 1, kfdia)
    for n in util.fields.OUTPUT_NAMES:
        g, o = util.defined(n, blk[n][None]), util.defined(n, ref1[n])
        assert np.array_equal(g[..., cols], o[..., cols]), n
        if n != "plude":
            assert np.all(g[..., :kidia - 1] == 7.0) and np.all(g[..., kfdia:] == 7.0), n
    assert np.all(blk["tendency_loc_cld"][4] == 7.0)


def _assert_mixed(stats):
    for k, v in stats.items():
        print(k, v)
        assert np.isfinite(v["normwise_max"]) and np.isfinite(v["rms_ratio"]), k
    for k in util.MIXED_BOUNDED:
        assert stats[k]["rms_ratio"] <= util.MIXED_RMS_TOL, (k, stats[k])
        assert stats[k]["normwise_max"] <= util.MIXED_MAX_TOL, (k, stats[k])


def test_mixed_precision_error(cuda):
    """FP32-mixed kernel vs the FP64 oracle on 3,200 columns: per-field
    normwise max error (max |err| / max |ref|) and RMS error ratio of the
    five species tendencies (liquid, ice, rain, snow; vapour = LOC_Q), the
    T tendency and the surface rain and snow fluxes, each within the bounds
    of tests/util.py."""
    p, po = util.params()
    arrs = inputs.generate(100, 32, p, seed=1)
    ref, _ = util.run_oracle(po, arrs, 32, 100, 3200, libm="plibm")
    gpu, _ = util.run_gpu(p, arrs, 32, 100, 3200, precision=cloudsc.MIXED)
    _assert_mixed(util.mixed_error_stats(gpu, ref))


def test_mixed_precision_error_config3_sample(cuda):
    """The FP32-mixed kernel over the whole 262,144-column workload, every
    8th block against the FP64 oracle: the same per-field bounds."""
    import torch
    from tests import test_cross_libm as X
    p, po, full, sub = X.config2_sample()
    cloudsc.setup(p)
    dev = {k: torch.from_numpy(v).to("cuda:0") for k, v in full.items()}
    cloudsc.cloudsc_batched(p, dev, 128, util.KLEV, 2048, 2048 * 128, util.PTSPHY, precision=cloudsc.MIXED)
    torch.cuda.synchronize()
    idx = torch.tensor(X.SAMPLE_BLOCKS, device="cuda:0")
    gsub = {k: v.index_select(0, idx).cpu().numpy() for k, v in dev.items()}
    del dev
    n = len(X.SAMPLE_BLOCKS)
    ref, _ = util.run_oracle(po, sub, 128, n, 128 * n, libm="plibm")
    _assert_mixed(util.mixed_error_stats(gsub, ref))


def test_phys32_form(cuda):
    """FP32-physics kernel (FP32 process rates; state, solve, saturation
    adjustment and budgets in FP64) vs the FP64 oracle: finite everywhere,
    RMS errors of the T and q tendencies and of the surface fluxes bounded
    (threshold flips make it far less accurate than the FP32-mixed form)."""
    p, po = util.params()
    arrs = inputs.generate(100, 32, p, seed=1)
    ref, _ = util.run_oracle(po, arrs, 32, 100, 3200, libm="plibm")
    gpu, _ = util.run_gpu(p, arrs, 32, 100, 3200, precision=cloudsc.PHYS32)
    stats = util.mixed_error_stats(gpu, ref)
    for k, v in stats.items():
        print(k, v)
        assert np.isfinite(v["normwise_max"]), k
    for k in ("tendency_loc_t", "tendency_loc_q"):
        assert stats[k]["rms_ratio"] < 0.1, (k, stats[k])


@pytest.mark.parametrize("name,value", [("rcl_x2r", 2.0), ("rcl_lam2s", 0.5)])
def test_direct_parameter_exponent(cuda, name, value):
    """A parameter used as a pow exponent set to one of 0.5, 1.5, 2 and 3:
    the host then launches the kernels that keep plibm's tests for those
    exponents (sqrt and products instead of exp(y ln x)), still bit-identical
    to the oracle; setting the default back returns to the faster kernels."""
    p, po = util.params()
    q, qo = util.with_flags(p, {name: value}), util.with_flags(po, {name: value})
    arrs = inputs.generate(6, 64, p, seed=83)
    try:
        _check(q, qo, arrs, 64, 6, 6 * 64 - 5)
    finally:
        cloudsc.setup(p)
    _check(p, po, arrs, 64, 6, 6 * 64 - 5)
