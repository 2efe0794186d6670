"""The single-precision interface (JPRB = REAL(4), the OpenIFS single-precision
build, contrib/fiat/src/parkind/parkind1.F90:41-44) on the B200 (GPU tests).

Exact property: with precision 0 each float input is widened to double, the
FP64 arithmetic runs unchanged and each output is rounded to float, so the
outputs equal the FP64 oracle's on the widened inputs, rounded to float, bit
for bit.  The other forms are checked for their error against the FP64
oracle on the double inputs the float ones were rounded from: the rounding of
the state to float is the single-precision build's own error, reported per
field beside the FP32 arithmetic's."""
import numpy as np
import pytest

from openifs_b200 import cloudsc, fields, inputs
from tests import util

pytestmark = pytest.mark.gpu


def _widened(sp):
    return {k: (v.astype(np.float64) if v.dtype == np.float32 else v.copy()) for k, v in sp.items()}


def _gpu_sp(p, sp, nproma, nblk, ngptot, precision):
    import torch
    cloudsc.setup(p)
    d = {k: torch.from_numpy(v).cuda() for k, v in sp.items()}
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    cloudsc.cloudsc_batched_sp(p, d, nproma, util.KLEV, nblk, ngptot, util.PTSPHY, precision=precision,
                               counter=cnt)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in d.items()}, int(cnt.item())


@pytest.mark.parametrize("nproma,nblk,cut", [(32, 100, 0), (37, 9, 11)])
def test_fp64_form_is_the_oracle_rounded(cuda, nproma, nblk, cut):
    p, po = util.params()
    arrs = inputs.generate(nblk, nproma, p, seed=61)
    sp = fields.to_single(arrs)
    ngptot = nproma * nblk - cut
    ref, nw = util.run_oracle(po, _widened(sp), nproma, nblk, ngptot)
    got, nwg = _gpu_sp(p, sp, nproma, nblk, ngptot, cloudsc.FP64)
    for n in fields.OUTPUT_NAMES:
        a = util.defined(n, util._valid_cols(got[n], ngptot, nproma))
        b = util.defined(n, util._valid_cols(ref[n].astype(np.float32), ngptot, nproma))
        assert np.array_equal(a, b), n
    assert nwg == nw


def test_host_entry_matches_device_entry(cuda):
    """cloudsc_b200_batched_host_sp (pipelined chunks, ragged last chunk and
    block) gives the device entry's bits; columns beyond NGPTOT untouched."""
    p, po = util.params()
    nproma, nblk, ngptot = 64, 7, 7 * 64 - 9
    sp = fields.to_single(inputs.generate(nblk, nproma, p, seed=62))
    dev, _ = _gpu_sp(p, sp, nproma, nblk, ngptot, cloudsc.FP64)
    host = {k: v.copy() for k, v in sp.items()}
    for n in fields.OUTPUT_NAMES:
        if n != "plude":
            host[n][:] = 7.0
    cloudsc.cloudsc_batched_host_sp(p, host, nproma, util.KLEV, nblk, ngptot, util.PTSPHY, chunk_blocks=3)
    for n in fields.OUTPUT_NAMES:
        a = util.defined(n, util._valid_cols(host[n], ngptot, nproma))
        b = util.defined(n, util._valid_cols(dev[n], ngptot, nproma))
        assert np.array_equal(a, b), n
    last = ngptot - (nblk - 1) * nproma
    assert np.all(host["tendency_loc_t"][-1, :, last:] == 7.0)


@pytest.mark.parametrize("precision", [cloudsc.FP64, cloudsc.MIXED])
def test_error_against_fp64_on_double_inputs(cuda, precision):
    """Per-field error of the single-precision interface against the FP64
    oracle on the double inputs (3,200 columns): the float rounding of the
    state moves the tendencies by far less than 1e-2 of their RMS."""
    p, po = util.params()
    arrs = inputs.generate(100, 32, p, seed=1)
    ref, _ = util.run_oracle(po, arrs, 32, 100, 3200)
    got, _ = _gpu_sp(p, fields.to_single(arrs), 32, 100, 3200, precision)
    stats = util.mixed_error_stats(_widened(got), ref)
    for k, v in stats.items():
        print(precision, k, v)
        assert np.isfinite(v["normwise_max"]), k
    for k in util.MIXED_BOUNDED:
        assert stats[k]["rms_ratio"] < 1e-2, (k, stats[k])


def test_rejects_double_arrays(cuda):
    p, _ = util.params()
    import torch
    arrs = inputs.generate(2, 32, p, seed=3)
    d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.cloudsc_batched_sp(p, d, 32, util.KLEV, 2, 64, util.PTSPHY)
    assert e.value.code == -2
