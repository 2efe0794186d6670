"""cloudsc_b200_block_noalloc, the per-block call that allocates no device
memory (one fixed array inside the library), against the allocating
per-block entry cloudsc_b200_block: bit-identical outputs on two calls in a
row (the second on a different block and column range), and the size limit
reported as CLOUDSC_E_TOO_LARGE before any device work.  This file is
collected last so that it also runs after every other GPU test."""
import numpy as np
import pytest

from openifs_b200 import cloudsc, fields, inputs
from tests import util


def _block(arrs, ib):
    return {k: v[ib].copy() for k, v in arrs.items()}


@pytest.mark.gpu
def test_noalloc_matches_block_entry_two_calls(cuda):
    p, _ = util.params()
    nproma = 64
    arrs = inputs.generate(2, nproma, p, seed=43)
    cloudsc.setup(p)
    for ib, (kidia, kfdia) in enumerate([(1, nproma), (5, 40)]):
        ref = _block(arrs, ib)
        out = _block(arrs, ib)
        for n in fields.OUTPUT_NAMES:
            if n != "plude":
                ref[n][:] = 7.0
                out[n][:] = 7.0
        nw_ref = cloudsc.cloudsc_block(p, kidia, kfdia, nproma, util.KLEV, util.PTSPHY, ref)
        nw = cloudsc.cloudsc_block_noalloc(p, kidia, kfdia, nproma, util.KLEV, util.PTSPHY, out)
        assert nw == nw_ref
        for n in fields.OUTPUT_NAMES:
            assert np.array_equal(ref[n], out[n]), (ib, n)


def test_noalloc_rejects_blocks_above_capacity(built):
    p = cloudsc.default_params()
    try:
        cloudsc.setup(p)  # without a GPU the upload fails (-4) but the parameters are kept
    except cloudsc.CloudscError as e:
        assert e.code == -4
    assert cloudsc.block_noalloc_capacity() == 16 << 20
    klon = 289  # one column more than fits at KLEV 137
    blk = {k: v[0] for k, v in fields.alloc(1, klon, util.KLEV).items()}
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.cloudsc_block_noalloc(p, 1, klon, klon, util.KLEV, util.PTSPHY, blk)
    assert e.value.code == -6
    assert "16777216" in str(e.value)
