"""cloudsc_b200_block_noalloc, the per-block call that allocates no device
memory (one fixed array inside the library), against the allocating
per-block entry cloudsc_b200_block: bit-identical outputs on two calls in a
row (the second on a different block and column range), the device's free
memory unchanged by a call, and the size limit reported as
CLOUDSC_E_TOO_LARGE before any device work.  This file is
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


@pytest.mark.gpu
def test_noalloc_takes_no_device_memory(cuda):
    """In a thread of its own (no per-thread workspace of the allocating
    entries), a second call of another shape leaves the device's free memory
    exactly where the first call left it: the entry allocates nothing, and its
    fixed array was reserved when the parameters were set up."""
    import threading

    import torch

    p, _ = util.params()
    cloudsc.setup(p)
    got = {}

    def run():
        try:
            for shape, (kidia, kfdia) in [(48, (1, 48)), (96, (3, 90))]:
                blk = _block(inputs.generate(1, shape, p, seed=44 + shape), 0)
                nw = cloudsc.cloudsc_block_noalloc(p, kidia, kfdia, shape, util.KLEV, util.PTSPHY, blk)
                torch.cuda.synchronize()
                got.setdefault("free", []).append(torch.cuda.mem_get_info()[0])
                got.setdefault("nw", []).append(nw)
        except Exception as e:  # reported in the main thread
            got["error"] = e

    t = threading.Thread(target=run)
    t.start()
    t.join()
    assert "error" not in got, got.get("error")
    first, second = got["free"]
    assert second == first, (first, second)
    assert got["nw"][0] >= 0 and got["nw"][1] >= 0


@pytest.mark.gpu
def test_noalloc_first_call_after_setup_takes_no_device_memory(cuda):
    """In a fresh process, the device's free memory right after
    cloudsc_b200_setup equals the free memory after the first no-allocation
    call: set-up has already reserved the fixed array and the column kernels'
    local memory, so a caller may reserve the rest of the GPU for its own
    pool between the two."""
    import os
    import subprocess
    import sys
    script = """
import numpy as np, torch
from openifs_b200 import cloudsc, inputs
from tests import util
torch.cuda.init(); torch.zeros(1, device="cuda"); torch.cuda.synchronize()
p, _ = util.params()
blk = {k: v[0].copy() for k, v in inputs.generate(1, 64, p, seed=45).items()}
cloudsc.setup(p)
torch.cuda.synchronize()
f0 = torch.cuda.mem_get_info()[0]
nw = cloudsc.cloudsc_block_noalloc(p, 1, 64, 64, util.KLEV, util.PTSPHY, blk)
torch.cuda.synchronize()
f1 = torch.cuda.mem_get_info()[0]
print("FREE", f0, f1, nw)
"""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", script], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("FREE")][-1]
    _, f0, f1, nw = line.split()
    assert int(f1) == int(f0), (f0, f1)
    assert int(nw) >= 0


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
