"""The per-block drop-in called from many host threads at once, as
EC_PHYS_DRV's OpenMP loop calls CLOUDSC (ec_phys_drv.F90:430-442,
SCHEDULE(DYNAMIC,1)): every thread takes the next block and calls
cloudsc_b200_block on it.  ctypes releases the GIL for the call, so the calls
overlap inside the library (per-thread workspace and stream).  Every block's
outputs must be bit-identical to the oracle's, and the warning counts must
add up to the oracle's total."""
import itertools
import threading

import numpy as np
import pytest

from openifs_b200 import cloudsc, inputs
from tests import util

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nthreads", [4, 16])
def test_block_entry_from_concurrent_threads(cuda, nthreads):
    p, po = util.params()
    nproma, nblk = 96, 48
    ngptot = nblk * nproma - 13  # ragged last block: KFDIA < KLON there
    arrs = inputs.generate(nblk, nproma, p, seed=77 + nthreads)
    ref, nw_ref = util.run_oracle(po, arrs, nproma, nblk, ngptot, libm="plibm")
    cloudsc.setup(p)

    blocks = [{k: v[ib].copy() for k, v in arrs.items()} for ib in range(nblk)]
    counter = itertools.count()
    warn = [0] * nblk
    errors = []

    def worker():
        try:
            while True:
                ib = next(counter)
                if ib >= nblk:
                    return
                kfdia = min(nproma, ngptot - ib * nproma)
                warn[ib] = cloudsc.cloudsc_block(p, 1, kfdia, nproma, util.KLEV, util.PTSPHY, blocks[ib])
        except Exception as e:  # reported on the main thread
            errors.append(repr(e))

    threads = [threading.Thread(target=worker) for _ in range(nthreads)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not any(t.is_alive() for t in threads), "a worker did not finish"
    assert not errors, errors

    last = ngptot - (nblk - 1) * nproma
    for ib in range(nblk):
        cols = slice(0, nproma if ib < nblk - 1 else last)
        for n in util.fields.OUTPUT_NAMES:
            g = util.defined(n, blocks[ib][n][None])[..., cols]
            o = util.defined(n, ref[n][ib:ib + 1])[..., cols]
            assert np.array_equal(g, o), (ib, n)
    assert sum(warn) == nw_ref
