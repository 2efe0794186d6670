"""The CPU oracle against the committed regression fixture
(tests/golden/cloudsc_l137_6col.npz, made by tests/golden/make_golden.py):
bit-identical outputs for both libm builds, six L137 columns including a
convective and a clear-sky column.  The GPU FP64 kernel against the same
fixture is in tests/test_gpu_golden.py."""
import os

import numpy as np

from openifs_b200 import fields
from oracle import oracle
from tests import util

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cloudsc_l137_6col.npz")


def load():
    z = np.load(PATH)
    nproma, nblk, seed, klev, nc = (int(x) for x in z["meta"])
    arrs = fields.alloc(nblk, nproma, klev)
    for k in fields.INPUT_NAMES:
        arrs[k][...] = z[f"in_{k}"]
    return z, arrs, nproma, nblk, nc


def test_fixture_shape():
    z, arrs, nproma, nblk, nc = load()
    assert (nproma, nblk) == (3, 2)
    assert int(arrs["ldcum"].sum()) >= 1
    assert np.all(arrs["pclv"][1, :4, :, 2] == 0.0)


def test_oracle_matches_fixture_glibc_and_plibm():
    z, arrs, nproma, nblk, nc = load()
    po = oracle.params_default(util.PTSPHY, nc)
    for libm in ("glibc", "plibm"):
        ref = {k: v.copy() for k, v in arrs.items()}
        nw = oracle.cloudsc_batched(po, ref, nproma, util.KLEV, nblk, nproma * nblk, util.PTSPHY, 1,
                                    libm=libm)
        assert nw == int(z[f"{libm}_nwarn"])
        for k in fields.OUTPUT_NAMES:
            a, b = util.defined(k, ref[k]), util.defined(k, z[f"{libm}_{k}"])
            assert np.array_equal(a, b), (libm, k, float(np.abs(a - b).max()))
