"""FP64 kernel against the committed oracle fixture (plibm build):
bit-identical on every defined output of the six fixture columns."""
import numpy as np
import pytest

from openifs_b200 import cloudsc, fields
from tests import util
from tests.test_golden import load

pytestmark = pytest.mark.gpu


def test_gpu_matches_fixture(cuda):
    z, arrs, nproma, nblk, nc = load()
    p = cloudsc.default_params(util.PTSPHY, nc)
    gpu, nw = util.run_gpu(p, arrs, nproma, nblk, nproma * nblk)
    assert nw == int(z["plibm_nwarn"])
    for k in fields.OUTPUT_NAMES:
        a, b = util.defined(k, gpu[k]), util.defined(k, z[f"plibm_{k}"])
        assert np.array_equal(a, b), (k, float(np.abs(a - b).max()))
