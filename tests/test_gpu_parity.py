"""FP64 GPU kernel vs the CPU oracle on identical seeded inputs.

Bar: max relative error <= 1e-12 on every defined output, with the
denominator floored at FLOOR_REL (1e-6) times the field's largest magnitude
(tests/util.py).  The only expected differences are the last-bit differences
between CUDA's and glibc's exp/pow (<= 2 ulp each), propagated through the
column recurrence.
"""
import numpy as np
import pytest

from openifs_b200 import cloudsc, inputs
from tests import util

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _check(p, po, arrs, nproma, ngpblks, ngptot, tol=TOL):
    ref, nw_ref = util.run_oracle(po, arrs, nproma, ngpblks, ngptot)
    gpu, nw_gpu = util.run_gpu(p, arrs, nproma, ngpblks, ngptot)
    rep, colmax = util.compare(gpu, ref, ngptot=ngptot, nproma=nproma)
    bad = {k: v for k, v in rep.items() if not v <= tol}
    nflip = int((colmax > tol).sum())
    assert not bad, f"fields above {tol}: {bad}; columns above: {nflip}"
    assert nw_gpu == nw_ref
    return rep


def test_config1_3200_columns(cuda):
    """100 NPROMA blocks of 32, L137, PTSPHY 3600 s."""
    p, po = util.params()
    arrs = inputs.generate(100, 32, p, seed=1)
    rep = _check(p, po, arrs, 32, 100, 3200)
    print({k: f"{v:.2e}" for k, v in rep.items()})


def test_partial_last_block_and_odd_nproma(cuda):
    """NPROMA not a multiple of 32 and NGPTOT ending inside the last block."""
    p, po = util.params()
    arrs = inputs.generate(5, 37, p, seed=7)
    _check(p, po, arrs, 37, 5, 4 * 37 + 11)


def test_single_column(cuda):
    p, po = util.params()
    arrs = inputs.generate(3, 1, p, seed=11)
    _check(p, po, arrs, 1, 3, 3)


@pytest.mark.parametrize("case", ["clear", "overcast", "warm", "cold", "no_convection",
                                  "all_convection", "land", "sea", "tiny_condensate"])
def test_edge_columns(cuda, case):
    """Edge-case columns the reference's branches single out."""
    p, po = util.params()
    arrs = inputs.generate(4, 64, p, seed=23)
    cl = arrs["pclv"]
    if case == "clear":
        cl[:] = 0.0
        arrs["pa"][:] = 0.0
        arrs["tendency_cml_cld"][:] = 0.0
    elif case == "overcast":
        arrs["pa"][:] = 1.0
    elif case == "warm":
        arrs["pt"][:] = np.maximum(arrs["pt"], 280.0)
    elif case == "cold":
        arrs["pt"][:] = np.minimum(arrs["pt"], 230.0)
    elif case == "no_convection":
        for n in ("ldcum", "ktype", "plu", "plude", "pludeli", "psnde", "pmfu", "pmfd"):
            arrs[n][:] = 0
    elif case == "all_convection":
        arrs["ldcum"][:] = 1
        arrs["ktype"][:] = np.where(arrs["ktype"] == 0, 2, arrs["ktype"])
    elif case == "land":
        arrs["plsm"][:] = 1.0
    elif case == "sea":
        arrs["plsm"][:] = 0.0
    elif case == "tiny_condensate":
        cl[:, :4] = np.where(cl[:, :4] > 0, 5e-9, 0.0)
    _check(p, po, arrs, 64, 4, 256)


def test_config2_sampled_blocks(cuda):
    """BASELINE config 2 shape (NPROMA 128, 2048 blocks, seed 2): the whole
    262,144-column launch runs on the GPU and a sample of its blocks is
    checked against the oracle."""
    import torch
    p, po = util.params()
    nproma, nblk = 128, 2048
    full = inputs.generate(nblk, nproma, p, seed=2)
    gpu, _ = util.run_gpu(p, full, nproma, nblk, nproma * nblk)
    sample = [0, 1, 517, 1024, 2046, 2047]
    sub = {k: np.ascontiguousarray(v[sample]) for k, v in full.items()}
    ref, _ = util.run_oracle(po, sub, nproma, len(sample), nproma * len(sample))
    gsub = {k: v[sample] for k, v in gpu.items()}
    rep, colmax = util.compare(gsub, ref)
    bad = {k: v for k, v in rep.items() if not v <= TOL}
    assert not bad, bad
    # size-independent property over the whole launch: finite outputs
    for k, v in gpu.items():
        assert np.isfinite(v).all(), k
    del torch
