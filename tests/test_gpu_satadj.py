"""CLOUD_SATADJ on the B200 against the CPU oracle (GPU tests): the batched
device-pointer entry and the per-block host entry, bit for bit with the
oracle built with the kernels' libm."""
import numpy as np
import pytest

from openifs_b200 import cloudsc, fields, inputs
from tests import util

pytestmark = pytest.mark.gpu


def _gpu(p, arrs, nproma, nblk, ngptot):
    import torch
    cloudsc.setup(p)
    d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    cloudsc.satadj_batched(p, d, nproma, util.KLEV, nblk, ngptot, util.PTSPHY, counter=cnt)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in d.items()}, int(cnt.item())


@pytest.mark.parametrize("nproma,nblk,cut", [(32, 100, 0), (37, 9, 11), (128, 3, 1)])
def test_batched_bit_exact(cuda, nproma, nblk, cut):
    p, po = util.params()
    arrs = inputs.generate_satadj(nblk, nproma, p, seed=21 + nproma)
    ngptot = nproma * nblk - cut
    ref, nw = util.run_oracle_satadj(po, arrs, nproma, nblk, ngptot)
    gpu, nwg = _gpu(p, arrs, nproma, nblk, ngptot)
    for n in fields.SATADJ_OUTPUTS:
        assert np.array_equal(gpu[n], ref[n]), n
    assert nw == nwg


def test_config2_sampled_blocks(cuda):
    """The full 262,144-column input (2,048 blocks of 128): 12 sampled blocks
    against the oracle bit for bit; every point closes its water and
    enthalpy budget."""
    import torch
    p, po = util.params()
    nproma, nblk = 128, 2048
    full = inputs.generate_satadj(nblk, nproma, p, seed=2)
    gpu, _ = _gpu(p, full, nproma, nblk, nproma * nblk)
    q, l, i, t = (gpu[f"tendency_loc_{s}"] for s in "qlit")
    assert np.abs(q + l + i).max() <= 1e-12 * np.abs(q).max()
    assert np.abs(t - p.ralvdcp * l - p.ralsdcp * i).max() <= 1e-12 * np.abs(t).max()
    blocks = [0, 1, 177, 512, 1023, 1024, 1500, 1777, 2000, 2045, 2046, 2047]
    sub = {k: np.ascontiguousarray(v[blocks]) for k, v in full.items()}
    ref, _ = util.run_oracle_satadj(po, sub, nproma, len(blocks), nproma * len(blocks))
    for n in fields.SATADJ_OUTPUTS:
        assert np.array_equal(gpu[n][blocks], ref[n]), n
    del full, gpu
    torch.cuda.empty_cache()


def test_block_entry(cuda):
    """cloudsc_b200_satadj_block (host pointers, the reference's argument
    list): columns KIDIA..KFDIA as the oracle, the other columns untouched;
    PLUDELI's unread components 1-2 may hold anything."""
    p, po = util.params()
    nproma = 48
    arrs = inputs.generate_satadj(1, nproma, p, seed=31)
    ref, nw = util.run_oracle_satadj(po, arrs, nproma, 1, nproma)
    blk = {k: np.ascontiguousarray(v[0]) for k, v in arrs.items()}
    for n in fields.SATADJ_OUTPUTS:
        blk[n][:] = 7.0
    blk["pludeli"][:2] = np.nan
    kidia, kfdia = 4, 41
    cloudsc.setup(p)
    cloudsc.satadj_block(p, kidia, kfdia, nproma, util.KLEV, util.PTSPHY, blk)
    cols = slice(kidia - 1, kfdia)
    for n in fields.SATADJ_OUTPUTS:
        assert np.array_equal(blk[n][:, cols], ref[n][0][:, cols]), n
        assert np.all(blk[n][:, :kidia - 1] == 7.0) and np.all(blk[n][:, kfdia:] == 7.0), n


@pytest.mark.parametrize("nproma,nblk,cut", [(32, 40, 0), (128, 6, 17)])
def test_sltend_supersat_bit_exact(cuda, nproma, nblk, cut):
    """SLTEND's supersaturation adjustment on the GPU against the oracle;
    with the diagnostics off the tendencies are the same."""
    import torch
    p, po = util.params()
    arrs = inputs.generate_sltend(nblk, nproma, p, seed=51 + nproma)
    ngptot = nproma * nblk - cut
    ref = util.run_oracle_sltend(po, arrs, nproma, nblk, ngptot)
    cloudsc.setup(p)
    for diag in (True, False):
        d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
        cloudsc.sltend_supersat_batched(p, d, nproma, util.KLEV, nblk, ngptot, util.PTSPHY, diagnostics=diag)
        torch.cuda.synchronize()
        for n in fields.SLTEND_OUTPUTS:
            g = d[n].cpu().numpy()
            if n.startswith("padj") and not diag:
                assert np.all(g == 0.0), n
                continue
            assert np.array_equal(g, ref[n]), (diag, n)
