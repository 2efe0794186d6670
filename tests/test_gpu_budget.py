"""The cloud budget diagnostics (LCLDBUDC/L/I/T, LCLDBUD_VERTINT;
cloudsc.F90:3832-4110) on the B200 against the oracle: PEXTRA and every
output bit for bit, through the batched entry and the per-block host entry."""
import numpy as np
import pytest

from openifs_b200 import cloudsc, fields, inputs
from tests import util

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flags", util.BUDGET_CASES)
def test_batched_diag_bit_exact(cuda, flags):
    import torch
    p0, po0 = util.params()
    p, po = util.with_flags(p0, flags), util.with_flags(po0, flags)
    nproma, nblk = 64, 5
    ngptot = nproma * nblk - 9
    arrs = inputs.generate(nblk, nproma, p, seed=37)
    diag = inputs.generate_diag(arrs, nproma, fields.budget_fields_needed(p) + 2, seed=37)
    ref, dref, nw = util.run_oracle_diag(po, arrs, diag, nproma, nblk, ngptot)
    try:
        cloudsc.setup(p)
        d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
        g = {k: torch.from_numpy(v).cuda() for k, v in diag.items()}
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        cloudsc.cloudsc_batched_diag(p, d, g, nproma, util.KLEV, nblk, ngptot, util.PTSPHY, counter=cnt)
        torch.cuda.synchronize()
        assert np.array_equal(g["pextra"].cpu().numpy(), dref["pextra"])
        for n in util.COMPARED:
            assert np.array_equal(util.defined(n, d[n].cpu().numpy()), util.defined(n, ref[n])), n
        assert int(cnt.item()) == nw
        # the plain batched entry refuses: it has no PEXTRA
        with pytest.raises(cloudsc.CloudscError):
            cloudsc.cloudsc_batched(p, d, nproma, util.KLEV, nblk, ngptot, util.PTSPHY)
    finally:
        cloudsc.setup(p0)


def test_block_entry_budgets(cuda):
    """cloudsc_b200_block with all budget sections on: PEXTRA(KIDIA:KFDIA,:,:)
    as the oracle, the other columns of PEXTRA untouched."""
    p0, po0 = util.params()
    flags = util.BUDGET_CASES[-1]
    p, po = util.with_flags(p0, flags), util.with_flags(po0, flags)
    nproma = 40
    arrs = inputs.generate(1, nproma, p, seed=41)
    kf = fields.budget_fields_needed(p)
    diag = inputs.generate_diag(arrs, nproma, kf, seed=41)
    ref, dref, _ = util.run_oracle_diag(po, arrs, diag, nproma, 1, nproma)
    blk = {k: np.ascontiguousarray(v[0]) for k, v in arrs.items()}
    blk.update({k: np.ascontiguousarray(v[0]) for k, v in diag.items()})
    kidia, kfdia = 3, 37
    try:
        cloudsc.setup(p)
        cloudsc.cloudsc_block(p, kidia, kfdia, nproma, util.KLEV, util.PTSPHY, blk, kfldx=kf)
    finally:
        cloudsc.setup(p0)
    cols = slice(kidia - 1, kfdia)
    assert np.array_equal(blk["pextra"][..., cols], dref["pextra"][0][..., cols])
    assert np.array_equal(blk["pextra"][..., :kidia - 1], diag["pextra"][0][..., :kidia - 1])
    assert np.array_equal(blk["pextra"][..., kfdia:], diag["pextra"][0][..., kfdia:])
    for n in util.COMPARED:
        g, o = util.defined(n, blk[n][None]), util.defined(n, ref[n])
        assert np.array_equal(g[..., cols], o[..., cols]), n


@pytest.mark.parametrize("case", util.OPT_CASES)
def test_spp_inhomogeneity_batched(cuda, case):
    """SPP perturbations and the cloud-inhomogeneity paths (PFSD) through
    cloudsc_b200_batched_diag, bit for bit with the oracle."""
    import torch
    p0, po0 = util.params()
    p, po = util.opt_params(p0, case), util.opt_params(po0, case)
    nproma, nblk = 64, 5
    ngptot = nproma * nblk - 9
    arrs = inputs.generate(nblk, nproma, p, seed=47)
    diag = inputs.generate_diag(arrs, nproma, fields.budget_fields_needed(p) + 1, seed=47)
    ref, dref, nw = util.run_oracle_diag(po, arrs, diag, nproma, nblk, ngptot)
    try:
        cloudsc.setup(p)
        d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
        g = {k: torch.from_numpy(v).cuda() for k, v in diag.items()}
        cloudsc.cloudsc_batched_diag(p, d, g, nproma, util.KLEV, nblk, ngptot, util.PTSPHY)
        torch.cuda.synchronize()
        for n in util.COMPARED:
            assert np.array_equal(util.defined(n, d[n].cpu().numpy()), util.defined(n, ref[n])), n
        assert np.array_equal(g["pfsd"].cpu().numpy(), dref["pfsd"])
        assert np.array_equal(g["pextra"].cpu().numpy(), dref["pextra"])
        with pytest.raises(cloudsc.CloudscError):  # no PGAW/PGP2DSPP in the plain entry
            cloudsc.cloudsc_batched(p, d, nproma, util.KLEV, nblk, ngptot, util.PTSPHY)
    finally:
        cloudsc.setup(p0)


def test_block_entry_spp_inhomogeneity(cuda):
    """cloudsc_b200_block with SPP, both inhomogeneity paths and the budgets:
    PFSD and every output over KIDIA..KFDIA as the oracle."""
    p0, po0 = util.params()
    p, po = util.opt_params(p0, "all+budgets"), util.opt_params(po0, "all+budgets")
    nproma = 40
    arrs = inputs.generate(1, nproma, p, seed=53)
    kf = fields.budget_fields_needed(p)
    diag = inputs.generate_diag(arrs, nproma, kf, seed=53)
    ref, dref, _ = util.run_oracle_diag(po, arrs, diag, nproma, 1, nproma)
    blk = {k: np.ascontiguousarray(v[0]) for k, v in arrs.items()}
    blk.update({k: np.ascontiguousarray(v[0]) for k, v in diag.items()})
    kidia, kfdia = 2, 39
    try:
        cloudsc.setup(p)
        cloudsc.cloudsc_block(p, kidia, kfdia, nproma, util.KLEV, util.PTSPHY, blk, kfldx=kf)
    finally:
        cloudsc.setup(p0)
    cols = slice(kidia - 1, kfdia)
    assert np.array_equal(blk["pfsd"][..., cols], dref["pfsd"][0][..., cols])
    assert np.array_equal(blk["pextra"][..., cols], dref["pextra"][0][..., cols])
    for n in util.COMPARED:
        g, o = util.defined(n, blk[n][None]), util.defined(n, ref[n])
        assert np.array_equal(g[..., cols], o[..., cols]), n


def test_optional_forms_more_levels_than_the_fast_pass_keeps(cuda):
    """300 levels: the budget, SPP and inhomogeneity form runs its plain
    kernel (no fast pass beyond 256 levels).  Outputs, PFSD and PEXTRA
    bit for bit with the oracle."""
    import torch
    klev = 300
    p0, po0 = util.params(inputs.ncldtop_for(klev))
    p, po = util.opt_params(p0, "all+budgets"), util.opt_params(po0, "all+budgets")
    nproma, nblk = 32, 4
    ngptot = nproma * nblk - 3
    arrs = inputs.generate(nblk, nproma, p, klev=klev, seed=37)
    diag = inputs.generate_diag(arrs, nproma, fields.budget_fields_needed(p) + 1, klev=klev, seed=37)
    ref, dref, nw = util.run_oracle_diag(po, arrs, diag, nproma, nblk, ngptot, klev=klev)
    try:
        cloudsc.setup(p)
        d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
        g = {k: torch.from_numpy(v).cuda() for k, v in diag.items()}
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        cloudsc.cloudsc_batched_diag(p, d, g, nproma, klev, nblk, ngptot, util.PTSPHY, counter=cnt)
        torch.cuda.synchronize()
        for n in util.COMPARED:
            a = util.defined(n, util._valid_cols(d[n].cpu().numpy(), ngptot, nproma))
            b = util.defined(n, util._valid_cols(ref[n], ngptot, nproma))
            assert np.array_equal(a, b), n
        assert np.array_equal(g["pfsd"].cpu().numpy(), dref["pfsd"])
        assert np.array_equal(g["pextra"].cpu().numpy(), dref["pextra"])
        assert int(cnt.item()) == nw
    finally:
        cloudsc.setup(p0)


@pytest.mark.parametrize("case", ["budgets", "spp", "all+budgets"])
def test_optional_forms_rerun_mid_column(cuda, case):
    """Forms 3-5 run the fast pass with its rerun.  Three columns get a
    pressure of 1e80 Pa at levels 60, 90 and 120, outside the fast division's
    window: they report there and run again with IEEE division, the fast pass
    having added PEXTRA's terms of the levels above.  Every output, PFSD and
    PEXTRA equal the oracle's bit for bit, and the warning count is counted
    once."""
    import torch
    p0, po0 = util.params()
    if case == "budgets":
        p, po = util.with_flags(p0, util.BUDGET_CASES[-1]), util.with_flags(po0, util.BUDGET_CASES[-1])
    else:
        p, po = util.opt_params(p0, case), util.opt_params(po0, case)
    nproma, nblk = 32, 6
    ngptot = nproma * nblk - 3
    arrs = util.with_out_of_window_pressure(inputs.generate(nblk, nproma, p, seed=43))
    diag = inputs.generate_diag(arrs, nproma, fields.budget_fields_needed(p) + 1, seed=43)
    ref, dref, nw = util.run_oracle_diag(po, arrs, diag, nproma, nblk, ngptot)
    try:
        cloudsc.setup(p)
        d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
        g = {k: torch.from_numpy(v).cuda() for k, v in diag.items()}
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        cloudsc.cloudsc_batched_diag(p, d, g, nproma, util.KLEV, nblk, ngptot, util.PTSPHY, counter=cnt)
        torch.cuda.synchronize()
        for n in util.COMPARED:
            a = util.defined(n, util._valid_cols(d[n].cpu().numpy(), ngptot, nproma))
            b = util.defined(n, util._valid_cols(ref[n], ngptot, nproma))
            assert np.array_equal(a, b), n
            assert np.isfinite(b).all(), n
        assert np.array_equal(g["pfsd"].cpu().numpy(), dref["pfsd"])
        assert np.array_equal(g["pextra"].cpu().numpy(), dref["pextra"])
        assert int(cnt.item()) == nw
    finally:
        cloudsc.setup(p0)
