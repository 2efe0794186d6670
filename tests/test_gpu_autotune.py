"""The launch-schedule autotuner on the B200: every compiled variant gives
bit-identical results, and tune() applies the fastest schedule it timed."""
import numpy as np
import pytest
import torch

from openifs_b200 import autotune, cloudsc, fields, inputs
from tests import util

pytestmark = pytest.mark.gpu


def test_variants_identical_and_tuned(cuda):
    p, _ = util.params()
    cloudsc.setup(p)
    nproma, nblk = 128, 24
    ncol = nproma * nblk - 5
    host = inputs.generate(nblk, nproma, p, seed=77, ngptot=ncol)
    saved = {pr: cloudsc.get_schedule(pr) for pr in (cloudsc.FP64, cloudsc.MIXED)}
    try:
        for prec in (cloudsc.FP64, cloudsc.MIXED):
            for v in range(cloudsc.num_variants()):
                info = cloudsc.variant_info(prec, v)
                assert 0 < info["regs"] <= 255 and info["local_bytes"] >= 0
            outs = []
            for sched in autotune.candidates(prec):
                d = {k: torch.from_numpy(a).cuda() for k, a in host.items()}
                cloudsc.set_schedule(prec, *sched)
                cloudsc.cloudsc_batched(p, d, nproma, util.KLEV, nblk, ncol, util.PTSPHY, precision=prec)
                torch.cuda.synchronize()
                outs.append((sched, {n: d[n].cpu().numpy() for n in fields.OUTPUT_NAMES}))
            ref = outs[0][1]
            for sched, o in outs[1:]:
                for n in fields.OUTPUT_NAMES:
                    a, b = util.defined(n, o[n]), util.defined(n, ref[n])
                    assert np.array_equal(a, b), (prec, sched, n)
            d = {k: torch.from_numpy(a).cuda() for k, a in host.items()}
            plude = d["plude"].clone()
            r = autotune.tune(p, d, nproma, util.KLEV, nblk, ncol, util.PTSPHY, prec, reps=1, cache=None)
            assert torch.equal(d["plude"], plude)  # INOUT restored
            best = min(r["trials"], key=lambda t: t["ms"])
            assert r["best"]["ms"] == best["ms"] > 0
            v, t, c = cloudsc.get_schedule(prec)
            info = cloudsc.variant_info(prec, v)
            assert (info["max_threads"], info["min_ctas"], t, c) == (
                best["max_threads"], best["min_ctas"], best["threads"], best["ctas_per_sm"])
    finally:
        for pr, s in saved.items():
            cloudsc.set_schedule(pr, *s)
