"""STATE_INCREMENT on the B200 (GPU tests): the batched entry and the
CLOUD_SATADJ kernel with the increment fused in, bit for bit against the
oracle (the separate SATADJ and STATE_INCREMENT restatements)."""
import numpy as np
import pytest

from openifs_b200 import cloudsc, fields, inputs, params as P
from oracle import oracle
from tests import util
from tests.test_state_increment import KLEV, NB, NP, make

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("keymask", [P.KEY_ALL, P.KEY_Q | P.KEY_QR])
@pytest.mark.parametrize("kidia,cut", [(1, 0), (6, 13)])
def test_batched_bit_exact(cuda, keymask, kidia, cut):
    """After CLOUDSC (callpar.F90:1308-1311): T, Q, A and the four condensate
    species of a CLD-shaped tendency; U, V, O3 and TKE as well."""
    import torch
    state, inc, loc_cld = make(11)
    ngptot = NB * NP - cut
    ref = {k: v.copy() for k, v in state.items()}
    oracle.state_increment_batched(ref, dict(inc, cld=loc_cld), NP, KLEV, NB, ngptot, kidia, keymask)
    d = {k: torch.from_numpy(v).cuda() for k, v in state.items()}
    di = {k: torch.from_numpy(v).cuda() for k, v in dict(inc, cld=loc_cld).items()}
    cloudsc.state_increment_batched(d, di, NP, KLEV, NB, ngptot, kidia, keymask)
    torch.cuda.synchronize()
    for n in ref:
        assert np.array_equal(d[n].cpu().numpy(), ref[n]), n


@pytest.mark.parametrize("keymask", [P.KEY_ALL, P.KEY_A | P.KEY_QI])
def test_satadj_with_increment_bit_exact(cuda, keymask):
    """CLOUD_SATADJ + STATE_INCREMENT in one kernel against the oracle's
    SATADJ followed by its STATE_INCREMENT (callpar.F90:1253-1280), ragged
    last block; the tendencies and the updated cumulative tendencies."""
    import torch
    p, po = util.params()
    nproma, nblk = 37, 9
    ngptot = nproma * nblk - 11
    arrs = inputs.generate_satadj(nblk, nproma, p, seed=71)
    ref, nw = util.run_oracle_satadj(po, arrs, nproma, nblk, ngptot)
    st = {"t": ref["tendency_cml_t"], "q": ref["tendency_cml_q"], "a": ref["tendency_cml_a"],
          "cld": np.ascontiguousarray(np.stack([ref["tendency_cml_l"], ref["tendency_cml_i"],
                                                np.zeros_like(ref["tendency_cml_l"]),
                                                np.zeros_like(ref["tendency_cml_l"])], axis=1))}
    incs = {"t": ref["tendency_loc_t"], "q": ref["tendency_loc_q"], "a": ref["tendency_loc_a"],
            "ql": ref["tendency_loc_l"], "qi": ref["tendency_loc_i"]}
    oracle.state_increment_batched(st, incs, nproma, util.KLEV, nblk, ngptot, 1, keymask)
    cloudsc.setup(p)
    d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    cloudsc.satadj_increment_batched(p, d, nproma, util.KLEV, nblk, ngptot, util.PTSPHY, keymask, counter=cnt)
    torch.cuda.synchronize()
    g = {k: v.cpu().numpy() for k, v in d.items()}
    for n in fields.SATADJ_OUTPUTS:
        assert np.array_equal(g[n], ref[n]), n
    for n, r in [("t", st["t"]), ("q", st["q"]), ("a", st["a"]), ("l", st["cld"][:, 0]), ("i", st["cld"][:, 1])]:
        assert np.array_equal(g[f"tendency_cml_{n}"], r), n
    assert int(cnt.item()) == nw
