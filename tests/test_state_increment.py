"""STATE_INCREMENT (state_increment.F90:9-105) on the CPU: the oracle's
restatement against a numpy statement of the same rule, the C structs'
layout against the ctypes mirrors, and the C ABI's argument checks (which
run before any device work, so no GPU is needed)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from openifs_b200 import cloudsc, params as P
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NP, KLEV, NB = 37, 19, 4


def make(seed, nclv_pa=5):
    rng = np.random.default_rng(seed)
    shp = (NB, KLEV, NP)
    state = {n: rng.standard_normal(shp) for n in ("u", "v", "t", "o3", "q", "a", "tke")}
    state["cld"] = rng.standard_normal((NB, 5, KLEV, NP))
    inc = {n: rng.standard_normal(shp) for n in ("u", "v", "t", "o3", "q", "a", "tke")}
    loc_cld = rng.standard_normal((NB, nclv_pa, KLEV, NP))
    return state, inc, loc_cld


def expected(state, inc, loc_cld, ngptot, kidia, keymask, species=(0, 1, 2, 3)):
    """The reference's rule, written with numpy slices."""
    out = {k: v.copy() for k, v in state.items()}
    gated = {"q": P.KEY_Q, "o3": P.KEY_O3, "a": P.KEY_A, "tke": P.KEY_TKE}
    keys = [P.KEY_QL, P.KEY_QI, P.KEY_QR, P.KEY_QS]
    for ib in range(NB):
        icend = min(NP, ngptot - ib * NP)
        cols = slice(kidia - 1, icend)
        for n in ("u", "v", "t", "q", "o3", "a", "tke"):
            if n in inc and (n not in gated or keymask & gated[n]):
                out[n][ib, :, cols] = out[n][ib, :, cols] + inc[n][ib, :, cols]
        for m in species:
            if keymask & keys[m]:
                out["cld"][ib, m, :, cols] = out["cld"][ib, m, :, cols] + loc_cld[ib, m, :, cols]
    return out


@pytest.mark.parametrize("keymask", [P.KEY_ALL, P.KEY_Q | P.KEY_QL | P.KEY_QS, 0])
@pytest.mark.parametrize("kidia,cut", [(1, 0), (4, 9)])
def test_oracle_matches_the_rule(built, keymask, kidia, cut):
    state, inc, loc_cld = make(3)
    ngptot = NB * NP - cut
    want = expected(state, inc, loc_cld, ngptot, kidia, keymask)
    got = {k: v.copy() for k, v in state.items()}
    oracle.state_increment_batched(got, dict(inc, cld=loc_cld), NP, KLEV, NB, ngptot, kidia, keymask)
    for n in want:
        assert np.array_equal(got[n], want[n]), n


def test_oracle_separate_species_arrays(built):
    """The call after CLOUD_SATADJ (callpar.F90:1278-1280): T, Q, A and the
    liquid and ice increments as arrays of their own."""
    state, inc, loc_cld = make(5)
    got = {k: v.copy() for k, v in state.items()}
    two = {"t": inc["t"], "q": inc["q"], "a": inc["a"], "ql": np.ascontiguousarray(loc_cld[:, 0]),
           "qi": np.ascontiguousarray(loc_cld[:, 1])}
    oracle.state_increment_batched(got, two, NP, KLEV, NB, NB * NP)
    want = expected(state, {k: inc[k] for k in ("t", "q", "a")}, loc_cld, NB * NP, 1, P.KEY_ALL, species=(0, 1))
    for n in want:
        assert np.array_equal(got[n], want[n]), n


def test_struct_layout_matches_header(tmp_path):
    """offsetof/sizeof of cloudsc_state and cloudsc_increments from the C
    compiler against the ctypes mirrors."""
    src = tmp_path / "layout.c"
    fields_s = list(P.STATE_FIELDS) + ["keymask", "nclv"]
    fields_i = ["pa_" + n for n in P.INCREMENT_FIELDS] + ["nclv_pa"]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cloudsc_b200.h"', "int main(void){"]
    lines.append('printf("%zu\\n", sizeof(cloudsc_state));')
    lines += [f'printf("%zu\\n", offsetof(cloudsc_state, {f}));' for f in fields_s]
    lines.append('printf("%zu\\n", sizeof(cloudsc_increments));')
    lines += [f'printf("%zu\\n", offsetof(cloudsc_increments, {f}));' for f in fields_i]
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(P.CloudscState)] + [getattr(P.CloudscState, f).offset for f in fields_s]
    want += [ctypes.sizeof(P.CloudscIncrements)] + [getattr(P.CloudscIncrements, f).offset for f in fields_i]
    assert vals == want


def test_abi_rejects_bad_arguments(built):
    """Checked before any device work: an increment for a field the state
    does not carry (-1), inconsistent shapes (-2)."""
    state, inc, _ = make(7)
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.state_increment_batched({"t": state["t"]}, {"q": inc["q"]}, NP, KLEV, NB, NB * NP)
    assert e.value.code == -1
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.state_increment_batched({"t": state["t"]}, {"t": inc["t"]}, NP, KLEV, NB, NB * NP + 1)
    assert e.value.code == -2
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.state_increment_batched({"t": state["t"]}, {"t": inc["t"]}, NP, KLEV, NB, NB * NP, kidia=NP + 1)
    assert e.value.code == -2
    # a field left out by the keymask needs no destination
    assert cloudsc.state_increment_batched({"t": None}, {"q": inc["q"]}, NP, KLEV, NB, NB * NP, keymask=0) == 0
