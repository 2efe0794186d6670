"""Write tests/golden/cloudsc_l137_6col.npz: a small regression fixture of the
CPU oracle (both libm builds) on a seeded 6-column L137 state.

The reference holds no CLOUDSC-level golden vectors and its Fortran cannot be
compiled here, so this fixture pins the oracle against itself over time: any
change to the restatement, the constants or the input generator that moves
a single bit of a defined output shows up in tests/test_golden.py.  Inputs are
stored too, so the fixture does not depend on the generator.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from openifs_b200 import fields, inputs  # noqa: E402
from oracle import oracle  # noqa: E402

NPROMA, NBLK, SEED, PTSPHY, KLEV = 3, 2, 5, 3600.0, 137
PATH = os.path.join(HERE, "cloudsc_l137_6col.npz")


def make():
    nc = inputs.ncldtop_l137()
    po = oracle.params_default(PTSPHY, nc)
    arrs = inputs.generate(NBLK, NPROMA, po, seed=SEED)
    # column 1 of block 0 is convective (LDCUM, KTYPE 2) as generated; make
    # column 3 of block 1 clear sky: no condensate, no cloud
    arrs["pclv"][1, :4, :, 2] = 0.0
    arrs["pa"][1, :, 2] = 0.0
    out = {f"in_{k}": v for k, v in arrs.items() if k in fields.INPUT_NAMES}
    for libm in ("glibc", "plibm"):
        ref = {k: v.copy() for k, v in arrs.items()}
        nw = oracle.cloudsc_batched(po, ref, NPROMA, KLEV, NBLK, NPROMA * NBLK, PTSPHY, 1, libm=libm)
        for k in fields.OUTPUT_NAMES:
            out[f"{libm}_{k}"] = ref[k]
        out[f"{libm}_nwarn"] = np.array(nw)
    out["meta"] = np.array([NPROMA, NBLK, SEED, KLEV, nc], dtype=np.int64)
    np.savez_compressed(PATH, **out)
    return PATH


if __name__ == "__main__":
    print(make(), os.path.getsize(PATH))
