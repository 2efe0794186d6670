"""Shared helpers for the parity tests: run the oracle and the GPU on the same
inputs and compare every defined output."""
import numpy as np

from openifs_b200 import cloudsc, fields, inputs
from oracle import oracle

KLEV = 137
PTSPHY = 3600.0

# Outputs compared.  PTENDENCY_LOC_CLD(:,:,NCLV) is left undefined by the
# reference (cloudsc.F90:971 loops to NCLV-1) and is excluded by slicing.
COMPARED = [n for n in fields.OUTPUT_NAMES]

# Relative-error denominator floor: an element's error is
# |gpu - ref| / max(|ref|, FLOOR_REL * max|ref over the field|).
FLOOR_REL = 1e-6


def params(ncldtop=None):
    nc = inputs.ncldtop_l137() if ncldtop is None else ncldtop
    return cloudsc.default_params(PTSPHY, nc), oracle.params_default(PTSPHY, nc)


def defined(name, a):
    if name == "tendency_loc_cld":
        return a[:, :4]
    return a


def rel_err(g, o):
    g = np.asarray(g, dtype=np.float64)
    o = np.asarray(o, dtype=np.float64)
    scale = np.max(np.abs(o)) if o.size else 0.0
    denom = np.maximum(np.abs(o), FLOOR_REL * scale)
    with np.errstate(invalid="ignore", divide="ignore"):
        e = np.where(denom > 0, np.abs(g - o) / denom, np.where(g == o, 0.0, np.inf))
    return e


def compare(gpu, ref, names=COMPARED, ngptot=None, nproma=None):
    """Per-field max relative error, plus the column-wise maximum used to
    count branch-flip columns."""
    report = {}
    colmax = None
    for n in names:
        g, o = defined(n, gpu[n]), defined(n, ref[n])
        if ngptot is not None:
            g = _valid_cols(g, ngptot, nproma)
            o = _valid_cols(o, ngptot, nproma)
        e = rel_err(g, o)
        report[n] = float(e.max()) if e.size else 0.0
        c = e.reshape(e.shape[0], -1, e.shape[-1]).max(axis=1)  # (blocks, columns)
        colmax = c if colmax is None else np.maximum(colmax, c)
    return report, colmax


def _valid_cols(a, ngptot, nproma):
    nb = a.shape[0]
    last = ngptot - (nb - 1) * nproma
    if last == nproma:
        return a
    a = a.copy()
    a[-1, ..., last:] = 0.0
    return a


def run_oracle(po, arrs, nproma, ngpblks, ngptot, nthreads=0):
    ref = {k: v.copy() for k, v in arrs.items()}
    nwarn = oracle.cloudsc_batched(po, ref, nproma, KLEV, ngpblks, ngptot, PTSPHY, nthreads)
    return ref, nwarn


def run_gpu(p, arrs, nproma, ngpblks, ngptot, precision=cloudsc.FP64, device="cuda:0"):
    import torch
    cloudsc.setup(p)
    dev = {k: torch.from_numpy(v).to(device) for k, v in arrs.items()}
    cnt = torch.zeros(1, dtype=torch.int32, device=device)
    cloudsc.cloudsc_batched(p, dev, nproma, KLEV, ngpblks, ngptot, PTSPHY, precision=precision,
                            counter=cnt)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in dev.items()}
    return out, int(cnt.item())
