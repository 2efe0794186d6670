"""Train the CLOUDSC surrogate on columns computed by the FP64 GPU kernel and
calibrate its guard.

    python -m openifs_b200.train_surrogate --chunks 8 --steps 40000 --widths 128,64

Each chunk is 262,144 seeded synthetic columns (2,048 NPROMA blocks of 128,
openifs_b200/inputs.py) that cloudsc_b200_batched (FP64) turns into targets.
A held-out chunk (another seed) gives the reported errors and the guard
thresholds: the head-spread, raw-closure and refilled-condensate tolerances are each set
at the `--flag-quantile` quantile of the held-out columns.  The weights, input/output normalisation, thresholds and
the held-out statistics go into one .npz (and a .json beside it).
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np


def _log(msg):
    print(msg, flush=True)


def evaluate(net, params, seed, nblk=2048, nproma=128, flag_quantile=0.99):
    """Held-out errors of the raw network and of the guarded surrogate."""
    import torch
    from . import cloudsc, inputs, surrogate as S
    host = inputs.generate(nblk, nproma, params, seed=seed)
    ref = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    cloudsc.setup(params)
    cloudsc.cloudsc_batched(params, ref, nproma, S.KLEV, nblk, nproma * nblk, 3600.0)
    dev = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    del host
    ncol = nproma * nblk
    plude0 = dev["plude"].clone()
    # calibration pass: nothing flagged, diagnostics only
    run = S.Runner(net, params, nproma, nblk, capacity=nproma, neg_tol=1e30, closure_tol=1e30, spread_tol=1e30)
    b = run.prepare(dev)
    run.run(b)
    torch.cuda.synchronize()
    diag = run.diag.cpu().numpy()
    spread_tol = float(np.quantile(diag[:, 2], flag_quantile))
    closure_tol = float(np.quantile(np.maximum(diag[:, 0], diag[:, 1]), flag_quantile))
    neg_tol = float(np.quantile(diag[:, 3], flag_quantile))
    raw_err = _errors(dev, ref)
    # guarded pass
    del run, b
    torch.cuda.empty_cache()
    dev["plude"].copy_(plude0)  # the first pass wrote PLUDE's output
    cap = int(math.ceil(0.0625 * ncol))
    run = S.Runner(net, params, nproma, nblk, capacity=cap, neg_tol=neg_tol, closure_tol=closure_tol,
                   spread_tol=spread_tol)
    b = run.prepare(dev)
    run.run(b)
    torch.cuda.synchronize()
    nflag = int(b.nflag.item())
    err = _errors(dev, ref)
    return {"columns": ncol, "spread_tol": spread_tol, "closure_tol": closure_tol, "neg_tol": neg_tol,
            "flagged": nflag, "flagged_fraction": nflag / ncol, "capacity": run.cap,
            "errors_unguarded": raw_err, "errors_guarded": err}


def _errors(dev, ref):
    out = {}
    for n in ["tendency_loc_t", "tendency_loc_q", "tendency_loc_a", "tendency_loc_cld", "pfplsl", "pfplsn"]:
        r, g = ref[n], dev[n]
        if n == "tendency_loc_cld":
            for m, s in enumerate("lirs"):
                rr, gg = r[:, m], g[:, m]
                out[f"{n}_{s}"] = float((gg - rr).pow(2).mean().sqrt() / rr.pow(2).mean().sqrt())
            continue
        if n in ("pfplsl", "pfplsn"):
            r, g = r[:, -1], g[:, -1]
        out[n] = float((g - r).pow(2).mean().sqrt() / r.pow(2).mean().sqrt())
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--chunks", type=int, default=8)
    ap.add_argument("--nblk", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=40000)
    ap.add_argument("--nb", type=int, default=512)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--widths", default="128", help="comma-separated, each 64 or 128")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--flag-quantile", type=float, default=0.99)
    ap.add_argument("--outdir", default=None)
    a = ap.parse_args(argv)
    import torch
    from . import cloudsc, surrogate as S
    from .build import build
    build()
    params = cloudsc.default_params()
    t0 = time.time()
    data = S.Dataset(params, a.chunks, nblk=a.nblk, seed0=1000, log=_log)
    norm, scale = data.normalisation()
    data.apply_scale(scale)
    _log(f"dataset: {data.ncol} columns in {time.time() - t0:.1f} s")
    nets = {}
    for width in [int(w) for w in a.widths.split(",")]:
        net = S.Net(width, seed=a.seed)
        net.norm, net.out_scale = norm, scale
        torch.cuda.synchronize()
        t1 = time.time()
        hist = S.train(net, data, a.steps, nb=a.nb, lr=a.lr, log=_log, log_every=1000)
        torch.cuda.synchronize()
        train_s = time.time() - t1
        _log(f"width {width}: {a.steps} steps of {a.nb} columns in {train_s:.1f} s")
        nets[width] = (net, hist, train_s)
    del data
    torch.cuda.empty_cache()
    outdir = a.outdir or os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
    for width, (net, hist, train_s) in nets.items():
        ev = evaluate(net, params, seed=5000, flag_quantile=a.flag_quantile)
        ev.update({"train_columns": int(a.chunks * a.nblk * 128), "steps": a.steps, "batch_columns": a.nb,
                   "train_seconds": train_s, "loss_history": hist, "width": width})
        _log(json.dumps({k: v for k, v in ev.items() if k != "loss_history"}, indent=1))
        out = os.path.join(outdir, f"surrogate_w{width}.npz")
        st = net.state()
        st["guard"] = np.array([ev["neg_tol"], ev["closure_tol"], ev["spread_tol"]])
        np.savez_compressed(out, **st)
        with open(os.path.splitext(out)[0] + ".json", "w") as f:
            json.dump(ev, f, indent=1)
        _log(f"saved {out}")
        torch.cuda.empty_cache()


if __name__ == "__main__":
    sys.exit(main())
