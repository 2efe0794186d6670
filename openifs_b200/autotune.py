"""Autotuner of the CLOUDSC kernels' launch schedule.

A schedule, per precision (FP64, FP32-mixed or FP32 physics), is

    variant      one of the compiled __launch_bounds__(max_threads, min_ctas)
                 pairs of the kernels, which fixes the registers per thread
                 (cloudsc.variant_info);
    threads      columns per CTA, a multiple of 32 up to the variant's
                 max_threads;
    ctas_per_sm  persistent CTAs per SM (0: one CTA per tile of `threads`
                 columns, the hardware schedules the tiles).

tune() runs every candidate schedule on the caller's own device arrays,
times it with CUDA events on the launching stream, applies the fastest with
cloudsc.set_schedule and records it in a JSON cache keyed by device name,
precision and (NPROMA, KLEV, NGPBLKS).  apply_cached() applies a recorded
schedule without running anything.  The reference has no counterpart: it
runs CLOUDSC on CPU threads, one NPROMA block per call
(ifs-source/arpifs/phys_ec/ec_phys_drv.F90:438).
"""
import json
import os
import statistics

from . import cloudsc

DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "schedules.json")
PREC_NAME = {cloudsc.FP64: "fp64", cloudsc.MIXED: "mixed", cloudsc.PHYS32: "phys32"}


def candidates(precision):
    """Every (variant, threads, ctas_per_sm) the tuner tries: each variant at
    its full CTA size and 64 columns below it, each both non-persistent and
    with min_ctas persistent CTAs per SM."""
    out = []
    for v in range(cloudsc.num_variants()):
        info = cloudsc.variant_info(precision, v)
        mt, mb = info["max_threads"], info["min_ctas"]
        for t in sorted({mt, mt - 64}, reverse=True):
            if t < 32:
                continue
            for ctas in (0, mb):
                out.append((v, t, ctas))
    return out


def key(precision, nproma, klev, ngpblks, device_name):
    return f"{device_name}|{PREC_NAME[precision]}|{nproma}x{klev}x{ngpblks}"


def _device_name():
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def load(cache=DEFAULT_CACHE):
    if cache and os.path.exists(cache):
        with open(cache) as f:
            return json.load(f)
    return {}


def _describe(precision, sched):
    v, t, c = sched
    info = cloudsc.variant_info(precision, v)
    return {"max_threads": info["max_threads"], "min_ctas": info["min_ctas"], "threads": t,
            "ctas_per_sm": c, "regs": info["regs"], "local_bytes": info["local_bytes"]}


def _variant_index(precision, max_threads, min_ctas):
    for v in range(cloudsc.num_variants()):
        info = cloudsc.variant_info(precision, v)
        if info["max_threads"] == max_threads and info["min_ctas"] == min_ctas:
            return v
    return None


def apply_cached(precision, nproma, klev, ngpblks, cache=DEFAULT_CACHE, device_name=None):
    """Apply the recorded schedule for this device and shape; returns its
    cache entry, or None (schedule unchanged) when there is none or its
    variant is not compiled into this library."""
    entry = load(cache).get(key(precision, nproma, klev, ngpblks, device_name or _device_name()))
    if not entry:
        return None
    v = _variant_index(precision, entry["max_threads"], entry["min_ctas"])
    if v is None:
        return None
    cloudsc.set_schedule(precision, v, entry["threads"], entry["ctas_per_sm"])
    return entry


def _event_timer(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision, reps, stream):
    import torch
    inout = {n: arrays[n].clone() for n in ("plude",)}  # PLUDE is INOUT

    def run_once():
        for n, v in inout.items():
            arrays[n].copy_(v)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cloudsc.cloudsc_batched(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy,
                                precision=precision, stream=stream)
        e1.record(stream)
        return e0, e1

    def timer(sched):
        cloudsc.set_schedule(precision, *sched)
        run_once()  # warm-up
        ev = [run_once() for _ in range(reps)]
        torch.cuda.synchronize()
        return statistics.median(a.elapsed_time(b) for a, b in ev)

    def restore():
        for n, v in inout.items():
            arrays[n].copy_(v)
        torch.cuda.synchronize()

    return timer, restore


def tune(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision, reps=3, cache=DEFAULT_CACHE,
         cands=None, timer=None, device_name=None, stream=None, log=None):
    """Time every candidate schedule, apply the fastest, record it in `cache`
    (None: do not record) and return {"best": entry, "trials": [...]}.

    `arrays` are the device arrays of one batched call; PLUDE (INOUT) is
    restored before every run and at the end.  `timer(sched) -> ms` replaces
    the CUDA-event timer (tests)."""
    restore = None
    if timer is None:
        import torch
        stream = stream or torch.cuda.current_stream()
        timer, restore = _event_timer(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision,
                                      reps, stream)
    before = cloudsc.get_schedule(precision)
    trials = []
    try:
        for sched in (cands or candidates(precision)):
            ms = float(timer(sched))
            trials.append(dict(_describe(precision, sched), ms=ms))
            if log:
                log(f"{PREC_NAME[precision]} {trials[-1]}")
    finally:
        cloudsc.set_schedule(precision, *before)
        if restore:
            restore()
    best = min(trials, key=lambda t: t["ms"])
    v = _variant_index(precision, best["max_threads"], best["min_ctas"])
    cloudsc.set_schedule(precision, v, best["threads"], best["ctas_per_sm"])
    entry = dict(best, columns=ngptot)
    if cache:
        data = load(cache)
        data[key(precision, nproma, klev, ngpblks, device_name or _device_name())] = entry
        os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
        with open(cache, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    return {"best": entry, "trials": trials}


def ensure(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision, cache=DEFAULT_CACHE, **kw):
    """The recorded schedule if there is one, else tune now.  Returns
    (entry, "cache" | "tuned")."""
    entry = apply_cached(precision, nproma, klev, ngpblks, cache=cache)
    if entry is not None:
        return entry, "cache"
    r = tune(params, arrays, nproma, klev, ngpblks, ngptot, ptsphy, precision, cache=cache, **kw)
    return r["best"], "tuned"


def main(argv=None):
    """python -m openifs_b200.autotune [--nproma 128 --ngpblks 2048]: tune
    every precision on seeded synthetic inputs of that shape and record the
    schedules in the cache."""
    import argparse
    import torch
    from . import inputs
    ap = argparse.ArgumentParser()
    ap.add_argument("--nproma", type=int, default=128)
    ap.add_argument("--ngpblks", type=int, default=2048)
    ap.add_argument("--ptsphy", type=float, default=3600.0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cache", default=DEFAULT_CACHE)
    a = ap.parse_args(argv)
    p = cloudsc.default_params(a.ptsphy, inputs.ncldtop_l137())
    cloudsc.setup(p)
    klev = inputs.KLEV_L137
    host = inputs.generate(a.ngpblks, a.nproma, p, klev=klev, seed=a.seed)
    d = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    ncol = a.nproma * a.ngpblks
    for prec in (cloudsc.FP64, cloudsc.MIXED, cloudsc.PHYS32):
        r = tune(p, d, a.nproma, klev, a.ngpblks, ncol, a.ptsphy, prec, reps=a.reps, cache=a.cache,
                 log=print)
        print(PREC_NAME[prec], "best", json.dumps(r["best"]))


if __name__ == "__main__":
    main()
