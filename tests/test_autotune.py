"""The launch-schedule autotuner's host logic (CPU: a fake timer stands in
for the CUDA-event timing; set_schedule only records host state)."""
import json

import pytest

from openifs_b200 import autotune, cloudsc


@pytest.fixture
def restore_schedule():
    saved = {p: cloudsc.get_schedule(p) for p in (cloudsc.FP64, cloudsc.MIXED)}
    yield
    for p, s in saved.items():
        cloudsc.set_schedule(p, *s)


def test_candidates_are_valid(restore_schedule):
    for prec in (cloudsc.FP64, cloudsc.MIXED):
        cands = autotune.candidates(prec)
        assert len(cands) == len(set(cands)) >= cloudsc.num_variants()
        for v, t, c in cands:
            info = cloudsc.variant_info(prec, v)
            assert t % 32 == 0 and 32 <= t <= info["max_threads"]
            assert c in (0, info["min_ctas"])
            cloudsc.set_schedule(prec, v, t, c)
            assert cloudsc.get_schedule(prec) == (v, t, c)


def test_schedule_limits(restore_schedule):
    n = cloudsc.num_variants()
    info = [cloudsc.variant_info(cloudsc.FP64, v) for v in range(n)]
    big = max(range(n), key=lambda v: info[v]["max_threads"])
    with pytest.raises(cloudsc.CloudscError):
        cloudsc.set_schedule(cloudsc.FP64, big, info[big]["max_threads"] + 32, 0)
    with pytest.raises(cloudsc.CloudscError):
        cloudsc.set_schedule(cloudsc.FP64, n, 128, 0)
    with pytest.raises(cloudsc.CloudscError):
        cloudsc.set_schedule(cloudsc.FP64, 0, 100, 0)
    # set_launch: the one-CTA-per-SM variant with the most registers that fits
    cloudsc.set_launch(cloudsc.FP64, 128, 0)
    v, t, c = cloudsc.get_schedule(cloudsc.FP64)
    fits = [u for u in range(n) if info[u]["min_ctas"] == 1 and info[u]["max_threads"] >= 128]
    assert t == 128 and info[v]["max_threads"] == min(info[u]["max_threads"] for u in fits)


def test_tune_picks_fastest_and_caches(tmp_path, restore_schedule):
    cache = str(tmp_path / "sched.json")
    cands = autotune.candidates(cloudsc.FP64)
    target = cands[len(cands) // 2]
    seen = []

    def timer(s):
        seen.append(s)
        return 1.0 if s == target else 2.0 + 0.01 * len(seen)

    before = cloudsc.get_schedule(cloudsc.FP64)
    r = autotune.tune(None, None, 128, 137, 2048, 262144, 3600.0, cloudsc.FP64, cache=cache, timer=timer,
                      device_name="fake")
    assert seen == cands
    assert cloudsc.get_schedule(cloudsc.FP64) == target
    assert r["best"]["ms"] == 1.0 and len(r["trials"]) == len(cands)
    data = json.load(open(cache))
    assert list(data) == ["fake|fp64|128x137x2048"]
    # applying the cached entry restores the tuned schedule
    cloudsc.set_schedule(cloudsc.FP64, *before)
    e = autotune.apply_cached(cloudsc.FP64, 128, 137, 2048, cache=cache, device_name="fake")
    assert e is not None and cloudsc.get_schedule(cloudsc.FP64) == target
    assert autotune.apply_cached(cloudsc.MIXED, 128, 137, 2048, cache=cache, device_name="fake") is None
    assert autotune.apply_cached(cloudsc.FP64, 64, 137, 2048, cache=cache, device_name="fake") is None


def test_tune_restores_schedule_on_error(tmp_path, restore_schedule):
    before = cloudsc.get_schedule(cloudsc.MIXED)

    def timer(s):
        raise RuntimeError("timer failed")

    with pytest.raises(RuntimeError):
        autotune.tune(None, None, 128, 137, 4, 512, 3600.0, cloudsc.MIXED, cache=None, timer=timer,
                      device_name="fake")
    assert cloudsc.get_schedule(cloudsc.MIXED) == before
