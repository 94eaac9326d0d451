"""Measured choice of launch parameters, remembered on disk.

sumpy tunes nothing at run time (its work-group sizes follow fixed rules,
e.g. ``min(256, max_ntargets_in_one_box)`` at ``sumpy/p2p.py:727``). Here the
schedule of an evaluation has knobs whose best values depend on the workload
(:attr:`SumpyExpansionWrangler.SCHEDULE_KNOBS`):

* ``m2l_item_groups``: M2L class groups per work item (one CTA): small items
  balance the 148 SMs better, large ones keep a tile's accumulators longer;
* ``item_rounds``: source boxes (List 3) or 32-source batches (List 4) per
  work item of the one-launch M2P / P2L;
* ``octant_split``: how many times the per-level M2M / L2L octant GEMMs are
  cut to cover the SMs (items and K parts);
* ``chain_levels``: those GEMMs as one persistent level-chained launch or one
  launch per level;
* ``concurrent_stages``: the independent stages on a second stream or not.

The tile shapes of the kernels are fixed by their instruction shapes (the
tensor-core M2L tile is the MMA's N = 128 target boxes by M = 128
coefficient rows, K streamed in 128-byte rows, 64 f16 or 32 TF32 values at a
time; smaller K steps and a TMA gather
loader were measured slower) and are not searched.

:func:`tune` times each candidate of one knob with CUDA events on the
current stream; :func:`tune_schedule` searches all knobs by coordinate
descent; both keep the best per workload key in a JSON file
(``$SUMPY_B200_AUTOTUNE_CACHE``, default ``~/.cache/sumpy_b200/autotune.json``).
"""
from __future__ import annotations

import json
import math
import os
import threading
from pathlib import Path

import torch

_lock = threading.Lock()


def cache_path(path=None) -> Path:
    if path is not None:
        return Path(path)
    env = os.environ.get("SUMPY_B200_AUTOTUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "sumpy_b200" / "autotune.json"


def _load(path):
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(path, data):
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(path.suffix + f".{os.getpid()}.tmp")
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def time_ms(fn, warmup=1, reps=3):
    """Median CUDA-event time of ``fn()`` on the current stream, in ms."""
    for _ in range(warmup):
        fn()
    times = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    times.sort()
    return times[len(times) // 2]


def tune(key, candidates, measure, path=None, refresh=False):
    """Return the candidate with the smallest ``measure(candidate)`` (ms),
    from the cache when ``key`` was tuned before. ``key`` is a string that
    names the device and the workload class."""
    p = cache_path(path)
    with _lock:
        data = _load(p)
        hit = data.get(key)
        if hit is not None and not refresh and hit.get("best") in list(candidates):
            return hit["best"]
    results = {}
    for c in candidates:
        results[c] = float(measure(c))
    best = min(results, key=results.get)
    with _lock:
        data = _load(p)
        data[key] = {"best": best, "ms": {str(c): t for c, t in results.items()}}
        _store(p, data)
    return best


def workload_key(wrangler, what):
    """Cache key: device, precision, expansion orders, size class of the tree."""
    dev = torch.cuda.get_device_name(wrangler.device) if wrangler.device.type == "cuda" else "cpu"
    nb = max(1, wrangler.tree.nboxes)
    orders = sorted(set(wrangler.level_orders))
    return (f"{what}|{dev}|{wrangler.precision}|p{','.join(map(str, orders))}"
            f"|nboxes~2^{int(round(math.log2(nb)))}")


def tune_m2l_item_groups(wrangler, run, candidates=(16, 32, 64, 128), path=None,
                         refresh=False):
    """Pick ``wrangler.m2l_item_groups`` by timing ``run()`` (one FMM
    evaluation with this wrangler) per candidate; sets and returns it."""
    def measure(c):
        wrangler.m2l_item_groups = int(c)
        return time_ms(run)

    best = tune(workload_key(wrangler, "m2l_item_groups"), list(candidates), measure, path,
                refresh)
    wrangler.m2l_item_groups = int(best)
    return best


SCHEDULE_SPACE = {
    "m2l_item_groups": (64, 96, 128, 192),
    "item_rounds": (4, 8, 16, 32),
    "octant_split": (1, 2, 4),
    "chain_levels": (False, True),
    "concurrent_stages": (True, False),
}


def coordinate_descent(start, space, measure, sweeps=2):
    """Minimise ``measure(config)`` over the product of ``space`` (knob ->
    candidate values) by coordinate descent from ``start``: each sweep tries
    every other value of each knob in turn and keeps a change that lowers the
    time; stops after a sweep without change. Returns (best config, its
    time, {config key: time} of every config tried)."""
    cur = dict(start)
    tried = {}

    def run(cfg):
        k = repr(sorted(cfg.items()))
        if k not in tried:
            tried[k] = float(measure(dict(cfg)))
        return tried[k]

    best = run(cur)
    for _ in range(sweeps):
        changed = False
        for knob, values in space.items():
            for v in values:
                if v == cur[knob]:
                    continue
                cand = dict(cur, **{knob: v})
                t = run(cand)
                if t < best:
                    best, cur, changed = t, cand, True
        if not changed:
            break
    return cur, best, tried


def tune_schedule(wrangler, run, space=None, path=None, refresh=False, reps=3):
    """Choose the wrangler's schedule knobs by timing ``run()`` (one
    evaluation with this wrangler) under each candidate schedule, coordinate
    descent over ``space`` (default :data:`SCHEDULE_SPACE`). The best
    schedule is applied, cached on disk per workload key, and returned."""
    space = dict(SCHEDULE_SPACE if space is None else space)
    p = cache_path(path)
    key = workload_key(wrangler, "schedule")
    with _lock:
        hit = _load(p).get(key)
    if hit is not None and not refresh and set(hit.get("best", {})) == set(space):
        wrangler.set_schedule(**hit["best"])
        return dict(hit["best"])

    def measure(cfg):
        wrangler.set_schedule(**cfg)
        run()                       # plans and graph for this schedule, untimed
        return time_ms(run, warmup=0, reps=reps)

    start = {k: getattr(wrangler, k) for k in space}
    best, t_best, tried = coordinate_descent(start, space, measure)
    wrangler.set_schedule(**best)
    with _lock:
        data = _load(p)
        data[key] = {"best": best, "ms": t_best, "tried": tried}
        _store(p, data)
    return best
