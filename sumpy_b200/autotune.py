"""Measured choice of launch parameters, remembered on disk.

sumpy tunes nothing at run time (its work-group sizes follow fixed rules,
e.g. ``min(256, max_ntargets_in_one_box)`` at ``sumpy/p2p.py:727``); here the one schedule knob with a
workload-dependent best value is the number of M2L class groups per work
item (``SumpyExpansionWrangler.m2l_item_groups``): small items balance the
148 SMs better, large ones reuse each target tile's accumulators longer.
:func:`tune` times each candidate with CUDA events on the current stream and
keeps the fastest per key in a JSON file (``$SUMPY_B200_AUTOTUNE_CACHE``,
default ``~/.cache/sumpy_b200/autotune.json``).
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
