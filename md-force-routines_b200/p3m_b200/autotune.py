"""Autotuner of the PP stage: threads per particle in the force kernel and the
Verlet-list skin (larger skins rebuild less often but visit more list
entries). It times short device-resident NVE runs of the caller's own
context -- so the state should already be equilibrated -- and installs the
fastest setting. Results are cached per workload signature in a JSON file.
"""
from __future__ import annotations

import json
import os

from ._lib import MODE_NVE

CANDIDATES = [(tpi, skin) for tpi in (1, 2, 4) for skin in (0.5, 0.8, 1.1, 1.4)]
CACHE = os.environ.get("P3M_B200_TUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "p3m_b200", "autotune.json"))


def signature(ctx) -> str:
    reps = ctx.replicas
    parts = sorted({(r.N, round(r.L, 6), r.rc, r.M) for r in reps})
    return f"p{ctx.precision}|R{len(reps)}|" + ";".join(f"{n},{l},{c},{m}" for n, l, c, m in parts)


def _load():
    try:
        return json.load(open(CACHE))
    except Exception:
        return {}


def _save(d):
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        json.dump(d, open(CACHE, "w"), indent=1)
    except OSError:
        pass


def tune(ctx, steps=150, warm=5, use_cache=True, candidates=None, finalists=3):
    """Time each (threads per particle, skin) candidate over `steps` NVE steps
    (CUDA events on the context's stream), time the `finalists` fastest again
    over 2 `steps` (list rebuilds come every few tens of steps, so short runs
    rank close candidates by chance) and install the fastest of those.
    Returns {"choice": (tpi, skin), "ms_per_step": {...}, "final_ms_per_step":
    {...}}. Advances the system by warm + steps per candidate and warm + 2
    steps per finalist."""
    import torch

    sig = signature(ctx)
    cache = _load() if use_cache else {}
    if use_cache and sig in cache:
        tpi, skin = cache[sig]["choice"]
        max_skin = min(0.5 * r.rc for r in ctx.replicas)
        ctx.set_pp_config(tpi, min(skin, max_skin))
        return cache[sig]
    stream = torch.cuda.ExternalStream(ctx.stream())
    max_skin = min(0.5 * r.rc for r in ctx.replicas)

    def timed(tpi, skin, n):
        ctx.set_pp_config(tpi, skin)
        ctx.run(warm, MODE_NVE, graph=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.run(n, MODE_NVE, graph=True, sync=False)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n

    times = {}
    for tpi, skin in (candidates or CANDIDATES):
        if skin <= max_skin:
            times[f"{tpi},{skin}"] = timed(tpi, skin, steps)
    final = {}
    for key in sorted(times, key=times.get)[:max(1, finalists)]:
        tpi, skin = key.split(",")
        final[key] = timed(int(tpi), float(skin), 2 * steps)
    best = min(final, key=final.get)
    tpi, skin = best.split(",")
    choice = (int(tpi), float(skin))
    ctx.set_pp_config(*choice)
    result = {"choice": choice, "ms_per_step": times, "final_ms_per_step": final}
    if use_cache:
        cache[sig] = result
        _save(cache)
    return result
