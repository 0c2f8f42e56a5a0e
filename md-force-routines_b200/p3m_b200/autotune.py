"""Autotuner of a context's kernel shapes, by timing its own NVE steps.

What it searches (p3m_tuning of the C ABI):

* the PP stage: threads per particle in the pair kernel and the Verlet-list
  skin (larger skins rebuild less often but visit more list entries) -- a
  grid of both, since they interact;
* the list cells: (rc + skin)/2 or (rc + skin) wide (cell_div 2 or 1: a
  125-cell stencil of small cells, or 27 larger cells whose candidates are
  staged once for many particles);
* the FFT tiles of meshes up to 64^3: the fused y/z plane kernel (a whole kx
  plane per CTA) or the y and z pencil passes (16 lines per CTA);
* the force gather: a CTA per mesh brick with one or two field-tile buffers
  (copy/compute overlap against CTAs per SM), or a CTA per brick and field
  component (three times the work items);
* on the FP32 path, inner lists (dynamic pruning): the pair kernel reads the
  Verlet entries closer than rc + prune_buf and rebuilds those lists itself
  every few steps, which makes larger skins (rarer Verlet rebuilds) cheap.

The list cells, FFT tiles and gather are searched one at a time from the
best PP setting (coordinate descent), then inner-list buffers with a few
skins from the best of those, each with both list-cell divisors; then the
fastest few settings are timed again over
four times the steps (list rebuilds come every few tens of steps, so short runs
rank close candidates by chance) and the fastest is installed. The state
should already be equilibrated: each timing advances the system. Results are
cached per workload signature in a JSON file.
"""
from __future__ import annotations

import json
import os

from ._lib import FP32, MODE_NVE, P3MError

CANDIDATES = [(tpi, skin) for tpi in (1, 2, 4) for skin in (0.5, 0.8, 1.1, 1.4)]
#: FP32 inner-list buffers, each tried with the best skin so far and larger ones
PRUNE_BUFS = (0.2, 0.3)
PRUNE_SKINS = (1.1, 1.4)
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


def _key(t):
    return (f"tpi{t['pp_tpi']},skin{t['skin']:g},div{t['cell_div']},plane{t['plane_max']},"
            f"gather{t['gather_mode']},prune{t.get('prune_buf', 0.0):g}")


def shape_options(ctx):
    """The values of each non-PP shape worth trying on this context."""
    opts = {"cell_div": (2, 1)}
    if any(0 < r.M <= 64 for r in ctx.replicas):
        opts["plane_max"] = (64, 0)
    if any(r.M > 0 for r in ctx.replicas):
        opts["gather_mode"] = (1, 0, 2) if ctx.precision == FP32 else (1, 0)
    return opts


def max_skin(ctx):
    """The largest skin every replica allows (half its cutoff)."""
    return min(0.5 * r.rc for r in ctx.replicas)


def pp_candidates(ctx, candidates=None):
    """(threads per particle, skin) pairs of the PP grid that every replica
    allows; with cutoffs too short for any of the grid's skins, each thread
    count at the largest skin allowed."""
    grid = list(candidates or CANDIDATES)
    cap = max_skin(ctx)
    fit = [(tpi, skin) for tpi, skin in grid if skin <= cap]
    return fit or sorted({(tpi, cap) for tpi, _ in grid})


def prune_options(ctx, skin, cap):
    """(skin, prune_buf) pairs worth trying from a best skin so far: FP32
    only, skins up to cap, each buffer below the skin."""
    if ctx.precision != FP32:
        return []
    skins = sorted({skin, *(x for x in PRUNE_SKINS if x <= cap)})
    return [(sk, pb) for pb in PRUNE_BUFS for sk in skins if pb < sk]


def tune(ctx, steps=150, warm=5, use_cache=True, candidates=None, finalists=3, shapes=True,
         prune=True):
    """Search the kernel shapes (see the module docstring) and install the
    fastest. Returns {"choice": {tuning}, "ms_per_step": {setting: ms},
    "final_ms_per_step": {setting: ms}, "prune_trials": n}."""
    import torch

    sig = signature(ctx)
    cache = _load() if use_cache else {}
    cap = max_skin(ctx)
    if use_cache and sig in cache and isinstance(cache[sig].get("choice"), dict):
        choice = dict(cache[sig]["choice"])
        choice["skin"] = min(choice["skin"], cap)
        ctx.set_tuning(**choice)
        return cache[sig]
    stream = torch.cuda.ExternalStream(ctx.stream())
    base = ctx.tuning()

    def timed(t, n):
        try:
            ctx.set_tuning(**t)
        except P3MError:  # e.g. an inner-list buffer not below a box-clamped skin
            return float("inf")
        ctx.run(warm, MODE_NVE, graph=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.run(n, MODE_NVE, graph=True, sync=False)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n

    times, settings = {}, {}

    def trial(t):
        k = _key(t)
        if k not in times:
            times[k] = timed(t, steps)
            settings[k] = dict(t)
        return times[k]

    base["prune_buf"] = 0.0
    for tpi, skin in pp_candidates(ctx, candidates):
        trial(dict(base, pp_tpi=tpi, skin=skin))
    best = dict(settings[min(times, key=times.get)])
    if shapes:
        for name, values in shape_options(ctx).items():
            for v in values:
                trial(dict(best, **{name: v}))
            best = dict(settings[min(times, key=times.get)])
    n_before = len(times)
    if prune:
        # the cell size follows the skin: each inner-list setting with every
        # list-cell divisor
        divs = shape_options(ctx)["cell_div"] if shapes else (best["cell_div"],)
        for skin, pb in prune_options(ctx, best["skin"], cap):
            for d in divs:
                trial(dict(best, skin=skin, prune_buf=pb, cell_div=d))
    n_prune = len(times) - n_before
    final = {}
    for k in sorted(times, key=times.get)[:max(1, finalists)]:
        final[k] = timed(settings[k], 4 * steps)
    win = min(final, key=final.get)
    choice = settings[win]
    ctx.set_tuning(**choice)
    result = {"choice": choice, "ms_per_step": times, "final_ms_per_step": final,
              "prune_trials": n_prune}
    if use_cache:
        cache[sig] = result
        _save(cache)
    return result
