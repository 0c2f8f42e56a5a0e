"""The autotuner's search (p3m_b200.autotune.tune) without a device: a fake
context whose step time follows a synthetic cost model of its kernel shapes,
and CUDA events that read the fake's clock. Checks the order of the search
(PP grid, then one shape at a time, then inner-list buffers with each list
cell divisor, then the finalists over four times the steps), that every
trial runs the shapes it names, that a setting the context refuses is
skipped, and that the fastest finalist is installed and cached."""
import json

import pytest

import p3m_b200.autotune as at
from p3m_b200 import FP32, FP64, P3MError, Replica

DEFAULT = {"pp_tpi": 2, "cell_div": 2, "plane_max": 64, "gather_mode": 1, "skin": 0.8,
           "prune_buf": 0.0}


def cost(t):
    """ms per step of a setting: best at tpi 2, skin 1.4, cell_div 1,
    pencil passes, gather mode 2, inner lists at 0.3."""
    c = 1.0
    c += {1: 0.30, 2: 0.0, 4: 0.10}[t["pp_tpi"]]
    c += 0.05 * abs(t["skin"] - 1.4)
    c += 0.0 if t["cell_div"] == 1 else 0.02
    c += 0.0 if t["plane_max"] == 0 else 0.01
    c += {0: 0.03, 1: 0.01, 2: 0.0}[t["gather_mode"]]
    c -= {0.0: 0.0, 0.2: 0.04, 0.3: 0.06}[t["prune_buf"]]
    return c


class FakeCtx:
    def __init__(self, precision=FP32, rc=6.0, refuse=None):
        self.precision = precision
        self.replicas = [Replica(N=10000, L=34.7, kappa=2.0, alpha=0.6, rc=rc, M=64)]
        self.cur = dict(DEFAULT)
        self.clock = 0.0
        self.timed_steps = []   # (tuning, n) of every run
        self.refuse = refuse or (lambda t: False)

    def tuning(self):
        return dict(self.cur)

    def set_tuning(self, **kw):
        new = dict(self.cur, **kw)
        if self.refuse(new):
            raise P3MError(-1, "refused")
        self.cur = new

    def run(self, n, mode, graph=True, sync=True, **kw):
        self.clock += n * cost(self.cur)
        self.timed_steps.append((dict(self.cur), n))

    def stream(self):
        return 0


class FakeEvent:
    ctx = None

    def __init__(self, enable_timing=True):
        self.t = None

    def record(self, stream=None):
        self.t = FakeEvent.ctx.clock

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return other.t - self.t


@pytest.fixture
def fake_cuda(monkeypatch):
    import torch

    monkeypatch.setattr(torch.cuda, "ExternalStream", lambda s: s)
    monkeypatch.setattr(torch.cuda, "Event", FakeEvent)


def _tune(ctx, **kw):
    FakeEvent.ctx = ctx
    return at.tune(ctx, steps=10, warm=1, use_cache=False, **kw)


def test_tune_installs_the_fastest_setting(fake_cuda):
    ctx = FakeCtx()
    res = _tune(ctx)
    want = {"pp_tpi": 2, "skin": 1.4, "cell_div": 1, "plane_max": 0, "gather_mode": 2,
            "prune_buf": 0.3}
    assert res["choice"] == want
    assert ctx.cur == want
    # every trial's time is its own setting's cost
    for k, ms in res["ms_per_step"].items():
        assert ms == pytest.approx(cost(
            next(t for t, n in ctx.timed_steps if at._key(t) == k)))
    # inner-list stage: buffers 0.2 and 0.3 at skins 1.4 (the best) and 1.1,
    # each with both cell divisors -- all new (the stages before ran none)
    assert res["prune_trials"] == 2 * 2 * 2


def test_tune_stage_order_and_finalists(fake_cuda):
    ctx = FakeCtx()
    res = _tune(ctx, finalists=3)
    timed = [(t, n) for t, n in ctx.timed_steps if n != 1]  # drop the warm-up runs
    n_grid = sum(1 for tpi, s in at.CANDIDATES if s <= 3.0)
    grid = timed[:n_grid]
    assert {(t["pp_tpi"], t["skin"]) for t, _ in grid} == set(at.CANDIDATES)
    assert all(t["prune_buf"] == 0.0 for t, _ in grid)
    assert all(n == 10 for _, n in timed[:-3])
    finals = timed[-3:]
    assert all(n == 40 for _, n in finals)                      # four times the steps
    ranked = sorted(res["ms_per_step"], key=res["ms_per_step"].get)[:3]
    assert [at._key(t) for t, _ in finals] == ranked
    assert set(res["final_ms_per_step"]) == set(ranked)


def test_tune_fp64_has_no_inner_lists_and_short_cutoffs_still_tune(fake_cuda):
    ctx = FakeCtx(precision=FP64, rc=0.8)
    res = _tune(ctx)
    assert res["prune_trials"] == 0
    assert res["choice"]["prune_buf"] == 0.0
    assert res["choice"]["skin"] == 0.4                          # rc / 2: the largest allowed
    assert all(t["gather_mode"] != 2 for t, _ in ctx.timed_steps)  # FP32-only mode


def test_tune_skips_refused_settings(fake_cuda):
    """A setting the context refuses (P3MError from set_tuning) is ranked
    last and never installed."""
    ctx = FakeCtx(refuse=lambda t: t["prune_buf"] == 0.3)
    res = _tune(ctx)
    assert res["choice"]["prune_buf"] == 0.2
    refused = [k for k in res["ms_per_step"] if k.endswith("prune0.3")]
    assert refused and all(res["ms_per_step"][k] == float("inf") for k in refused)


def test_tune_cache_round_trip(fake_cuda, tmp_path, monkeypatch):
    monkeypatch.setattr(at, "CACHE", str(tmp_path / "tune.json"))
    ctx = FakeCtx()
    FakeEvent.ctx = ctx
    first = at.tune(ctx, steps=10, warm=1)
    saved = json.load(open(tmp_path / "tune.json"))
    assert saved[at.signature(ctx)]["choice"] == first["choice"]
    other = FakeCtx()
    FakeEvent.ctx = other
    again = at.tune(other, steps=10, warm=1)
    assert again["choice"] == first["choice"] and other.cur == first["choice"]
    assert other.timed_steps == []                               # from the cache: nothing timed
