"""The benchmark workloads: Yukawa OCP ensembles in the units of
yukawa_MD_p3m_ord6.py (lengths in a_ws, n = 3/(4 pi), L = (4 pi N / 3)^(1/3),
time in 1/omega_p, T = 1/Gamma, af = 1/3, uf = 1, kf = 1.5)."""
from __future__ import annotations

import numpy as np

from .context import Replica


def box(N):
    return (4.0 * np.pi * N / 3.0) ** (1.0 / 3.0)


def replica(N, Gamma, kappa, M, alpha, rc, dt=0.1, seed=0):
    return Replica(N=int(N), L=box(N), kappa=float(kappa), alpha=float(alpha), rc=float(rc),
                   M=int(M), dt=float(dt), T_desired=1.0 / float(Gamma), seed=int(seed))


def cfg1():
    """Plain method, single replica: N=1e4, Gamma=100, kappa=2, 64^3, alpha=0.6,
    rc=6, dt=0.1, seed 1 (1000 thermostat + 1000 NVE steps)."""
    return [replica(10000, 100.0, 2.0, 64, 0.6, 6.0, seed=1)]


def cfg2():
    """Single replica, FP32 bulk: N=1e5, Gamma=50, kappa=1, 128^3, alpha=0.5,
    rc=7, dt=0.1, seed 2 (2000 steps)."""
    return [replica(100000, 50.0, 1.0, 128, 0.5, 7.0, seed=2)]


def cfg3(n_replicas=20, first_seed=1):
    """Batched ensemble: 20 replicas identical but for the seed (1..20), each
    cfg1's system; n(q,t) on the 32 smallest q = m 2 pi/L, m = 1..32."""
    return [replica(10000, 100.0, 2.0, 64, 0.6, 6.0, seed=first_seed + i) for i in range(n_replicas)]


#: cfg4's replicas: one per seed 100..163
CFG4_SEEDS = tuple(range(100, 164))


def cfg4_system(seed):
    """(N, Gamma, kappa) of the cfg4 replica with this seed: numpy's default
    generator (PCG64, ``np.random.default_rng(seed)``), three draws in this
    order: ln N ~ U[ln 2000, ln 50000] (rounded to an integer), ln Gamma ~
    U[ln 10, ln 200], kappa ~ U[0.5, 3]."""
    rng = np.random.default_rng(int(seed))
    N = int(round(float(np.exp(rng.uniform(np.log(2000.0), np.log(50000.0))))))
    Gamma = float(np.exp(rng.uniform(np.log(10.0), np.log(200.0))))
    kappa = float(rng.uniform(0.5, 3.0))
    return N, Gamma, kappa


def cfg4(n_replicas=64, tol=None, device=0, **pick_kw):
    """Uneven ensemble: replicas with N, Gamma and kappa drawn per seed
    (cfg4_system), each with the (M in {32, 64, 128}, alpha, r_c <= L/3) of
    least modelled cost whose estimated RMS force error is within ``tol``
    (params.pick_params; default 1e-6 in reduced units); 500 NVE steps of
    dt = 0.1. Returns (replicas, choices)."""
    from .params import DEFAULT_TOL, pick_params

    seeds = CFG4_SEEDS[:n_replicas]
    systems = [cfg4_system(s) for s in seeds]
    choices = pick_params([(N, box(N), kappa) for N, _, kappa in systems],
                          tol=DEFAULT_TOL if tol is None else tol, device=device, **pick_kw)
    reps = [replica(N, Gamma, kappa, c.M, c.alpha, c.rc, seed=s)
            for (N, Gamma, kappa), c, s in zip(systems, choices, seeds)]
    return reps, choices


def cfg5():
    """Large single replica: N=1e6, Gamma=100, kappa=2, 256^3, alpha=0.6, rc=6,
    200 NVE steps from seed 7."""
    return [replica(1000000, 100.0, 2.0, 256, 0.6, 6.0, seed=7)]


CFG3_QMULT = np.arange(1, 33, dtype=np.float64)

WORKLOADS = {"cfg1": cfg1, "cfg2": cfg2, "cfg3": cfg3, "cfg4": lambda: cfg4()[0], "cfg5": cfg5}
