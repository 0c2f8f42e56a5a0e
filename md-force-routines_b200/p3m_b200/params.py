"""PPPM parameter choice from error estimates.

The reference sets the Ewald parameter alpha, the cutoff r_c and the mesh M
by hand for each run (yukawa_MD_p3m_ord6.py:52-68, README.md:27); its only
error measure is A_pm (yukawa_gf_opt.py:96). Here the RMS per-particle force
errors of the two parts are estimated (``pp_error``: the Yukawa-Ewald force
beyond r_c over a uniform background, Kolafa & Perram 1992; ``pm_error``:
Hockney & Eastwood's Q functional at the optimal influence function), both
in the reference's reduced units (force per charge^2 / a_ws^2), and
``pick_params`` chooses, per system, the (M, alpha, r_c) of least modelled
step time whose total error sqrt(dF_pp^2 + dF_pm^2) is within a tolerance.
The reference's hand-set parameters sit near 1e-6 (N=1e4, kappa=0.1,
alpha=0.46, r_c=7.8, 64^3: 1.1e-6), the default tolerance here.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import check, dptr, lib

#: modelled step time, ms: COST_PP * N * (r_c + skin)^3 for the pair loop and
#: COST_MESH * M^3 for the mesh transforms; from the stage timings of the
#: 20 x 1e4-particle, 64^3 ensemble on one B200 (pair loop 0.319 ms at
#: r_c + skin = 6.8, both FFT directions 0.219 ms). Assignment and gather
#: scale with N alone and do not move the choice.
COST_PP = 5.1e-9
COST_MESH = 4.2e-8
MESHES = (32, 64, 128)
DEFAULT_TOL = 1e-6


def pp_error(N, L, kappa, alpha, rc):
    """RMS PP truncation error at r_c (host, FP64)."""
    out = ctypes.c_double()
    check(lib().p3m_pp_error(float(N), float(L), float(kappa), float(alpha), float(rc),
                             ctypes.byref(out)), None)
    return out.value


def pp_cutoff(N, L, kappa, alpha, tol, rc_max):
    """Smallest r_c <= rc_max with pp_error <= tol, or None."""
    out = ctypes.c_double()
    check(lib().p3m_pp_cutoff(float(N), float(L), float(kappa), float(alpha), float(tol),
                              float(rc_max), ctypes.byref(out)), None)
    return None if out.value < 0 else out.value


def pm_error(N, L, kappa, alpha, M, p=6, m_alias=3, device=0):
    """RMS PM error of each parameter set (arrays broadcast together), on the
    device in FP64 -> (dF_pm, A_pm) arrays; A_pm is the reference's sum for
    the same parameters."""
    b = np.broadcast_arrays(*(np.asarray(v, dtype=np.float64) for v in (N, L, kappa, alpha, M)))
    n, box, ka, al = (np.ascontiguousarray(v.ravel()) for v in b[:4])
    Ms = np.ascontiguousarray(b[4].ravel().astype(np.int32))
    dF = np.empty(n.size)
    A = np.empty(n.size)
    check(lib().p3m_pm_error(int(device), int(n.size), dptr(n), dptr(box), dptr(ka), dptr(al),
                             Ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(p), int(m_alias),
                             dptr(dF), dptr(A)), None)
    return dF.reshape(b[0].shape), A.reshape(b[0].shape)


@dataclass
class Choice:
    M: int
    alpha: float
    rc: float
    dF_pp: float
    dF_pm: float
    cost_ms: float
    feasible: bool

    @property
    def dF(self):
        return float(np.hypot(self.dF_pp, self.dF_pm))


def _alpha_grid(L, M, rc_max, n):
    # from alpha r_c = 2 at the largest cutoff (the PP tail is ~1e-2 there)
    # to alpha h = 1.2 (the order-6 PM error is ~1e-2 there)
    return np.geomspace(2.0 / rc_max, 1.2 * M / L, n)


def pick_params(systems, tol=DEFAULT_TOL, meshes=MESHES, p=6, m_alias=3, skin=0.5, n_alpha=24,
                rc_frac=1.0 / 3.0, device=0, pm_fn=None, cutoff_fn=None, pp_fn=None):
    """systems: iterable of (N, L, kappa). For each, over M in ``meshes`` and
    a geometric alpha grid refined once around the best point: the PM error
    (one batched device call per pass), the smallest r_c <= rc_frac * L whose
    PP error fits sqrt(tol^2 - dF_pm^2), and the modelled cost; returns one
    Choice per system, the cheapest feasible one, or the most accurate
    candidate with feasible=False when none fits. ``pm_fn``, ``cutoff_fn``
    and ``pp_fn`` replace pm_error, pp_cutoff and pp_error (same
    signatures)."""
    pm_fn = pm_fn or (lambda *a: pm_error(*a, p=p, m_alias=m_alias, device=device)[0])
    cutoff_fn = cutoff_fn or pp_cutoff
    pp_fn = pp_fn or pp_error
    systems = [(int(N), float(L), float(k)) for N, L, k in systems]
    grids = {}
    for i, (N, L, k) in enumerate(systems):
        for M in meshes:
            grids[i, M] = _alpha_grid(L, M, rc_frac * L, n_alpha)
    best = {}
    for refine in (False, True):
        keys = sorted(grids)
        Ns = np.concatenate([np.full(len(grids[key]), systems[key[0]][0]) for key in keys])
        Ls = np.concatenate([np.full(len(grids[key]), systems[key[0]][1]) for key in keys])
        ks = np.concatenate([np.full(len(grids[key]), systems[key[0]][2]) for key in keys])
        Ms = np.concatenate([np.full(len(grids[key]), key[1]) for key in keys])
        als = np.concatenate([grids[key] for key in keys])
        pms = np.asarray(pm_fn(Ns, Ls, ks, als, Ms), dtype=np.float64).ravel() if len(als) else []
        j = 0
        for (i, M) in keys:
            N, L, k = systems[i]
            rc_max = rc_frac * L
            for a in grids[i, M]:
                pm = float(pms[j])
                j += 1
                if pm < tol:
                    rc = cutoff_fn(N, L, k, a, float(np.sqrt(tol * tol - pm * pm)), rc_max)
                    if rc is not None:
                        c = Choice(M, float(a), float(rc), float(pp_fn(N, L, k, a, rc)), pm,
                                   COST_PP * N * (rc + skin) ** 3 + COST_MESH * M ** 3, True)
                        if i not in best or not best[i].feasible or c.cost_ms < best[i].cost_ms:
                            best[i] = c
                        continue
                if i not in best or not best[i].feasible:
                    c = Choice(M, float(a), rc_max, float(pp_fn(N, L, k, a, rc_max)), pm,
                               COST_PP * N * (rc_max + skin) ** 3 + COST_MESH * M ** 3, False)
                    if i not in best or c.dF < best[i].dF:
                        best[i] = c
        if refine:
            break
        # second pass: a finer grid between the neighbours of each best alpha
        new = {}
        for i, c in best.items():
            g = grids[i, c.M]
            step = g[1] / g[0] if len(g) > 1 else 1.0
            new[i, c.M] = np.geomspace(c.alpha / step, c.alpha * step, 9)[1:-1]
        grids = new
    return [best[i] for i in range(len(systems))]
