"""Host logic of the PPPM parameter picker and of cfg4's draws (no GPU: the
error estimators are replaced by closed-form stand-ins)."""
import numpy as np

from oracle import oracle as O


def _fake_pm(N, L, kappa, alpha, M):
    # grows with alpha h, like the order-6 PM error
    h = np.asarray(L) / np.asarray(M)
    return 1e-3 * (np.asarray(alpha) * h) ** 7 * np.sqrt(np.asarray(N) / 1e4)


def _fake_pp(N, L, kappa, alpha, rc):
    return 2.0 * np.sqrt(N / L ** 3 / rc) * np.exp(-(alpha * rc) ** 2 - kappa ** 2 / (4 * alpha ** 2))


def _fake_cutoff(N, L, kappa, alpha, tol, rc_max):
    if _fake_pp(N, L, kappa, alpha, rc_max) > tol:
        return None
    lo, hi = 1e-9, rc_max
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if _fake_pp(N, L, kappa, alpha, mid) <= tol:
            hi = mid
        else:
            lo = mid
    return hi


def _pick(systems, **kw):
    from p3m_b200.params import pick_params

    return pick_params(systems, pm_fn=_fake_pm, cutoff_fn=_fake_cutoff, pp_fn=_fake_pp, **kw)


def test_picker_meets_tolerance_at_least_cost():
    from p3m_b200.configs import box
    from p3m_b200.params import COST_MESH, COST_PP

    systems = [(N, box(N), k) for N, k in ((2000, 0.5), (10000, 2.0), (50000, 3.0))]
    tol = 1e-6
    for (N, L, k), c in zip(systems, _pick(systems, tol=tol)):
        assert c.feasible and c.M in (32, 64, 128)
        assert c.dF <= tol * (1 + 1e-9)
        assert c.rc <= L / 3 + 1e-12
        # no candidate on a fine brute-force grid is cheaper by more than the
        # refinement's resolution
        best = np.inf
        for M in (32, 64, 128):
            for a in np.geomspace(3.0 / L, 1.2 * M / L, 400):
                pm = float(_fake_pm(N, L, k, a, M))
                if pm >= tol:
                    continue
                rc = _fake_cutoff(N, L, k, a, np.sqrt(tol * tol - pm * pm), L / 3)
                if rc is not None:
                    best = min(best, COST_PP * N * (rc + 0.5) ** 3 + COST_MESH * M ** 3)
        assert c.cost_ms <= best * 1.02


def test_picker_flags_infeasible():
    # a tolerance no candidate reaches: flagged, and the most accurate one kept
    (c,) = _pick([(2000, 20.3, 1.0)], tol=1e-30)
    assert not c.feasible
    assert c.dF > 1e-30


def test_cfg4_draws():
    from p3m_b200.configs import CFG4_SEEDS, box, cfg4_system

    assert CFG4_SEEDS == tuple(range(100, 164))
    d = [cfg4_system(s) for s in CFG4_SEEDS]
    assert d == [cfg4_system(s) for s in CFG4_SEEDS]  # seeded, repeatable
    N = np.array([x[0] for x in d])
    G = np.array([x[1] for x in d])
    k = np.array([x[2] for x in d])
    assert N.min() >= 2000 and N.max() <= 50000 and len(set(N.tolist())) == 64
    assert G.min() >= 10 and G.max() <= 200
    assert k.min() >= 0.5 and k.max() <= 3.0
    assert box(2000) > 20.3 and box(50000) < 59.4
    # log-uniform N: the median sits near the geometric mean of the range
    assert 4000 < np.median(N) < 25000


def test_oracle_estimators_match_measured_small():
    """The oracle's PP and PM estimates against the errors they predict,
    measured directly (truncated minimum-image sum; PM force against the
    exact k-space Ewald force) on 600 random unit charges."""
    N = 600
    L = (4 * np.pi * N / 3) ** (1 / 3)
    rng = np.random.default_rng(3)
    pos = rng.random((N, 3)) * L
    kappa, alpha, rc, M = 1.0, 0.7, 3.0, 16
    d = pos[:, None, :] - pos[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d * d).sum(-1))
    np.fill_diagonal(r, np.inf)
    m = (r > rc) & (r < L / 2)
    F = np.zeros_like(r)
    F[m] = O.pair_force_sr(r[m], kappa, alpha) / r[m]
    meas_pp = np.sqrt(np.mean(np.sum(np.sum(F[:, :, None] * d, axis=1) ** 2, axis=1)))
    est_pp = O.pp_error(N, L, kappa, alpha, rc)
    assert 0.8 < est_pp / meas_pp < 1.25
    P = O.Params(N, kappa, alpha, rc, M)
    G_k, kx, ky, kz, A_ref = P.green()
    h = L / M
    _, acc_pm, _ = O.pm(pos, P.Z, G_k, kx, ky, kz, M, M, M, h, h, h, L, L, L)
    meas_pm = np.sqrt(np.mean(np.sum((acc_pm - O.ewald_lr_acc(pos, L, kappa, alpha)) ** 2, 1)))
    est_pm, A = O.pm_error(N, L, kappa, alpha, M)
    assert 0.8 < est_pm / meas_pm < 1.25
    # its A term is the reference's A_pm
    assert abs(A - A_ref) <= 1e-12 * abs(A_ref)
