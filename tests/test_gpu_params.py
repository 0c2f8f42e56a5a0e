"""PPPM error estimates and the parameter picker on the device, against the
oracle and against errors measured directly."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SETS = [  # N, kappa, alpha, M
    (1000, 1.0, 0.6, 16),
    (1000, 1.0, 0.9, 32),
    (2500, 2.5, 0.45, 32),
    (600, 0.5, 1.4, 32),
]


def test_pm_error_matches_oracle():
    from p3m_b200.params import pm_error

    N = np.array([s[0] for s in SETS], dtype=float)
    L = (4 * np.pi * N / 3) ** (1 / 3)
    k = np.array([s[1] for s in SETS])
    a = np.array([s[2] for s in SETS])
    M = np.array([s[3] for s in SETS])
    dF, A = pm_error(N, L, k, a, M)
    for i in range(len(SETS)):
        ref, A_ref = O.pm_error(N[i], L[i], k[i], a[i], int(M[i]))
        # the oracle forms sum R^2 - sum A directly; with Q / A_pm down to
        # 1e-8 here that keeps about 8 digits of dF^2 (the device sums the
        # alias terms apart and cancels the central one exactly)
        assert abs(dF[i] - ref) <= 1e-6 * ref, (dF[i], ref)
        # sum_k A(k) is the reference's A_pm (yukawa_gf_opt.py:96)
        h = L[i] / M[i]
        _, _, _, _, A_gf = O.gf_opt(k[i], a[i], 6, 3, 3, 3, int(M[i]), int(M[i]), int(M[i]),
                                    h, h, h, L[i], L[i], L[i])
        assert abs(A[i] - A_gf) <= 1e-11 * abs(A_gf)
        assert abs(A[i] - A_ref) <= 1e-11 * abs(A_ref)


def test_pp_error_and_cutoff_match_oracle():
    from p3m_b200.params import pp_cutoff, pp_error

    for N, kappa, alpha, rc in [(1000, 1.0, 0.6, 3.0), (10000, 2.0, 0.6, 6.0), (2000, 3.0, 0.3, 5.5),
                                (50000, 0.5, 1.2, 2.5)]:
        L = (4 * np.pi * N / 3) ** (1 / 3)
        est = pp_error(N, L, kappa, alpha, rc)
        assert abs(est - O.pp_error(N, L, kappa, alpha, rc)) <= 1e-4 * est
        tol = est * 0.37
        r = pp_cutoff(N, L, kappa, alpha, tol, L / 3)
        assert r is not None and r > rc
        assert pp_error(N, L, kappa, alpha, r) <= tol
        assert pp_error(N, L, kappa, alpha, r * (1 - 1e-3)) > tol
        worst = pp_error(N, L, kappa, alpha, L / 3)
        assert worst == 0.0 or pp_cutoff(N, L, kappa, alpha, 0.5 * worst, L / 3) is None


def test_picked_parameters_reach_tolerance():
    """Pick (alpha, r_c) at 32^3 for a tolerance, run the library's FP64 force
    with them, and measure its error against the exact Yukawa-Ewald force (a
    minimum-image short-range sum plus the k-space sum): within 25% of the
    estimate that the picker held to the tolerance."""
    from p3m_b200 import FP64, Context, Replica
    from p3m_b200.params import pick_params, pp_error

    N, kappa, tol = 1500, 1.0, 2e-5
    L = (4 * np.pi * N / 3) ** (1 / 3)
    (c,) = pick_params([(N, L, kappa)], tol=tol, meshes=(32,))
    assert c.feasible and c.dF <= tol * (1 + 1e-9) and c.rc <= L / 3
    # the minimum-image sum is complete: the tail beyond L/2 is far below tol
    assert pp_error(N, L, kappa, c.alpha, L / 2) < 1e-3 * tol
    rng = np.random.default_rng(4)
    pos = rng.random((N, 3)) * L
    r = Replica(N=N, L=L, kappa=kappa, alpha=c.alpha, rc=c.rc, M=32)
    with Context(r, precision=FP64) as ctx:
        _, acc, _ = ctx.force(pos)
    d = pos[:, None, :] - pos[None, :, :]
    d -= L * np.round(d / L)
    rr = np.sqrt((d * d).sum(-1))
    np.fill_diagonal(rr, np.inf)
    m = rr < L / 2
    F = np.zeros_like(rr)
    F[m] = O.pair_force_sr(rr[m], kappa, c.alpha) / rr[m]
    exact = np.sum(F[:, :, None] * d, axis=1) + O.ewald_lr_acc(pos, L, kappa, c.alpha)
    meas = np.sqrt(np.mean(np.sum((acc / r.af - exact) ** 2, axis=1)))
    assert 0.75 * c.dF < meas < 1.25 * c.dF, (meas, c)


def test_cfg4_parameters():
    """All 64 cfg4 replicas reach 1e-6 within M <= 128 and L/r_c >= 3."""
    from p3m_b200.configs import cfg4

    reps, choices = cfg4()
    assert len(reps) == 64
    for r, c in zip(reps, choices):
        assert c.feasible and c.dF <= 1e-6 * (1 + 1e-9)
        assert r.M in (32, 64, 128) and r.L / r.rc >= 3.0 - 1e-9
        assert (r.M, r.alpha, r.rc) == (c.M, c.alpha, c.rc)
