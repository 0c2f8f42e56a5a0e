"""The CPU oracle against the reference's own outputs (tests/golden/*.npz,
generated by tests/golden/make_golden.py from the reference's numba code)."""
import numpy as np
import pytest

from oracle import oracle as O


def _params(g):
    return O.Params(int(g["N"]), float(g["kappa"]), float(g["alpha"]), float(g["rc"]), int(g["M"]),
                    Gamma=float(g["Gamma"]), dt=float(g["dt"]))


def test_pp_bitexact(golden):
    g = golden
    L = float(g["L"])
    U, acc = O.pp(float(g["kappa"]), float(g["alpha"]), float(g["rc"]), [L] * 3, g["pos0"])
    assert U == g["U_pp"]
    assert np.array_equal(acc, g["acc_pp"])


def test_assign(golden):
    g = golden
    M, L = int(g["M"]), float(g["L"])
    h = L / M
    rho = O.assign6(g["pos0"], np.ones(int(g["N"])), M, M, M, h, h, h)
    np.testing.assert_allclose(rho, g["rho"], rtol=0, atol=1e-15)
    assert abs(rho.sum() - int(g["N"])) < 1e-9


def test_gf_opt(golden):
    g = golden
    M, L = int(g["M"]), float(g["L"])
    h = L / M
    G, kx, ky, kz, A = O.gf_opt(float(g["kappa"]), float(g["alpha"]), 6, 3, 3, 3, M, M, M, h, h, h,
                                L, L, L)
    np.testing.assert_allclose(G, g["G_k"], rtol=1e-13, atol=1e-18)
    assert A == pytest.approx(float(g["A_pm"]), rel=1e-13)


def test_gather(golden):
    g = golden
    M, L, N = int(g["M"]), float(g["L"]), int(g["N"])
    h = L / M
    rng = np.random.default_rng(int(g["seed"]) + 1000)
    Em = [rng.standard_normal((M, M, M)) for _ in range(3)]
    acc, _ = O.gather6(g["pos0"], np.ones(N), M, M, M, h, h, h, *Em)
    np.testing.assert_allclose(acc, g["acc_gather"], rtol=0, atol=1e-14)


def test_pm(golden):
    g = golden
    M, L, N = int(g["M"]), float(g["L"]), int(g["N"])
    h = L / M
    P = _params(g)
    _, kx, ky, kz, _ = P.green()
    U, acc, Ep = O.pm(g["pos0"], np.ones(N), g["G_k"], kx, ky, kz, M, M, M, h, h, h, L, L, L)
    assert U == pytest.approx(float(g["U_pm"]), rel=1e-14)
    np.testing.assert_allclose(acc, g["acc_pm"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(Ep, g["E_p"], rtol=0, atol=1e-14)


def test_force_pot(golden):
    g = golden
    U, acc, _ = O.force_pot(_params(g), g["pos0"])
    assert U == pytest.approx(float(g["U0"]), rel=1e-14)
    np.testing.assert_allclose(acc, g["acc0"], rtol=0, atol=1e-14)


def test_trace(golden):
    """vscale x S then update x S from the golden initial state."""
    g = golden
    P = _params(g)
    S = int(g["trace_steps"])
    _, acc, _ = O.force_pot(P, g["pos0"])
    p, v = g["pos0"].copy(), g["vel0"].copy()
    tr = []
    for it in range(S):
        p, v, acc, U, _ = O.vscale(P, p, v, acc, it)
        tr.append([U, P.kf * np.sum(v ** 2)])
    for _ in range(S):
        p, v, acc, U = O.update(P, p, v, acc)
        tr.append([U, P.kf * np.sum(v ** 2)])
    np.testing.assert_allclose(np.array(tr), g["trace"], rtol=1e-12)
    np.testing.assert_allclose(p, g["pos_final"], rtol=0, atol=1e-12)


def test_nqt_and_sqw(golden):
    g = golden
    nq = O.nqt(g["pos_final"], g["qv"])
    np.testing.assert_allclose(nq, g["nq_final"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(O.q_vectors_reference(float(g["L"])), g["qv"], rtol=0, atol=0)
    N, dt = int(g["N"]), float(g["dt"])
    s = O.sqw(g["nqt_series"], N, dt, 64 * dt)
    np.testing.assert_allclose(s, g["sqw"], rtol=1e-14)
