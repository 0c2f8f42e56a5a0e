"""Per-stage parity of the CUDA path (through the C ABI) with the reference's
outputs (golden vectors) and the CPU oracle.

Tolerances: FP64 path ("plain method") -- PP to 1e-12 relative, mesh stages
to 1e-9 relative (the deterministic assignment accumulates in 2^-40 fixed
point); FP32 path -- RMS force error <= 1e-5 relative to the FP64 result.
"""
import numpy as np
import pytest

from gpu_util import golden_kvecs, oracle_params, rel_max, rel_rms, replica_from_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["fp64", "fp32"])
def prec(request):
    from p3m_b200 import FP32, FP64

    return {"fp64": FP64, "fp32": FP32}[request.param]


def _ctx(g, prec, mesh=True):
    from p3m_b200 import Context

    r = replica_from_golden(g)
    if not mesh:
        r.M = 0
    return Context(r, precision=prec)


def test_pp(golden, prec):
    from p3m_b200 import FP64

    g = golden
    with _ctx(g, prec, mesh=False) as c:
        U, acc = c.pp(g["pos0"])
    if prec == FP64:
        assert U == pytest.approx(float(g["U_pp"]), rel=1e-12)
        assert rel_rms(acc, g["acc_pp"]) < 1e-12
    else:
        assert U == pytest.approx(float(g["U_pp"]), rel=1e-6)
        assert rel_rms(acc, g["acc_pp"]) < 1e-6


def test_assign(golden, prec):
    from p3m_b200 import FP64

    g = golden
    with _ctx(g, prec) as c:
        rho = c.assign(g["pos0"])
    tol = 1e-11 if prec == FP64 else 1e-6
    assert np.max(np.abs(rho - g["rho"])) < tol * np.max(np.abs(g["rho"]))
    assert abs(rho.sum() - int(g["N"])) < (1e-9 if prec == FP64 else 1e-7) * int(g["N"])


def test_gather(golden, prec):
    from p3m_b200 import FP64

    g = golden
    M = int(g["M"])
    rng = np.random.default_rng(int(g["seed"]) + 1000)
    Em = [rng.standard_normal((M, M, M)) for _ in range(3)]
    with _ctx(g, prec) as c:
        acc, Ep = c.gather(g["pos0"], np.ones(int(g["N"])), *Em)
    tol = 1e-12 if prec == FP64 else 2e-6
    assert rel_rms(acc, g["acc_gather"]) < tol
    np.testing.assert_allclose(Ep.T, acc, rtol=0, atol=0)


def test_gf_opt_device(golden):
    import yukawa_gf_opt

    g = golden
    M, L = int(g["M"]), float(g["L"])
    h = L / M
    G, kx, ky, kz, A = yukawa_gf_opt.gf_opt(float(g["kappa"]), float(g["alpha"]), 6, 3, 3, 3,
                                            M, M, M, h, h, h, L, L, L)
    assert np.max(np.abs(G - g["G_k"])) < 1e-12 * np.max(np.abs(g["G_k"]))
    assert A == pytest.approx(float(g["A_pm"]), rel=1e-11)
    gx, gy, gz = golden_kvecs(g)
    assert np.array_equal(kx, gx) and np.array_equal(ky, gy) and np.array_equal(kz, gz)


def test_pm(golden, prec):
    from p3m_b200 import FP64

    g = golden
    with _ctx(g, prec) as c:
        c.set_green(g["G_k"])
        U, acc, Ep, rho = c.pm(g["pos0"], want_rho=True)
    if prec == FP64:
        assert U == pytest.approx(float(g["U_pm"]), rel=1e-9)
        assert rel_rms(acc, g["acc_pm"]) < 1e-9
        assert rel_rms(Ep, g["E_p"]) < 1e-9
    else:
        assert U == pytest.approx(float(g["U_pm"]), rel=1e-5)
        assert rel_rms(acc, g["acc_pm"]) < 5e-6


def test_pm_device_green(golden):
    """PM with the influence function computed by the context itself."""
    from p3m_b200 import FP64

    g = golden
    with _ctx(g, FP64) as c:
        U, acc, _, _ = c.pm(g["pos0"])
    assert U == pytest.approx(float(g["U_pm"]), rel=1e-9)
    assert rel_rms(acc, g["acc_pm"]) < 1e-9


def test_force(golden, prec):
    from p3m_b200 import FP64

    g = golden
    with _ctx(g, prec) as c:
        U, acc, parts = c.force(g["pos0"])
    if prec == FP64:
        assert U == pytest.approx(float(g["U0"]), rel=1e-10)
        assert rel_rms(acc, g["acc0"]) < 1e-9
    else:
        assert U == pytest.approx(float(g["U0"]), rel=1e-5)
        assert rel_rms(acc, g["acc0"]) <= 1e-5
        assert rel_max(acc, g["acc0"]) <= 1e-4
    assert parts[2] == pytest.approx(-int(g["N"]) * float(g["alpha"]) / np.sqrt(np.pi), rel=1e-15)


def test_trace_compat(golden, prec):
    """vscale x S then update x S through the compat calls, against the
    reference's energy trace."""
    from p3m_b200 import FP64

    g = golden
    S = int(g["trace_steps"])
    with _ctx(g, prec) as c:
        c.set_green(g["G_k"])
        _, acc, _ = c.force(g["pos0"])
        p, v = g["pos0"].copy(), g["vel0"].copy()
        tr = []
        for it in range(S):
            U, _ = c.vscale(it, p, v, acc)
            tr.append([U, 1.5 * np.sum(v ** 2)])
        for _ in range(S):
            U = c.update(p, v, acc)
            tr.append([U, 1.5 * np.sum(v ** 2)])
    tr = np.array(tr)
    tol = 1e-9 if prec == FP64 else 1e-5
    np.testing.assert_allclose(tr, g["trace"], rtol=tol)
    assert np.max(np.abs(p - g["pos_final"])) < (1e-10 if prec == FP64 else 1e-5)


def test_reference_modules_force_pot(golden, capsys):
    """force_pot / update / vscale through the reference-named modules."""
    import thermostat_p3m_ord6 as th
    import velocity_verlet_p3m_ord6 as vv
    import yukawa_p3m_ord6
    from p3m_b200 import set_compat_precision

    set_compat_precision("fp64")
    g = golden
    N, M, L = int(g["N"]), int(g["M"]), float(g["L"])
    h = L / M
    k, a, rc = float(g["kappa"]), float(g["alpha"]), float(g["rc"])
    kx, ky, kz = golden_kvecs(g)
    Lv = np.array([L] * 3)
    Z = np.ones(N)
    scratch = [np.zeros((N, 3)), np.zeros((N, 3)), np.zeros((M, M, M)), np.zeros(N), np.zeros(N),
               np.zeros(N)]
    args = (g["G_k"], kx, ky, kz, M, M, M, h, h, h, L, L, L, 6, 3, 3, 3, *scratch)
    U0, acc = yukawa_p3m_ord6.force_pot(k, a, N, rc, Lv, 1 / 3, 1.0, g["pos0"], None, Z, *args)
    assert U0 == pytest.approx(float(g["U0"]), rel=1e-10)
    assert rel_rms(acc, g["acc0"]) < 1e-9
    pos, vel = g["pos0"], g["vel0"]
    S = int(g["trace_steps"])
    tr = []
    T_d = 1.0 / float(g["Gamma"])
    for it in range(S):
        pos, vel, acc, U = th.vscale(pos, vel, acc, T_d, 1, it, float(g["dt"]), N, 3, Lv, Lv,
                                     np.zeros(3), k, a, rc, 1 / 3, 1.0, 1.5, Z, *args)
        tr.append([U, 1.5 * np.sum(vel ** 2)])
    for _ in range(S):
        pos, vel, acc, U = vv.update(pos, vel, acc, float(g["dt"]), 1, k, N, 3, Lv, Lv, np.zeros(3),
                                     a, rc, 1 / 3, 1.0, Z, *args)
        tr.append([U, 1.5 * np.sum(vel ** 2)])
    np.testing.assert_allclose(np.array(tr), g["trace"], rtol=1e-9)
    out = capsys.readouterr().out
    assert "U_short, U_long, U_self =" in out


def test_reference_modules_pp_pm(golden):
    import yukawa_pm_ord6
    import yukawa_pp
    from p3m_b200 import set_compat_precision

    set_compat_precision("fp64")
    g = golden
    N, M, L = int(g["N"]), int(g["M"]), float(g["L"])
    h = L / M
    acc = np.zeros((N, 3))
    U, acc2 = yukawa_pp.particle_particle(float(g["kappa"]), float(g["alpha"]), float(g["rc"]),
                                          np.array([L] * 3), g["pos0"], acc)
    assert acc2 is acc
    assert U == pytest.approx(float(g["U_pp"]), rel=1e-12)
    rho = np.zeros((M, M, M))
    out = yukawa_pm_ord6.charge_assgn_6_numba(rho, g["pos0"], np.ones(N), N, M, M, M, h, h, h)
    assert out is rho and np.max(np.abs(rho - g["rho"])) < 1e-11 * np.max(np.abs(g["rho"]))
    kx, ky, kz = golden_kvecs(g)
    Ex, Ey, Ez = np.zeros(N), np.zeros(N), np.zeros(N)
    Uf, accf = yukawa_pm_ord6.particle_mesh_fft_r(
        float(g["kappa"]), float(g["alpha"]), g["pos0"], np.ones(N), N, g["G_k"], kx, ky, kz, M, M,
        M, h, h, h, L, L, L, 6, 3, 3, 3, np.zeros((M, M, M)), np.zeros((N, 3)), Ex, Ey, Ez)
    assert Uf == pytest.approx(float(g["U_pm"]), rel=1e-9)
    assert rel_rms(np.stack([Ex, Ey, Ez]), g["E_p"]) < 1e-9


def test_nqt(golden, prec):
    g = golden
    with _ctx(g, prec) as c:
        nq = c.nqt(g["pos_final"], g["qv"])
    ref = g["nq_final"]
    scale = np.sqrt(int(g["N"]))
    assert np.max(np.abs(nq - ref)) < (1e-9 if prec == 0 else 2e-3) * scale
