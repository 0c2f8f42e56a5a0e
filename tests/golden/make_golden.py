"""Generate the golden vectors in this directory from the reference's own code.

Run where the reference tree is present, naming it in $P3M_REFERENCE_DIR:

    P3M_REFERENCE_DIR=<reference tree> python tests/golden/make_golden.py

It imports the reference's numba modules unchanged, with two shims:
``numba.autojit`` (removed from numba) is aliased to ``numba.jit``, and a
stand-in ``pyfftw`` module whose builders return numpy.fft calls (pyFFTW is not
installed). The Python-2 driver-level modules (yukawa_p3m_ord6,
velocity_verlet_p3m_ord6, thermostat_p3m_ord6) are loaded with their ``print``
statements rewritten as calls and their output discarded; nothing else is
changed. No file is written into the reference tree (bytecode writing is off).

The outputs (``*.npz``) are the fixtures the oracle is pinned against; they
are small (a few hundred KB) and committed. Nothing at test time reads the
reference tree.
"""
from __future__ import annotations

import contextlib
import io
import os
import re
import sys
import types

sys.dont_write_bytecode = True

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("P3M_REFERENCE_DIR", "")


def _install_shims():
    import numba

    if not hasattr(numba, "autojit"):
        numba.autojit = numba.jit
    fake = types.ModuleType("pyfftw")
    fake.builders = types.SimpleNamespace(
        fftn=lambda a: (lambda: np.fft.fftn(a)),
        ifftn=lambda a: (lambda: np.fft.ifftn(a)),
    )
    sys.modules["pyfftw"] = fake
    sys.modules["pyfftw.builders"] = fake.builders


_PRINT = re.compile(r"^(\s*)print\s+(?!\()(.*)$")


def _load_py2(name):
    """Load a reference module whose only Python-2 construct is the print
    statement, rewriting ``print a, b`` into ``print(a, b)``."""
    src = open(os.path.join(REF, name + ".py")).read()
    lines = [_PRINT.sub(r"\1print(\2)", ln) for ln in src.splitlines()]
    mod = types.ModuleType(name)
    mod.__file__ = os.path.join(REF, name + ".py")
    sys.modules[name] = mod
    exec(compile("\n".join(lines) + "\n", mod.__file__, "exec"), mod.__dict__)
    return mod


def load_reference():
    _install_shims()
    sys.path.insert(0, REF)
    import initialize_pos_vel
    import s_of_q_w
    import yukawa_gf_opt
    import yukawa_pm_ord6
    import yukawa_pp

    p3m = _load_py2("yukawa_p3m_ord6")
    vv = _load_py2("velocity_verlet_p3m_ord6")
    th = _load_py2("thermostat_p3m_ord6")
    return types.SimpleNamespace(
        initial=initialize_pos_vel.initial, pp=yukawa_pp.particle_particle,
        assign=yukawa_pm_ord6.charge_assgn_6_numba, gather=yukawa_pm_ord6.field_assgn_6_numba,
        pm=yukawa_pm_ord6.particle_mesh_fft_r, gf_opt=yukawa_gf_opt.gf_opt,
        force_pot=p3m.force_pot, update=vv.update, vscale=th.vscale, sqw=s_of_q_w.n_of_q_w)


# name: (N, Gamma, kappa, alpha, rc, M, seed, dt)
CASES = {
    "n500_m32": (500, 100.0, 1.0, 0.8, 4.0, 32, 11, 0.1),
    "n2000_m32": (2000, 100.0, 2.0, 0.6, 6.0, 32, 1, 0.1),
}
TRACE_STEPS = 6  # thermostat steps, then the same number of NVE steps


def make_case(R, name, N, Gamma, kappa, alpha, rc, M, seed, dt):
    L = (4.0 * np.pi * N / 3.0) ** (1.0 / 3.0)
    Lv = np.array([L, L, L])
    h = L / M
    T_d = 1.0 / Gamma
    pos = np.zeros((N, 3))
    vel = np.zeros((N, 3))
    pos, vel = R.initial(seed, N, Lv, pos, vel, T_d)
    pos0, vel0 = pos.copy(), vel.copy()
    Z = np.ones(N)

    U_pp, acc_pp = R.pp(kappa, alpha, rc, Lv, pos, np.zeros((N, 3)))
    acc_pp = acc_pp.copy()
    rho = R.assign(np.zeros((M, M, M)), pos, Z, N, M, M, M, h, h, h).copy()
    G_k, kx_v, ky_v, kz_v, A_pm = R.gf_opt(kappa, alpha, 6, 3, 3, 3, M, M, M, h, h, h, L, L, L)
    Exp, Eyp, Ezp = np.zeros(N), np.zeros(N), np.zeros(N)
    U_pm, acc_pm = R.pm(kappa, alpha, pos, Z, N, G_k, kx_v, ky_v, kz_v, M, M, M, h, h, h,
                        L, L, L, 6, 3, 3, 3, np.zeros((M, M, M)), np.zeros((N, 3)),
                        Exp, Eyp, Ezp)
    acc_pm = acc_pm.copy()
    E_p = np.stack([Exp, Eyp, Ezp]).copy()

    # A gather on a known (non-physical) mesh pins the gather on its own.
    rng = np.random.default_rng(seed + 1000)
    Em = [rng.standard_normal((M, M, M)) for _ in range(3)]
    acc_g = R.gather(np.zeros((N, 3)), np.zeros(N), np.zeros(N), np.zeros(N),
                     Em[0], Em[1], Em[2], pos, Z, N, M, M, M, h, h, h).copy()

    scratch = dict(acc_s_r=np.zeros((N, 3)), acc_fft=np.zeros((N, 3)),
                   rho_r=np.zeros((M, M, M)), E_x_p=np.zeros(N), E_y_p=np.zeros(N),
                   E_z_p=np.zeros(N))
    af, uf, kf = 1.0 / 3.0, 1.0, 1.5
    sink = io.StringIO()
    with contextlib.redirect_stdout(sink):
        U0, acc = R.force_pot(kappa, alpha, N, rc, Lv, af, uf, pos, np.zeros((N, 3)), Z, G_k,
                              kx_v, ky_v, kz_v, M, M, M, h, h, h, L, L, L, 6, 3, 3, 3,
                              *scratch.values())
        acc0 = acc.copy()
        Lmax, Lmin = Lv.copy(), np.zeros(3)
        trace = []
        for it in range(TRACE_STEPS):
            pos, vel, acc, U = R.vscale(pos, vel, acc, T_d, 1, it, dt, N, 3, Lv, Lmax, Lmin,
                                        kappa, alpha, rc, af, uf, kf, Z, G_k, kx_v, ky_v, kz_v,
                                        M, M, M, h, h, h, L, L, L, 6, 3, 3, 3,
                                        *scratch.values())
            trace.append([U, kf * np.sum(vel ** 2)])
        for it in range(TRACE_STEPS):
            pos, vel, acc, U = R.update(pos, vel, acc, dt, 1, kappa, N, 3, Lv, Lmax, Lmin,
                                        alpha, rc, af, uf, Z, G_k, kx_v, ky_v, kz_v, M, M, M,
                                        h, h, h, L, L, L, 6, 3, 3, 3, *scratch.values())
            trace.append([U, kf * np.sum(vel ** 2)])

    # n(q,t) on the final positions with the driver's q list, and S(q,w) of a
    # short synthetic n(q,t) series through the reference's n_of_q_w.
    dq = 2.0 * np.pi / L
    Nq = 3 * int(2.5 / dq)
    qv = np.zeros(Nq)
    for iqv in range(0, Nq, 3):
        iq = iqv / 3.0
        qv[iqv] = (iq + 1.0) * dq
        qv[iqv + 1] = (iq + 1.0) * np.sqrt(2.0) * dq
        qv[iqv + 2] = (iq + 1.0) * np.sqrt(3.0) * dq
    nq = np.zeros((Nq, 3), dtype=np.complex128)
    for iqv in range(Nq):
        for ax in range(3):
            nq[iqv, ax] = np.sum(np.exp(-1j * qv[iqv] * pos[:, ax]))
    nqt_series = (rng.standard_normal((64, 3)) + 1j * rng.standard_normal((64, 3)))
    sqw = R.sqw(nqt_series, N, dt, 64 * dt)

    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(
        out, N=N, Gamma=Gamma, kappa=kappa, alpha=alpha, rc=rc, M=M, seed=seed, dt=dt, L=L,
        pos0=pos0, vel0=vel0, U_pp=U_pp, acc_pp=acc_pp, rho=rho, G_k=G_k, A_pm=A_pm,
        U_pm=U_pm, acc_pm=acc_pm, E_p=E_p, acc_gather=acc_g,
        U0=U0, acc0=acc0, trace=np.array(trace), trace_steps=TRACE_STEPS,
        pos_final=pos, vel_final=vel, acc_final=acc, qv=qv, nq_final=nq,
        nqt_series=nqt_series, sqw=sqw)
    print("wrote", out, os.path.getsize(out), "bytes")


def main():
    if not REF or not os.path.isdir(REF):
        raise SystemExit("set P3M_REFERENCE_DIR to the reference tree")
    R = load_reference()
    for name, args in CASES.items():
        make_case(R, name, *args)


if __name__ == "__main__":
    main()
