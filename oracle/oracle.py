"""CPU oracle for the P3M force step and integrator -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``, the smoke check
in ``__graft_entry__.py`` and the CPU-baseline leg of ``bench.py`` import it.
The product path (``md-force-routines_b200``) never imports anything under
``oracle/`` and fails loudly when its CUDA library is missing.

It restates, in Python 3 + numpy over the plain-C kernels of ``oracle.c``, the
FP64 algorithm of the reference (xgdhar/MD-force-routines):

* ``pp``           yukawa_pp.py:6-139            (C: oracle_pp)
* ``assign6``      yukawa_pm_ord6.py:6-95         (C: oracle_assign6)
* ``gather6``      yukawa_pm_ord6.py:213-312      (C: oracle_gather6)
* ``pm``           yukawa_pm_ord6.py:440-484      (numpy FFT chain)
* ``gf_opt``       yukawa_gf_opt.py:5-98          (C: oracle_gf_opt)
* ``gf_opt_points`` the same at chosen k points   (C: oracle_gf_opt_points)
* ``force_pot``    yukawa_p3m_ord6.py:6-29
* ``update``       velocity_verlet_p3m_ord6.py:5-26
* ``vscale``       thermostat_p3m_ord6.py:5-25
* ``nqt``          yukawa_MD_p3m_ord6.py:121-137, 214-219
* ``sqw``          s_of_q_w.py:3-20 and s_of_q_w_avg.py:5-20

Pinning: ``tests/golden/*.npz`` hold the reference's own numba outputs on the
same inputs (generated by ``tests/golden/make_golden.py``); the tests check
this restatement against them. The reference's FFT goes through pyFFTW (FFTW
>= 3.3, no pinned version); neither is installed here, so the FFT step here and
in the golden vectors is numpy.fft (pocketfft) -- that library boundary is
the one place where parity is unpinned.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    """Compile oracle.c into liboracle.so (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.oracle_pp.argtypes = [ctypes.c_int, dp, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, dp, dp]
        lib.oracle_pp.restype = ctypes.c_int
        lib.oracle_assign6.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, dp]
        lib.oracle_assign6.restype = ctypes.c_int
        lib.oracle_gather6.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, dp, dp, dp, dp, dp]
        lib.oracle_gather6.restype = ctypes.c_int
        lib.oracle_gf_opt.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      dp, dp]
        lib.oracle_gf_opt.restype = None
        lib.oracle_gf_opt_points.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_int), dp]
        lib.oracle_gf_opt_points.restype = None
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def pp(kappa, G, rc, Lv, pos):
    """yukawa_pp.py:6-139 -> (U_s_r, acc_s_r)."""
    pos = _c64(pos)
    n = pos.shape[0]
    acc = np.zeros((n, 3))
    U = np.zeros(1)
    st = _load().oracle_pp(n, _p(pos), float(Lv[0]), float(Lv[1]), float(Lv[2]),
                           float(kappa), float(G), float(rc), _p(acc), _p(U))
    if st != 0:
        raise ValueError("oracle_pp: particle outside the cell grid")
    return float(U[0]), acc


def assign6(pos, Z, Mx, My, Mz, hx, hy, hz):
    """yukawa_pm_ord6.py:6-95 -> rho_r (Mz,My,Mx)."""
    pos, Z = _c64(pos), _c64(Z)
    rho = np.zeros((Mz, My, Mx))
    st = _load().oracle_assign6(pos.shape[0], _p(pos), _p(Z), Mx, My, Mz, hx, hy, hz, _p(rho))
    if st != 0:
        raise ValueError("oracle_assign6: particle outside [-L, 2L)")
    return rho


def gather6(pos, Z, Mx, My, Mz, hx, hy, hz, Ex, Ey, Ez):
    """yukawa_pm_ord6.py:213-312 -> (acc (N,3), E_p (3,N))."""
    pos, Z = _c64(pos), _c64(Z)
    Ex, Ey, Ez = _c64(Ex), _c64(Ey), _c64(Ez)
    n = pos.shape[0]
    acc = np.zeros((n, 3))
    Ep = np.zeros((3, n))
    st = _load().oracle_gather6(n, _p(pos), _p(Z), Mx, My, Mz, hx, hy, hz,
                                _p(Ex), _p(Ey), _p(Ez), _p(acc), _p(Ep))
    if st != 0:
        raise ValueError("oracle_gather6: particle outside [-L, 2L)")
    return acc, Ep


def gf_opt(kappa, Gew, p, mx_max, my_max, mz_max, Mx, My, Mz, hx, hy, hz, Lx, Ly, Lz):
    """yukawa_gf_opt.py:5-98 -> (G_k, kx_v, ky_v, kz_v, A_pm)."""
    G_k = np.zeros((Mz, My, Mx))
    A = np.zeros(1)
    _load().oracle_gf_opt(kappa, Gew, p, mx_max, my_max, mz_max, Mx, My, Mz,
                          hx, hy, hz, Lx, Ly, Lz, _p(G_k), _p(A))
    nx_mid = Mx // 2 if Mx % 2 == 0 else (Mx - 1) // 2
    ny_mid = My // 2 if My % 2 == 0 else (My - 1) // 2
    nz_mid = Mz // 2 if Mz % 2 == 0 else (Mz - 1) // 2
    kx_v = 2 * np.pi * (np.arange(Mx).reshape((1, Mx)) - nx_mid) / Lx
    ky_v = 2 * np.pi * (np.arange(My).reshape((My, 1)) - ny_mid) / Ly
    kz_v = 2 * np.pi * (np.arange(Mz).reshape((Mz, 1, 1)) - nz_mid) / Lz
    return G_k, kx_v, ky_v, kz_v, float(A[0])


def gf_opt_points(kappa, Gew, p, m_max, M, L, idx):
    """yukawa_gf_opt.py:5-98 on a cubic M^3 mesh at chosen points only:
    idx (n, 3) integer (nz, ny, nx) of the fftshifted layout -> G_k there
    (same arithmetic as gf_opt, point by point)."""
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    out = np.zeros(idx.shape[0])
    _load().oracle_gf_opt_points(float(kappa), float(Gew), int(p), int(m_max), int(M),
                                 float(L) / M, float(L), idx.shape[0],
                                 idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _p(out))
    return out


def pm_fields(pos, Z, G_k, kx_v, ky_v, kz_v, Mx, My, Mz, hx, hy, hz, Lx, Ly, Lz):
    """The mesh part of yukawa_pm_ord6.py:440-480: returns (U_f, rho, E_x, E_y, E_z).

    assign (:445) -> fftn + fftshift (:447-449) -> phi = G_k rho_k (:451) ->
    U_f = 1/2 sum |rho_k|^2 G_k / V (:453-457) -> E_k = -i k phi (:459-461) ->
    ifftshift + ifftn (:463-472) -> scale M^3/V and real part (:474-480).
    """
    V = Lx * Ly * Lz
    M_V = Mx * My * Mz
    rho = assign6(pos, Z, Mx, My, Mz, hx, hy, hz)
    rho_k = np.fft.fftshift(np.fft.fftn(rho))
    phi_k = G_k * rho_k
    rho_k_sq = np.real(rho_k) * np.real(rho_k) + np.imag(rho_k) * np.imag(rho_k)
    U_f = 0.5 * np.sum(rho_k_sq * G_k) / V
    E = []
    for kv in (kx_v, ky_v, kz_v):
        E_k = -1j * kv * phi_k
        E_r = np.fft.ifftn(np.fft.ifftshift(E_k))
        E.append(np.real(M_V * E_r / V))
    return float(U_f), rho, E[0], E[1], E[2]


def pm(pos, Z, G_k, kx_v, ky_v, kz_v, Mx, My, Mz, hx, hy, hz, Lx, Ly, Lz):
    """yukawa_pm_ord6.py:440-484 (particle_mesh_fft_r) -> (U_f, acc_f, E_p)."""
    U_f, _, Ex, Ey, Ez = pm_fields(pos, Z, G_k, kx_v, ky_v, kz_v, Mx, My, Mz,
                                   hx, hy, hz, Lx, Ly, Lz)
    acc, Ep = gather6(pos, Z, Mx, My, Mz, hx, hy, hz, Ex, Ey, Ez)
    return U_f, acc, Ep


class Params:
    """The run constants the reference's driver passes down the call stack
    (yukawa_MD_p3m_ord6.py:26-79)."""

    def __init__(self, N, kappa, G, rc, M, L=None, Gamma=1.0, dt=0.1, p=6, m_max=3,
                 af=1.0 / 3.0, uf=1.0, kf=1.5):
        self.N = int(N)
        self.L = float(L) if L is not None else (4.0 * np.pi * N / 3.0) ** (1.0 / 3.0)
        self.Lv = np.array([self.L] * 3)
        self.kappa, self.G, self.rc = float(kappa), float(G), float(rc)
        self.M = int(M)
        self.h = self.L / self.M
        self.Gamma = float(Gamma)
        self.T_desired = 1.0 / self.Gamma
        self.dt = float(dt)
        self.p, self.m_max = int(p), int(m_max)
        self.af, self.uf, self.kf = af, uf, kf
        self.Z = np.ones(self.N)
        self._gk = None

    def green(self):
        if self._gk is None:
            M, h, L = self.M, self.h, self.L
            self._gk = gf_opt(self.kappa, self.G, self.p, self.m_max, self.m_max,
                              self.m_max, M, M, M, h, h, h, L, L, L)
        return self._gk


def force_pot(P: Params, pos):
    """yukawa_p3m_ord6.py:6-29 -> (U, acc, (U_short, U_fft, U_self)).

    acc = af*(acc_pp + acc_pm) (:21), U = uf*(U_short+U_fft+U_self) with
    U_self = -N G / sqrt(pi) (:23-24).
    """
    G_k, kx_v, ky_v, kz_v, _ = P.green()
    U_short, acc_s_r = pp(P.kappa, P.G, P.rc, P.Lv, pos)
    M, h, L = P.M, P.h, P.L
    U_fft, acc_fft, _ = pm(pos, P.Z, G_k, kx_v, ky_v, kz_v, M, M, M, h, h, h, L, L, L)
    acc = P.af * (acc_s_r + acc_fft)
    U_self = -P.N * P.G / np.sqrt(np.pi)
    U = P.uf * (U_short + U_fft + U_self)
    return U, acc, (U_short, U_fft, U_self)


def wrap(P: Params, pos):
    """Single periodic wrap of velocity_verlet_p3m_ord6.py:12-19 (vectorised;
    the same comparisons in the same order per element)."""
    pos = pos.copy()
    L = P.Lv
    hi = pos > L[None, :]
    pos[hi] = (pos - L[None, :])[hi]
    lo = pos < 0.0
    pos[lo] = (pos + L[None, :])[lo]
    return pos


def update(P: Params, pos, vel, acc):
    """velocity_verlet_p3m_ord6.py:5-26 -> (pos, vel, acc, U)."""
    vel = vel + 0.5 * acc * P.dt
    pos = pos + vel * P.dt
    pos = wrap(P, pos)
    U, acc, _ = force_pot(P, pos)
    vel = vel + 0.5 * acc * P.dt
    return pos, vel, acc, U


def vscale(P: Params, pos, vel, acc, it):
    """thermostat_p3m_ord6.py:5-25 -> (pos, vel, acc, U, T).

    T = kf*sum(v^2)/kf/N; for it <= 1999 v *= sqrt(T_d/T), otherwise
    v *= sqrt((20 T_d/T - 1)/20).
    """
    pos, vel, acc, U = update(P, pos, vel, acc)
    K = P.kf * np.sum(vel ** 2)
    T = K / P.kf / float(P.N)
    if it <= 1999:
        fact = np.sqrt(P.T_desired / T)
    else:
        fact = np.sqrt((20.0 * P.T_desired / T - 1.0) / 20.0)
    vel = vel * fact
    return pos, vel, acc, U, T


def q_vectors_reference(L):
    """The q list of yukawa_MD_p3m_ord6.py:122-137: (iq+1) dq {1, sqrt2, sqrt3}."""
    dq = 2.0 * np.pi / L
    Nq = 3 * int(2.5 / dq)
    qv = np.zeros(Nq)
    for iqv in range(0, Nq, 3):
        iq = iqv / 3.0
        qv[iqv] = (iq + 1.0) * dq
        qv[iqv + 1] = (iq + 1.0) * np.sqrt(2.0) * dq
        qv[iqv + 2] = (iq + 1.0) * np.sqrt(3.0) * dq
    return qv


def nqt(pos, qv):
    """One row of n(q,t), yukawa_MD_p3m_ord6.py:215-219: n[iq, ax] =
    sum_i exp(-i q x_{i,ax}) -> complex128 (Nq, 3)."""
    out = np.zeros((len(qv), 3), dtype=np.complex128)
    for iq, q in enumerate(qv):
        for ax in range(3):
            out[iq, ax] = np.sum(np.exp(-1j * q * pos[:, ax]))
    return out


def sqw(n_q_t, N, dt, T):
    """s_of_q_w.py:3-20: S(q,w) = |dt FFT_t n(q,t)|^2/(N T) per axis -> (Nt, 3)."""
    out = np.zeros((n_q_t.shape[0], 3))
    for ax in range(3):
        out[:, ax] = np.absolute(np.fft.fft(n_q_t[:, ax]) * dt) ** 2 / (N * T)
    return out


def sqw_avg(n_q_t_array, Nq, N, dt, T, stride=3):
    """s_of_q_w_avg.py:5-20 plus the replica mean of s_of_q_w_script.py:37:
    mean over axes of sqw() on every ``stride``-th q column, then over runs."""
    R = n_q_t_array.shape[0]
    out = np.zeros((R, Nq, n_q_t_array.shape[1]))
    for j in range(R):
        for i in range(Nq):
            out[j, i, :] = np.mean(sqw(n_q_t_array[j][:, i * stride, :], N, dt, T), axis=1)
    return out.mean(axis=0)


# ---------------------------------------------------------------------------
# PPPM error estimates (the reference sets alpha, r_c and M by hand,
# yukawa_MD_p3m_ord6.py:52-68; its only error measure is A_pm,
# yukawa_gf_opt.py:96). Restated from the published methods, for checking the
# library's estimator.
# ---------------------------------------------------------------------------

_erfc_v = np.frompyfunc(math.erfc, 1, 1)


def pair_force_sr(r, kappa, alpha):
    """Radial short-range Yukawa-Ewald force -d phi/dr of
    phi = (1/2r)[e^{kr} erfc(ar + b) + e^{-kr} erfc(ar - b)], b = k/(2a)
    (yukawa_pp.py:115-124)."""
    r = np.asarray(r, dtype=np.float64)
    b = kappa / (2.0 * alpha)
    ep = np.exp(kappa * r) * _erfc_v(alpha * r + b).astype(np.float64)
    em = np.exp(-kappa * r) * _erfc_v(alpha * r - b).astype(np.float64)
    phi = 0.5 * (ep + em) / r
    return (phi / r - 0.5 * kappa * (ep - em) / r
            + 2.0 * alpha / (r * np.sqrt(np.pi)) * np.exp(-alpha * alpha * r * r - b * b))


def pp_error(N, L, kappa, alpha, rc, n_int=4000):
    """RMS per-particle force error of cutting the short-range force at r_c
    for N unit charges placed at random (Kolafa & Perram, Mol. Sim. 9 (1992)
    351, with the Yukawa-Ewald force): sqrt(4 pi n int_rc^inf F(r)^2 r^2 dr),
    n = N / L^3, by Simpson's rule on [r_c, sqrt(r_c^2 + 40/alpha^2)]."""
    n = N / L ** 3
    r_end = np.sqrt(rc * rc + 40.0 / (alpha * alpha))
    r = np.linspace(rc, r_end, n_int + 1)
    f = pair_force_sr(r, kappa, alpha) ** 2 * r * r
    w = np.ones(n_int + 1)
    w[1:-1:2] = 4.0
    w[2:-1:2] = 2.0
    integral = (r[1] - r[0]) / 3.0 * np.sum(w * f)
    return float(np.sqrt(4.0 * np.pi * n * integral))


def pm_error(N, L, kappa, alpha, M, p=6, m_max=3):
    """RMS per-particle PM force error with the optimal influence function
    (Hockney & Eastwood, Computer Simulation Using Particles, eq. 8-22):
    sqrt(N / V^2 sum_k [sum_m k_m^2 G_m^2 - A(k)]), G_m the Yukawa-Ewald
    long-range kernel 4 pi e^{-(kappa^2+k_m^2)/(4 alpha^2)}/(kappa^2+k_m^2),
    A(k) the term yukawa_gf_opt.py:92-94 sums into A_pm. Returns
    (dF_pm, A_pm)."""
    h = L / M
    s = np.arange(M) - M // 2
    kx = (2 * np.pi * s / L).reshape((1, 1, M))
    ky = (2 * np.pi * s / L).reshape((1, M, 1))
    kz = (2 * np.pi * s / L).reshape((M, 1, 1))
    ksq = kx * kx + ky * ky + kz * kz
    UG = np.zeros((M, M, M))
    Usq = np.zeros((M, M, M))
    R2 = np.zeros((M, M, M))

    def sinc(x):
        return np.where(x != 0.0, np.sin(0.5 * x * h) / np.where(x != 0.0, 0.5 * x * h, 1.0), 1.0)

    for mz in range(-m_max, m_max + 1):
        kmz = kz + 2 * np.pi * mz * M / L
        for my in range(-m_max, m_max + 1):
            kmy = ky + 2 * np.pi * my * M / L
            for mx in range(-m_max, m_max + 1):
                kmx = kx + 2 * np.pi * mx * M / L
                kmsq = kmx * kmx + kmy * kmy + kmz * kmz
                u2 = (sinc(kmx) * sinc(kmy) * sinc(kmz)) ** (2 * p)
                g = 4 * np.pi * np.exp(-0.25 * (kappa ** 2 + kmsq) / alpha ** 2) / (kappa ** 2 + kmsq)
                UG += u2 * g * (kx * kmx + ky * kmy + kz * kmz)
                Usq += u2
                R2 += kmsq * g * g
    nz = ksq != 0.0
    A = np.where(nz, UG ** 2 / np.where(nz, Usq ** 2 * ksq, 1.0), 0.0)
    Q = np.sum(np.where(nz, R2, 0.0)) - np.sum(A)
    V = L ** 3
    return float(np.sqrt(max(Q, 0.0) * N / (V * V))), float(np.sum(A))


def ewald_lr_acc(pos, L, kappa, alpha, kcut_exp=40.0):
    """Exact long-range field at each particle, E_i = -(1/V) sum_{k!=0}
    i k G(k) e^{i k.r_i} sum_j e^{-i k.r_j}, over all k with
    (k^2+kappa^2)/(4 alpha^2) < kcut_exp (the remainder is below e^-40)."""
    V = L ** 3
    kmax = 2.0 * alpha * np.sqrt(kcut_exp)
    nmax = int(np.ceil(kmax * L / (2 * np.pi)))
    n = np.arange(-nmax, nmax + 1)
    g = np.stack(np.meshgrid(n, n, n, indexing="ij"), -1).reshape(-1, 3).astype(np.float64)
    k = 2 * np.pi * g / L
    ksq = np.sum(k * k, axis=1)
    keep = (ksq > 0) & ((ksq + kappa ** 2) / (4 * alpha ** 2) < kcut_exp)
    k, ksq = k[keep], ksq[keep]
    G = 4 * np.pi * np.exp(-(ksq + kappa ** 2) / (4 * alpha ** 2)) / (ksq + kappa ** 2)
    acc = np.zeros_like(pos)
    for c0 in range(0, len(k), 2048):
        kc, Gc = k[c0:c0 + 2048], G[c0:c0 + 2048]
        ph = pos @ kc.T                       # (N, K)
        cs, sn = np.cos(ph), np.sin(ph)
        S_re, S_im = cs.sum(0), -sn.sum(0)    # S(k) = sum_j e^{-i k r_j}
        # Re(-i e^{i k r_i} S) = sin(k r_i) S_re + cos(k r_i) S_im
        w = (sn * S_re + cs * S_im) * Gc      # (N, K)
        acc += w @ kc
    return acc / V
