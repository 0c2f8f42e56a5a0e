"""Particle-mesh (PM) part of the P3M force -- drop-in for the reference's
yukawa_pm_ord6.py (charge_assgn_6_numba :6-95, field_assgn_6_numba :213-312,
particle_mesh_fft_r :440-484, Efield_fourier :202-209).

Assignment, the 3-D FFTs, the influence-function multiply, ik differentiation,
the inverse FFTs and the gather run in libp3m_b200's sm_100a kernels.
"""
import numpy as np

from p3m_b200.context import compat_context


def _cubic(Mx, My, Mz, hx, hy, hz):
    if not (Mx == My == Mz and hx == hy == hz):
        raise ValueError("only cubic meshes are supported")
    return int(Mx), float(hx)


def _ctx(pos, M, h, kappa=0.0, alpha=1.0):
    L = M * h
    # the PP cut-off does not enter the mesh stages; any value giving >= 3
    # cells per side is accepted
    return compat_context(len(pos), L, kappa, alpha, L / 3.0, M=M)


def charge_assgn_6_numba(rho_r, pos, Z, N, Mx, My, Mz, hx, hy, hz):
    """Order-6 charge assignment onto rho_r[z,y,x] (filled in place and returned)."""
    M, h = _cubic(Mx, My, Mz, hx, hy, hz)
    rho_r[...] = _ctx(pos, M, h).assign(np.asarray(pos)[:N], None if Z is None else np.asarray(Z)[:N])
    return rho_r


def field_assgn_6_numba(acc, E_x_p, E_y_p, E_z_p, E_x_r, E_y_r, E_z_r, pos, Z, N, Mx, My, Mz,
                        hx, hy, hz):
    """Order-6 gather of the field meshes at the particles; fills E_*_p and acc = Z E."""
    M, h = _cubic(Mx, My, Mz, hx, hy, hz)
    a, Ep = _ctx(pos, M, h).gather(np.asarray(pos)[:N], np.asarray(Z)[:N], E_x_r, E_y_r, E_z_r)
    E_x_p[...] = Ep[0]
    E_y_p[...] = Ep[1]
    E_z_p[...] = Ep[2]
    acc[...] = a
    return acc


def Efield_fourier(phi_k, kx_v, ky_v, kz_v):
    """E_k = -i k phi_k per component (yukawa_pm_ord6.py:202-209; the
    reference's driver does not call it)."""
    return -1j * kx_v * phi_k, -1j * ky_v * phi_k, -1j * kz_v * phi_k


def particle_mesh_fft_r(kappa, G_ew, pos, Z, N, G_k, kx_v, ky_v, kz_v, Mx, My, Mz, hx, hy, hz,
                        Lx, Ly, Lz, p, mx_max, my_max, mz_max, rho_r, acc_f, E_x_p, E_y_p, E_z_p):
    """PM force and energy -> (U_f, acc_f), as yukawa_pm_ord6.py:440.

    acc_f, E_*_p and rho_r are filled in place like the reference's. ``G_k``
    (fftshifted, as returned by gf_opt) is installed on the device once and
    reused while the same array is passed.
    """
    M, h = _cubic(Mx, My, Mz, hx, hy, hz)
    ctx = _ctx(pos, M, h, kappa, G_ew)
    ctx.set_green_cached(G_k)
    U, a, Ep, rho = ctx.pm(np.asarray(pos)[:N], np.asarray(Z)[:N], want_rho=True)
    rho_r[...] = rho
    E_x_p[...] = Ep[0]
    E_y_p[...] = Ep[1]
    E_z_p[...] = Ep[2]
    acc_f[...] = a
    return U, acc_f
