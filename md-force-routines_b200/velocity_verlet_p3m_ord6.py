"""Velocity-Verlet step -- drop-in for the reference's
velocity_verlet_p3m_ord6.py (update, :5-26), run on the device: half kick,
drift, single periodic wrap, P3M force, half kick."""
import numpy as np

from p3m_b200.context import compat_context


def _check_box(PBC, Lv, Lmax_v, Lmin_v):
    if int(PBC) != 1:
        raise NotImplementedError("only periodic boundaries (PBC == 1) are supported")
    L = float(Lv[0])
    if not (np.all(np.asarray(Lv) == L) and np.all(np.asarray(Lmax_v) == L)
            and np.all(np.asarray(Lmin_v) == 0.0)):
        raise ValueError("expected a cubic box [0, L)^3")
    return L


def _context(N, L, kappa, G, rc, dt, af, uf, Mx, My, Mz, p, mx_max, G_k, T_desired=0.01, kf=1.5):
    if not (Mx == My == Mz):
        raise ValueError("only cubic meshes are supported")
    ctx = compat_context(N, L, kappa, G, rc, M=int(Mx), dt=dt, T_desired=T_desired, af=af, uf=uf,
                         kf=kf, p=p, m_alias=mx_max)
    ctx.set_green_cached(G_k)
    return ctx


def update(pos, vel, acc, dt, PBC, kappa, N, d, Lv, Lmax_v, Lmin_v, G, rc, acc_fact, U_fact, Z,
           G_k, kx_v, ky_v, kz_v, Mx, My, Mz, hx, hy, hz, Lx, Ly, Lz, p, mx_max, my_max, mz_max,
           acc_s_r, acc_fft, rho_r, E_x_p, E_y_p, E_z_p):
    """-> (pos, vel, acc, U) as NEW arrays (the inputs are not modified)."""
    L = _check_box(PBC, Lv, Lmax_v, Lmin_v)
    ctx = _context(N, L, kappa, G, rc, dt, acc_fact, U_fact, Mx, My, Mz, p, mx_max, G_k)
    pos = np.array(pos, dtype=np.float64, order="C")
    vel = np.array(vel, dtype=np.float64, order="C")
    acc = np.array(acc, dtype=np.float64, order="C")
    U = ctx.update(pos, vel, acc)
    return pos, vel, acc, U
