"""Velocity-rescaling thermostat step -- drop-in for the reference's
thermostat_p3m_ord6.py (vscale, :5-25): one velocity-Verlet step, then
T = kf sum v^2 / kf / N and v *= sqrt(T_d/T) for it <= 1999, otherwise
v *= sqrt((20 T_d/T - 1)/20), all on the device."""
import numpy as np

from velocity_verlet_p3m_ord6 import _check_box, _context

#: print "dt*it, T" on every call, as the reference does (:13)
VERBOSE = True


def vscale(pos, vel, acc, T_desired, PBC, it, dt, N, d, Lv, Lmax_v, Lmin_v, kappa, G, rc, af, uf,
           kf, Z, G_k, kx_v, ky_v, kz_v, Mx, My, Mz, hx, hy, hz, Lx, Ly, Lz, p, mx_max, my_max,
           mz_max, acc_s_r, acc_fft, rho_r, E_x_p, E_y_p, E_z_p):
    """-> (pos, vel, acc, U) as NEW arrays."""
    L = _check_box(PBC, Lv, Lmax_v, Lmin_v)
    ctx = _context(N, L, kappa, G, rc, dt, af, uf, Mx, My, Mz, p, mx_max, G_k,
                   T_desired=T_desired, kf=kf)
    pos = np.array(pos, dtype=np.float64, order="C")
    vel = np.array(vel, dtype=np.float64, order="C")
    acc = np.array(acc, dtype=np.float64, order="C")
    U, T = ctx.vscale(it, pos, vel, acc)
    if VERBOSE:
        print(dt * it, T)
    return pos, vel, acc, U
