"""P3M force facade -- drop-in for the reference's yukawa_p3m_ord6.py
(force_pot, yukawa_p3m_ord6.py:6-29): PP + PM in one device pass."""
import numpy as np

from p3m_b200.context import compat_context

#: print the three energy terms on every call, as the reference does (:27)
VERBOSE = True


def force_pot(kappa, G, N, rc, Lv, af, uf, pos, acc, Z, G_k, kx_v, ky_v, kz_v, Mx, My, Mz,
              hx, hy, hz, Lx, Ly, Lz, p, mx_max, my_max, mz_max, acc_s_r, acc_fft, rho_r,
              E_x_p, E_y_p, E_z_p):
    """-> (U, acc) with acc = af*(acc_pp + acc_pm) a NEW array and
    U = uf*(U_short + U_fft + U_self), U_self = -N G/sqrt(pi) (:21-24).

    The scratch arrays are zeroed as in the reference (:8-14); the device keeps
    its own copies of the intermediate results.
    """
    if not (Mx == My == Mz and Lx == Ly == Lz and mx_max == my_max == mz_max):
        raise ValueError("force_pot: only cubic meshes/boxes are supported")
    for a in (acc_s_r, acc_fft, rho_r, E_x_p, E_y_p, E_z_p):
        a.fill(0.0)
    ctx = compat_context(N, float(Lv[0]), kappa, G, rc, M=int(Mx), af=af, uf=uf, p=p,
                         m_alias=mx_max)
    ctx.set_green_cached(G_k)
    U, acc_new, (U_short, U_fft, U_self) = ctx.force(np.asarray(pos)[:N], np.asarray(Z)[:N])
    if VERBOSE:
        print('U_short, U_long, U_self =', [U_short, U_fft, U_self])
    return U, acc_new
