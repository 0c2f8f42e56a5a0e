"""Optimal influence function -- drop-in for the reference's yukawa_gf_opt.py
(gf_opt, yukawa_gf_opt.py:5-98), computed in FP64 by an sm_100a kernel."""
import numpy as np

from p3m_b200.context import gf_opt_device


def _mid(M):
    return M // 2 if M % 2 == 0 else (M - 1) // 2


def gf_opt(kappa, Gew, p, mx_max, my_max, mz_max, Mx, My, Mz, hx, hy, hz, Lx, Ly, Lz):
    """-> (G_k, kx_v, ky_v, kz_v, A_pm), as yukawa_gf_opt.py:5.

    G_k is (Mz,My,Mx) in the fftshifted layout (index n <-> k = 2 pi (n - M/2)/L);
    kx_v (1,Mx), ky_v (My,1), kz_v (Mz,1,1) are the broadcastable wave-vector
    components (:27-33). The GPU path needs a cubic mesh and box and equal
    alias ranges.
    """
    if not (Mx == My == Mz and Lx == Ly == Lz and mx_max == my_max == mz_max):
        raise ValueError("gf_opt: only cubic meshes/boxes with equal alias ranges are supported")
    M, L = int(Mx), float(Lx)
    G_k, A_pm = gf_opt_device(kappa, Gew, int(p), int(mx_max), M, L)
    kx_v = 2 * np.pi * (np.arange(Mx).reshape((1, Mx)) - _mid(Mx)) / Lx
    ky_v = 2 * np.pi * (np.arange(My).reshape((My, 1)) - _mid(My)) / Ly
    kz_v = 2 * np.pi * (np.arange(Mz).reshape((Mz, 1, 1)) - _mid(Mz)) / Lz
    return G_k, kx_v, ky_v, kz_v, A_pm
