"""Dynamic structure factor of one run -- drop-in for the reference's
s_of_q_w.py (n_of_q_w, :3-20): S(q,w) = |dt FFT_t n(q,t)|^2 / (N T) for each
of the three axes, computed on the device in FP64."""
from p3m_b200 import sqw_series


def n_of_q_w(n_q_t, N, dt, T):
    """(Nt, 3) complex n(q,t) of one q -> (Nt, 3) float S(q,w)."""
    return sqw_series(n_q_t, N, dt, T)
