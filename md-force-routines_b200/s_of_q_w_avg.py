"""S(q,w) of several runs -- drop-in for the reference's s_of_q_w_avg.py
(s_of_q_w_avg_mat, :5-20): for runs j < N_avg and q columns 3i (i < Nq), the
mean over axes of n_of_q_w, written into sqw_mat[j, i, :]. All runs and
columns go to the device in one call."""
from p3m_b200 import sqw_runs


def s_of_q_w_avg_mat(n_q_t_array, Nq, sqw_mat, N_avg, N, dt, T):
    """n_q_t_array (>= N_avg, Nt, >= 3 Nq, 3) complex; fills and returns
    sqw_mat (N_avg, Nq, Nt)."""
    sqw_mat[:N_avg] = sqw_runs(n_q_t_array[:N_avg], Nq, N, dt, T, col0=0, col_stride=3)
    return sqw_mat
