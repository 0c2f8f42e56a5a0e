"""S(q, omega) on the device against the oracle (s_of_q_w.py:3-20,
s_of_q_w_avg.py:5-20, s_of_q_w_script.py:37)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# FP64 FFTs of length <= 2^15 on O(1) data: a few ulps per stage of the
# largest spectral value; the bound below is far above that and far below
# any indexing or normalisation error.
RTOL = 1e-10


def _series(rng, nt, nq=1):
    return rng.standard_normal((nt, nq, 3)) + 1j * rng.standard_normal((nt, nq, 3))


def _close(got, ref):
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) <= RTOL * scale, np.max(np.abs(got - ref)) / scale


@pytest.mark.parametrize("nt", [1024, 1000, 16384, 16000, 3])
def test_series_matches_oracle(nt):
    """Power-of-two and Bluestein lengths, in shared memory (P <= 8192) and
    in the global-memory scratch (16384; 16000 -> P = 32768, the length of
    the reference's own S(q,w) script)."""
    import s_of_q_w

    rng = np.random.default_rng(nt)
    x = _series(rng, nt)[:, 0, :]
    N, dt = 10000.0, 0.05
    for T in (nt * dt, 123.0):
        got = s_of_q_w.n_of_q_w(x, N, dt, T)
        assert got.shape == (nt, 3)
        _close(got, O.sqw(x, N, dt, T))


def test_runs_match_oracle():
    import s_of_q_w_avg

    rng = np.random.default_rng(5)
    R, nt, nq, Nq = 3, 500, 10, 4
    arr = np.stack([_series(rng, nt, nq) for _ in range(R)])
    N, dt = 1000.0, 0.1
    T = nt * dt
    mat = np.zeros((R, Nq, nt))
    got = s_of_q_w_avg.s_of_q_w_avg_mat(arr, Nq, mat, R, N, dt, T)
    assert got is mat
    ref = np.zeros((R, Nq, nt))
    for j in range(R):
        for i in range(Nq):
            ref[j, i] = O.sqw(arr[j][:, 3 * i, :], N, dt, T).mean(axis=1)
    _close(got, ref)
    _close(got.mean(axis=0), O.sqw_avg(arr, Nq, N, dt, T))


def _init_state(r, seed):
    import initialize_pos_vel

    pos, vel = np.zeros((r.N, 3)), np.zeros((r.N, 3))
    initialize_pos_vel.initial(seed, r.N, [r.L] * 3, pos, vel, r.T_desired)
    return pos, vel


def test_ensemble_ring_matches_oracle():
    """Two replicas of different N record into a ring that wraps; S(q,w) of
    the last nt rows, every other q column, per replica and averaged."""
    from p3m_b200 import FP32, MODE_NVE, Context, Replica

    reps = []
    for N in (500, 800):
        L = (4 * np.pi * N / 3) ** (1 / 3)
        reps.append(Replica(N=N, L=L, kappa=1.0, alpha=0.7, rc=L / 3.0, M=32, dt=0.1))
    qmult = np.arange(1, 9, dtype=np.float64)
    cap, steps = 256, 300
    with Context(reps, precision=FP32) as c:
        for i, r in enumerate(reps):
            c.set_state(i, *_init_state(r, 11 + i))
        c.init_forces()
        c.set_nqt(qmult, cap)
        c.run(steps, MODE_NVE, record_nqt=True)
        series = [c.get_nqt(i, len(qmult)) for i in range(len(reps))]
        for nt in (256, 200):
            got, got_rep = c.sqw(0.1, nt, col0=1, col_stride=2, per_replica=True)
            assert got.shape == (4, nt) and got_rep.shape == (2, 4, nt)
            ref_rep = np.zeros((2, 4, nt))
            for j, r in enumerate(reps):
                s = series[j][-nt:]
                for i in range(4):
                    ref_rep[j, i] = O.sqw(s[:, 1 + 2 * i, :], r.N, 0.1, nt * 0.1).mean(axis=1)
            _close(got_rep, ref_rep)
            _close(got, ref_rep.mean(axis=0))
        with pytest.raises(Exception):
            c.sqw(0.1, cap + 1)
        with pytest.raises(Exception):
            c.sqw(0.1, 64, col0=8)
