"""The statistics of the accuracy statement (p3m_b200.validate), on
synthetic inputs with known answers: the force-error norms, the energy-drift
measures, the S(q, w) peak finder and its replica-bootstrap error bars. No
device: these are the host-side reductions of what the device runs return."""
import numpy as np
import pytest

from p3m_b200.validate import _bootstrap_peaks, _drift_stats, _force_errors, _sqw_peaks


def test_force_errors_per_replica():
    rng = np.random.default_rng(3)
    a64 = rng.normal(size=(300, 3))
    offs = [0, 100, 300]
    a32 = a64.copy()
    a32[:100] *= 1 + 1e-6                    # replica 0: a uniform relative error
    a32[150] += np.array([0.0, 0.0, 1e-3])   # replica 1: one particle off
    (rms0, max0), (rms1, max1) = _force_errors(a32, a64, offs)
    assert rms0 == pytest.approx(1e-6, rel=1e-6)
    # the largest per-particle error over the replica's RMS force
    y = a64[:100]
    assert max0 == pytest.approx(1e-6 * np.sqrt((y ** 2).sum(1).max() / (y ** 2).sum(1).mean()),
                                 rel=1e-6)
    y1 = a64[100:]
    assert rms1 == pytest.approx(1e-3 / np.sqrt((y1 ** 2).sum()), rel=1e-9)
    assert max1 == pytest.approx(1e-3 / np.sqrt((y1 ** 2).sum(1).mean()), rel=1e-9)
    assert _force_errors(a64, a64, offs) == [(0.0, 0.0), (0.0, 0.0)]


def test_drift_stats_separates_drift_from_fluctuation():
    T = 4000
    t = np.arange(1, T + 1, dtype=np.float64)
    E0 = np.array([-100.0, 50.0])
    K0 = np.array([2.0, 4.0])
    slope = np.array([1e-6, 0.0])
    wiggle = np.array([0.0, 1e-3]) * np.sin(t / 7.0)[:, None]  # replica 1: no drift, fluctuates
    E = E0[None, :] + slope[None, :] * t[:, None] + wiggle
    K = np.tile(K0, (T, 1)) * 1.01
    d = _drift_stats(E, K, E0, K0)
    assert d["fit_drift_rel_E0"][0] == pytest.approx(1e-6 * T / 100.0, rel=1e-6)
    # fluctuation only: the drift proper is far below the largest deviation
    assert d["fit_drift_rel_E0"][1] < 0.05 * d["max_abs_dev_rel_E0"][1]
    assert d["max_abs_dev_rel_E0"][0] == pytest.approx(1e-6 * T / 100.0, rel=1e-9)
    assert d["max_abs_dev_rel_E0"][1] == pytest.approx(1e-3 / 50.0, rel=1e-3)
    assert d["max_abs_dev_rel_K0"][1] == pytest.approx(1e-3 / 4.0, rel=1e-3)
    assert d["K_mean_rel_K0"] == pytest.approx([1.01, 1.01])


def test_sqw_peaks_skip_zero_and_negative_frequencies():
    nq, nw, dw = 3, 64, 0.25
    S = np.zeros((nq, nw))
    S[:, 0] = 100.0                       # w = 0 (excluded)
    S[:, nw - 3] = 50.0                   # negative frequencies (excluded)
    S[0, 5], S[1, 9], S[2, 31] = 2.0, 3.0, 4.0
    w, h = _sqw_peaks(S, dw)
    assert w.tolist() == [5 * dw, 9 * dw, 31 * dw]
    assert h.tolist() == [2.0, 3.0, 4.0]


def test_bootstrap_peaks_zero_for_identical_replicas():
    S1 = np.zeros((2, 32))
    S1[0, 4], S1[1, 7] = 1.0, 2.0
    sw, sh = _bootstrap_peaks(np.stack([S1] * 5), 0.5, n_boot=50)
    assert np.all(sw == 0.0) and np.all(sh == 0.0)


def test_bootstrap_peaks_spread_of_the_replica_mean():
    """Replica peaks of height 1 +- 0.1 at a fixed frequency: the bootstrap
    SD of the mean height is close to 0.1 / sqrt(R), the frequency's zero."""
    rng = np.random.default_rng(11)
    R = 40
    S = np.zeros((R, 1, 64))
    S[:, 0, 10] = 1.0 + 0.1 * rng.standard_normal(R)
    S[:, 0, 20] = 0.2
    sw, sh = _bootstrap_peaks(S, 1.0, n_boot=2000, seed=5)
    sd = S[:, 0, 10].std() / np.sqrt(R)
    assert sw[0] == 0.0
    assert sh[0] == pytest.approx(sd, rel=0.1)
