"""Host-side logic that needs no GPU."""
import numpy as np
import pytest

from conftest import have_gpu


def test_initial_state_bitexact(golden):
    import initialize_pos_vel

    g = golden
    N, L = int(g["N"]), float(g["L"])
    pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
    initialize_pos_vel.initial(int(g["seed"]), N, [L] * 3, pos, vel, 1.0 / float(g["Gamma"]))
    assert np.array_equal(pos, g["pos0"])
    assert np.array_equal(vel, g["vel0"])


def test_replica_desc_layout():
    import ctypes

    from p3m_b200._lib import ReplicaDesc

    assert ctypes.sizeof(ReplicaDesc) == 4 * 4 + 10 * 8


def test_non_cubic_rejected_before_device():
    import yukawa_pm_ord6

    with pytest.raises(ValueError):
        yukawa_pm_ord6.charge_assgn_6_numba(np.zeros((4, 4, 8)), np.zeros((3, 3)), np.ones(3), 3,
                                            8, 4, 4, 1.0, 1.0, 1.0)


@pytest.mark.skipif(have_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    import yukawa_pp
    from p3m_b200 import P3MError

    pos = np.random.default_rng(0).random((100, 3)) * 10.0
    with pytest.raises(P3MError):
        yukawa_pp.particle_particle(1.0, 0.8, 3.0, np.array([10.0] * 3), pos, np.zeros((100, 3)))
