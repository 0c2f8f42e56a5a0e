"""Device status paths raised from host-made inputs: neighbour-list overflow
and non-finite velocities. Neither needs a device fault: the kernels check,
raise a status bit and carry on with in-bounds work; the host turns the bit
into P3MError, and the context stays usable.

The reference checks none of this (yukawa_pp.py:46-52 indexes its cell grid
without bounds checks; a NaN in velocity_verlet_p3m_ord6.py:7-19 propagates
silently).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 2000
L = (4 * np.pi * N / 3) ** (1 / 3)


def _state(seed=3):
    import initialize_pos_vel

    pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
    initialize_pos_vel.initial(seed, N, [L] * 3, pos, vel, 0.01)
    return pos, vel


def _replica():
    from p3m_b200 import Replica

    return Replica(N=N, L=L, kappa=1.0, alpha=0.7, rc=L / 3.2, M=32, dt=0.1, T_desired=0.01)


def _clustered(pos, count, radius, seed=0):
    """The first `count` particles moved into a ball of `radius` at the box
    centre: each of them then has about count - 1 neighbours."""
    rng = np.random.default_rng(seed)
    p = pos.copy()
    d = rng.normal(size=(count, 3))
    d *= (radius * rng.random(count) ** (1 / 3) / np.linalg.norm(d, axis=1))[:, None]
    p[:count] = 0.5 * L + d
    return p


@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_list_overflow_raises_and_context_recovers(prec_name):
    from p3m_b200 import FP32, FP64, Context, P3MError

    prec = {"fp32": FP32, "fp64": FP64}[prec_name]
    pos, _ = _state()
    with Context(_replica(), precision=prec) as c:
        _, _, maxnb = c.pp_config()
        dense = _clustered(pos, maxnb + 200, 1.5)
        with pytest.raises(P3MError) as e:
            c.force(dense)
        assert e.value.code == -7
        U, acc, _ = c.force(pos)  # a uniform state goes through on the same context
        assert np.isfinite(U) and np.all(np.isfinite(acc))


def test_list_overflow_in_device_run():
    from p3m_b200 import FP32, MODE_NVE, Context, P3MError

    pos, vel = _state()
    with Context(_replica(), precision=FP32) as c:
        _, _, maxnb = c.pp_config()
        c.set_state(0, _clustered(pos, maxnb + 200, 1.5), vel)
        with pytest.raises(P3MError) as e:
            c.init_forces()
            c.run(2, MODE_NVE)
        assert e.value.code == -7


@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_nonfinite_velocity_raises(prec_name):
    from p3m_b200 import FP32, FP64, MODE_NVE, Context, P3MError

    prec = {"fp32": FP32, "fp64": FP64}[prec_name]
    pos, vel = _state()
    with Context(_replica(), precision=prec) as c:
        c.set_state(0, pos, vel)
        c.init_forces()
        c.run(2, MODE_NVE)
        p, v, a = c.get_state(0)
        v[11, 1] = np.nan
        c.set_state(0, p, v, a)
        with pytest.raises(P3MError) as e:
            c.run(1, MODE_NVE)
        assert e.value.code == -5
        # a finite state runs again on the same context
        c.set_state(0, pos, vel)
        c.init_forces()
        c.run(2, MODE_NVE)
        c.check()
        assert np.all(np.isfinite(c.get_state(0)[0]))


def test_nonfinite_charge_rejected_on_host():
    from p3m_b200 import FP64, Context, P3MError

    pos, _ = _state()
    Z = np.ones(N)
    Z[5] = np.nan
    with Context(_replica(), precision=FP64) as c:
        with pytest.raises(P3MError) as e:
            c.force(pos, Z)
        assert e.value.code == -1
        U, _, _ = c.force(pos, np.ones(N))
        assert np.isfinite(U)
