"""Host side of the driver's input and output files (no GPU)."""
import io as _io

import numpy as np

from oracle import oracle as O

IN_TEXT = """100.0      Gamma
1.5       kappa
2000       Number of particles
0.1      dt
5         Number of equilibration steps
12       Number of post-equilibration steps
1         Periodic boundary condition (1=yes, 0=no)
4        snapshot interval
0         intial conditions (1=file, 0=random)
1         write to output (irp.out) file (1=yes, 0=no)
1         write to Ovito (irp.xyz) file (1=yes, 0=no)
7       seed for random number generator for initial positions and velocities
"""


def test_read_input(tmp_path):
    from p3m_b200.io import read_input

    p = tmp_path / "yukawa_MD_p3m.in"
    p.write_text(IN_TEXT)
    d = read_input(str(p))
    assert d == {"Gamma": 100.0, "kappa": 1.5, "N": 2000, "dt": 0.1, "Neq": 5, "Nt": 12, "PBC": 1,
                 "snap_int": 4, "init": 0.0, "write_output": 1.0, "write_xyz": 1.0, "seed": 7}
    assert isinstance(d["N"], int) and isinstance(d["Gamma"], float)


def test_reference_q_list():
    from p3m_b200.io import reference_qmult

    for N in (2000, 10000, 10 ** 6):
        L = (4 * np.pi * N / 3) ** (1 / 3)
        q = reference_qmult(L) * 2 * np.pi / L
        ref = O.q_vectors_reference(L)
        assert q.shape == ref.shape
        np.testing.assert_allclose(q, ref, rtol=1e-15, atol=0)


def test_read_initial_conditions(tmp_path):
    import read

    rng = np.random.default_rng(1)
    rows = rng.standard_normal((7, 9))
    f = tmp_path / "init.out"
    np.savetxt(f, rows)
    pos, vel = read.initL(np.zeros((5, 3)), np.zeros((5, 3)), str(f))
    assert np.array_equal(pos, rows[:5, 0:3]) and np.array_equal(vel, rows[:5, 3:6])
    pos, vel = read.init0(np.zeros((5, 3)), np.zeros((5, 3)), str(f))
    assert np.array_equal(vel, rows[:5, 0:3]) and np.array_equal(pos, rows[:5, 3:6])
    # a one-particle file
    np.savetxt(f, rows[:1])
    pos, vel = read.initL(np.zeros((1, 3)), np.zeros((1, 3)), str(f))
    assert np.array_equal(pos, rows[:1, 0:3]) and np.array_equal(vel, rows[:1, 3:6])


def test_output_writer_formats():
    from p3m_b200.io import OutputWriter, state_rows

    rng = np.random.default_rng(2)
    snaps = [(rng.standard_normal((4, 3)), rng.standard_normal((4, 3)), rng.standard_normal((4, 3)))
             for _ in range(3)]
    fs, fe, fx = _io.StringIO(), _io.StringIO(), _io.StringIO()
    w = OutputWriter(fs, fe, fx)
    for k, (p, v, a) in enumerate(snaps):
        w.put(state_rows(p, v, a), (0.1 * k, 1.0 + k, 2.0, 3.0, -1.0))
    w.close()
    # what the reference's driver writes (yukawa_MD_p3m_ord6.py:221-229)
    rs, re_, rx = _io.StringIO(), _io.StringIO(), _io.StringIO()
    for k, (p, v, a) in enumerate(snaps):
        irp = np.hstack((p, v, a))
        np.savetxt(rs, irp)
        np.savetxt(re_, np.array([0.1 * k, 1.0 + k, 2.0, 3.0, -1.0]).reshape(1, 5))
        rx.writelines("{0:d}\n".format(4))
        rx.writelines("x y z vx vy vz ax ay az\n")
        np.savetxt(rx, irp)
    assert fs.getvalue() == rs.getvalue()
    assert fe.getvalue() == re_.getvalue()
    assert fx.getvalue() == rx.getvalue()
