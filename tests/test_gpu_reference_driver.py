"""The reference's own MD driver running over this package's modules.

yukawa_MD_p3m_ord6.py (the reference's driver, :1-256) is a Python-2 script;
oracle/make_ref_driver.py writes a copy with only its print statements turned
into calls (into oracle/_ref/, next to the compiled reference PP routine,
wherever the reference tree is present at build time). Run from a directory
holding its input file, with md-force-routines_b200/ first on the module
path, it imports this package's read, initialize_pos_vel,
velocity_verlet_p3m_ord6, thermostat_p3m_ord6, yukawa_gf_opt and
yukawa_p3m_ord6 in place of the reference's, and calls them with the
reference's own arguments (:152-229): the drop-in boundary. Its output files
are compared with the oracle's trajectory for the same input and the
driver's hand-set parameters (G = 0.46, r_c = 7.8, 64^3, p = 6,
yukawa_MD_p3m_ord6.py:52-68).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "md-force-routines_b200")
DRIVER = os.path.join(ROOT, "oracle", "_ref", "yukawa_MD_p3m_ord6_py3.py")

# the input file's fields (yukawa_MD_p3m_ord6.py:26-38); N >= 3063 keeps
# floor(L / 7.8) >= 3 for the driver's r_c
GAMMA, KAPPA, N, DT, NEQ, NT, PBC, SNAP, INIT, WRITE, XYZ, SEED = (
    100.0, 0.5, 4000, 0.1, 4, 6, 1, 2, 0, 1, 1, 5)
ALPHA, RC, M = 0.46, 7.8, 64  # hard-coded in the driver


def _close(a, b, rtol=1e-9):
    scale = np.max(np.abs(b))
    err = np.max(np.abs(np.asarray(a) - np.asarray(b))) / scale
    assert err <= rtol, err


@pytest.mark.skipif(not os.path.isfile(DRIVER),
                    reason="the Python-3 copy of the reference's driver was not built "
                           "(the reference tree was absent at build time)")
def test_reference_driver_over_package_modules(tmp_path):
    vals = [GAMMA, KAPPA, N, DT, NEQ, NT, PBC, SNAP, INIT, WRITE, XYZ, SEED]
    names = ["Gamma", "kappa", "N", "dt", "Neq", "Nt", "PBC", "snap", "init", "write", "xyz",
             "seed"]
    (tmp_path / "yukawa_MD_p3m.in").write_text(
        "".join(f"{v}      {n}\n" for v, n in zip(vals, names)))
    env = dict(os.environ, PYTHONPATH=os.pathsep.join([PKG, ROOT]), P3M_B200_PRECISION="fp64",
               PYTHONDONTWRITEBYTECODE="1")
    res = subprocess.run([sys.executable, DRIVER], cwd=tmp_path, env=env, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    assert "Total elapsed time" in res.stdout

    # the oracle, step for step as the driver calls the modules
    import initialize_pos_vel

    P = O.Params(N, KAPPA, ALPHA, RC, M, Gamma=GAMMA, dt=DT)
    pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
    initialize_pos_vel.initial(SEED, N, P.Lv, pos, vel, P.T_desired)
    _, acc, _ = O.force_pot(P, pos)
    for it in range(NEQ):
        pos, vel, acc, U, _ = O.vscale(P, pos, vel, acc, it)
    qv = O.q_vectors_reference(P.L)
    snaps, energies, nqt, lines = [], [], [], []
    for it in range(NT):
        pos, vel, acc, U = O.update(P, pos, vel, acc)
        K = P.kf * np.sum(vel ** 2)
        lines.append([DT * it, K + U, K, U])
        nqt.append(O.nqt(pos, qv))
        if (it + 1) % SNAP == 0:
            snaps.append(np.hstack((pos, vel, acc)))
            energies.append([DT * it, K / P.kf / N, K + U, K, U])

    # the production lines it prints: time, E, K, U (:202-203)
    printed = [ln.split() for ln in res.stdout.splitlines()]
    rows = [list(map(float, p)) for p in printed if len(p) == 4 and p[0][0].isdigit()]
    assert len(rows) == NT
    _close(np.array(rows)[:, 1:], np.array(lines)[:, 1:])
    out = np.loadtxt(tmp_path / "pos_vel_acc.out").reshape(-1, N, 9)
    assert out.shape[0] == len(snaps) == NT // SNAP
    for got, ref in zip(out, snaps):
        _close(got, ref)
    E = np.loadtxt(tmp_path / "time_temp_totalEnergy_kinEnergy_potEnergy.out")
    _close(E, np.array(energies))
    xyz = (tmp_path / "pos_vel_acc.xyz").read_text().splitlines()
    assert len(xyz) == (NT // SNAP) * (N + 2) and xyz[0] == str(N)
    q = np.load(tmp_path / "n_q_t_1.npy")
    assert q.shape == (NT, len(qv), 3)
    _close(q, np.array(nqt))
    _close(np.loadtxt(tmp_path / "pos_vel_acc_final.out"), np.hstack((pos, vel, acc)))
