"""The MD driver end to end on the device against the oracle's trajectory:
its output files, n(q,t), and a resume from its final file."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

N, KAPPA, ALPHA, RC, M, GAMMA, DT, SEED = 2000, 1.5, 0.7, 4.0, 32, 100.0, 0.1, 7


def _input(path, Neq, Nt, snap, init, write, xyz):
    vals = [GAMMA, KAPPA, N, DT, Neq, Nt, 1, snap, init, write, xyz, SEED]
    path.write_text("".join(f"{v}    field\n" for v in vals))


def _oracle_start():
    import initialize_pos_vel

    P = O.Params(N, KAPPA, ALPHA, RC, M, Gamma=GAMMA, dt=DT)
    pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
    initialize_pos_vel.initial(SEED, N, [P.L] * 3, pos, vel, P.T_desired)
    _, acc, _ = O.force_pot(P, pos)
    return P, pos, vel, acc


def _close(a, b, rtol=1e-9):
    scale = np.max(np.abs(b))
    assert np.max(np.abs(a - b)) <= rtol * scale, np.max(np.abs(a - b)) / scale


def _run(tmp_path, *extra):
    import yukawa_MD_p3m_ord6 as drv

    drv.run(["--input", str(tmp_path / "in"), "--dir", str(tmp_path), "--alpha", str(ALPHA),
             "--rc", str(RC), "--mesh", str(M), "--quiet", *extra])


def test_driver_files_match_oracle(tmp_path):
    Neq, Nt, snap = 5, 12, 4
    _input(tmp_path / "in", Neq, Nt, snap, 0, 1, 1)
    _run(tmp_path, "--chunk", "5")  # chunks that do not line up with the snapshots
    P, pos, vel, acc = _oracle_start()
    for it in range(Neq):
        pos, vel, acc, U, T = O.vscale(P, pos, vel, acc, it)
    qv = O.q_vectors_reference(P.L)
    snaps, energies, nqt = [], [], []
    for it in range(Nt):
        pos, vel, acc, U = O.update(P, pos, vel, acc)
        nqt.append(O.nqt(pos, qv))
        if (it + 1) % snap == 0:
            K = P.kf * np.sum(vel ** 2)
            snaps.append(np.hstack((pos, vel, acc)))
            energies.append([DT * it, K / P.kf / N, K + U, K, U])
    out = np.loadtxt(tmp_path / "pos_vel_acc.out").reshape(-1, N, 9)
    assert out.shape[0] == len(snaps) == 3
    for got, ref in zip(out, snaps):
        _close(got, ref)
    E = np.loadtxt(tmp_path / "time_temp_totalEnergy_kinEnergy_potEnergy.out")
    assert E.shape == (3, 5)
    np.testing.assert_allclose(E[:, 0], [r[0] for r in energies], rtol=1e-12)
    _close(E[:, 1:], np.array(energies)[:, 1:])
    lines = (tmp_path / "pos_vel_acc.xyz").read_text().splitlines()
    assert len(lines) == 3 * (N + 2) and lines[0] == str(N) and lines[1] == "x y z vx vy vz ax ay az"
    q = np.load(tmp_path / "n_q_t_1.npy")
    assert q.shape == (Nt, len(qv), 3) and q.dtype == np.complex128
    _close(q, np.array(nqt))
    final = np.loadtxt(tmp_path / "pos_vel_acc_final.out")
    _close(final, np.hstack((pos, vel, acc)))

    # resume: the final file as init.out, 4 more steps, no thermostat
    (tmp_path / "init.out").write_text((tmp_path / "pos_vel_acc_final.out").read_text())
    _input(tmp_path / "in", 0, 4, 1, 1, 0, 0)
    _run(tmp_path)
    for it in range(4):
        pos, vel, acc, U = O.update(P, pos, vel, acc)
    _close(np.loadtxt(tmp_path / "pos_vel_acc_final.out"), np.hstack((pos, vel, acc)))
    assert (tmp_path / "pos_vel_acc.out").read_text() == ""  # write_output = 0


def test_driver_replicas_name_files_by_seed(tmp_path):
    _input(tmp_path / "in", 2, 6, 3, 0, 1, 0)
    _run(tmp_path, "--replicas", "2", "--precision", "fp32")
    for s in (SEED, SEED + 1):
        assert np.load(tmp_path / f"n_q_t_{s}.npy").shape[0] == 6
        assert np.loadtxt(tmp_path / f"pos_vel_acc_{s}.out").shape == (2 * N, 9)
        assert np.loadtxt(tmp_path / f"pos_vel_acc_final_{s}.out").shape == (N, 9)
    # different seeds, different states
    a = np.loadtxt(tmp_path / f"pos_vel_acc_final_{SEED}.out")
    b = np.loadtxt(tmp_path / f"pos_vel_acc_final_{SEED + 1}.out")
    assert not np.allclose(a, b)
