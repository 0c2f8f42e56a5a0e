"""Input and output files of the reference's MD driver (host side).

* ``read_input``: the run parameters of ``yukawa_MD_p3m.in``
  (yukawa_MD_p3m_ord6.py:25-37, the first field of each line).
* ``reference_qmult``: the driver's n(q,t) wave numbers (:119-137),
  (iq+1) dq {1, sqrt 2, sqrt 3}, in units of dq = 2 pi / L.
* ``OutputWriter``: ``pos_vel_acc.out`` (n rows of pos, vel, acc per
  snapshot), ``time_temp_totalEnergy_kinEnergy_potEnergy.out`` (one row per
  snapshot), ``pos_vel_acc.xyz`` (n, a header line, the rows), written as
  :221-229 writes them (``np.savetxt`` defaults), on a background thread so
  that formatting text does not hold up the GPU.
"""
from __future__ import annotations

import queue
import threading

import numpy as np

INPUT_FIELDS = ("Gamma", "kappa", "N", "dt", "Neq", "Nt", "PBC", "snap_int", "init",
                "write_output", "write_xyz", "seed")
_INT_FIELDS = {"N", "Neq", "Nt", "PBC", "snap_int", "seed"}


def read_input(path):
    """yukawa_MD_p3m.in -> dict of the twelve run parameters (ints where the
    reference converts with int(), :28-37)."""
    c = np.loadtxt(path, delimiter=" ", usecols=(0,), unpack=True)
    c = np.atleast_1d(c)
    if c.size < len(INPUT_FIELDS):
        raise ValueError(f"{path}: {c.size} values, {len(INPUT_FIELDS)} expected")
    return {k: (int(v) if k in _INT_FIELDS else float(v)) for k, v in zip(INPUT_FIELDS, c)}


def reference_qmult(L):
    """q / dq of the driver's list: 3 int(2.5/dq) values, dq = 2 pi / L."""
    dq = 2.0 * np.pi / L
    nq = 3 * int(2.5 / dq)
    m = np.repeat(np.arange(1, nq // 3 + 1, dtype=np.float64), 3)
    return m * np.tile(np.array([1.0, np.sqrt(2.0), np.sqrt(3.0)]), nq // 3)


def state_rows(pos, vel, acc):
    """hstack((pos, vel, acc)), the reference's row layout (:223)."""
    return np.hstack((pos, vel, acc))


def write_state(f, rows):
    np.savetxt(f, rows)


def write_energy(f, t, Tp, E, K, U):
    np.savetxt(f, np.array([[t, Tp, E, K, U]]))


def write_xyz(f, rows):
    f.write("{0:d}\n".format(rows.shape[0]))
    f.write("x y z vx vy vz ax ay az\n")
    np.savetxt(f, rows)


class OutputWriter:
    """Writes snapshots handed to ``put`` in order on a worker thread.

    ``files``: open text files (or None) for the state rows, the energy rows
    and the .xyz frames."""

    def __init__(self, state_file, energy_file, xyz_file=None):
        self.files = (state_file, energy_file, xyz_file)
        self.q = queue.Queue(maxsize=8)
        self.err = None
        self.t = threading.Thread(target=self._loop, daemon=True)
        self.t.start()

    def _loop(self):
        while True:
            item = self.q.get()
            if item is None:
                return
            try:
                rows, (t, Tp, E, K, U) = item
                fs, fe, fx = self.files
                if fs is not None:
                    write_state(fs, rows)
                if fe is not None:
                    write_energy(fe, t, Tp, E, K, U)
                if fx is not None:
                    write_xyz(fx, rows)
            except Exception as e:  # reported by close()
                self.err = e

    def put(self, rows, energy_row):
        if self.err is not None:
            raise self.err
        self.q.put((rows, energy_row))

    def close(self):
        self.q.put(None)
        self.t.join()
        if self.err is not None:
            raise self.err
