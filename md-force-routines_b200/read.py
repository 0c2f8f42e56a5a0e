"""Initial conditions from a file -- drop-in for the reference's read.py
(:3-74). Host-side text reading, as the reference does it.

``initL`` reads columns x y z vx vy vz ax ay az (the layout of
pos_vel_acc.out and pos_vel_acc_final.out, so a run resumes from its final
file); ``init0`` reads vx vy vz x y z ax ay az. Both keep the first N rows,
N = len(pos), and return NEW (pos, vel) arrays; the accelerations are read
and dropped (the driver recomputes the forces)."""
import numpy as np


def _columns(table, N, order):
    t = np.asarray(table, dtype=np.float64)
    if t.ndim == 1:  # a one-row file: nine scalars
        t = t.reshape(-1, 1)
    cols = {name: t[k, :N] for k, name in enumerate(order)}
    pos = np.stack([cols["x"], cols["y"], cols["z"]], axis=1)
    vel = np.stack([cols["vx"], cols["vy"], cols["vz"]], axis=1)
    return pos, vel


def init0(pos, vel, f_input):
    """read.py:3-36 (np.genfromtxt, columns vx vy vz x y z ax ay az)."""
    N = len(pos[:, 0])
    t = np.genfromtxt(f_input, usecols=(0, 1, 2, 3, 4, 5, 6, 7, 8), unpack=True)
    return _columns(t, N, ("vx", "vy", "vz", "x", "y", "z", "ax", "ay", "az"))


def initL(pos, vel, f_input):
    """read.py:39-74 (np.loadtxt, columns x y z vx vy vz ax ay az)."""
    N = len(pos[:, 0])
    t = np.loadtxt(f_input, usecols=(0, 1, 2, 3, 4, 5, 6, 7, 8), unpack=True)
    return _columns(t, N, ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"))
