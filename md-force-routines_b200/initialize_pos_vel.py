"""Initial state -- the reference's initialize_pos_vel.initial
(initialize_pos_vel.py:4-35), kept on the host because parity needs numpy's
legacy MT19937 stream drawn in the same order: u1..u4 (N each) for
Box-Muller velocities of standard deviation sqrt(T/3), mean removal, then
three uniform draws for the positions."""
import numpy as np


def initial(seed_int, N, Lv, pos, vel, T_desired):
    """Fill pos (N,3) uniform in the box and vel (N,3) Maxwell-Boltzmann at
    T_desired with zero mean; returns (pos, vel)."""
    np.random.seed(seed=seed_int)
    sig = np.sqrt(T_desired / 3)
    u = [np.random.random(N) for _ in range(4)]
    radial_xy = sig * np.sqrt(-2 * np.log(u[0]))
    vel[:, 0] = radial_xy * np.cos(2 * np.pi * u[1])
    vel[:, 1] = radial_xy * np.sin(2 * np.pi * u[1])
    vel[:, 2] = sig * np.sqrt(-2 * np.log(u[2])) * np.cos(2 * np.pi * u[3])
    for ax in range(3):
        vel[:, ax] = vel[:, ax] - np.mean(vel[:, ax])
    for ax in range(3):
        pos[:, ax] = Lv[ax] * np.random.random(N)
    return pos, vel
