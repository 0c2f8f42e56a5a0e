"""Yukawa OCP molecular dynamics run -- the reference's driver
yukawa_MD_p3m_ord6.py (a Python 2 script) as a Python 3 program over the
device-resident path.

Reads ``yukawa_MD_p3m.in`` (:25-37), sets the P3M parameters the reference
sets by hand (alpha = 0.46, r_c = 7.8, 64^3, p = 6, aliases 3; :52-68) or
picks them from the error estimates (``--tol``), starts from
``initialize_pos_vel.initial(seed)`` or, with init = 1, from ``init.out``
(``read.initL``, :143-148), runs Neq thermostat steps (thermostat_p3m_ord6
.vscale) and Nt velocity-Verlet steps recording n(q,t) on the reference's q
list (:119-137, :214-219), and writes what the reference writes (:187-241):

  pos_vel_acc.out                                 every snap_int steps (write_output = 1)
  time_temp_totalEnergy_kinEnergy_potEnergy.out   the same steps
  pos_vel_acc.xyz                                 the same steps (write_xyz = 1)
  n_q_t_1.npy                                     (Nt, Nq, 3) complex128
  pos_vel_acc_final.out                           the last state

Steps run as CUDA graphs in chunks; snapshots are copied into a device ring
inside the steps and written by a host thread while the next chunk runs.
With ``--replicas R`` the seeds seed .. seed+R-1 run as one batch and every
file name gets the suffix ``_<seed>`` (``n_q_t_<seed>.npy``, the names
s_of_q_w_script.py:27-28 loads).

  python yukawa_MD_p3m_ord6.py [--input yukawa_MD_p3m.in] [--dir .] [--replicas R]
                              [--precision fp64|fp32] [--alpha A --rc RC --mesh M | --tol TOL]
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
if _HERE not in sys.path:
    sys.path.insert(0, _HERE)

import initialize_pos_vel  # noqa: E402
import read  # noqa: E402
from p3m_b200 import FP32, FP64, MODE_NVE, MODE_THERMOSTAT, Context, Replica  # noqa: E402
from p3m_b200.io import OutputWriter, read_input, reference_qmult, state_rows  # noqa: E402

#: the reference driver's hand-set P3M parameters (yukawa_MD_p3m_ord6.py:52-68)
ALPHA, RC, MESH = 0.46, 7.8, 64


def parse(argv):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--input", default="yukawa_MD_p3m.in")
    ap.add_argument("--dir", default=".", help="where init.out is read and the outputs go")
    ap.add_argument("--replicas", type=int, default=1)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--alpha", type=float, default=ALPHA)
    ap.add_argument("--rc", type=float, default=RC)
    ap.add_argument("--mesh", type=int, default=MESH)
    ap.add_argument("--tol", type=float, default=None,
                    help="choose alpha, r_c and the mesh for this RMS force error instead")
    ap.add_argument("--quench", type=int, default=0,
                    help="thermostat steps at T_desired/100 before the equilibration (not in the "
                         "reference; damps runaway particles of random starts)")
    ap.add_argument("--chunk", type=int, default=1000, help="steps per launch batch")
    ap.add_argument("--quiet", action="store_true", help="no per-step lines on stdout")
    return ap.parse_args(argv)


def run(argv=None):
    t1 = time.time()
    a = parse(argv)
    inp = read_input(a.input)
    Gamma, kappa, N, dt = inp["Gamma"], inp["kappa"], inp["N"], inp["dt"]
    Neq, Nt, PBC, snap_int = inp["Neq"], inp["Nt"], inp["PBC"], inp["snap_int"]
    if PBC != 1:
        raise ValueError("only periodic boundaries are supported (README.md:21)")
    T_desired = 1.0 / Gamma
    L = (4.0 * np.pi * N / 3.0) ** (1.0 / 3.0)
    alpha, rc, M = a.alpha, a.rc, a.mesh
    if a.tol is not None:
        from p3m_b200.params import pick_params

        (c,) = pick_params([(N, L, kappa)], tol=a.tol)
        alpha, rc, M = c.alpha, c.rc, c.M
    seeds = [inp["seed"] + k for k in range(a.replicas)]
    reps = [Replica(N=N, L=L, kappa=kappa, alpha=alpha, rc=rc, M=M, dt=dt, T_desired=T_desired,
                    seed=s) for s in seeds]
    say = (lambda *x: None) if a.quiet else print
    say("\n\n----------- Molecular Dynamics Simulation of Yukawa System ----------------------")
    say("Gamma = ", Gamma)
    say("kappa = ", kappa)
    say("Temperature = ", T_desired)
    say("No. of particles = ", N)
    for ax in "xyz":
        say(f"Box length along {ax} axis = ", L)
    say("No. of non-zero box dimensions = ", 3)
    say("time step = ", dt)
    say("No. of equilibration steps = ", Neq)
    say("No. of post-equilibration steps = ", Nt)
    say("snapshot interval = ", snap_int)
    say("Periodic boundary condition{1=yes, 0=no} =", PBC)
    say("grid_size * Ewald_parameter (h * alpha) = ", L / M * alpha)
    qmult = reference_qmult(L)
    dq = 2.0 * np.pi / L
    say("smallest interval in Fourier space for S(q,w): dq = ", dq)
    suffix = (lambda s: "") if len(seeds) == 1 else (lambda s: f"_{s}")

    t2 = time.time()
    ctx = Context(reps, precision=FP64 if a.precision == "fp64" else FP32)
    t3 = time.time()
    try:
        states = []
        for r in reps:
            pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
            if inp["init"] == 1:
                say("\nReading initial particle positions and velocities from file...")
                pos, vel = read.initL(pos, vel, os.path.join(a.dir, "init.out"))
            else:
                say("\nAssigning random initial positions and velocities...")
                initialize_pos_vel.initial(r.seed, N, [L] * 3, pos, vel, T_desired)
            states.append((pos, vel))
        ctx.set_state_all(np.concatenate([p for p, _ in states]),
                          np.concatenate([v for _, v in states]))
        ctx.init_forces()
        t4 = time.time()

        say("\n------------- Equilibration -------------")
        say("time - temperature")
        chunk = max(1, min(a.chunk, 8192))
        if a.quench > 0:
            ctx.equilibrate(0, quench_steps=a.quench)
        for k0 in range(0, Neq, chunk):
            k = min(chunk, Neq - k0)
            ctx.run(k, MODE_THERMOSTAT, it0=k0)
            if not a.quiet:
                E = ctx.energies(max_steps=k)
                for j in range(k):
                    print(dt * (k0 + j), E[j, 0, 2])
        t5 = time.time()

        say("\n------------- Production -------------")
        say("time - total energy - kinetic energy - potential energy")
        write = inp["write_output"] == 1 and snap_int > 0
        if write:
            # at most ~512 MB of snapshot ring: fewer steps per chunk for
            # large ensembles written often
            per_snap = sum(r.N for r in reps) * 9 * 8
            chunk = max(1, min(chunk, max(1, (1 << 29) // per_snap) * snap_int))
        # the three files are opened (and left empty) whatever the flags, as
        # the reference does (:201-203)
        files, writers = [], []
        for s in seeds:
            f = [open(os.path.join(a.dir, f"pos_vel_acc{suffix(s)}.out"), "w"),
                 open(os.path.join(a.dir, f"time_temp_totalEnergy_kinEnergy_potEnergy{suffix(s)}.out"),
                      "w"),
                 open(os.path.join(a.dir, f"pos_vel_acc{suffix(s)}.xyz"), "w")]
            files.append(f)
            if write:
                writers.append(OutputWriter(f[0], f[1], f[2] if inp["write_xyz"] == 1 else None))
        if write:
            ctx.set_snapshots(snap_int, capacity=chunk // snap_int + 1)
        ctx.set_nqt(qmult, max(Nt, 1))
        offs = np.cumsum([0] + [N] * len(reps))
        try:
            for k0 in range(0, Nt, chunk):
                k = min(chunk, Nt - k0)
                ctx.run(k, MODE_NVE, it0=k0, record_nqt=True)
                E = ctx.energies(max_steps=k)  # (k, R, 4): U, K, T, factor
                if not a.quiet:
                    for j in range(k):
                        U, K = E[j, 0, 0], E[j, 0, 1]
                        print(dt * (k0 + j), K + U, K, U)
                if write:
                    snaps, steps = ctx.get_snapshots()
                    for snap, it in zip(snaps, steps):
                        U, K, T = E[it - k0, :, 0], E[it - k0, :, 1], E[it - k0, :, 2]
                        for i, w in enumerate(writers):
                            w.put(snap[offs[i]:offs[i + 1]].copy(),
                                  (dt * it, T[i], K[i] + U[i], K[i], U[i]))
        finally:
            for w in writers:
                w.close()
            for f in files:
                for x in f:
                    if x is not None:
                        x.close()
            if write:
                ctx.set_snapshots(0)
        for i, s in enumerate(seeds):
            name = "n_q_t_1" if len(seeds) == 1 else f"n_q_t_{s}"
            np.save(os.path.join(a.dir, name), ctx.get_nqt(i, len(qmult), max_steps=max(Nt, 1)))
        pos, vel, acc = ctx.get_state_all()
        for i, s in enumerate(seeds):
            sl = slice(offs[i], offs[i + 1])
            np.savetxt(os.path.join(a.dir, f"pos_vel_acc_final{suffix(s)}.out"),
                       state_rows(pos[sl], vel[sl], acc[sl]))
        t6 = time.time()
    finally:
        ctx.close()
    say("Time for importing required libraries = ", t2 - t1)
    say("Time for computing converged Greens function = ", t3 - t2)
    say("Time for initialization = ", t4 - t3)
    say("Time for equilibration = ", t5 - t4)
    say("Time for production = ", t6 - t5)
    say("Total elapsed time = ", t6 - t1)


if __name__ == "__main__":
    run()
