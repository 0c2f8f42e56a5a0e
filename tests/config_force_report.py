"""Force and energy errors of the device paths against the oracle, at every
benchmark configuration's own size -- a measurement script beside the
parity tests (it imports the oracle, so it lives with them).

For each workload (one replica, the 20-replica ensemble, the 64-replica
uneven ensemble, the N = 1e6 / 256^3 replica) and two sets of positions per
replica -- the seeded initial state (uniform positions, the reference's
initialize_pos_vel) and the state after the equilibration the benchmark uses
(200 thermostat steps at T_desired/100, then 300 of the reference's
thermostat, on the FP64 device path) -- it computes the total acceleration
and potential energy of every replica three ways:

* the oracle (the reference's FP64 algorithm on the CPU: PP and mesh stages
  in C, the FFT chain in numpy), with the influence function of the device
  checked against the oracle's gf_opt at sampled points;
* the FP64 device path, batched;
* the FP32 device path, batched,

and prints one JSON line per workload with, per path, the largest (over
replicas and the two states) eps_rms = sqrt(sum |a - a_o|^2 / sum |a_o|^2),
eps_max = max_i |a - a_o|_i / rms |a_o| and |U - U_o| / |U_pp,o|.

    python tests/config_force_report.py [cfg1 cfg2 cfg3 cfg4 cfg5]
"""
import json
import multiprocessing as mp
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "md-force-routines_b200")
for _p in (ROOT, PKG, os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def _oracle_force(args):
    N, L, kappa, alpha, rc, M, Gamma, G, pos = args
    from oracle import oracle as O

    P = O.Params(N, kappa, alpha, rc, M, L=L, Gamma=Gamma)
    kv = 2 * np.pi * (np.arange(M) - M // 2) / L
    P._gk = (G, kv.reshape(1, M), kv.reshape(M, 1), kv.reshape(M, 1, 1), 0.0)
    return O.force_pot(P, pos)


def _checked_green(kappa, alpha, M, L, seed):
    from oracle import oracle as O
    from p3m_b200 import gf_opt_device

    G, _ = gf_opt_device(kappa, alpha, 6, 3, M, L)
    idx = np.random.default_rng(seed).integers(0, M, size=(500, 3))
    ref = O.gf_opt_points(kappa, alpha, 6, 3, M, L, idx)
    err = np.max(np.abs(G[idx[:, 0], idx[:, 1], idx[:, 2]] - ref)) / np.max(np.abs(ref))
    assert err <= 1e-12, err
    return G


def _device_forces(reps, greens, pos_all, prec):
    from p3m_b200 import Context

    with Context(reps, precision=prec) as c:
        for i, G in enumerate(greens):
            c.set_green(G, replica=i)
        c.set_state_all(pos_all, np.zeros_like(pos_all))
        c.init_forces()
        _, _, acc = c.get_state_all()
        U = [c.replica_stats(i)["U"] for i in range(len(reps))]
    return acc, U


def report(name, pool):
    import initialize_pos_vel
    from p3m_b200 import FP32, FP64, Context
    from p3m_b200.configs import WORKLOADS

    reps = WORKLOADS[name]()
    offs = np.cumsum([0] + [r.N for r in reps])
    pos0, vel0 = [], []
    for r in reps:
        p, v = np.zeros((r.N, 3)), np.zeros((r.N, 3))
        initialize_pos_vel.initial(r.seed, r.N, [r.L] * 3, p, v, r.T_desired)
        pos0.append(p)
        vel0.append(v)
    pos0, vel0 = np.concatenate(pos0), np.concatenate(vel0)
    with Context(reps, precision=FP64) as c:
        c.set_state_all(pos0, vel0)
        c.init_forces()
        c.equilibrate(300, quench_steps=200)
        pos_eq = c.get_state_all()[0]
    gcache, greens = {}, []
    for r in reps:
        key = (r.kappa, r.alpha, r.M, r.L)
        if key not in gcache:
            gcache[key] = _checked_green(r.kappa, r.alpha, r.M, r.L, seed=len(gcache))
        greens.append(gcache[key])
    worst = {p: {"rms": 0.0, "max": 0.0, "U_rel_Upp": 0.0} for p in ("fp64", "fp32")}
    for pos_all in (pos0, pos_eq):
        tasks = [(r.N, r.L, r.kappa, r.alpha, r.rc, r.M, 1.0 / r.T_desired, greens[i],
                  pos_all[offs[i]:offs[i + 1]]) for i, r in enumerate(reps)]
        orc = pool.map(_oracle_force, tasks, chunksize=1)
        for pname, prec in (("fp64", FP64), ("fp32", FP32)):
            acc, U = _device_forces(reps, greens, pos_all, prec)
            w = worst[pname]
            for i, (Uo, ao, parts) in enumerate(orc):
                a = acc[offs[i]:offs[i + 1]]
                d2 = np.sum((a - ao) ** 2, axis=1)
                w["rms"] = max(w["rms"], float(np.sqrt(d2.sum() / np.sum(ao ** 2))))
                w["max"] = max(w["max"], float(np.sqrt(d2.max() / np.mean(np.sum(ao ** 2, axis=1)))))
                w["U_rel_Upp"] = max(w["U_rel_Upp"], abs(U[i] - Uo) / abs(parts[0]))
    return {"workload": name, "replicas": len(reps), "particles": int(offs[-1]),
            "vs_oracle": worst,
            "states": ["initial (seeded uniform)",
                       "equilibrated (200 quench + 300 thermostat steps, FP64 device path)"]}


def main(argv):
    names = argv or ["cfg1", "cfg2", "cfg3", "cfg4", "cfg5"]
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(16, os.cpu_count() or 1)) as pool:  # before any GPU call
        pool.map(abs, [0])
        for n in names:
            print(json.dumps(report(n, pool)), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
