"""Accuracy of the batched FP32 path on a workload, measured on the device.

The FP64 device path is the reference here (the parity tests pin it to the
CPU restatement of the reference's algorithm). For a workload of
``configs`` this measures:

* force error of the FP32 path at identical positions: eps_rms =
  sqrt(sum |a32 - a64|^2 / sum |a64|^2) and eps_max = max_i |a32 - a64|_i /
  rms |a64|, on the total acceleration, at the first step and every 100 steps
  of the FP64 trajectory;
* energy conservation of the FP32 path: the drift of E = K + U over
  ``drift_steps`` NVE steps from the equilibrated state, per replica (the
  largest |E(t) - E(0)| relative to |E(0)| and to the kinetic energy -- E(0)
  nears zero in weakly coupled replicas -- and the change from the first to
  the last 100-step mean);
* for the ensemble with n(q,t) (cfg3): S(q, w) of the FP32 and the FP64
  ensembles, both from their own trajectories (which part after a few hundred
  steps: the comparison is statistical), the frequency and height of the peak
  of each q.

  python -m p3m_b200.validate --workload cfg1 [--drift-steps 10000]
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import FP32, FP64, MODE_NVE, MODE_THERMOSTAT, Context
from .configs import CFG3_QMULT, WORKLOADS


def _initial(reps):
    import initialize_pos_vel

    pos, vel = [], []
    for r in reps:
        p, v = np.zeros((r.N, 3)), np.zeros((r.N, 3))
        initialize_pos_vel.initial(r.seed, r.N, [r.L] * 3, p, v, r.T_desired)
        pos.append(p)
        vel.append(v)
    return np.concatenate(pos), np.concatenate(vel)


def _force_errors(a32, a64, offs):
    out = []
    for i in range(len(offs) - 1):
        x, y = a32[offs[i]:offs[i + 1]], a64[offs[i]:offs[i + 1]]
        d2 = np.sum((x - y) ** 2, axis=1)
        y2 = np.sum(y ** 2, axis=1)
        out.append((float(np.sqrt(d2.sum() / y2.sum())), float(np.sqrt(d2.max() / y2.mean()))))
    return out


def _run_energies(ctx, steps, chunk=8000):
    """E = K + U of every replica after each of `steps` NVE steps."""
    E = []
    for k0 in range(0, steps, chunk):
        k = min(chunk, steps - k0)
        ctx.run(k, MODE_NVE)
        e = ctx.energies(max_steps=k)
        E.append(e[:, :, 0] + e[:, :, 1])
    return np.concatenate(E)


def _sqw_peaks(S, dw):
    """(frequency, height) of the largest value of S(q, w) for w in (0, w_N)."""
    half = S.shape[1] // 2
    k = 1 + np.argmax(S[:, 1:half], axis=1)
    return k * dw, S[np.arange(S.shape[0]), k]


def validate(workload="cfg1", equil=1000, traj_steps=1000, drift_steps=10000, sqw_steps=4096,
             quench=200, device=0):
    reps = WORKLOADS[workload]()
    offs = np.cumsum([0] + [r.N for r in reps])
    res = {"workload": workload, "replicas": len(reps), "particles": int(offs[-1])}
    pos0, vel0 = _initial(reps)
    with Context(reps, precision=FP64, device=device) as c64, \
            Context(reps, precision=FP32, device=device) as c32:
        # equilibrate in FP64: a quench, then the reference's thermostat
        c64.set_state_all(pos0, vel0)
        c64.init_forces()
        c64.equilibrate(equil, quench_steps=quench)
        pos_eq, vel_eq, _ = c64.get_state_all()
        # force error along the FP64 trajectory
        samples = []
        for k in range(0, traj_steps + 1, 100):
            if k:
                c64.run(100, MODE_NVE)
            p, _, a64 = c64.get_state_all()
            c32.set_state_all(p)
            c32.init_forces()
            _, _, a32 = c32.get_state_all()
            samples.append(_force_errors(a32, a64, offs))
        s = np.array(samples)  # (samples, replicas, 2)
        res["force_err"] = {"rms_max_over_samples": float(s[:, :, 0].max()),
                            "rms_mean": float(s[:, :, 0].mean()),
                            "max_rel_max_over_samples": float(s[:, :, 1].max()),
                            "samples": int(s.shape[0]),
                            "definition": "eps_rms = sqrt(sum|a32-a64|^2/sum|a64|^2), eps_max = "
                                          "max_i |a32-a64|_i / rms|a64|, total acceleration"}
        # FP32 energy conservation from the equilibrated state
        c32.set_state_all(pos_eq, vel_eq)
        c32.init_forces()
        E = _run_energies(c32, drift_steps)
        E0 = E[0]
        dev = np.max(np.abs(E - E0[None, :]), axis=0) / np.abs(E0)
        n = min(100, len(E) // 2)
        trend = np.abs(E[-n:].mean(axis=0) - E[:n].mean(axis=0)) / np.abs(E0)
        K0 = c32.energies(max_steps=1)[0, :, 1]
        res["nve_drift"] = {"steps": drift_steps, "max_abs_rel_dev": float(dev.max()),
                            "first_to_last_100_mean_rel": float(trend.max()),
                            "max_abs_dev_over_K": float(
                                (np.max(np.abs(E - E0[None, :]), axis=0) / K0).max()),
                            "dt": reps[0].dt}
        if workload == "cfg3" and sqw_steps:
            dt = reps[0].dt
            peaks = {}
            for name, c in (("fp32", c32), ("fp64", c64)):
                c.set_state_all(pos_eq, vel_eq)
                c.init_forces()
                c.set_nqt(CFG3_QMULT, sqw_steps)
                c.run(sqw_steps, MODE_NVE, record_nqt=True)
                S = c.sqw(dt, sqw_steps)
                peaks[name] = _sqw_peaks(S[:6], 2 * np.pi / (sqw_steps * dt))
            w32, h32 = peaks["fp32"]
            w64, h64 = peaks["fp64"]
            res["sqw_peaks"] = {"q_multiples": [1, 2, 3, 4, 5, 6],
                                "w_fp32": w32.tolist(), "w_fp64": w64.tolist(),
                                "dw": 2 * np.pi / (sqw_steps * dt),
                                "height_rel_diff": ((h32 - h64) / h64).tolist()}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cfg1", choices=sorted(WORKLOADS))
    ap.add_argument("--equil", type=int, default=1000)
    ap.add_argument("--traj-steps", type=int, default=1000)
    ap.add_argument("--drift-steps", type=int, default=10000)
    ap.add_argument("--sqw-steps", type=int, default=4096)
    ap.add_argument("--quench", type=int, default=200)
    a = ap.parse_args(argv)
    print(json.dumps(validate(a.workload, a.equil, a.traj_steps, a.drift_steps, a.sqw_steps,
                              a.quench)))


if __name__ == "__main__":
    main()
