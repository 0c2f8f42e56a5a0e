"""Accuracy of the batched FP32 path on a workload, measured on the device.

The FP64 device path is the reference here (the parity tests pin it to the
CPU restatement of the reference's algorithm). For a workload of
``configs`` this measures:

* force error of the FP32 path at identical positions: eps_rms =
  sqrt(sum |a32 - a64|^2 / sum |a64|^2) and eps_max = max_i |a32 - a64|_i /
  rms |a64|, on the total acceleration, at the first step and every 100 steps
  of the FP64 trajectory;
* energy conservation of the FP32 path, and of the FP64 path from the same
  equilibrated state as the control: per replica, the largest |E(t) - E(0)|
  over ``drift_steps`` NVE steps relative to |E(0)| and to the kinetic
  energy (E(0) nears zero in weakly coupled replicas), and the drift proper,
  the least-squares slope of E(t) times the run length over |E(0)|;
* the FP32 path runs with the kernel shapes the autotuner installs on the
  equilibrated ensemble (inner lists included), as the benchmark does;
* for the ensemble with n(q,t) (cfg3): S(q, w) of the FP32 and the FP64
  ensembles, both from their own trajectories (which part after a few hundred
  steps: the comparison is statistical), the frequency and height of the peak
  of each q, with replica-bootstrap standard deviations.

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
    """(E, K) of every replica after each of `steps` NVE steps: (steps, R)."""
    E, K = [], []
    for k0 in range(0, steps, chunk):
        k = min(chunk, steps - k0)
        ctx.run(k, MODE_NVE)
        e = ctx.energies(max_steps=k)
        E.append(e[:, :, 0] + e[:, :, 1])
        K.append(e[:, :, 1])
    return np.concatenate(E), np.concatenate(K)


def _drift_stats(E, K, E0, K0):
    """Per replica: the largest |E(t) - E(0)| relative to |E(0)| and to K(0),
    and the drift proper -- the least-squares slope of E(t) times the run
    length, relative to |E(0)| (fluctuations about a level, which the
    largest deviation also counts, do not grow with the run)."""
    t = np.arange(1, E.shape[0] + 1, dtype=np.float64)
    dev = np.max(np.abs(E - E0[None, :]), axis=0)
    slope = np.polyfit(t, E, 1)[0]  # per replica
    return {"max_abs_dev_rel_E0": (dev / np.abs(E0)).tolist(),
            "max_abs_dev_rel_K0": (dev / K0).tolist(),
            "fit_drift_rel_E0": (np.abs(slope) * E.shape[0] / np.abs(E0)).tolist(),
            "E0": E0.tolist(), "K0": K0.tolist(),
            "K_mean_rel_K0": (K.mean(axis=0) / K0).tolist()}


def _sqw_peaks(S, dw):
    """(frequency, height) of the largest value of S(q, w) for w in (0, w_N)."""
    half = S.shape[1] // 2
    k = 1 + np.argmax(S[:, 1:half], axis=1)
    return k * dw, S[np.arange(S.shape[0]), k]


def _bootstrap_peaks(S_rep, dw, n_boot=400, seed=0):
    """Standard deviation of the replica-mean S(q,w) peak frequency and height
    over bootstrap resamples of the replicas."""
    rng = np.random.default_rng(seed)
    R = S_rep.shape[0]
    ws, hs = [], []
    for _ in range(n_boot):
        S = S_rep[rng.integers(0, R, size=R)].mean(axis=0)
        w, h = _sqw_peaks(S, dw)
        ws.append(w)
        hs.append(h)
    return np.std(ws, axis=0), np.std(hs, axis=0)


def validate(workload="cfg1", equil=1000, traj_steps=1000, drift_steps=10000, sqw_steps=4096,
             quench=200, device=0, fp64_drift=True, tune=True):
    reps = WORKLOADS[workload]()
    offs = np.cumsum([0] + [r.N for r in reps])
    res = {"workload": workload, "replicas": len(reps), "particles": int(offs[-1]),
           "equil": {"quench_steps": quench, "thermostat_steps": equil}}
    pos0, vel0 = _initial(reps)
    with Context(reps, precision=FP64, device=device) as c64, \
            Context(reps, precision=FP32, device=device) as c32:
        # equilibrate in FP64: a quench, then the reference's thermostat
        c64.set_state_all(pos0, vel0)
        c64.init_forces()
        c64.equilibrate(equil, quench_steps=quench)
        pos_eq, vel_eq, _ = c64.get_state_all()
        if tune:  # the FP32 kernel shapes the benchmark would install
            from .autotune import tune as _tune

            c32.set_state_all(pos_eq, vel_eq)
            c32.init_forces()
            _tune(c32, use_cache=False)
        res["fp32_tuning"] = c32.tuning()
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
                                          "max_i |a32-a64|_i / rms|a64|, total acceleration, "
                                          "FP32 against the FP64 device path"}
        # energy conservation from the equilibrated state: FP32, and FP64 as
        # the control that separates the integrator's error (dt) from FP32's
        drift = {"steps": drift_steps, "dt": reps[0].dt}
        for name, c in (("fp32", c32), ("fp64", c64)) if fp64_drift else (("fp32", c32),):
            c.set_state_all(pos_eq, vel_eq)
            c.init_forces()
            E, K = _run_energies(c, drift_steps)
            E0, K0 = E[0], K[0]  # after the first step
            st = _drift_stats(E, K, E0, K0)
            drift[name] = {"max_abs_dev_rel_E0_max": float(np.max(st["max_abs_dev_rel_E0"])),
                           "fit_drift_rel_E0_max": float(np.max(st["fit_drift_rel_E0"])),
                           "max_abs_dev_rel_K0_max": float(np.max(st["max_abs_dev_rel_K0"])),
                           "per_replica": st}
        res["nve_drift"] = drift
        if workload == "cfg3" and sqw_steps:
            dt = reps[0].dt
            dw = 2 * np.pi / (sqw_steps * dt)
            peaks = {}
            for name, c in (("fp32", c32), ("fp64", c64)):
                c.set_state_all(pos_eq, vel_eq)
                c.init_forces()
                c.set_nqt(CFG3_QMULT, sqw_steps)
                c.run(sqw_steps, MODE_NVE, record_nqt=True)
                S, S_rep = c.sqw(dt, sqw_steps, per_replica=True)
                w, h = _sqw_peaks(S[:6], dw)
                sw, sh = _bootstrap_peaks(S_rep[:, :6], dw)
                peaks[name] = (w, h, sw, sh)
            w32, h32, sw32, sh32 = peaks["fp32"]
            w64, h64, sw64, sh64 = peaks["fp64"]
            dh = h32 - h64
            sd = np.sqrt(sh32 ** 2 + sh64 ** 2)
            res["sqw_peaks"] = {"q_multiples": [1, 2, 3, 4, 5, 6], "dw": dw,
                                "w_fp32": w32.tolist(), "w_fp64": w64.tolist(),
                                "w_boot_sd_fp32": sw32.tolist(), "w_boot_sd_fp64": sw64.tolist(),
                                "h_fp32": h32.tolist(), "h_fp64": h64.tolist(),
                                "h_boot_sd_fp32": sh32.tolist(), "h_boot_sd_fp64": sh64.tolist(),
                                "height_rel_diff": (dh / h64).tolist(),
                                "height_diff_in_sd": (dh / sd).tolist(),
                                "note": "each ensemble from its own trajectories; sd: replica "
                                        "bootstrap (400 resamples) of the replica-mean peak"}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cfg1", choices=sorted(WORKLOADS))
    ap.add_argument("--equil", type=int, default=1000)
    ap.add_argument("--traj-steps", type=int, default=1000)
    ap.add_argument("--drift-steps", type=int, default=10000)
    ap.add_argument("--sqw-steps", type=int, default=4096)
    ap.add_argument("--quench", type=int, default=200)
    ap.add_argument("--no-fp64-drift", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the FP32 context's default kernel shapes instead of autotuning")
    a = ap.parse_args(argv)
    print(json.dumps(validate(a.workload, a.equil, a.traj_steps, a.drift_steps, a.sqw_steps,
                              a.quench, fp64_drift=not a.no_fp64_drift, tune=not a.no_tune)))


if __name__ == "__main__":
    main()
