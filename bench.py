#!/usr/bin/env python
"""Throughput of the P3M MD step on B200, in particle-steps/s.

Workload (default): the batched ensemble of 20 Yukawa OCP replicas, each
N = 10^4, Gamma = 100, kappa = 2, 64^3 mesh, p = 6, alpha = 0.6, r_c = 6,
dt = 0.1, seeds 1..20, advanced together (FP32 bulk arithmetic, FP64
reductions and positions) by CUDA-graph-captured NVE steps that also record
n(q,t) on 32 wave numbers x 3 axes. A "step" is one velocity-Verlet step of
every replica.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Ours: one process per GPU (torchrun for N > 1), each with its own 20-replica
ensemble (replicas only: no data-path collective; weak scaling). The timed
region is K graph launches between CUDA events on the context's stream,
after a barrier and device synchronisation; the max over ranks is taken.
The line also carries the plain FP64 single-replica path on the same
ensemble, the FP32-vs-FP64 force error, the end-to-end number through the
C ABI with host buffers, the PP kernel's roofline and the CPU baseline (the
oracle port on one host core).

--impl reference: the reference's CPU path for the same workload, run as the
oracle port (the reference's own code is Python/numba that does not travel
to the GPU box) over all host cores, each process owning a fixed set of
replicas that it sets up and warms up before the timed region.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "md-force-routines_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "particle-steps/s on 1 B200: batched FP32 vs plain FP64 P3M at force err<=1e-5"
UNIT = "particle-steps/s"
WORKLOAD = ("cfg3 ensemble: 20 replicas x N=1e4, Gamma=100, kappa=2, 64^3 mesh, p=6, "
            "alpha=0.6, rc=6, dt=0.1, NVE steps with n(q,t) (32 q x 3 axes)")
WORKLOADS_TEXT = {
    "cfg1": "cfg1: 1 replica N=1e4, Gamma=100, kappa=2, 64^3 mesh, p=6, alpha=0.6, rc=6, dt=0.1",
    "cfg2": "cfg2: 1 replica N=1e5, Gamma=50, kappa=1, 128^3 mesh, p=6, alpha=0.5, rc=7, dt=0.1",
    "cfg3": WORKLOAD,
    "cfg4": ("cfg4: 64 uneven replicas (seeds 100-163; N 2031-48336, Gamma 10-198, kappa 0.50-2.92; "
             "M in {32,64,128}, alpha, rc picked for 1e-6 RMS force error), dt=0.1"),
    "cfg5": "cfg5: 1 replica N=1e6, Gamma=100, kappa=2, 256^3 mesh, p=6, alpha=0.6, rc=6, dt=0.1",
}
FLOP_PER_PAIR = 48  # fixed convention for the PP roofline (unique pairs)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg3", choices=sorted(WORKLOADS_TEXT),
                    help="the configuration to time (default: the 20-replica ensemble)")
    ap.add_argument("--replicas", type=int, default=20, help="cfg3's ensemble size")
    ap.add_argument("--equil", type=int, default=300,
                    help="untimed thermostat steps before the NVE warm-up")
    ap.add_argument("--quench", type=int, default=200,
                    help="thermostat steps at T_desired/100 before --equil (damps the runaway "
                         "particles that random initial positions launch)")
    ap.add_argument("--no-tune", action="store_true", help="skip the kernel-shape autotuner")
    ap.add_argument("--pp-config", default=None, metavar="TPI,SKIN",
                    help="set threads per particle and Verlet skin instead of autotuning")
    ap.add_argument("--prune-buf", type=float, default=0.0,
                    help="with --pp-config: FP32 inner-list buffer beyond rc (0: none)")
    ap.add_argument("--e2e-parts", type=int, default=5,
                    help="contexts the ensemble is split into for the end-to-end number")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the FP64, e2e, roofline and CPU-baseline legs")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.25)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        self.proc.wait()
        with open(self.path) as f:
            lines = f.readlines()
        os.unlink(self.path)
        return summarise_clocks(lines)


def summarise_clocks(lines):
    """The clocks record of a timed region from nvidia-smi rows of
    ClockSampler.FIELDS (csv, no header, no units): the median SM clock of the
    samples under load (above half the highest), the highest max clock, the
    highest power draw, and every throttle reason seen active."""
    rows = []
    for line in lines:
        parts = [p.strip() for p in line.split(",")]
        if len(parts) >= 9:
            rows.append(parts)
    if not rows:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
    sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
    mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
    pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
    loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
    return {"sm_mhz": float(np.median(loaded)) if loaded else None,
            "sm_max_mhz": max(mx) if mx else None,
            "power_w_max": max(pw) if pw else None,
            "samples": len(rows), "reasons": reasons}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def initial_states(reps):
    import initialize_pos_vel

    out = []
    for r in reps:
        pos, vel = np.zeros((r.N, 3)), np.zeros((r.N, 3))
        initialize_pos_vel.initial(r.seed, r.N, [r.L] * 3, pos, vel, r.T_desired)
        out.append((pos, vel))
    return out


def pp_flop(reps):
    """Algorithmic PP work of one step: N rc^3/2 unique in-cutoff pairs per
    replica (number density 3/(4 pi)) x 48 FLOP."""
    return float(sum(r.N * r.rc ** 3 / 2.0 * FLOP_PER_PAIR for r in reps))


def hbm_peak_gbs():
    """HBM copy bandwidth: the measured figure of MEASURED_PEAKS.json where
    the file is present, else this pool's earlier measurement (fallback)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        v = float(json.load(open(path))["hbm_gbs"])
        return v, "of measured (MEASURED_PEAKS.json)"
    except Exception:
        return 6650.0, "of fallback (6.65 TB/s: MEASURED_PEAKS.json absent)"


def step_roofline_s(reps, fp32_tflops, hbm_gbs, nq=32):
    """Time of one step of every replica at the roofline: the PP pairs and
    the n(q,t) sums on the FP32 pipe, the mesh arrays (each FP32 stage array
    written and read once: 66 M^3 bytes) and the particle state (FP64
    pos/vel read and written, FP32 accelerations: 120 N bytes) at HBM speed."""
    flop = pp_flop(reps) + sum(r.N * 3 * nq * 8.0 for r in reps)
    byts = sum(66.0 * r.M ** 3 + 120.0 * r.N for r in reps)
    return flop / (fp32_tflops * 1e12) + byts / (hbm_gbs * 1e9)


def working_set_mb(reps):
    b = 0
    for r in reps:
        M = r.M
        spec = (M // 2 + 1) * M * M
        nb = (M // 16) ** 3
        b += r.N * (3 * 3 * 8 + 32 + 16 + 16 + 40)        # state, staged, acc_pp/pm, keys
        b += spec * 8 * 4 + spec * 4 + 3 * M ** 3 * 4      # spectra, green, fields
        b += nb * 21 ** 3 * 8                              # assignment tiles
    return b / 1e6


def rank_first_seed(rank, n_replicas):
    """Seeds of rank r's ensemble: 1 + r R .. (r + 1) R (disjoint over ranks)."""
    return 1 + rank * n_replicas


def max_over_ranks(x, world, device):
    """The largest x over all ranks (every rank calls it, in the same order)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload_replicas(name, n_replicas, rank):
    """The replicas rank `rank` runs: cfg3's ensemble with the rank's seeds,
    or the named configuration with its seeds shifted by 1000 per rank."""
    import dataclasses

    from p3m_b200.configs import WORKLOADS, cfg3

    if name == "cfg3":
        return cfg3(n_replicas, first_seed=rank_first_seed(rank, n_replicas))
    reps = WORKLOADS[name]()
    return [dataclasses.replace(r, seed=r.seed + 1000 * rank) for r in reps]


def job_value(n_part_per_rank, steps, world, ms_max):
    """Whole-job particle-steps/s: every rank's particles over the slowest
    rank's time (weak scaling: each rank has the same work)."""
    return n_part_per_rank * steps * world / (ms_max * 1e-3)


def dist_setup(backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


# ---------------------------------------------------------------------------
# reference arm: the oracle port on the host cores
# ---------------------------------------------------------------------------
def _green_slab(args):
    """Planes z0 <= nz < z1 of the influence function (oracle, FP64)."""
    kappa, alpha, M, L, z0, z1 = args
    from oracle import oracle as O

    nz, ny, nx = np.meshgrid(np.arange(z0, z1), np.arange(M), np.arange(M), indexing="ij")
    idx = np.stack([nz.ravel(), ny.ravel(), nx.ravel()], axis=1)
    return z0, O.gf_opt_points(kappa, alpha, 6, 3, M, L, idx).reshape(z1 - z0, M, M)


def _ref_greens(pool, reps):
    """The influence function of every distinct (kappa, alpha, M, L), by the
    oracle's gf_opt (yukawa_gf_opt.py:5-98) split over the pool in z slabs.
    Set-up, outside the timed region (the reference times it apart too)."""
    keys = sorted({(r.kappa, r.alpha, r.M, r.L) for r in reps})
    tasks = []
    for key in keys:
        M = key[2]
        step = max(1, M // 16)
        tasks += [key + (z0, min(M, z0 + step)) for z0 in range(0, M, step)]
    out = {k: np.zeros((k[2],) * 3) for k in keys}
    for t, (z0, slab) in zip(tasks, pool.map(_green_slab, tasks, chunksize=1)):
        out[t[:4]][z0:z0 + slab.shape[0]] = slab
    return out


def _ref_group(wid, items, warm, steps, barrier, queue):
    """One worker process: its own fixed set of replicas, each set up
    (initial state, first force call) and warmed up before the barrier; then
    the timed NVE steps of all of them. Puts (wid, t_start, t_end, error)."""
    try:
        from oracle import oracle as O

        import initialize_pos_vel

        states = []
        for (N, L, kappa, alpha, rc, M, dt, Gamma, seed), G in items:
            P = O.Params(N, kappa, alpha, rc, M, L=L, Gamma=Gamma, dt=dt)
            kv = 2 * np.pi * (np.arange(M) - M // 2) / L
            P._gk = (G, kv.reshape(1, M), kv.reshape(M, 1), kv.reshape(M, 1, 1), 0.0)
            pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
            initialize_pos_vel.initial(seed, N, [L] * 3, pos, vel, 1.0 / Gamma)
            _, acc, _ = O.force_pot(P, pos)
            states.append([P, pos, vel, acc])
        for _ in range(warm):
            for st in states:
                st[1], st[2], st[3], _ = O.update(st[0], st[1], st[2], st[3])
        barrier.wait()
        t0 = time.monotonic()
        for _ in range(steps):
            for st in states:
                st[1], st[2], st[3], _ = O.update(st[0], st[1], st[2], st[3])
        queue.put((wid, t0, time.monotonic(), None))
    except Exception as e:  # reported by the parent
        try:
            barrier.abort()
        finally:
            queue.put((wid, 0.0, 0.0, repr(e)))


def balance(sizes, nproc):
    """Replica indices per process: largest first, each onto the process
    with the fewest particles so far (ties: the lowest process)."""
    groups = [[] for _ in range(nproc)]
    load = [0] * nproc
    for i in sorted(range(len(sizes)), key=lambda i: -sizes[i]):
        k = load.index(min(load))
        groups[k].append(i)
        load[k] += sizes[i]
    return groups


def run_reference(args):
    world, rank, _ = dist_setup("gloo")
    if rank != 0:
        return 0
    import multiprocessing as mp

    from oracle import oracle as O

    O.build()
    reps = workload_replicas(args.workload, args.replicas, 0)
    cores = os.cpu_count() or 1
    nproc = min(len(reps), cores)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        greens = _ref_greens(pool, reps)
    params = [(r.N, r.L, r.kappa, r.alpha, r.rc, r.M, r.dt, 1.0 / r.T_desired, r.seed) for r in reps]
    # each process owns a fixed set of replicas, so nothing is set up inside
    # the timed region
    owned = balance([r.N for r in reps], nproc)
    groups = [[(params[i], greens[(reps[i].kappa, reps[i].alpha, reps[i].M, reps[i].L)])
               for i in idx] for idx in owned]
    load = [sum(reps[i].N for i in idx) for idx in owned]
    # bounded sample: the GPU arm's step and warm-up counts, capped so the arm
    # ends within a few minutes (about 0.15 s per 1e4-particle replica step)
    big = max(load) > 2 * 10 ** 5
    steps = max(1, min(args.steps, 2 if big else 20))
    warm = max(1, min(args.warmup, 1 if big else 5))
    barrier = ctx.Barrier(nproc, timeout=1800)
    queue = ctx.Queue()
    procs = [ctx.Process(target=_ref_group, args=(k, groups[k], warm, steps, barrier, queue))
             for k in range(nproc)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=3600) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    errors = [r[3] for r in results if r[3]]
    if errors:
        raise RuntimeError(f"reference arm worker failed: {errors[0]}")
    wall = max(r[2] for r in results) - min(r[1] for r in results)
    total = sum(r.N for r in reps) * steps
    value = total / wall
    sample = (f"{len(reps)} replicas ({args.workload}) advanced {steps} NVE steps each "
              f"(after {warm} untimed) by the oracle port (C PP + numpy FFT/PM; the "
              f"reference's FP64 algorithm) in {nproc} spawned processes, each owning a fixed "
              f"set of replicas set up before the timed region; wall {wall:.2f} s from the "
              "first process's start to the last one's end")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * wall / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded initialize_pos_vel states)",
            "config": {"workload": WORKLOADS_TEXT[args.workload], "replicas": len(reps),
                       "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def cpu_baseline_port(rep, G, n_steps=None):
    """The oracle port on one core for replica `rep` (bounded sample)."""
    from oracle import oracle as O

    if n_steps is None:
        n_steps = 1 if rep.N > 2 * 10 ** 5 else 4

    M = rep.M
    P = O.Params(rep.N, rep.kappa, rep.alpha, rep.rc, M, L=rep.L, Gamma=1.0 / rep.T_desired,
                 dt=rep.dt)
    kv = 2 * np.pi * (np.arange(M) - M // 2) / rep.L
    P._gk = (G, kv.reshape(1, M), kv.reshape(M, 1), kv.reshape(M, 1, 1), 0.0)
    (pos, vel), = initial_states([rep])
    _, acc, _ = O.force_pot(P, pos)
    times = []
    for _ in range(n_steps):
        t0 = time.perf_counter()
        pos, vel, acc, _ = O.update(P, pos, vel, acc)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    return {"value": rep.N / t, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 replica (N={rep.N}, {M}^3) x {n_steps} NVE steps, median step "
                      f"{t * 1e3:.1f} ms, oracle port (C PP + numpy FFT/PM), 1 thread"}


def run_ours(args):
    import torch

    world, rank, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    from p3m_b200 import FP32, MODE_NVE, MODE_THERMOSTAT, Context
    from p3m_b200.configs import CFG3_QMULT

    reps = workload_replicas(args.workload, args.replicas, rank)
    states = initial_states(reps)
    ctx = Context(reps, precision=FP32, device=local)
    for i, (p, v) in enumerate(states):
        ctx.set_state(i, p, v)
    ctx.init_forces()
    ctx.set_nqt(CFG3_QMULT, 4096)
    stream = torch.cuda.ExternalStream(ctx.stream())

    # equilibration with the reference's thermostat (thermostat_p3m_ord6.vscale)
    # from the random initial state, then NVE warm-up (also builds the graph)
    ctx.equilibrate(args.equil, quench_steps=args.quench)
    tuned = None
    if args.pp_config:
        tpi, skin = args.pp_config.split(",")
        ctx.set_tuning(pp_tpi=int(tpi), skin=float(skin), prune_buf=args.prune_buf)
    elif not args.no_tune:
        from p3m_b200.autotune import tune

        tuned = tune(ctx, use_cache=False)
    ctx.run(max(args.warmup, 3), MODE_NVE, record_nqt=True, graph=True)
    rb0 = sum(ctx.replica_stats(i)["rebuilds"] for i in range(len(reps)))
    ib0 = sum(ctx.inner_builds(i) for i in range(len(reps)))

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    ctx.sync()
    n0 = ctx.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.run(args.steps, MODE_NVE, record_nqt=True, graph=True, sync=False)
    e1.record(stream)
    e1.synchronize()
    ctx.sync()
    ms = e0.elapsed_time(e1)
    launches = ctx.launch_count() - n0
    rebuilds = sum(ctx.replica_stats(i)["rebuilds"] for i in range(len(reps))) - rb0
    inner_builds = sum(ctx.inner_builds(i) for i in range(len(reps))) - ib0
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ctx.check()
    ms = max_over_ranks(ms, world, "cuda")
    n_part = sum(r.N for r in reps)
    value = job_value(n_part, args.steps, world, ms)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded initialize_pos_vel: uniform positions, Maxwell-Boltzmann "
                    "velocities)",
            "config": {"workload": WORKLOADS_TEXT[args.workload], "replicas": len(reps),
                       "N_per_replica": reps[0].N if len({r.N for r in reps}) == 1 else "varies",
                       "mesh": reps[0].M if len({r.M for r in reps}) == 1 else "varies", "parallelism": f"replicas x{world}" if world > 1 else "replicas",
                       "l2": (f"inputs larger than L2 (working set {working_set_mb(reps):.0f} MB > 126 MB)"
                              if working_set_mb(reps) > 126 else
                              f"working set {working_set_mb(reps):.0f} MB fits L2; no flush"),
                       "pp_config": dict(zip(("threads_per_particle", "skin", "list_capacity"),
                                             ctx.pp_config())),
                       "tuning": ctx.tuning(),
                       "list_rebuilds_per_replica_step": rebuilds / (len(reps) * args.steps),
                       "inner_list_builds_per_replica_step": inner_builds / (len(reps) * args.steps),
                       "autotune_ms_per_step": tuned["ms_per_step"] if tuned else None,
                       "autotune_final_ms_per_step": tuned.get("final_ms_per_step") if tuned else None},
            "gpu_launches": launches, "clocks": clocks}

    if not args.no_extras and rank == 0:
        eq_states = [ctx.get_state(i)[:2] for i in range(len(reps))]
        extras(args, line, ctx, reps, eq_states, local)
    ctx.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def extras(args, line, ctx, reps, states, device):
    import torch

    from p3m_b200 import FP32, FP64, MODE_NVE, Context, fp32_peak_tflops, gf_opt_device, lib

    # -- per-stage device times and the PP roofline (FP32 pipe) ------------------
    try:
        stages = ctx.profile_stages(iters=20)
    except Exception as e:  # measurement only: report and carry on
        print(f"profile_stages: {e}", file=sys.stderr)
        stages = {}
    flagged = [k for k, v in stages.items() if v < 0]
    if flagged:
        print(f"profile_stages: status raised in {flagged}: "
              f"{lib().p3m_last_error(ctx.handle).decode()}", file=sys.stderr)
        stages = {k: abs(v) for k, v in stages.items()}
    peak = fp32_peak_tflops(device)
    pp_ms = stages.get("pp", 0.0)
    flop = pp_flop(reps)
    traffic, traffic_src = None, None
    tpath = os.path.join(ROOT, "profiles", "pp_traffic.json")
    if os.path.exists(tpath) and args.workload == "cfg3":
        try:
            tj = json.load(open(tpath))
            traffic = tj.get("cfg3_bytes_per_launch")
            traffic_src = f"profiles/pp_traffic.json: {tj.get('source', 'ncu capture')}"
        except Exception:
            traffic = None
    achieved = flop / (pp_ms * 1e-3) / 1e12 if pp_ms > 0 else None
    hbm, hbm_src = hbm_peak_gbs()
    t_roof = step_roofline_s(reps, peak, hbm)
    line["roofline"] = {"kernel": "k_pp_f32 (PP pair loop, FP32)", "bound": "fp32",
                        "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                        "traffic_source": traffic_src,
                        "peak_source": "measured FP32 FMA probe (p3m_fp32_peak) on this GPU; "
                                       "MEASURED_PEAKS.json has no FP32 figure",
                        "work": f"{flop:.3e} FLOP per launch = sum N rc^3/2 pairs x {FLOP_PER_PAIR}",
                        "step_t_roof_ms": t_roof * 1e3,
                        "step_frac": t_roof * 1e3 / line["ms_per_step"],
                        "step_roof_how": (f"sum over replicas of N rc^3/2 x {FLOP_PER_PAIR} FLOP and "
                                          f"n(q,t) N x 3 x Nq x 8 FLOP at {peak:.1f} TFLOP/s, plus "
                                          f"66 M^3 + 120 N bytes at {hbm:.0f} GB/s ({hbm_src})")}
    if "fft_both" in stages and "fft_forward" in stages:
        stages["fft_inverse"] = stages["fft_both"] - stages["fft_forward"]
    line["stages_ms"] = {k: round(v, 5) for k, v in stages.items()}

    # -- FP32 force error against the FP64 path on replica 0's initial state -----
    r0 = reps[0]
    with Context(r0, precision=FP64, device=device) as c64, \
            Context(r0, precision=FP32, device=device) as c32:
        _, a64, _ = c64.force(states[0][0])
        _, a32, _ = c32.force(states[0][0])
    ref_rms = np.sqrt(np.mean(np.sum(a64 ** 2, axis=1)))
    line["force_err"] = {
        "rms_rel": float(np.sqrt(np.sum((a32 - a64) ** 2) / np.sum(a64 ** 2))),
        "max_rel": float(np.max(np.sqrt(np.sum((a32 - a64) ** 2, axis=1))) / ref_rms),
        "vs": "FP64 device path (pinned to the FP64 oracle by the parity tests)"}

    # -- the plain FP64 single-replica path on the same ensemble -------------------
    t_tot, ps = 0.0, 0
    nrun = min(args.steps, 20)
    for r, (p, v) in zip(reps, states):
        with Context(r, precision=FP64, device=device) as c:
            c.set_state(0, p, v)
            c.init_forces()
            c.run(3, MODE_NVE, graph=True)
            s = torch.cuda.ExternalStream(c.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            c.run(nrun, MODE_NVE, graph=True, sync=False)
            e1.record(s)
            e1.synchronize()
            t_tot += e0.elapsed_time(e1) * 1e-3
            ps += r.N * nrun
    fp64 = ps / t_tot
    line["fp64_plain"] = {"value": fp64, "unit": UNIT,
                          "how": f"each replica alone, FP64 bulk, graph-captured NVE steps "
                                 f"({nrun} per replica, device-timed)",
                          "batched_fp32_over_fp64": line["value"] / line["n_gpus"] / fp64}

    # -- end to end through the C ABI with host buffers ----------------------------
    # per step: H2D of the whole ensemble's (pos, vel, acc) from pinned host
    # memory, one step, D2H of the state and of the step's energies. An
    # ensemble of several replicas is held as up to five contexts on their
    # own streams with asynchronous copies, so one part's copies overlap the
    # others' steps (the copy engines and the SMs work at the same time).
    ntot = sum(r.N for r in reps)
    nparts = min(args.e2e_parts, len(reps))
    cuts = [round(k * len(reps) / nparts) for k in range(nparts + 1)]
    halves = [reps[cuts[k]:cuts[k + 1]] for k in range(nparts)]
    offs = np.cumsum([0] + [sum(r.N for r in h) for h in halves])
    pos_all = np.concatenate([st[0] for st in states])
    vel_all = np.concatenate([st[1] for st in states])
    host = []
    for k in range(len(halves)):
        n = int(offs[k + 1] - offs[k])
        hb = [torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
        hb[0][:] = pos_all[offs[k]:offs[k + 1]]
        hb[1][:] = vel_all[offs[k]:offs[k + 1]]
        host.append(hb)
    ctxs = [Context(h, precision=FP32, device=device) for h in halves]
    try:
        # descending stream priorities: the first part finishes its step first
        # and its copies back overlap the later parts' steps; every part runs
        # the kernel shapes installed on the timed ensemble
        shapes = ctx.tuning()
        for k, c in enumerate(ctxs):
            c.set_priority(k)
            c.set_tuning(**shapes)
        for c, hb in zip(ctxs, host):
            c.set_state_all(hb[0], hb[1])
            c.init_forces()
            c.get_state_all(*hb)
            c.run(2, MODE_NVE, graph=True)
            c.get_state_all(*hb)
        n_e2e = min(args.steps, 200)
        ebuf = [torch.empty((len(h), 4), dtype=torch.float64, pin_memory=True).numpy()
                for h in halves]
        s = torch.cuda.ExternalStream(ctxs[0].stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        # each context's step k+1 starts from the host arrays its step k
        # wrote back: wait for that context only (the host reads its result,
        # then hands it in again), so while one context's copies run the
        # others compute and no step waits for the whole ensemble
        for k in range(n_e2e):
            for c, hb, eb in zip(ctxs, host, ebuf):
                if k:
                    c.sync()  # this context's previous step is in hb, eb
                c.set_state_all(*hb, keep_lists=True, sync=False)
                c.run(1, MODE_NVE, graph=True, sync=False)
                c.get_step_async(*hb, eb)
        for c in ctxs:
            c.sync()
        e1.record(s)  # after every context's work: the host synchronised on all
        e1.synchronize()
        t = e0.elapsed_time(e1) * 1e-3
    finally:
        for c in ctxs:
            c.close()
    nb = ntot * 3 * 8
    line["e2e"] = {"value": ntot * n_e2e / t, "unit": UNIT,
                   "h2d_bytes_per_step": 3 * nb, "d2h_bytes_per_step": 3 * nb + 8 * 8 * len(reps) + 4 * len(halves),
                   "how": ("p3m_set_state_all_async (pinned host -> device, lists kept), "
                           "p3m_run(1, sync=0), p3m_get_step_async (state and energies back) "
                           f"per step on each of {len(halves)} contexts (its own streams, "
                           "priority levels 0, 1, ...); a context's next step is queued after "
                           "p3m_sync on that context alone (its result back in the host "
                           "arrays it hands in again)")}

    # -- CPU baseline: the oracle port on one host core ------------------------------
    G, _ = gf_opt_device(r0.kappa, r0.alpha, 6, 3, r0.M, r0.L, device=device)
    line["cpu_baseline"] = cpu_baseline_port(r0, G)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
