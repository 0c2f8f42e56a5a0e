"""Python wrapper of a p3m_b200 context (one or more replicas on one GPU)."""
from __future__ import annotations

import ctypes
import os
from collections import OrderedDict
from dataclasses import dataclass, field

import numpy as np

from ._lib import (FP32, FP64, MODE_NVE, MODE_THERMOSTAT, P3MError, ReplicaDesc, Tuning, check,
                   dptr, lib)


@dataclass
class Replica:
    """One independent system: the constants of yukawa_MD_p3m_ord6.py:26-79."""

    N: int
    L: float
    kappa: float
    alpha: float
    rc: float
    M: int = 0
    dt: float = 0.1
    T_desired: float = 0.01
    af: float = 1.0 / 3.0
    uf: float = 1.0
    kf: float = 1.5
    p: int = 6
    m_alias: int = 3
    skin: float = -1.0  # Verlet-list skin; negative: the library's default
    seed: int = field(default=0, compare=False)

    def desc(self) -> ReplicaDesc:
        return ReplicaDesc(int(self.N), int(self.M), int(self.p), int(self.m_alias),
                           float(self.L), float(self.kappa), float(self.alpha), float(self.rc),
                           float(self.dt), float(self.T_desired), float(self.af),
                           float(self.uf), float(self.kf), float(self.skin))


def _out(a, shape):
    """An output array: a new one, or the caller's if it is FP64, C-order and
    of the right shape."""
    if a is None:
        return np.empty(shape)
    if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != tuple(shape):
        raise ValueError(f"output array must be float64, C-contiguous, shape {tuple(shape)}")
    return a


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


class Context:
    """Device buffers, stream and CUDA graphs for a batch of replicas."""

    def __init__(self, replicas, precision=FP32, device=0):
        if isinstance(replicas, Replica):
            replicas = [replicas]
        self.replicas = list(replicas)
        self.precision = precision
        self.device = device
        R = len(self.replicas)
        arr = (ReplicaDesc * R)(*[r.desc() for r in self.replicas])
        h = ctypes.c_void_p()
        rc = lib().p3m_create(arr, R, int(precision), int(device), ctypes.byref(h))
        check(rc, None)
        self._h = h
        self._green_key = [None] * R
        self._nq = 0
        self._nqt_cap = 0
        self._snap_cap = 0

    # -- lifetime -------------------------------------------------------------
    @property
    def handle(self):
        if self._h is None:
            raise P3MError(-6, "context is closed")
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().p3m_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, rc):
        return check(rc, self.handle)

    # -- compat calls (single replica) -----------------------------------------
    def pp(self, pos):
        """yukawa_pp.particle_particle -> (U, acc)."""
        pos = _f64(pos)
        acc = np.empty_like(pos)
        U = np.zeros(1)
        self._ck(lib().p3m_pp(self.handle, 0, dptr(pos), dptr(acc), dptr(U)))
        return float(U[0]), acc

    def assign(self, pos, Z=None):
        """charge_assgn_6_numba -> rho (M,M,M)."""
        M = self.replicas[0].M
        pos = _f64(pos)
        rho = np.empty((M, M, M))
        self._ck(lib().p3m_assign(self.handle, 0, dptr(pos), dptr(None if Z is None else _f64(Z)),
                                  dptr(rho)))
        return rho

    def gather(self, pos, Z, Ex, Ey, Ez):
        """field_assgn_6_numba -> (acc (N,3), E_p (3,N))."""
        pos = _f64(pos)
        n = pos.shape[0]
        acc = np.empty((n, 3))
        Ep = np.empty((3, n))
        self._ck(lib().p3m_gather(self.handle, 0, dptr(pos), dptr(None if Z is None else _f64(Z)),
                                  dptr(_f64(Ex)), dptr(_f64(Ey)), dptr(_f64(Ez)), dptr(acc),
                                  dptr(Ep)))
        return acc, Ep

    def set_green(self, G_k=None, replica=0):
        """Install an influence function (fftshifted (M,M,M) FP64), or compute
        it on the device when G_k is None."""
        self._ck(lib().p3m_set_green(self.handle, replica,
                                     dptr(None if G_k is None else _f64(G_k))))

    def set_green_cached(self, G_k, replica=0):
        """set_green, skipped when the same array (same buffer and sampled
        contents) was installed last."""
        G = _f64(G_k)
        flat = G.reshape(-1)
        idx = np.linspace(0, flat.size - 1, 61).astype(np.int64)
        key = (G.ctypes.data, G.shape, flat[idx].tobytes())
        if self._green_key[replica] != key:
            self.set_green(G, replica)
            self._green_key[replica] = key

    def pm(self, pos, Z=None, want_rho=False):
        """particle_mesh_fft_r -> (U_f, acc (N,3), E_p (3,N), rho or None)."""
        M = self.replicas[0].M
        pos = _f64(pos)
        n = pos.shape[0]
        acc = np.empty((n, 3))
        Ep = np.empty((3, n))
        U = np.zeros(1)
        rho = np.empty((M, M, M)) if want_rho else None
        self._ck(lib().p3m_pm(self.handle, 0, dptr(pos), dptr(None if Z is None else _f64(Z)),
                              dptr(acc), dptr(U), dptr(Ep), dptr(rho)))
        return float(U[0]), acc, Ep, rho

    def force(self, pos, Z=None):
        """force_pot -> (U, acc, (U_short, U_fft, U_self))."""
        pos = _f64(pos)
        acc = np.empty_like(pos)
        U = np.zeros(1)
        parts = np.zeros(3)
        self._ck(lib().p3m_force(self.handle, 0, dptr(pos), dptr(None if Z is None else _f64(Z)),
                                 dptr(acc), dptr(U), dptr(parts)))
        return float(U[0]), acc, tuple(float(x) for x in parts)

    def update(self, pos, vel, acc):
        """velocity_verlet update, in place on the given float64 arrays -> U."""
        U = np.zeros(1)
        self._ck(lib().p3m_update(self.handle, 0, dptr(pos), dptr(vel), dptr(acc), dptr(U)))
        return float(U[0])

    def vscale(self, it, pos, vel, acc):
        """thermostat vscale, in place -> (U, T before rescale)."""
        U = np.zeros(1)
        T = np.zeros(1)
        self._ck(lib().p3m_vscale(self.handle, 0, int(it), dptr(pos), dptr(vel), dptr(acc),
                                  dptr(U), dptr(T)))
        return float(U[0]), float(T[0])

    def nqt(self, pos, qv, replica=0):
        """One n(q,t) row: complex128 (nq, 3)."""
        pos = _f64(pos)
        qv = _f64(qv)
        out = np.empty((len(qv), 3, 2))
        self._ck(lib().p3m_nqt(self.handle, replica, dptr(pos), dptr(qv), len(qv), dptr(out)))
        return out[..., 0] + 1j * out[..., 1]

    # -- device-resident path ------------------------------------------------------
    def set_state(self, replica, pos=None, vel=None, acc=None):
        self._ck(lib().p3m_set_state(self.handle, replica,
                                     dptr(None if pos is None else _f64(pos)),
                                     dptr(None if vel is None else _f64(vel)),
                                     dptr(None if acc is None else _f64(acc))))

    def get_state(self, replica, pos=None, vel=None, acc=None):
        """-> (pos, vel, acc) of one replica, into the given (n,3) FP64
        C-order arrays where passed (e.g. pinned buffers)."""
        n = self.replicas[replica].N
        pos, vel, acc = (_out(a, (n, 3)) for a in (pos, vel, acc))
        self._ck(lib().p3m_get_state(self.handle, replica, dptr(pos), dptr(vel), dptr(acc)))
        return pos, vel, acc

    def set_state_all(self, pos=None, vel=None, acc=None, keep_lists=False, sync=True):
        """State of every replica from (sum N, 3) arrays in replica order.
        keep_lists: keep the neighbour lists (continuing a trajectory).
        sync=False: only queue the copies (the arrays must be FP64 C-order,
        ideally pinned, and untouched until sync())."""
        n = sum(r.N for r in self.replicas)
        if not sync:
            for x in (pos, vel, acc):
                if x is not None and (x.dtype != np.float64 or not x.flags.c_contiguous
                                      or x.shape != (n, 3)):
                    raise ValueError("asynchronous copies need (sum N, 3) float64 C-order arrays")
            self._ck(lib().p3m_set_state_all_async(self.handle, dptr(pos), dptr(vel), dptr(acc),
                                                   int(bool(keep_lists))))
            return
        self._ck(lib().p3m_set_state_all(self.handle,
                                         dptr(None if pos is None else _f64(pos, (n, 3))),
                                         dptr(None if vel is None else _f64(vel, (n, 3))),
                                         dptr(None if acc is None else _f64(acc, (n, 3))),
                                         int(bool(keep_lists))))

    def get_state_all(self, pos=None, vel=None, acc=None, sync=True):
        """-> (pos, vel, acc) of every replica, (sum N, 3) in replica order.
        sync=False: only queue the copies into the given arrays (valid after
        sync())."""
        n = sum(r.N for r in self.replicas)
        if not sync and any(a is None for a in (pos, vel, acc)):
            raise ValueError("asynchronous reads need the three output arrays")
        pos, vel, acc = (_out(a, (n, 3)) for a in (pos, vel, acc))
        fn = lib().p3m_get_state_all if sync else lib().p3m_get_state_all_async
        self._ck(fn(self.handle, dptr(pos), dptr(vel), dptr(acc)))
        return pos, vel, acc

    def get_step_async(self, pos, vel, acc, energies):
        """Queue the copies of the state and of every replica's (U, K, T,
        thermostat factor) after the last step, (R, 4), into the given arrays;
        they hold the values once sync() returns (which then needs no further
        device read). Pass pinned arrays for full copy speed."""
        if any(a is None for a in (pos, vel, acc, energies)):
            raise ValueError("asynchronous reads need the four output arrays")
        n = sum(r.N for r in self.replicas)
        for a in (pos, vel, acc):
            _out(a, (n, 3))
        _out(energies, (len(self.replicas), 4))
        self._ck(lib().p3m_get_step_async(self.handle, dptr(pos), dptr(vel), dptr(acc),
                                          dptr(energies)))

    def set_t_desired(self, t_desired):
        """Thermostat targets for the following thermostat-mode runs: one
        value per replica, or one for all."""
        t = np.broadcast_to(np.asarray(t_desired, dtype=np.float64), (len(self.replicas),)).copy()
        self._ck(lib().p3m_set_t_desired(self.handle, dptr(t)))

    def equilibrate(self, steps, quench_steps=200, quench_factor=0.01):
        """Thermostat phase from seeded random positions: `quench_steps` of
        the reference's thermostat at quench_factor * T_desired, then `steps`
        at T_desired. Uniformly random initial positions leave close pairs
        whose repulsion launches a few particles at tens of times the thermal
        speed; in weakly coupled, strongly screened replicas the reference's
        rescaling alone does not slow them within thousands of steps (their
        collisions weaken as the speed grows), and at dt = 0.1 they heat the
        system. The quench damps them with everything else."""
        td = np.array([r.T_desired for r in self.replicas])
        if quench_steps > 0:
            self.set_t_desired(td * quench_factor)
            try:
                self.run(quench_steps, MODE_THERMOSTAT, it0=0)
            finally:
                self.set_t_desired(td)
        if steps > 0:
            self.run(steps, MODE_THERMOSTAT, it0=0)

    def init_forces(self):
        self._ck(lib().p3m_init_forces(self.handle))

    def set_nqt(self, qmult, capacity):
        qm = None if qmult is None or len(qmult) == 0 else _f64(qmult)
        self._nq = 0 if qm is None else len(qm)
        self._nqt_cap = int(capacity)
        self._ck(lib().p3m_set_nqt(self.handle, dptr(qm), 0 if qm is None else len(qm),
                                   int(capacity)))

    def run(self, n_steps, mode=MODE_NVE, it0=0, record_nqt=False, graph=True, sync=True):
        self._ck(lib().p3m_run(self.handle, int(n_steps), int(mode), int(it0), int(bool(record_nqt)),
                               int(bool(graph)), int(bool(sync))))

    def thermostat(self, n_steps, it0=0, **kw):
        self.run(n_steps, MODE_THERMOSTAT, it0=it0, **kw)

    def energies(self, max_steps=1 << 20):
        """Per-step (U, K, T, factor) of every replica: (steps, R, 4)."""
        R = len(self.replicas)
        cap = min(max_steps, 8192)
        out = np.empty((cap, R, 4))
        n = ctypes.c_int()
        self._ck(lib().p3m_get_energies(self.handle, dptr(out), cap, ctypes.byref(n)))
        return out[: n.value]

    def get_nqt(self, replica, nq, max_steps=None):
        """The recorded n(q,t) rows of one replica, oldest first: (steps, nq, 3)
        complex."""
        if max_steps is None:
            max_steps = max(1, self._nqt_cap)
        out = np.empty((max_steps, nq, 3, 2))
        n = ctypes.c_int()
        self._ck(lib().p3m_get_nqt(self.handle, replica, dptr(out), max_steps, ctypes.byref(n)))
        o = out[: n.value]
        return o[..., 0] + 1j * o[..., 1]

    def set_snapshots(self, interval, capacity=64):
        """Copy [pos | vel | acc] of every replica into a device ring after
        each step it of run() with (it + 1) % interval == 0 (0: off)."""
        self._ck(lib().p3m_set_snapshots(self.handle, int(interval), int(capacity)))
        self._snap_cap = int(capacity) if interval > 0 else 0

    def get_snapshots(self, max_snaps=None):
        """The snapshots taken since the last call, oldest first ->
        (array (n, sum N, 9), step indices (n,))."""
        ntot = sum(r.N for r in self.replicas)
        m = self._snap_cap if max_snaps is None else int(max_snaps)
        out = np.empty((max(m, 1), ntot, 9))
        steps = np.empty(max(m, 1), dtype=np.int32)
        n = ctypes.c_int()
        self._ck(lib().p3m_get_snapshots(self.handle, dptr(out),
                                         steps.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), m,
                                         ctypes.byref(n)))
        return out[: n.value], steps[: n.value]

    def sqw(self, dt, nt, col0=0, col_stride=1, ncols=None, per_replica=False):
        """S(q,w) of the last nt recorded n(q,t) rows, averaged over axes and
        replicas: (ncols, nt); with per_replica also (R, ncols, nt)."""
        nq = self._nq
        if ncols is None:
            ncols = (nq - col0 + col_stride - 1) // col_stride
        out = np.empty((ncols, nt))
        rep = np.empty((len(self.replicas), ncols, nt)) if per_replica else None
        self._ck(lib().p3m_sqw(self.handle, float(dt), int(col0), int(col_stride), int(ncols),
                               int(nt), dptr(out), dptr(rep)))
        return (out, rep) if per_replica else out

    def replica_stats(self, replica=0):
        """{U_short, U_fft, U_self, U, K, T, factor, rebuilds} of one replica."""
        out = np.zeros(8)
        self._ck(lib().p3m_get_replica_stats(self.handle, int(replica), dptr(out)))
        keys = ("U_short", "U_fft", "U_self", "U", "K", "T", "factor", "rebuilds")
        return dict(zip(keys, (float(x) for x in out)))

    def inner_builds(self, replica=0):
        """Inner-list builds of one replica between Verlet-list rebuilds
        (prune_buf > 0)."""
        out = np.zeros(1)
        self._ck(lib().p3m_get_inner_builds(self.handle, int(replica), dptr(out)))
        return float(out[0])

    def check(self):
        self._ck(lib().p3m_check(self.handle))

    def sync(self):
        self._ck(lib().p3m_sync(self.handle))

    def set_priority(self, level):
        """Scheduling priority of this context's streams: 0 is the device's
        highest, larger levels are lower. For several contexts sharing a GPU
        (copies of one overlapping steps of another). Recreates the streams:
        query stream() afterwards."""
        self._ck(lib().p3m_set_priority(self.handle, int(level)))

    def launch_count(self):
        return int(lib().p3m_launch_count(self.handle))

    def stream(self):
        return lib().p3m_stream(self.handle)

    def profile_stages(self, iters=20):
        """{stage name: average ms per launch} (perturbs the state: call after
        the measured run)."""
        ms = np.zeros(16)
        n = ctypes.c_int()
        self._ck(lib().p3m_profile_stages(self.handle, int(iters), dptr(ms), 16, ctypes.byref(n)))
        return {lib().p3m_stage_name(i).decode(): float(ms[i]) for i in range(n.value)}

    def set_pp_config(self, tpi, skin=-1.0):
        """Threads per particle of the PP force kernel and the list skin."""
        self._ck(lib().p3m_set_pp_config(self.handle, int(tpi), float(skin)))

    def tuning(self):
        """{pp_tpi, cell_div, plane_max, gather_mode, skin, prune_buf}: the kernel shapes."""
        t = Tuning()
        self._ck(lib().p3m_get_tuning(self.handle, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        """Change some of the kernel shapes (the others keep their values):
        pp_tpi (1, 2, 4, 8), cell_div (1, 2), plane_max (0, 32, 64),
        gather_mode (0, 1, 2), skin, prune_buf (FP32: 0, or the inner-list
        buffer beyond rc, below the skin)."""
        cur = self.tuning()
        unknown = set(kw) - set(cur)
        if unknown:
            raise ValueError(f"unknown tuning keys {sorted(unknown)}")
        cur.update(kw)
        t = Tuning(int(cur["pp_tpi"]), int(cur["cell_div"]), int(cur["plane_max"]),
                   int(cur["gather_mode"]), float(cur["skin"]), float(cur["prune_buf"]))
        self._ck(lib().p3m_set_tuning(self.handle, ctypes.byref(t)))

    def pp_config(self):
        """-> (threads per particle, skin, list capacity)."""
        t, s, m = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        self._ck(lib().p3m_get_pp_config(self.handle, ctypes.byref(t), ctypes.byref(s),
                                         ctypes.byref(m)))
        return t.value, s.value, m.value


def gf_opt_device(kappa, alpha, p, m_alias, M, L, device=0):
    """yukawa_gf_opt on the GPU in FP64 -> (G_k (M,M,M) fftshifted, A_pm)."""
    G = np.empty((M, M, M))
    A = np.zeros(1)
    check(lib().p3m_gf_opt(int(device), float(kappa), float(alpha), int(p), int(m_alias), int(M),
                           float(L), dptr(G), dptr(A)), None)
    return G, float(A[0])


def _complex_ptr(a):
    return a.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def sqw_series(n_q_t, N, dt, T, device=0):
    """s_of_q_w.n_of_q_w on the device: (nt, 3) complex -> (nt, 3) =
    |dt FFT_t n|^2 / (N T) per axis."""
    a = np.ascontiguousarray(n_q_t, dtype=np.complex128)
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError("n_q_t must have shape (nt, 3)")
    nt = a.shape[0]
    out = np.empty((nt, 3))
    check(lib().p3m_sqw_series(int(device), _complex_ptr(a), nt, float(N), float(dt), float(T),
                               dptr(out)), None)
    return out


def sqw_runs(n_q_t_array, Nq, N, dt, T, col0=0, col_stride=3, device=0):
    """s_of_q_w_avg.s_of_q_w_avg_mat on the device: (runs, nt, nq, 3)
    complex -> (runs, Nq, nt), the mean over axes of S(q,w) on q columns
    col0 + i*col_stride."""
    a = np.ascontiguousarray(n_q_t_array, dtype=np.complex128)
    if a.ndim != 4 or a.shape[3] != 3:
        raise ValueError("n_q_t_array must have shape (runs, nt, nq, 3)")
    R, nt, nq = a.shape[:3]
    out = np.empty((R, int(Nq), nt))
    check(lib().p3m_sqw_runs(int(device), _complex_ptr(a), R, nt, nq, int(col0), int(col_stride),
                             int(Nq), float(N), float(dt), float(T), dptr(out)), None)
    return out


def fp32_peak_tflops(device=0):
    """Measured FP32 FMA throughput of the device (TFLOP/s)."""
    t = np.zeros(1)
    check(lib().p3m_fp32_peak(int(device), dptr(t)), None)
    return float(t[0])


# -- contexts of the compat (reference-signature) functions --------------------------

_PRECISIONS = {"fp64": FP64, "fp32": FP32}
_compat_precision = _PRECISIONS[os.environ.get("P3M_B200_PRECISION", "fp64").lower()]
_compat_cache: "OrderedDict[tuple, Context]" = OrderedDict()
_COMPAT_MAX = 8


def set_compat_precision(name: str):
    """Arithmetic of the reference-signature functions: 'fp64' (default, the
    plain method) or 'fp32' (FP32 bulk stages, FP64 reductions)."""
    global _compat_precision
    _compat_precision = _PRECISIONS[name.lower()]


def compat_precision():
    return _compat_precision


def compat_context(N, L, kappa, alpha, rc, M=0, dt=0.1, T_desired=0.01, af=1.0 / 3.0, uf=1.0,
                   kf=1.5, p=6, m_alias=3):
    key = (int(N), float(L), float(kappa), float(alpha), float(rc), int(M), float(dt),
           float(T_desired), float(af), float(uf), float(kf), int(p), int(m_alias),
           _compat_precision)
    ctx = _compat_cache.get(key)
    if ctx is None:
        ctx = Context(Replica(N=N, L=L, kappa=kappa, alpha=alpha, rc=rc, M=M, dt=dt,
                              T_desired=T_desired, af=af, uf=uf, kf=kf, p=p, m_alias=m_alias),
                      precision=_compat_precision)
        _compat_cache[key] = ctx
        while len(_compat_cache) > _COMPAT_MAX:
            _, old = _compat_cache.popitem(last=False)
            old.close()
    else:
        _compat_cache.move_to_end(key)
    return ctx
