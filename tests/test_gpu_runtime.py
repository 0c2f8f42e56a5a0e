"""Device-resident stepping, batching, graphs, determinism and robustness."""
import numpy as np
import pytest

from gpu_util import oracle_params, rel_rms, replica_from_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _init_state(r, seed):
    import initialize_pos_vel

    pos, vel = np.zeros((r.N, 3)), np.zeros((r.N, 3))
    initialize_pos_vel.initial(seed, r.N, [r.L] * 3, pos, vel, r.T_desired)
    return pos, vel


def test_run_matches_compat_steps(golden):
    """p3m_run (graph) == the compat vscale/update loop, bit for bit."""
    from p3m_b200 import FP64, MODE_NVE, MODE_THERMOSTAT, Context

    g = golden
    r = replica_from_golden(g)
    S = int(g["trace_steps"])
    with Context(r, precision=FP64) as c:
        c.set_green(g["G_k"])
        c.set_state(0, g["pos0"], g["vel0"])
        c.init_forces()
        c.run(S, MODE_THERMOSTAT, it0=0, graph=True)
        c.run(S, MODE_NVE, graph=True)
        pos, vel, acc = c.get_state(0)
        E = c.energies()
    with Context(r, precision=FP64) as c:
        c.set_green(g["G_k"])
        _, a, _ = c.force(g["pos0"])
        p, v = g["pos0"].copy(), g["vel0"].copy()
        for it in range(S):
            c.vscale(it, p, v, a)
        for _ in range(S):
            c.update(p, v, a)
    # the compat calls rebuild the neighbour lists on every call (the caller's
    # arrays may hold any state); p3m_run rebuilds on the skin criterion, so
    # the pair summation order -- and the last bits -- can differ
    np.testing.assert_allclose(pos, p, rtol=0, atol=1e-12)
    np.testing.assert_allclose(vel, v, rtol=0, atol=1e-12)
    np.testing.assert_allclose(acc, a, rtol=1e-10, atol=1e-13)
    assert E.shape == (2 * S, 1, 4)
    np.testing.assert_allclose(E[:, 0, 0], g["trace"][:, 0], rtol=1e-9)


@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_graph_equals_eager_and_deterministic(prec_name):
    from p3m_b200 import FP32, FP64, MODE_NVE, Context, Replica

    prec = {"fp32": FP32, "fp64": FP64}[prec_name]
    N = 3000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=2.0, alpha=0.6, rc=L / 3.2, M=32, dt=0.1, T_desired=0.01)
    pos, vel = _init_state(r, 5)
    outs = []
    for graph in (True, False, True):
        with Context(r, precision=prec) as c:
            c.set_state(0, pos, vel)
            c.init_forces()
            c.run(10, MODE_NVE, graph=graph)
            outs.append(c.get_state(0))
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert np.array_equal(a, b)


def test_batch_replica_equals_alone():
    """A replica inside an uneven batch is bit-identical to the same replica
    run alone (FP32 path)."""
    from p3m_b200 import FP32, MODE_NVE, MODE_THERMOSTAT, Context, Replica

    reps = []
    # meshes of 32 and 64 take the fused plane FFT, 128 the multi-pass one
    for N, kappa, M in [(2000, 1.0, 32), (5000, 2.0, 128), (3000, 0.5, 64)]:
        L = (4 * np.pi * N / 3) ** (1 / 3)
        reps.append(Replica(N=N, L=L, kappa=kappa, alpha=0.7, rc=min(5.0, L / 3.01), M=M, dt=0.1,
                            T_desired=0.02))
    states = [_init_state(r, 11 + i) for i, r in enumerate(reps)]
    # bit-identity holds at equal PP configuration (threads per particle fix
    # the order in which a particle's neighbours are summed)
    with Context(reps, precision=FP32) as c:
        c.set_pp_config(2)
        for i, (p, v) in enumerate(states):
            c.set_state(i, p, v)
        c.init_forces()
        c.run(5, MODE_THERMOSTAT)
        c.run(5, MODE_NVE)
        batch = [c.get_state(i) for i in range(len(reps))]
        E = c.energies()
    for i, r in enumerate(reps):
        with Context(r, precision=FP32) as c:
            c.set_pp_config(2)
            c.set_state(0, *states[i])
            c.init_forces()
            c.run(5, MODE_THERMOSTAT)
            c.run(5, MODE_NVE)
            alone = c.get_state(0)
            Ea = c.energies()
        for a, b in zip(batch[i], alone):
            assert np.array_equal(a, b)
        assert np.array_equal(E[:, i, :], Ea[:, 0, :])


def test_fp32_force_error_cfg1_size():
    """FP32 total-force error against the FP64 oracle at the N=1e4, 64^3,
    kappa=2, alpha=0.6, rc=6 configuration (RMS <= 1e-5)."""
    from p3m_b200 import FP32, FP64, Context, Replica

    N = 10000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=2.0, alpha=0.6, rc=6.0, M=64, T_desired=0.01)
    pos, _ = _init_state(r, 1)
    with Context(r, precision=FP64) as c:
        U64, a64, parts64 = c.force(pos)
        G, A = None, None
    with Context(r, precision=FP32) as c:
        U32, a32, _ = c.force(pos)
    # the FP64 device result against the oracle (PP in C, PM in numpy, G from
    # the device gf_opt which is pinned to the reference at 16^3 and 32^3)
    from p3m_b200 import gf_opt_device

    P = O.Params(N, 2.0, 0.6, 6.0, 64, Gamma=100.0)
    Gk, _ = gf_opt_device(2.0, 0.6, 6, 3, 64, L)
    mid = 32
    kv = 2 * np.pi * (np.arange(64) - mid) / L
    P._gk = (Gk, kv.reshape(1, 64), kv.reshape(64, 1), kv.reshape(64, 1, 1), 0.0)
    Uo, ao, _ = O.force_pot(P, pos)
    assert U64 == pytest.approx(Uo, rel=1e-10)
    assert rel_rms(a64, ao) < 1e-9
    assert rel_rms(a32, ao) <= 1e-5
    # U = U_pp + U_pm + U_self cancels ~18x here: judge it against |U_pp|
    assert abs(U32 - Uo) < 1e-6 * abs(parts64[0])


def test_edge_particle_at_box_edge():
    """x = L exactly is the periodic image of x = 0 for the mesh (as the
    reference's single wrap makes it) and for the PP cells."""
    from p3m_b200 import FP64, Context, Replica

    N = 2000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=1.0, alpha=0.7, rc=L / 3.0, M=32)
    pos, _ = _init_state(r, 3)
    pos_edge = pos.copy()
    pos_edge[7] = [L, 0.5 * L, L]
    pos_zero = pos_edge.copy()
    pos_zero[7] = [0.0, 0.5 * L, 0.0]
    with Context(r, precision=FP64) as c:
        U1, a1, _ = c.force(pos_edge)
        U2, a2, _ = c.force(pos_zero)
        rho_e = c.assign(pos_edge)
    assert U1 == pytest.approx(U2, rel=1e-12)
    assert rel_rms(a1, a2) < 1e-12
    h = L / 32
    rho_o = O.assign6(pos_edge, np.ones(N), 32, 32, 32, h, h, h)
    assert np.max(np.abs(rho_e - rho_o)) < 1e-11


def test_out_of_box_raises():
    from p3m_b200 import FP64, Context, P3MError, Replica

    N = 2000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=1.0, alpha=0.7, rc=L / 3.0, M=32)
    pos, _ = _init_state(r, 3)
    pos[5, 1] = 2.5 * L
    with Context(r, precision=FP64) as c:
        with pytest.raises(P3MError) as e:
            c.force(pos)
        assert e.value.code == -4
        pos[5, 1] = 0.5 * L
        c.force(pos)  # the context stays usable


def test_bad_descriptors_rejected():
    from p3m_b200 import FP32, Context, P3MError, Replica

    L = 10.0
    with pytest.raises(P3MError):
        Context(Replica(N=100, L=L, kappa=1, alpha=1, rc=4.0, M=32), precision=FP32)  # 2 cells
    with pytest.raises(P3MError):
        Context(Replica(N=100, L=L, kappa=1, alpha=1, rc=3.0, M=48), precision=FP32)  # not 2^k
    with pytest.raises(P3MError):
        Context(Replica(N=0, L=L, kappa=1, alpha=1, rc=3.0, M=32), precision=FP32)


def test_nqt_ring_matches_oracle():
    from p3m_b200 import FP64, MODE_NVE, Context, Replica

    N = 2000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=1.0, alpha=0.7, rc=L / 3.0, M=32)
    pos, vel = _init_state(r, 9)
    qmult = np.arange(1, 9, dtype=np.float64)
    with Context(r, precision=FP64) as c:
        c.set_state(0, pos, vel)
        c.init_forces()
        c.set_nqt(qmult, 16)
        c.run(4, MODE_NVE, record_nqt=True)
        nqt = c.get_nqt(0, len(qmult))
        p, _, _ = c.get_state(0)
    assert nqt.shape == (4, 8, 3)
    ref = O.nqt(p, qmult * 2 * np.pi / L)
    np.testing.assert_allclose(nqt[-1], ref, rtol=0, atol=1e-9)


def test_launch_count_grows():
    from p3m_b200 import FP32, MODE_NVE, Context, Replica

    N = 2000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=1.0, alpha=0.7, rc=L / 3.0, M=32)
    pos, vel = _init_state(r, 2)
    with Context(r, precision=FP32) as c:
        c.set_state(0, pos, vel)
        c.init_forces()
        n0 = c.launch_count()
        c.run(3, MODE_NVE)
        assert c.launch_count() - n0 >= 3 * 15


@pytest.mark.parametrize("M", [32, 64, 128])
def test_pm_fp64_against_oracle_mesh_paths(M):
    """PM force and energy at M = 32 and 64 (fused plane FFT) and M = 128
    (multi-pass FFT) against the oracle's numpy chain on the same influence
    function."""
    from p3m_b200 import FP64, Context, Replica, gf_opt_device

    N = 4000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=1.0, alpha=0.8, rc=L / 3.2, M=M)
    pos, _ = _init_state(r, 21)
    G, _ = gf_opt_device(r.kappa, r.alpha, 6, 3, M, L)
    with Context(r, precision=FP64) as c:
        c.set_green(G)
        U, acc, Ep, _ = c.pm(pos)
    kv = 2 * np.pi * (np.arange(M) - M // 2) / L
    h = L / M
    Uo, ao, Epo = O.pm(pos, np.ones(N), G, kv.reshape(1, M), kv.reshape(M, 1), kv.reshape(M, 1, 1),
                       M, M, M, h, h, h, L, L, L)
    assert U == pytest.approx(Uo, rel=1e-10)
    assert rel_rms(acc, ao) < 1e-10


def test_state_all_round_trip_and_kept_lists():
    """p3m_set_state_all / p3m_get_state_all move the whole ensemble; reading
    the state back and setting it again with the lists kept continues the
    trajectory bit for bit."""
    from p3m_b200 import FP32, MODE_NVE, Context, Replica

    reps = []
    for N, M in ((1500, 32), (2500, 64)):
        L = (4 * np.pi * N / 3) ** (1 / 3)
        reps.append(Replica(N=N, L=L, kappa=1.0, alpha=0.7, rc=4.0, M=M))
    states = [_init_state(r, 21 + i) for i, r in enumerate(reps)]
    pos0 = np.concatenate([s[0] for s in states])
    vel0 = np.concatenate([s[1] for s in states])

    def start(c):
        c.set_state_all(pos0, vel0)
        c.init_forces()

    with Context(reps, precision=FP32) as a, Context(reps, precision=FP32) as b:
        start(a)
        start(b)
        # per-replica reads agree with the batched read
        p, v, ac = a.get_state_all()
        off = 0
        for i, r in enumerate(reps):
            pi, vi, ai = a.get_state(i)
            assert np.array_equal(pi, p[off:off + r.N]) and np.array_equal(ai, ac[off:off + r.N])
            off += r.N
        a.run(10, MODE_NVE)
        b.run(5, MODE_NVE)
        out = [np.empty((len(pos0), 3)) for _ in range(3)]
        b.get_state_all(*out)
        b.set_state_all(*out, keep_lists=True)
        b.run(5, MODE_NVE)
        for x, y in zip(a.get_state_all(), b.get_state_all()):
            assert np.array_equal(x, y)


def test_set_t_desired_and_quench():
    """The thermostat follows p3m_set_t_desired; the quench + thermostat
    equilibration leaves a hot, strongly screened replica of the uneven
    ensemble (the cfg4 draw of seed 163) with a thermal velocity tail and a
    conserved energy, where the reference's thermostat alone leaves runaway
    particles from the random start."""
    from p3m_b200 import FP32, MODE_NVE, MODE_THERMOSTAT, Context, Replica
    from p3m_b200.configs import box, cfg4_system

    N, Gamma, kappa = cfg4_system(163)
    r = Replica(N=N, L=box(N), kappa=kappa, alpha=0.54, rc=5.96, M=64, dt=0.1,
                T_desired=1.0 / Gamma, seed=163)
    pos, vel = _init_state(r, 163)
    with Context(r, precision=FP32) as c:
        c.set_state(0, pos, vel)
        c.init_forces()
        c.set_t_desired(2.0 * r.T_desired)
        c.run(20, MODE_THERMOSTAT)
        v = c.get_state(0)[1]
        assert abs(np.sum(v ** 2) / N / (2.0 * r.T_desired) - 1.0) < 1e-9  # rescaled to 2 T_d
        c.set_t_desired(r.T_desired)
        c.equilibrate(300)
        v = c.get_state(0)[1]
        vm = np.sqrt(np.sum(v ** 2, axis=1))
        assert vm.max() / np.sqrt(np.mean(vm ** 2)) < 6.0
        c.run(300, MODE_NVE)
        e = c.energies(max_steps=300)
        E = e[:, 0, 0] + e[:, 0, 1]
        assert np.max(np.abs(E - E[0])) / e[-1, 0, 1] < 1e-3


def test_async_state_copies_on_two_contexts():
    """Two contexts on their own streams, driven with queued copies and
    asynchronous runs, produce what the synchronous calls produce."""
    from p3m_b200 import FP32, MODE_NVE, Context, Replica

    def reps_of(seeds):
        L = (4 * np.pi * 1500 / 3) ** (1 / 3)
        return [Replica(N=1500, L=L, kappa=1.0, alpha=0.7, rc=4.0, M=32, seed=s) for s in seeds]

    halves = [reps_of([31, 32]), reps_of([33, 34])]
    states = []
    for h in halves:
        st = [_init_state(r, r.seed) for r in h]
        states.append((np.concatenate([x[0] for x in st]), np.concatenate([x[1] for x in st])))
    ref = []
    for h, (p, v) in zip(halves, states):
        with Context(h, precision=FP32) as c:
            c.set_state_all(p, v)
            c.init_forces()
            for _ in range(3):
                out = c.get_state_all()
                c.set_state_all(*out, keep_lists=True)
                c.run(1, MODE_NVE)
            ref.append(c.get_state_all())
    ctxs = [Context(h, precision=FP32) for h in halves]
    try:
        bufs = []
        for c, (p, v) in zip(ctxs, states):
            c.set_state_all(p, v)
            c.init_forces()
            bufs.append(list(c.get_state_all()))
        for _ in range(3):
            for c, b in zip(ctxs, bufs):
                c.set_state_all(*b, keep_lists=True, sync=False)
                c.run(1, MODE_NVE, sync=False)
                c.get_state_all(*b, sync=False)
            for c in ctxs:
                c.sync()
        for b, r in zip(bufs, ref):
            for x, y in zip(b, r):
                assert np.array_equal(x, y)
    finally:
        for c in ctxs:
            c.close()



def test_autotune_installs_a_finalist():
    """The autotuner times the PP candidates, then each other kernel shape
    from the best of them, re-times the fastest settings and installs the
    best finalist."""
    from p3m_b200 import FP32, Context, Replica
    from p3m_b200.autotune import shape_options, tune

    N = 3000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=1.0, alpha=0.8, rc=L / 4, M=32)  # skins up to L/3 - rc = 1.2
    pos, vel = _init_state(r, 9)
    with Context([r, r], precision=FP32) as c:
        c.set_state_all(np.concatenate([pos, pos]), np.concatenate([vel, vel]))
        c.init_forces()
        assert set(shape_options(c)) == {"cell_div", "plane_max", "gather_mode"}
        res = tune(c, steps=10, use_cache=False, candidates=[(1, 0.5), (2, 0.8), (4, 1.1)],
                   finalists=2)
        # 3 PP settings, then one new setting per other shape value, then
        # the inner-list buffers
        assert res["prune_trials"] >= 2
        assert len(res["ms_per_step"]) == 3 + 1 + 1 + 2 + res["prune_trials"]
        assert len(res["final_ms_per_step"]) == 2
        assert any(k.endswith("prune0.2") for k in res["ms_per_step"])
        best = min(res["final_ms_per_step"], key=res["final_ms_per_step"].get)
        assert best in res["ms_per_step"]
        assert c.tuning() == res["choice"]


@pytest.mark.parametrize("prec_name", ["fp32", "fp64"])
def test_kernel_shapes_agree(prec_name):
    """Every kernel shape computes the same forces and energies: cell divisor
    1 or 2, the fused plane FFT or the pencil passes for a 32^3 and a 64^3
    replica, every gather mode, FP32 inner lists -- to rounding (FP64: 1e-12; FP32:
    1e-6 of the RMS force) -- and the pencil FFT path matches the oracle."""
    from p3m_b200 import FP32, FP64, Context, Replica, gf_opt_device

    prec = {"fp32": FP32, "fp64": FP64}[prec_name]
    reps = []
    for N, M in ((2500, 32), (4000, 64)):
        L = (4 * np.pi * N / 3) ** (1 / 3)
        reps.append(Replica(N=N, L=L, kappa=1.0, alpha=0.8, rc=L / 3.4, M=M))
    states = [_init_state(r, 30 + i)[0] for i, r in enumerate(reps)]
    pos = np.concatenate(states)
    out = {}
    shapes = [{}, {"cell_div": 1}, {"plane_max": 0}, {"plane_max": 32}, {"gather_mode": 0},
              {"gather_mode": 2}]
    if prec_name == "fp32":
        shapes.append({"prune_buf": 0.2})  # inner lists, built by this force evaluation
    for shape in shapes:
        with Context(reps, precision=prec) as c:
            c.set_tuning(**shape)
            assert all(c.tuning()[k] == v for k, v in shape.items()) or prec_name == "fp64"
            c.set_state_all(pos, np.zeros_like(pos))
            c.init_forces()
            acc = c.get_state_all()[2]
            st = [c.replica_stats(i) for i in range(2)]
        out[str(shape)] = (acc, st)
    acc0, st0 = out["{}"]
    tol = 1e-12 if prec_name == "fp64" else 1e-6
    for k, (acc, st) in out.items():
        assert rel_rms(acc, acc0) < tol, k
        for a, b in zip(st, st0):  # U = U_short + U_fft + U_self cancels: judge on U_short
            assert abs(a["U"] - b["U"]) <= tol * abs(b["U_short"]), k
    if prec_name == "fp64":
        # the pencil passes on the 64^3 replica against the oracle's chain
        r, p = reps[1], states[1]
        G, _ = gf_opt_device(r.kappa, r.alpha, 6, 3, r.M, r.L)
        with Context(r, precision=FP64) as c:
            c.set_tuning(plane_max=0)
            c.set_green(G)
            U, acc, _, _ = c.pm(p)
        kv = 2 * np.pi * (np.arange(r.M) - r.M // 2) / r.L
        h = r.L / r.M
        Uo, ao, _ = O.pm(p, np.ones(r.N), G, kv.reshape(1, r.M), kv.reshape(r.M, 1),
                         kv.reshape(r.M, 1, 1), r.M, r.M, r.M, h, h, h, r.L, r.L, r.L)
        assert U == pytest.approx(Uo, rel=1e-10)
        assert rel_rms(acc, ao) < 1e-10


@pytest.mark.parametrize("tpi", [1, 2, 4, 8])
def test_inner_lists_follow_the_trajectory(tpi):
    """With inner lists (prune_buf > 0) the steps read lists of the Verlet
    entries closer than rc + prune_buf, rebuilt whenever a particle moved
    prune_buf/2: over a trajectory with several such builds between Verlet
    rebuilds, the last step's forces equal a fresh evaluation at the same
    positions (every list layout: 1, 2, 4, 8 threads per particle), and
    graph and eager runs stay bit-identical."""
    from p3m_b200 import FP32, MODE_NVE, Context, Replica

    reps = []
    for N, kappa, M in [(3000, 2.0, 32), (5000, 1.0, 64)]:
        L = (4 * np.pi * N / 3) ** (1 / 3)
        reps.append(Replica(N=N, L=L, kappa=kappa, alpha=0.7, rc=min(5.0, L / 3.6), M=M, dt=0.1,
                            T_desired=0.02))
    states = [_init_state(r, 41 + i) for i, r in enumerate(reps)]
    with Context(reps, precision=FP32) as c:
        for i, (p, v) in enumerate(states):
            c.set_state(i, p, v)
        c.init_forces()
        c.equilibrate(100, quench_steps=100)
        eq = c.get_state_all()
    outs = []
    for graph in ((True, False) if tpi == 2 else (True,)):
        with Context(reps, precision=FP32) as c:
            skin = min(0.9, min(r.L / 3 - r.rc for r in reps) * 0.99)
            c.set_tuning(pp_tpi=tpi, skin=skin, prune_buf=0.15)
            assert c.tuning()["prune_buf"] == pytest.approx(0.15)
            c.set_state_all(eq[0], eq[1])
            c.init_forces()
            rb0 = [c.replica_stats(i)["rebuilds"] for i in range(2)]
            c.run(150, MODE_NVE, graph=graph)
            builds = [c.inner_builds(i) for i in range(2)]
            rebuilds = [c.replica_stats(i)["rebuilds"] - rb0[i] for i in range(2)]
            st = c.get_state_all()
            U = [c.replica_stats(i)["U_short"] for i in range(2)]
        outs.append(st)
        assert all(b >= 2 for b in builds), (builds, rebuilds)
        assert all(b > rb for b, rb in zip(builds, rebuilds)), (builds, rebuilds)
        with Context(reps, precision=FP32) as c:  # the Verlet lists themselves
            c.set_tuning(pp_tpi=tpi, skin=skin)
            c.set_state_all(st[0], st[1])
            c.init_forces()
            acc = c.get_state_all()[2]
            U0 = [c.replica_stats(i)["U_short"] for i in range(2)]
        assert rel_rms(st[2], acc) < 1e-6
        for a, b in zip(U, U0):
            assert a == pytest.approx(b, rel=1e-6)
    if len(outs) == 2:
        for a, b in zip(outs[0], outs[1]):
            assert np.array_equal(a, b)


def test_inner_list_settings_are_checked():
    """prune_buf: FP32 only, non-negative, below every replica's skin; a
    rejected setting leaves the context's shapes as they were."""
    from p3m_b200 import FP32, FP64, Context, P3MError, Replica

    N = 2000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=1.0, alpha=0.8, rc=L / 4, M=32)
    with Context(r, precision=FP64) as c:
        with pytest.raises(P3MError):
            c.set_tuning(prune_buf=0.2)
    with Context(r, precision=FP32) as c:
        c.set_tuning(skin=0.5)
        before = c.tuning()
        for bad in (-0.1, 0.5, 0.7, float("nan")):
            with pytest.raises(P3MError):
                c.set_tuning(prune_buf=bad)
            assert c.tuning() == before
        c.set_tuning(prune_buf=0.3)
        c.set_tuning(prune_buf=0.0)
        assert c.tuning()["prune_buf"] == 0.0


def test_get_step_async_matches_sync_reads():
    """p3m_get_step_async + p3m_sync deliver the state and the last step's
    (U, K, T, factor) that the synchronous reads give, and a device status
    raised by the step (a particle still outside [-L, 2L) after the step's
    periodic wrap) still surfaces at p3m_sync."""
    import torch

    from p3m_b200 import FP32, MODE_NVE, Context, P3MError, Replica

    N = 3000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    reps = [Replica(N=N, L=L, kappa=1.0, alpha=0.8, rc=L / 3.2, M=32, seed=s) for s in (4, 5)]
    st = [_init_state(r, r.seed) for r in reps]
    pos = np.concatenate([p for p, _ in st])
    vel = np.concatenate([v for _, v in st])
    hb = [torch.empty((2 * N, 3), dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
    en = torch.empty((2, 4), dtype=torch.float64, pin_memory=True).numpy()
    with Context(reps, precision=FP32) as c:
        c.set_state_all(pos, vel)
        c.init_forces()
        c.run(3, MODE_NVE, sync=False)
        c.get_step_async(*hb, en)
        c.sync()
        p, v, a = c.get_state_all()
        E = c.energies(max_steps=1)[0]
        for x, y in zip(hb, (p, v, a)):
            assert np.array_equal(x, y)
        assert np.array_equal(en, E)
        bad = p.copy()
        bad[7, 0] = 3.5 * L  # one wrap (velocity_verlet_p3m_ord6.py:16-19) leaves 2.5 L
        c.set_state_all(bad, v, a, keep_lists=True, sync=False)
        c.run(1, MODE_NVE, sync=False)
        c.get_step_async(*hb, en)
        with pytest.raises(P3MError) as e:
            c.sync()
        assert e.value.code == -4


def test_set_priority_keeps_results():
    """Recreating a context's streams at another priority level changes no
    result: the steps after it equal those of a context left at the default."""
    from p3m_b200 import FP32, MODE_NVE, Context, Replica

    N = 3000
    L = (4 * np.pi * N / 3) ** (1 / 3)
    r = Replica(N=N, L=L, kappa=1.0, alpha=0.8, rc=L / 3.2, M=32)
    pos, vel = _init_state(r, 12)
    out = []
    for level in (None, 3):
        with Context(r, precision=FP32) as c:
            c.set_state(0, pos, vel)
            c.init_forces()
            c.run(2, MODE_NVE)
            if level is not None:
                c.set_priority(level)
            c.run(3, MODE_NVE)
            out.append(c.get_state(0) + (c.energies(max_steps=5),))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
