"""Host-side logic that needs no GPU."""
import numpy as np
import pytest

from conftest import have_gpu


def test_initial_state_bitexact(golden):
    import initialize_pos_vel

    g = golden
    N, L = int(g["N"]), float(g["L"])
    pos, vel = np.zeros((N, 3)), np.zeros((N, 3))
    initialize_pos_vel.initial(int(g["seed"]), N, [L] * 3, pos, vel, 1.0 / float(g["Gamma"]))
    assert np.array_equal(pos, g["pos0"])
    assert np.array_equal(vel, g["vel0"])


def test_replica_desc_layout():
    import ctypes

    from p3m_b200._lib import ReplicaDesc

    assert ctypes.sizeof(ReplicaDesc) == 4 * 4 + 10 * 8


def test_non_cubic_rejected_before_device():
    import yukawa_pm_ord6

    with pytest.raises(ValueError):
        yukawa_pm_ord6.charge_assgn_6_numba(np.zeros((4, 4, 8)), np.zeros((3, 3)), np.ones(3), 3,
                                            8, 4, 4, 1.0, 1.0, 1.0)


@pytest.mark.skipif(have_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    import yukawa_pp
    from p3m_b200 import P3MError

    pos = np.random.default_rng(0).random((100, 3)) * 10.0
    with pytest.raises(P3MError):
        yukawa_pp.particle_particle(1.0, 0.8, 3.0, np.array([10.0] * 3), pos, np.zeros((100, 3)))


def test_reference_driver_calls_bind_to_package_modules():
    """Every call the reference's driver makes into the modules this package
    shadows (yukawa_MD_p3m_ord6.py:15-21 imports, :152-229 calls) binds to
    this package's function of the same name with the same arguments. Reads
    the Python-3 copy of the driver that the build writes into oracle/_ref/
    where the reference tree is present."""
    import ast
    import importlib
    import inspect
    import os

    from conftest import ROOT

    path = os.path.join(ROOT, "oracle", "_ref", "yukawa_MD_p3m_ord6_py3.py")
    if not os.path.isfile(path):
        pytest.skip("the copy of the reference's driver was not built here")
    tree = ast.parse(open(path).read())
    alias = {}
    for node in ast.walk(tree):
        if isinstance(node, ast.Import):
            for a in node.names:
                if a.name not in ("numpy", "time"):
                    alias[a.asname or a.name] = a.name
    assert set(alias.values()) == {"read", "initialize_pos_vel", "velocity_verlet_p3m_ord6",
                                   "thermostat_p3m_ord6", "yukawa_gf_opt", "yukawa_p3m_ord6"}
    seen = set()
    for node in ast.walk(tree):
        if (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute)
                and isinstance(node.func.value, ast.Name) and node.func.value.id in alias):
            mod = importlib.import_module(alias[node.func.value.id])
            fn = getattr(mod, node.func.attr)
            assert not node.keywords
            inspect.signature(fn).bind(*range(len(node.args)))
            seen.add((mod.__name__, node.func.attr))
    assert seen == {("yukawa_gf_opt", "gf_opt"), ("yukawa_p3m_ord6", "force_pot"),
                    ("thermostat_p3m_ord6", "vscale"), ("velocity_verlet_p3m_ord6", "update"),
                    ("read", "initL"), ("initialize_pos_vel", "initial")}


def test_tuning_struct_layout():
    """p3m_tuning of the C header: four int32 shapes, then the skin and the
    inner-list buffer as doubles."""
    import ctypes

    from p3m_b200._lib import Tuning

    assert ctypes.sizeof(Tuning) == 4 * 4 + 2 * 8
    assert [f for f, _ in Tuning._fields_] == ["pp_tpi", "cell_div", "plane_max", "gather_mode",
                                             "skin", "prune_buf"]


class _FakeCtx:
    def __init__(self, precision, Ms, rc=3.0):
        from p3m_b200 import Replica

        self.precision = precision
        self.replicas = [Replica(N=1000, L=10.0, kappa=1.0, alpha=0.7, rc=rc, M=M)
                         for M in Ms]


def test_autotune_search_space():
    """The autotuner's options: inner-list buffers only on FP32 and below the
    skin, larger skins only up to the cap, plane/pencil only for meshes up
    to 64^3, the two-buffer gather only on FP32, and keys that tell every
    setting apart."""
    from p3m_b200 import FP32, FP64
    from p3m_b200.autotune import PRUNE_BUFS, _key, prune_options, shape_options

    c32, c64 = _FakeCtx(FP32, [32, 128]), _FakeCtx(FP64, [128])
    assert prune_options(c64, 0.8, 1.5) == []
    opts = prune_options(c32, 0.8, 1.5)
    assert all(pb < sk <= 1.5 for sk, pb in opts)
    assert {pb for _, pb in opts} == set(PRUNE_BUFS)
    assert {sk for sk, _ in opts} == {0.8, 1.1, 1.4}
    assert {sk for sk, _ in prune_options(c32, 0.5, 1.2)} == {0.5, 1.1}
    assert shape_options(c32) == {"cell_div": (2, 1), "plane_max": (64, 0), "gather_mode": (1, 0, 2)}
    assert shape_options(c64) == {"cell_div": (2, 1), "gather_mode": (1, 0)}
    base = {"pp_tpi": 2, "cell_div": 2, "plane_max": 64, "gather_mode": 1, "skin": 0.8,
            "prune_buf": 0.0}
    keys = {_key(dict(base, **kw)) for kw in ({}, {"prune_buf": 0.3}, {"cell_div": 1},
                                              {"skin": 1.1}, {"gather_mode": 2})}
    assert len(keys) == 5


def test_autotune_pp_grid_fits_the_cutoffs():
    """The PP grid keeps the skins every replica allows (at most rc/2); with
    cutoffs too short for all of them, each thread count is tried at the
    largest skin allowed instead of nothing."""
    from p3m_b200 import FP32
    from p3m_b200.autotune import CANDIDATES, max_skin, pp_candidates

    wide = _FakeCtx(FP32, [64], rc=3.0)
    assert max_skin(wide) == 1.5 and pp_candidates(wide) == CANDIDATES
    mid = _FakeCtx(FP32, [64], rc=2.0)
    assert {sk for _, sk in pp_candidates(mid)} == {0.5, 0.8}
    short = _FakeCtx(FP32, [64], rc=0.8)
    assert pp_candidates(short) == [(1, 0.4), (2, 0.4), (4, 0.4)]
    assert pp_candidates(short, [(2, 0.8)]) == [(2, 0.4)]
