"""ctypes binding of libp3m_b200.so (the C ABI declared in include/p3m_b200.h).

The library is the product path: every force, mesh and integrator stage runs
in its sm_100a kernels. There is no CPU fallback -- if the library is missing
or no B200 is visible, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libp3m_b200.so")

P3M_OK = 0
P3M_EARG = -1
P3M_ECUDA = -2
P3M_ENODEV = -3
P3M_EBOX = -4
P3M_ENONFINITE = -5
P3M_ESTATE = -6
P3M_ENBOVF = -7

FP64 = 0
FP32 = 1
MODE_NVE = 0
MODE_THERMOSTAT = 1


class P3MError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code, msg):
        super().__init__(f"p3m_b200 error {code}: {msg}")
        self.code = code


class Tuning(ctypes.Structure):
    """p3m_tuning of include/p3m_b200.h: the kernel shapes of a context."""

    _fields_ = [
        ("pp_tpi", ctypes.c_int32),
        ("cell_div", ctypes.c_int32),
        ("plane_max", ctypes.c_int32),
        ("gather_mode", ctypes.c_int32),
        ("skin", ctypes.c_double),
        ("prune_buf", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ReplicaDesc(ctypes.Structure):
    """p3m_replica_desc of include/p3m_b200.h."""

    _fields_ = [
        ("n", ctypes.c_int32),
        ("mesh", ctypes.c_int32),
        ("order", ctypes.c_int32),
        ("m_alias", ctypes.c_int32),
        ("box", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("alpha", ctypes.c_double),
        ("rc", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("t_desired", ctypes.c_double),
        ("af", ctypes.c_double),
        ("uf", ctypes.c_double),
        ("kf", ctypes.c_double),
        ("skin", ctypes.c_double),
    ]


_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.c_int
_V = ctypes.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "p3m_create": (_I, [ctypes.POINTER(ReplicaDesc), _I, _I, _I, ctypes.POINTER(_V)]),
    "p3m_destroy": (_I, [_V]),
    "p3m_last_error": (ctypes.c_char_p, [_V]),
    "p3m_version": (_I, []),
    "p3m_launch_count": (ctypes.c_int64, [_V]),
    "p3m_pp": (_I, [_V, _I, _D, _D, _D]),
    "p3m_assign": (_I, [_V, _I, _D, _D, _D]),
    "p3m_gather": (_I, [_V, _I, _D, _D, _D, _D, _D, _D, _D]),
    "p3m_gf_opt": (_I, [_I, ctypes.c_double, ctypes.c_double, _I, _I, _I, ctypes.c_double, _D, _D]),
    "p3m_set_green": (_I, [_V, _I, _D]),
    "p3m_pm": (_I, [_V, _I, _D, _D, _D, _D, _D, _D]),
    "p3m_force": (_I, [_V, _I, _D, _D, _D, _D, _D]),
    "p3m_update": (_I, [_V, _I, _D, _D, _D, _D]),
    "p3m_vscale": (_I, [_V, _I, _I, _D, _D, _D, _D, _D]),
    "p3m_nqt": (_I, [_V, _I, _D, _D, _I, _D]),
    "p3m_set_state": (_I, [_V, _I, _D, _D, _D]),
    "p3m_get_state": (_I, [_V, _I, _D, _D, _D]),
    "p3m_set_state_all": (_I, [_V, _D, _D, _D, _I]),
    "p3m_get_state_all": (_I, [_V, _D, _D, _D]),
    "p3m_set_state_all_async": (_I, [_V, _D, _D, _D, _I]),
    "p3m_get_state_all_async": (_I, [_V, _D, _D, _D]),
    "p3m_get_step_async": (_I, [_V, _D, _D, _D, _D]),
    "p3m_set_t_desired": (_I, [_V, _D]),
    "p3m_init_forces": (_I, [_V]),
    "p3m_set_nqt": (_I, [_V, _D, _I, _I]),
    "p3m_run": (_I, [_V, _I, _I, _I, _I, _I, _I]),
    "p3m_get_energies": (_I, [_V, _D, _I, ctypes.POINTER(_I)]),
    "p3m_get_nqt": (_I, [_V, _I, _D, _I, ctypes.POINTER(_I)]),
    "p3m_set_snapshots": (_I, [_V, _I, _I]),
    "p3m_get_snapshots": (_I, [_V, _D, ctypes.POINTER(ctypes.c_int), _I, ctypes.POINTER(ctypes.c_int)]),
    "p3m_check": (_I, [_V]),
    "p3m_sqw": (_I, [_V, ctypes.c_double, _I, _I, _I, _I, _D, _D]),
    "p3m_sqw_series": (_I, [_I, _D, _I, ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]),
    "p3m_pp_error": (_I, [ctypes.c_double] * 5 + [_D]),
    "p3m_pp_cutoff": (_I, [ctypes.c_double] * 6 + [_D]),
    "p3m_pm_error": (_I, [_I, _I, _D, _D, _D, _D, ctypes.POINTER(ctypes.c_int), _I, _I, _D, _D]),
    "p3m_sqw_runs": (_I, [_I, _D, _I, _I, _I, _I, _I, _I, ctypes.c_double, ctypes.c_double,
                          ctypes.c_double, _D]),
    "p3m_get_replica_stats": (_I, [_V, _I, _D]),
    "p3m_sync": (_I, [_V]),
    "p3m_set_priority": (_I, [_V, _I]),
    "p3m_stream": (_V, [_V]),
    "p3m_set_pp_config": (_I, [_V, _I, ctypes.c_double]),
    "p3m_get_pp_config": (_I, [_V, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(_I)]),
    "p3m_set_tuning": (_I, [_V, ctypes.POINTER(Tuning)]),
    "p3m_get_tuning": (_I, [_V, ctypes.POINTER(Tuning)]),
    "p3m_get_inner_builds": (_I, [_V, _I, _D]),
    "p3m_profile_stages": (_I, [_V, _I, _D, _I, ctypes.POINTER(_I)]),
    "p3m_stage_name": (ctypes.c_char_p, [_I]),
    "p3m_fp32_peak": (_I, [_I, _D]),
    "p3m_gf_opt_static": (_I, [ctypes.c_double, ctypes.c_double, _I, _I, _I, ctypes.c_double, _V,
                               _V, _V]),
    "p3m_gf_opt_static_error": (ctypes.c_char_p, []),
}


def lib():
    """Load libp3m_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise P3MError(P3M_ENODEV, f"{LIB_PATH} is missing: build it with "
                           "`make -C md-force-routines_b200/csrc` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def dptr(a):
    """Pointer to a C-contiguous float64 array (or NULL for None)."""
    if a is None:
        return None
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
        raise TypeError("expected a C-contiguous float64 numpy array")
    return a.ctypes.data_as(_D)


def check(rc, ctx=None):
    if rc != P3M_OK:
        msg = lib().p3m_last_error(ctx)
        raise P3MError(rc, msg.decode() if msg else "")
    return rc
