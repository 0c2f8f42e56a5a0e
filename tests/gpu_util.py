"""Helpers shared by the GPU parity tests."""
import numpy as np

from oracle import oracle as O


def rel_rms(a, ref):
    return float(np.sqrt(np.sum((a - ref) ** 2) / np.sum(ref ** 2)))


def rel_max(a, ref):
    """max_i |a_i - ref_i| / rms|ref| (the force-error definition used for
    the FP32 path)."""
    ref_rms = np.sqrt(np.mean(np.sum(ref ** 2, axis=1)))
    return float(np.max(np.sqrt(np.sum((a - ref) ** 2, axis=1))) / ref_rms)


def replica_from_golden(g, **kw):
    from p3m_b200 import Replica

    return Replica(N=int(g["N"]), L=float(g["L"]), kappa=float(g["kappa"]), alpha=float(g["alpha"]),
                   rc=float(g["rc"]), M=int(g["M"]), dt=float(g["dt"]),
                   T_desired=1.0 / float(g["Gamma"]), **kw)


def golden_kvecs(g):
    M, L = int(g["M"]), float(g["L"])
    mid = M // 2
    kx = 2 * np.pi * (np.arange(M).reshape((1, M)) - mid) / L
    ky = 2 * np.pi * (np.arange(M).reshape((M, 1)) - mid) / L
    kz = 2 * np.pi * (np.arange(M).reshape((M, 1, 1)) - mid) / L
    return kx, ky, kz


def oracle_params(g):
    return O.Params(int(g["N"]), float(g["kappa"]), float(g["alpha"]), float(g["rc"]), int(g["M"]),
                    Gamma=float(g["Gamma"]), dt=float(g["dt"]))
