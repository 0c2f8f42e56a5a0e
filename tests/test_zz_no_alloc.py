"""p3m_gf_opt_static -- the influence function for callers that cannot
allocate device memory (for example code that owns a fixed device-memory
budget and hands out every byte through its own pool). The caller
passes device output buffers and a stream; the library keeps its scratch in
a fixed device array instead of calling cudaMalloc.

This file is named so that pytest collects it last. It compares the
allocation-free entry point with p3m_gf_opt, through the C ABI, on calls in a
row with different parameters, within the tolerance the other gf_opt tests
use. The largest mesh goes first: its 8192 block partials stay in the shared
array, and the smaller meshes after it read only the first of those slots,
which they wrote themselves (the A_pm comparison would catch a sum that
picked up stale partials).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [  # kappa, alpha, M, L -- largest mesh first
    (1.0, 0.5, 128, 74.8),
    (2.0, 0.6, 32, 20.31),
    (1.0, 0.5, 64, 34.73),
]


def _static_call(lib, torch, kappa, alpha, M, L):
    G = torch.empty(M ** 3, dtype=torch.float64, device="cuda")
    A = torch.empty(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.p3m_gf_opt_static(kappa, alpha, 6, 3, M, L, ctypes.c_void_p(G.data_ptr()),
                               ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, lib.p3m_gf_opt_static_error().decode()
    torch.cuda.synchronize()
    return G.cpu().numpy().reshape(M, M, M), float(A.cpu().numpy()[0])


def test_static_matches_allocating_entry_point_twice():
    import torch

    from p3m_b200 import gf_opt_device, lib

    L = lib()
    torch.cuda.init()
    for kappa, alpha, M, box in CASES:
        G_s, A_s = _static_call(L, torch, kappa, alpha, M, box)
        G_a, A_a = gf_opt_device(kappa, alpha, 6, 3, M, box)
        assert np.max(np.abs(G_s - G_a)) <= 1e-12 * np.max(np.abs(G_a))
        assert A_s == pytest.approx(A_a, rel=1e-12)


def test_static_rejects_oversized_mesh():
    import torch

    from p3m_b200 import lib

    L = lib()
    G = torch.empty(1, dtype=torch.float64, device="cuda")
    rc = L.p3m_gf_opt_static(1.0, 0.5, 6, 3, 256, 50.0, ctypes.c_void_p(G.data_ptr()),
                             ctypes.c_void_p(G.data_ptr()), None)
    assert rc == -1
    assert "128" in L.p3m_gf_opt_static_error().decode()
