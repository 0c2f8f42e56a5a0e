"""The oracle's PP against the reference's own C PP routine (yukawa_p3m.c),
compiled unchanged into oracle/_ref by oracle/Makefile where the reference
tree is present. Skipped where that library was not built."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

REF_SO = os.path.join(os.path.dirname(O.__file__), "_ref", "libyukawa_p3m_ref.so")


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference C library not built here")
@pytest.mark.parametrize("kappa", [0.0, 1.3])
def test_oracle_pp_matches_reference_c(kappa):
    from conftest import load_golden

    g = load_golden("n2000_m32")
    pos = np.ascontiguousarray(g["pos0"])
    n = pos.shape[0]
    L, alpha, rc = float(g["L"]), float(g["alpha"]), float(g["rc"])
    lib = ctypes.CDLL(REF_SO)
    rows_p = (ctypes.POINTER(ctypes.c_double) * n)()
    acc = np.zeros((n, 3))
    rows_a = (ctypes.POINTER(ctypes.c_double) * n)()
    for i in range(n):
        rows_p[i] = pos[i].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        rows_a[i] = acc[i].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    Z = np.ones(n)
    lib.particle_particle.restype = None
    lib.particle_particle(rows_p, rows_a, Z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                          ctypes.c_int(n), ctypes.c_double(L), ctypes.c_double(kappa),
                          ctypes.c_double(alpha), ctypes.c_double(rc))
    _, acc_o = O.pp(kappa, alpha, rc, [L] * 3, pos)
    np.testing.assert_allclose(acc_o, acc, rtol=0, atol=1e-13)
