"""The oracle's point-wise influence function (gf_opt_points, which the
256^3 parity tests use to check the device's G_k at chosen k points, where
the oracle's full alias sum takes minutes) against the oracle's whole-mesh
gf_opt, which tests/test_oracle_golden.py pins to the reference's output:
every point of a 32^3 mesh, both for the reference's hand-set parameters
and for a strongly screened system."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("kappa,alpha,L", [(0.1, 0.46, 20.31), (2.0, 0.6, 34.73)])
def test_gf_opt_points_equal_the_whole_mesh(kappa, alpha, L):
    M = 32
    h = L / M
    G_k = O.gf_opt(kappa, alpha, 6, 3, 3, 3, M, M, M, h, h, h, L, L, L)[0]
    iz, iy, ix = np.meshgrid(np.arange(M), np.arange(M), np.arange(M), indexing="ij")
    idx = np.stack([iz.ravel(), iy.ravel(), ix.ravel()], axis=1)
    pts = O.gf_opt_points(kappa, alpha, 6, 3, M, L, idx).reshape(M, M, M)
    assert np.array_equal(pts, G_k)
    assert np.count_nonzero(G_k) > 0.99 * M ** 3
