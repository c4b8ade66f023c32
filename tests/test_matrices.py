"""The synthetic workload matrices have the values the benchmark configurations name."""
import numpy as np

from pastix_b200 import matrices as M


def test_laplacian_7pt_values():
    A = M.laplacian(4, 3, 5, 7, 6.0)
    D = A.to_dense()
    assert np.allclose(np.diag(D), 6.0)
    assert np.allclose(D, D.T)
    off = D - np.diag(np.diag(D))
    assert set(np.unique(off)) <= {0.0, -1.0}
    # interior point has 6 neighbours
    i = 1 + 4 * (1 + 3 * 2)
    assert (off[i] == -1).sum() == 6


def test_laplacian_27pt_values():
    A = M.laplacian(5, 5, 5, 27, 26.0, shift=1e-3)
    D = A.to_dense()
    assert np.allclose(np.diag(D), 26.001)
    i = 2 + 5 * (2 + 5 * 2)
    assert (D[i] == -1).sum() == 26
    assert np.linalg.eigvalsh(D).min() > 0


def test_convection_diffusion_pattern_symmetric_values_not():
    A = M.convection_diffusion(5, 4, 3, seed=1)
    D = A.to_dense()
    assert np.array_equal(D != 0, (D != 0).T)
    assert not np.allclose(D, D.T)
    assert np.all(np.diag(D) >= 6.0)


def test_shifted_2d_is_indefinite():
    side = 12
    lam = M.lambda_max_5pt(side)
    A = M.shifted_laplacian_2d(side, 0.3 * lam)
    ev = np.linalg.eigvalsh(A.to_dense())
    assert ev.min() < 0 < ev.max()


def test_matvec_and_rhs():
    A = M.laplacian(4, 4, 4, 27, 26.0)
    x, b = M.rhs_from_xtrue(A, 3, seed=0)
    assert np.allclose(A.to_dense() @ x, b)
    assert x.min() >= -1 and x.max() <= 1
    assert np.allclose(A.full().to_dense(), A.to_dense())
