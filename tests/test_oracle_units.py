"""The oracle's building blocks against independent numpy/scipy references
(the LAPACK/deal.II stand-ins restated in oracle/cp_oracle.cpp)."""
import numpy as np
import pytest
import scipy.linalg as sla

from plasticity_b200 import materials as M


def test_odfpoint_is_rotation(oracle_lib):
    rng = np.random.default_rng(0)
    for r in M.random_rodrigues(rng, 50):
        R = oracle_lib.odfpoint(r)
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-13)
        assert np.isclose(np.linalg.det(R), 1.0, atol=1e-13)
        # rotation angle theta with tan(theta/2) = |r|, axis r
        th = 2 * np.arctan(np.linalg.norm(r))
        assert np.isclose(np.trace(R), 1 + 2 * np.cos(th), atol=1e-12)
        assert np.allclose(R @ r, r, atol=1e-12)


def test_elasticmoduli_rotates_stiffness(oracle_lib):
    """N(R) C N(R)^T equals the tensor rotation of C (Voigt, tensor shear
    on the strain side as the reference's Dmat2 uses)."""
    rng = np.random.default_rng(1)
    C6 = M.cubic_stiffness(170e3, 124e3, 75e3)
    voigt = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
    C4 = np.zeros((3, 3, 3, 3))
    for I, (i, j) in enumerate(voigt):
        for J, (k, l) in enumerate(voigt):
            for a, b in ((i, j), (j, i)):
                for c, d in ((k, l), (l, k)):
                    C4[a, b, c, d] = C6[I, J]
    for r in M.random_rodrigues(rng, 10):
        R = oracle_lib.odfpoint(r)
        Cr = oracle_lib.elasticmoduli(R, C6)
        C4r = np.einsum("ai,bj,ck,dl,ijkl->abcd", R, R, R, R, C4)
        ref = np.array([[C4r[i, j, k, l] for (k, l) in voigt] for (i, j) in voigt])
        assert np.allclose(Cr, ref, rtol=0, atol=1e-9 * np.abs(C6).max())
        assert np.allclose(Cr, Cr.T, atol=1e-9)


def test_matrix_exponential_series(oracle_lib):
    rng = np.random.default_rng(2)
    for scale in (1e-4, 1e-2, 0.3, 1.5):
        A = rng.standard_normal((3, 3)) * scale
        E, terms = oracle_lib.matrix_exponential(A)
        assert np.allclose(E, sla.expm(A), rtol=0, atol=5e-10 * max(1, np.abs(sla.expm(A)).max()))
        assert terms >= 1


def test_pinv_and_invert(oracle_lib):
    rng = np.random.default_rng(3)
    for n in (1, 2, 3, 4, 7, 12, 32):
        A = rng.standard_normal((n, n)) + n * np.eye(n)
        Ai, sing = oracle_lib.pinv_svd(A)
        assert sing == 0
        assert np.allclose(Ai, np.linalg.inv(A), atol=1e-12 * np.abs(np.linalg.inv(A)).max())
        Bi, sing2 = oracle_lib.invert(A)
        assert sing2 == 0
        assert np.allclose(Bi, np.linalg.inv(A), atol=1e-12 * np.abs(np.linalg.inv(A)).max())
    # compute_inverse_svd(0.0) zeroes only singular values that are exactly 0
    A = np.diag([3.0, 2.0, 0.0])
    Ai, sing = oracle_lib.pinv_svd(A)
    assert sing == 1
    assert np.array_equal(Ai, np.diag([1 / 3.0, 0.5, 0.0]))


def test_eig_sym3(oracle_lib):
    rng = np.random.default_rng(4)
    for _ in range(20):
        F = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
        C = F.T @ F
        ev, V = oracle_lib.eig_sym3(C)
        assert np.allclose(V @ np.diag(ev) @ V.T, C, atol=1e-13)
        assert np.allclose(np.sort(ev), np.linalg.eigvalsh(C), atol=1e-13)
