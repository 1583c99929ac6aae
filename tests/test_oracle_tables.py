"""Known-answer checks of the oracle's 1D tables (quadrature, shape values, derivatives,
transfer matrices).  These pin the tables every other oracle result is built on."""
import numpy as np
import pytest


def test_gauss_known_values(oracle):
    x, w = oracle.gauss(2)
    np.testing.assert_allclose(x, [0.5 - 0.5 / np.sqrt(3), 0.5 + 0.5 / np.sqrt(3)], rtol=0, atol=1e-16)
    np.testing.assert_allclose(w, [0.5, 0.5], atol=1e-16)
    x, w = oracle.gauss(3)
    np.testing.assert_allclose(x, [0.5 - 0.5 * np.sqrt(0.6), 0.5, 0.5 + 0.5 * np.sqrt(0.6)], atol=1e-16)
    np.testing.assert_allclose(w, [5 / 18, 8 / 18, 5 / 18], atol=1e-16)


def test_gauss_lobatto_known_values(oracle):
    x, w = oracle.gauss_lobatto(3)
    np.testing.assert_allclose(x, [0, 0.5, 1], atol=1e-16)
    np.testing.assert_allclose(w, [1 / 6, 4 / 6, 1 / 6], atol=1e-16)
    x, w = oracle.gauss_lobatto(5)
    t = np.sqrt(3 / 7)
    np.testing.assert_allclose(x, [0, 0.5 - 0.5 * t, 0.5, 0.5 + 0.5 * t, 1], atol=1e-16)
    np.testing.assert_allclose(w, np.array([9, 49, 64, 49, 9]) / 180, atol=1e-15)


@pytest.mark.parametrize("n", range(1, 9))
def test_gauss_exactness(oracle, n):
    x, w = oracle.gauss(n)
    for k in range(2 * n):
        assert abs(np.dot(w, x ** k) - 1.0 / (k + 1)) < 1e-15


@pytest.mark.parametrize("p", range(1, 7))
def test_shape_tables_reproduce_polynomials(oracle, p):
    S, SD, D, W = oracle.shape_tables(p)
    xl, _ = oracle.gauss_lobatto(p + 1)
    xg, _ = oracle.gauss(p + 1)
    for k in range(p + 1):
        # interpolation of x^k at the Gauss points, and its derivative
        np.testing.assert_allclose(S.T @ xl ** k, xg ** k, atol=1e-14)
        np.testing.assert_allclose(SD.T @ xl ** k, k * xg ** max(k - 1, 0) * (k > 0), atol=2e-13)
        # collocation derivative on the Gauss points
        np.testing.assert_allclose(D.T @ xg ** k, k * xg ** max(k - 1, 0) * (k > 0), atol=2e-13)
    # S^T * D == SD (derivative of the interpolant at the Gauss points)
    np.testing.assert_allclose(S @ D, SD, atol=2e-13)


@pytest.mark.parametrize("pc,pf", [(1, 2), (2, 3), (3, 4), (2, 4), (3, 6), (1, 6)])
def test_projection_matrix_is_interpolation(oracle, pc, pf):
    P = oracle.projection_matrix(pc, pf)
    xc, _ = oracle.gauss_lobatto(pc + 1)
    xf, _ = oracle.gauss_lobatto(pf + 1)
    np.testing.assert_allclose(P.sum(0), 1.0, atol=1e-14)  # partition of unity
    for k in range(pc + 1):
        np.testing.assert_allclose(P.T @ xc ** k, xf ** k, atol=1e-14)


@pytest.mark.parametrize("p", range(1, 7))
def test_h_prolongation_matrix(oracle, p):
    P = oracle.h_prolongation_matrix(p)
    x, _ = oracle.gauss_lobatto(p + 1)
    y = np.concatenate([0.5 * x, 0.5 + 0.5 * x[1:]])
    for k in range(p + 1):
        np.testing.assert_allclose(P.T @ x ** k, y ** k, atol=1e-14)
