"""Gauss-type quadrature rules and Legendre bases on [-1, 1] (host, FP64).

Host-side setup used by the velocity meshes (radial Gauss-Jacobi rule,
dgfs1D/quadratures.py:205-208 ``zwgj``) and by the DG bases (Gauss-Lobatto
points and nodal Lagrange operators, dgfs1D/quadratures.py:39-65, 209-220).
Nodes are eigenvalues of the symmetric Jacobi matrix of the monic Jacobi
polynomials (Golub & Welsch, Math. Comp. 23, 1969); Lobatto rules modify the
last recurrence coefficient so that +-1 are nodes (Golub, SIAM Rev. 15, 1973).
"""
import math

import numpy as np
from scipy.linalg import eigh_tridiagonal


def _jacobi_coeffs(n, a, b):
    """Diagonal alpha_k and squared off-diagonal beta_k (k < n), mu0."""
    k = np.arange(n, dtype=np.float64)
    s = 2 * k + a + b
    alpha = np.empty(n)
    with np.errstate(invalid='ignore', divide='ignore'):
        alpha[:] = (b * b - a * a) / (s * (s + 2))
    if n > 0 and abs(a + b) < 1e-300:
        alpha[0] = (b - a) / (a + b + 2)
    elif n > 0:
        alpha[0] = (b - a) / (a + b + 2)
    beta = np.zeros(n)
    kk = k[1:]
    s1 = 2 * kk + a + b
    beta[1:] = (4 * kk * (kk + a) * (kk + b) * (kk + a + b)
                / (s1 * s1 * (s1 + 1) * (s1 - 1)))
    mu0 = 2.0 ** (a + b + 1) * math.gamma(a + 1) * math.gamma(b + 1) \
        / math.gamma(a + b + 2)
    return alpha, beta, mu0


def _from_jacobi_matrix(alpha, beta, mu0):
    z, V = eigh_tridiagonal(alpha, np.sqrt(beta[1:]))
    return z, mu0 * V[0, :] ** 2


def gauss_jacobi(n, a=0.0, b=0.0):
    """n-point Gauss-Jacobi nodes and weights for (1-x)^a (1+x)^b."""
    alpha, beta, mu0 = _jacobi_coeffs(n, a, b)
    return _from_jacobi_matrix(alpha, beta, mu0)


def gauss_lobatto_jacobi(n, a=0.0, b=0.0):
    """n-point Gauss-Lobatto-Jacobi rule (both end points are nodes)."""
    if n < 2:
        raise ValueError('Lobatto rules need at least two points')
    alpha, beta, mu0 = _jacobi_coeffs(n, a, b)
    N = n - 2
    apb1 = a + b + 1.
    alpha[n - 1] = (a - b) / (2. * N + apb1 + 1.)
    beta[n - 1] = (4. * (N + a + 1.) * (N + b + 1.) * (N + apb1)
                   / ((2. * N + apb1) * (2 * N + apb1 + 1) ** 2))
    return _from_jacobi_matrix(alpha, beta, mu0)


def legendre_orthonormal(order, x):
    """Orthonormal Legendre polynomials sqrt(k+1/2) P_k(x), shape (order, len(x))."""
    x = np.asarray(x, dtype=np.float64)
    P = np.zeros((order, x.size))
    if order > 0:
        P[0] = 1.0
    if order > 1:
        P[1] = x
    for k in range(2, order):
        P[k] = ((2 * k - 1) * x * P[k - 1] - (k - 1) * P[k - 2]) / k
    return P * np.sqrt(np.arange(order) + 0.5)[:, None]


def legendre_orthonormal_deriv(order, x):
    """d/dx of ``legendre_orthonormal``."""
    x = np.asarray(x, dtype=np.float64)
    P = np.zeros((order, x.size))
    dP = np.zeros((order, x.size))
    if order > 0:
        P[0] = 1.0
    if order > 1:
        P[1] = x
        dP[1] = 1.0
    for k in range(2, order):
        P[k] = ((2 * k - 1) * x * P[k - 1] - (k - 1) * P[k - 2]) / k
        dP[k] = dP[k - 2] + (2 * k - 1) * P[k - 1]
    return dP * np.sqrt(np.arange(order) + 0.5)[:, None]


def lagrange_at(nodes, x):
    """Lagrange basis on ``nodes`` evaluated at ``x``: shape (len(x), len(nodes))."""
    K = len(nodes)
    return np.linalg.solve(legendre_orthonormal(K, nodes),
                           legendre_orthonormal(K, x)).T


def lagrange_deriv_at(nodes, x):
    """Derivative matrix D[i, j] = l_i'(x_j): shape (len(nodes), len(x))."""
    K = len(nodes)
    return np.linalg.solve(legendre_orthonormal(K, nodes),
                           legendre_orthonormal_deriv(K, x))
