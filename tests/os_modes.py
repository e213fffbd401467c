"""Orr-Sommerfeld eigenmodes of plane Poiseuille flow (test helper).

Chebyshev collocation with clamped boundary conditions (the formulation of
Trefethen, Spectral Methods in MATLAB, program 40).  Used to build known-answer
initial fields; the published benchmark is Orszag (1971), J. Fluid Mech. 50:
Re = 10000, alpha = 1  ->  c = 0.23752649 + 0.00373967 i.
"""
import numpy as np
import scipy.linalg as sl


def cheb(n):
    x = np.cos(np.pi * np.arange(n + 1) / n)
    c = np.hstack([2, np.ones(n - 1), 2]) * (-1) ** np.arange(n + 1)
    X = np.tile(x, (n + 1, 1)).T
    dX = X - X.T
    D = np.outer(c, 1 / c) / (dX + np.eye(n + 1))
    return D - np.diag(D.sum(1)), x


def least_stable_mode(n, re, alpha):
    """(c, v, dv) of the least stable 2-D mode on the n+1 Gauss-Lobatto points."""
    D, x = cheb(n)
    D2 = D @ D
    D3 = D2 @ D
    D4 = D3 @ D
    S = np.diag(np.hstack([0, 1 / (1 - x[1:n] ** 2), 0]))
    D4c = (np.diag(1 - x ** 2) @ D4 - 8 * np.diag(x) @ D3 - 12 * D2) @ S
    I = np.eye(n - 1)
    D2i, D4i = D2[1:n, 1:n], D4c[1:n, 1:n]
    a2 = alpha * alpha
    U = np.diag(1 - x[1:n] ** 2)
    A = U @ (D2i - a2 * I) + 2 * I - (D4i - 2 * a2 * D2i + a2 * a2 * I) / (1j * alpha * re)
    B = D2i - a2 * I
    ev, V = sl.eig(A, B)
    ok = np.isfinite(ev) & (np.abs(ev) < 1.5)
    idx = np.where(ok)[0]
    k = idx[np.argmax(ev[idx].imag)]
    v = np.zeros(n + 1, complex)
    v[1:n] = V[:, k]
    v /= v[np.argmax(np.abs(v))]
    return ev[k], v, D @ v
