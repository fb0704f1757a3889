"""Shared helpers for the parity tests: seeded column-major inputs and error metrics."""
import numpy as np

EPS = np.finfo(np.float64).eps


def colmajor(a, ld=None):
    """Column-major copy of `a`; with ld > rows the matrix is a view into a taller buffer."""
    a = np.asarray(a, dtype=np.float64)
    r, c = a.shape
    ld = max(r, 1) if ld is None else ld
    buf = np.zeros((ld, max(c, 1)), order="F")
    buf[:r, :c] = a
    return buf[:r, :c]


def even_ld(r):
    return r + (r % 2)


def spd(rng, n, shift=0.5):
    g = rng.standard_normal((n, n))
    return g @ g.T / max(n, 1) + shift * np.eye(n)


def fro(a):
    return float(np.linalg.norm(a))


def gemm_bound(k, alpha, beta, A, B, C0):
    return 4 * max(k, 1) * EPS * (abs(alpha) * fro(A) * fro(B) + abs(beta) * fro(C0)) + 1e-300
