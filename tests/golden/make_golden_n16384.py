"""Generate tests/golden/n16384.npz: the reference's own results at the benchmark's order.

Runs the oracle drivers linked against the reference's calgo/*.c (oracle/_ref, built by
`make -C oracle ref` from the reference sources) on the configured n = 16384 inputs, with
NumWorkers = this host's cores and nb = 64 (the reference's baseline block size):
  * DecomposeLU + SolveLU on A iid N(0,1) (numpy PCG64 seed 4, generated column by column,
    so every machine builds the same bits), 64 RHS iid U[-1,1] (seed 5): the full pivot
    vector, the factor at 4096 sampled positions and 256 sampled rows of X;
  * DecomposeCHOL + SolveCHOL on A = G G^T / n + 0.5 I (G iid N(0,1), seed 2), 64 RHS iid
    U[-1,1] (seed 3): L at 4096 sampled lower-triangle positions and 256 rows of X.
The factors themselves (2 GiB each) are not stored.  Takes several minutes of CPU.

    python tests/golden/make_golden_n16384.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.oracle import Oracle, build  # noqa: E402

N, NRHS, NB = 16384, 64, 64
LO = 0x4


def lu_input(n=N):
    return np.asfortranarray(np.random.default_rng(4).standard_normal((n, n)).T)


def chol_g(n=N):
    return np.random.default_rng(2).standard_normal((n, n))


def rhs(seed, n=N, nrhs=NRHS):
    return np.asfortranarray(np.random.default_rng(seed).uniform(-1, 1, (nrhs, n)).T)


def sample_positions(n=N, count=4096, lower=False):
    rng = np.random.default_rng(99 if not lower else 98)
    i = rng.integers(0, n, count)
    j = rng.integers(0, n, count)
    if lower:
        i, j = np.maximum(i, j), np.minimum(i, j)
    return i.astype(np.int64), j.astype(np.int64)


def sample_rows(n=N, count=256):
    return np.sort(np.random.default_rng(97).choice(n, count, replace=False)).astype(np.int64)


def main():
    build(ref=True)
    ref = Oracle("ref")
    cores = os.cpu_count() or 1
    ref.NumWorkers(cores)
    out = {"n": N, "nb": NB, "num_workers": cores}
    rows = sample_rows()

    A = lu_input()
    B = rhs(5)
    piv = np.zeros(N, np.int64)
    t0 = time.time()
    assert ref.DecomposeLU(A, piv, NB) == 0
    t1 = time.time()
    assert ref.SolveLU(B, A, piv, 0) == 0
    t2 = time.time()
    i, j = sample_positions()
    out.update(lu_piv=piv, lu_i=i, lu_j=j, lu_val=A[i, j], lu_x_rows=rows, lu_x=B[rows],
               lu_factor_s=t1 - t0, lu_solve_s=t2 - t1)
    print(f"LU {t1 - t0:.1f} s, SolveLU {t2 - t1:.1f} s", flush=True)
    del A, B

    G = chol_g()
    A = np.asfortranarray(G @ G.T / N + 0.5 * np.eye(N))
    del G
    B = rhs(3)
    t0 = time.time()
    assert ref.DecomposeCHOL(A, LO, NB) == 0
    t1 = time.time()
    ref.SolveCHOL(B, A, LO)
    t2 = time.time()
    i, j = sample_positions(lower=True)
    out.update(chol_i=i, chol_j=j, chol_val=A[i, j], chol_x_rows=rows, chol_x=B[rows],
               chol_factor_s=t1 - t0, chol_solve_s=t2 - t1)
    print(f"Cholesky {t1 - t0:.1f} s, SolveCHOL {t2 - t1:.1f} s", flush=True)
    path = os.path.join(HERE, "n16384.npz")
    np.savez_compressed(path, **out)
    print(path)


if __name__ == "__main__":
    main()
