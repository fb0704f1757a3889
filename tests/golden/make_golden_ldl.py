"""Generate tests/golden/ldl.npz from the reference's own C kernels (LDL^T path).

Runs the restated Go sweeps of ldlnp.go / ldl.go / ldlbk.go / ldlbks.go (oracle/drivers.c)
linked against hrautila/matops's calgo/ C files compiled from their sources
(oracle/_ref/libmatops_ref.so, `make -C oracle ref`) on
  * the 7 x 7 lower-triangle tables of the reference's Bunch-Kaufman tests
    (ldlbkl_test.go:62-69 and :111-118) with the right-hand sides of those tests (columns
    10 and 20 times the matrix, ldlbkl_test.go:71-84), and
  * seeded symmetric uniform inputs (orders 7, 40, 80; LOWER and UPPER; the 7 x 7
    A = A0 A0^T of ldl_test.go:58-61 for DecomposeLDL).
Every case stores its inputs and the reference outputs (factor, pivots, solution).

    python tests/golden/make_golden_ldl.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.oracle import Oracle, build  # noqa: E402

LO, UP = 0x4, 0x8


def F(a):
    a = np.asarray(a, dtype=np.float64)
    r, c = a.shape
    buf = np.zeros((r + (r % 2), max(c, 1)), order="F")
    buf[:r, :c] = a
    return buf[:r, :c]


def main():
    build(ref=True)
    ref = Oracle("ref")
    rng = np.random.default_rng(20261205)
    out = {}

    def put(name, **arrs):
        for k, v in arrs.items():
            out[f"{name}/{k}"] = np.asarray(v)

    t1 = [[1, 0, 0, 0, 0, 0, 0], [1, 2, 0, 0, 0, 0, 0], [1, 2, 3, 0, 0, 0, 0],
          [1, 2, 3, 4, 0, 0, 0], [1, 5, 3, 4, 5, 0, 0], [1, 2, 3, 4, 9, 6, 0],
          [1, 2, 3, 4, 5, 6, 7]]                            # ldlbkl_test.go:62-69
    t2 = [r[:] for r in t1]
    t2[6] = [1, 2, 3, 9, 5, 6, 7]                           # ldlbkl_test.go:111-118
    for name, t in (("ka_bk7a", t1), ("ka_bk7b", t2)):
        L = np.array(t, dtype=np.float64)
        S = np.tril(L) + np.tril(L, -1).T
        X = np.tile([10.0, 20.0], (7, 1))
        B = S @ X                                           # MultSym(B, A, X, LOWER|LEFT)
        A, p = F(L), np.zeros(7, np.int64)
        assert ref.DecomposeBK(A, p, LO) == 0
        Bs = F(B)
        ref.SolveBK(Bs, A, p, LO)
        put(name, A=L, flags=LO, LDL=A, piv=p, B=B, X=Bs)
    for n in (7, 40, 80):
        for fl in (LO, UP):
            g = rng.uniform(-1, 1, (n, n))
            S = g + g.T
            B = rng.uniform(-1, 1, (n, 3))
            A, p = F(S), np.zeros(n, np.int64)
            assert ref.DecomposeBK(A, p, fl) == 0
            Bs = F(B)
            ref.SolveBK(Bs, A, p, fl)
            put(f"bk_{n}_{fl}", A=S, flags=fl, LDL=A, piv=p, B=B, X=Bs)
            A, p = F(S), np.zeros(n, np.int64)
            assert ref.DecomposeLDL(A, p, fl) == 0
            Bs = F(B)
            ref.SolveLDL(Bs, A, p, fl)
            put(f"ldl_{n}_{fl}", A=S, flags=fl, LDL=A, piv=p, B=B, X=Bs)
            Sd = S + 2.0 * n * np.eye(n)
            A = F(Sd)
            assert ref.DecomposeLDLnoPiv(A, fl) == 0
            Bs = F(B)
            ref.SolveLDLnoPiv(Bs, A, fl)
            put(f"np_{n}_{fl}", A=Sd, flags=fl, LDL=A, B=B, X=Bs)
    A0 = rng.uniform(size=(7, 7))
    S = A0 @ A0.T                                           # ldl_test.go:58-61
    A, p = F(S), np.zeros(7, np.int64)
    assert ref.DecomposeLDL(A, p, LO) == 0
    put("ka_ldl7", A=S, flags=LO, LDL=A, piv=p)
    np.savez_compressed(os.path.join(HERE, "ldl.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
