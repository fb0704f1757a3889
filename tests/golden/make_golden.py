"""Generate tests/golden/golden.npz from the reference's own C kernels.

Runs the oracle drivers (oracle/drivers.c) linked against hrautila/matops's calgo/ C
files compiled from their sources (oracle/_ref/libmatops_ref.so, built by
`make -C oracle ref`), on
  * the deterministic matrices of the reference's tests (decomp_test.go:85-89 and
    :110-114 LU inputs, :150-155 Cholesky factor, calgo_test.go:48-70 triangles), and
  * seeded random inputs for every entry point and flag combination.
Every case stores its inputs and the reference outputs.  Buffers use an even leading
dimension so the reference takes its aligned GEMV path (calgo/dmvec_gemv.c:241 offsets
Y by the X stride in the unaligned path).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.oracle import Oracle, build  # noqa: E402

TA, TB, LO, UP, LEFT, RIGHT, UNIT = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40


def F(a, ld=None):
    a = np.asarray(a, dtype=np.float64)
    r, c = a.shape
    ld = ld or r + (r % 2)
    buf = np.zeros((ld, max(c, 1)), order="F")
    buf[:r, :c] = a
    return buf[:r, :c]


def table(rows):
    return F(np.array(rows, dtype=np.float64))


def main():
    build(ref=True)
    ref = Oracle("ref")
    rng = np.random.default_rng(20240601)
    out = {}

    def put(name, **arrs):
        for k, v in arrs.items():
            out[f"{name}/{k}"] = np.asarray(v)

    # ---- known-answer inputs from the reference's tests ----
    lu3 = [[3.0, 2.0, 2.0], [6.0, 4.0, 1.0], [4.0, 6.0, 3.0]]          # decomp_test.go:85-89
    lu34 = [[3.0, 2.0, 2.0, 1.0], [6.0, 4.0, 1.0, 2.0], [4.0, 6.0, 3.0, 3.0]]  # :110-114
    for name, t in [("ka_lu3x3", lu3), ("ka_lu3x4", lu34)]:
        A = table(t)
        R = F(A)
        p = np.zeros(min(A.shape), np.int64)
        assert ref.DecomposeLU(R, p, 0) == 0
        put(name, A=A, LU=R, piv=p, nb=0)
    L3 = np.array([[3.0, 0.0, 0.0], [6.0, 4.0, 0.0], [4.0, 6.0, 3.0]])   # decomp_test.go:150-155
    A = F(L3 @ L3.T)
    R = F(A)
    assert ref.DecomposeCHOL(R, LO, 0) == 0
    put("ka_chol3x3", A=A, L=R, flags=LO, nb=0, Lexact=L3)
    lower7 = np.tril(np.ones((7, 7)) * np.arange(1, 8)[None, :])          # calgo_test.go:55-62
    upper7 = np.triu(np.ones((7, 7)) * np.arange(1, 8)[:, None])          # calgo_test.go:46-53
    data7 = np.ones((7, 7)) * np.arange(1, 8)[:, None]                     # calgo_test.go:21-28
    for tname, T in [("lower7", lower7), ("upper7", upper7)]:
        for flags in [LEFT, LEFT | TA, RIGHT, RIGHT | TA]:
            fl = flags | (LO if tname == "lower7" else UP)
            A = F(T)
            B = F(data7)
            X = F(B)
            assert ref.SolveTrm(X, A, 1.0, fl) == 0
            put(f"ka_trsm_{tname}_{fl:#x}", A=A, B=B, X=X, flags=fl, alpha=1.0)

    # ---- seeded random cases ----
    for fl in [0, TA, TB, TA | TB]:
        m, n, k = 37, 29, 41
        A = F(rng.uniform(-1, 1, (k, m) if fl & TA else (m, k)))
        B = F(rng.uniform(-1, 1, (n, k) if fl & TB else (k, n)))
        C = F(rng.uniform(-1, 1, (m, n)))
        for beta in [-0.5, 0.0]:
            R = F(C)
            assert ref.Mult(R, A, B, 1.5, beta, fl) == 0
            put(f"mult_{fl}_{beta}", A=A, B=B, C=C, R=R, alpha=1.5, beta=beta, flags=fl)
    for fl in [LO, UP | TA, UP, LO | TA]:
        for beta in [1.0, 0.5]:
            n, k = 70, 5   # n > 68: exercises the diagonal-block beta of dmmat_rank.c
            A = F(rng.standard_normal((k, n) if fl & TA else (n, k)))
            C = F(rng.standard_normal((n, n)))
            R = F(C)
            assert ref.RankUpdateSym(R, A, -1.0, beta, fl) == 0
            put(f"syrk_{fl}_{beta}", A=A, C=C, R=R, alpha=-1.0, beta=beta, flags=fl)
    for side in [LEFT, RIGHT]:
        for uplo in [LO, UP]:
            for tr in [0, TA]:
                for unit in [0, UNIT]:
                    fl = side | uplo | tr | unit
                    n, nrhs = 45, 5
                    T = rng.uniform(-0.3, 0.3, (n, n)) + np.diag(rng.uniform(1.0, 2.0, n))
                    A = F(T)
                    B = F(rng.standard_normal((nrhs, n) if side == RIGHT else (n, nrhs)))
                    X = F(B)
                    assert ref.SolveTrm(X, A, 0.75, fl) == 0
                    put(f"trsm_{fl:#x}", A=A, B=B, X=X, flags=fl, alpha=0.75)
    for fl in [LO, UP]:
        for n, nb in [(61, 16), (33, 0), (1, 0), (2, 16), (69, 68)]:
            G = rng.standard_normal((n, n))
            A = F(G @ G.T / n + 0.5 * np.eye(n))
            R = F(A)
            assert ref.DecomposeCHOL(R, fl, nb) == 0
            B = F(rng.uniform(-1, 1, (n, 7)))
            X = F(B)
            ref.SolveCHOL(X, R, fl)
            put(f"chol_{fl}_{n}_{nb}", A=A, L=R, B=B, X=X, flags=fl, nb=nb)
    for (m, n, nb) in [(60, 60, 12), (40, 40, 0), (70, 50, 16), (64, 96, 16), (101, 101, 64),
                       (1, 1, 0), (2, 2, 0)]:
        A = F(rng.standard_normal((m, n)))
        R = F(A)
        p = np.zeros(min(m, n), np.int64)
        assert ref.DecomposeLU(R, p, nb) == 0
        case = dict(A=A, LU=R, piv=p, nb=nb)
        if m == n:
            for tr in [0, TA]:
                B = F(rng.uniform(-1, 1, (n, 5)))
                X = F(B)
                assert ref.SolveLU(X, R, p, tr) == 0
                case[f"B{tr}"] = B
                case[f"X{tr}"] = X
        put(f"lu_{m}_{n}_{nb}", **case)
    # ---- the rest of the level-3 surface (mmult.go:266, :338, :453, :501) ----
    for fl in [LEFT | LO, LEFT | UP, LEFT | LO | TA, RIGHT | LO, RIGHT | UP]:
        n, p = (45, 7) if fl & LEFT else (45, 45)
        A = F(rng.uniform(-1, 1, (n, n)))
        B = F(rng.uniform(-1, 1, (n, p) if fl & LEFT else (p, n)))
        C = F(rng.uniform(-1, 1, (n, p) if fl & LEFT else (p, n)))
        R = F(C)
        assert ref.MultSym(R, A, B, 1.5, -0.5, fl) == 0
        put(f"symm_{fl:#x}", A=A, B=B, C=C, R=R, alpha=1.5, beta=-0.5, flags=fl)
    for fl in [LEFT | LO, LEFT | UP | TA, RIGHT | LO | UNIT, RIGHT | UP | TA, LO | TA | UNIT]:
        n = 75
        A = F(rng.uniform(-1, 1, (n, n)))
        B = F(rng.uniform(-1, 1, (6, n) if fl & RIGHT else (n, 6)))
        R = F(B)
        assert ref.MultTrm(R, A, 0.75, fl) == 0
        put(f"trmm_{fl:#x}", A=A, B=B, R=R, alpha=0.75, flags=fl)
    for fl in [LO, UP, LO | TA, UP | TA]:
        for beta in [1.0, 0.5]:
            n, k = 75, 6
            A = F(rng.standard_normal((k, n) if fl & TA else (n, k)))
            B = F(rng.standard_normal(A.shape))
            C = F(rng.standard_normal((n, n)))
            R = F(C)
            assert ref.RankUpdate2Sym(R, A, B, 1.5, beta, fl) == 0
            put(f"syr2k_{fl}_{beta}", A=A, B=B, C=C, R=R, alpha=1.5, beta=beta, flags=fl)
    for fl in [LO, UP, LO | TA, UP | TB]:
        for beta in [1.0, 0.5]:
            n, k = 75, 6
            A = F(rng.standard_normal((k, n) if fl & TA else (n, k)))
            B = F(rng.standard_normal((n, k) if fl & TB else (k, n)))
            C = F(rng.standard_normal((n, n)))
            R = F(C)
            assert ref.UpdateTrm(R, A, B, 1.5, beta, fl) == 0
            put(f"trmupd_{fl}_{beta}", A=A, B=B, C=C, R=R, alpha=1.5, beta=beta, flags=fl)
    for fl in [LO, UP, LO | UNIT, UP | UNIT]:
        for n, nb in [(40, 0), (75, 16)]:
            T = rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n) + np.diag(rng.uniform(1.0, 2.0, n))
            A = F(T)
            R = F(A)
            assert ref.InverseTrm(R, fl, nb) == 0
            put(f"trinv_{fl}_{n}_{nb}", A=A, R=R, flags=fl, nb=nb)
    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **out)
    print(path, len(out), "arrays")


if __name__ == "__main__":
    main()
