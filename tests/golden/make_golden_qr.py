"""Generate tests/golden/qr.npz from the reference's own C kernels (QR path).

Runs the restated Go drivers of qrwy.go / qrwym.go / house.go (oracle/drivers.c) linked
against hrautila/matops's calgo/ C files compiled from their sources
(oracle/_ref/libmatops_ref.so, `make -C oracle ref`), on seeded uniform [0, 1) inputs of
the shapes of the reference's own QR tests (qr_test.go:13-205: 60 x 40 with nb 4 and 12,
30 right-hand sides, a 40 x 40 minimum-norm system, BuildQ / BuildQT of qrwyk.go) and on
a 200 x 120 case where more
than 68 rows lie below the first columns, so that the reference's transposed GEMV scales
by beta once per 68-row block (calgo/dmvec_gemv.c:379-393).  Every case stores its inputs
and the reference outputs.

    python tests/golden/make_golden_qr.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.oracle import LEFT, RIGHT, TRANS, Oracle, build  # noqa: E402


def F(a):
    a = np.asarray(a, dtype=np.float64)
    r, c = a.shape
    buf = np.zeros((r + (r % 2), max(c, 1)), order="F")
    buf[:r, :c] = a
    return buf[:r, :c]


def main():
    build(ref=True)
    ref = Oracle("ref")
    rng = np.random.default_rng(20261204)
    out = {}

    def put(name, **arrs):
        for k, v in arrs.items():
            out[f"{name}/{k}"] = np.asarray(v)

    for name, (M, N, nb) in {"qrt_60x40_nb12": (60, 40, 12), "qrt_60x40_nb4": (60, 40, 4),
                             "qrt_60x40_unb": (60, 40, 0), "qrt_200x120_nb32": (200, 120, 32)}.items():
        A = F(rng.uniform(size=(M, N)))
        R, T = F(A), F(np.zeros((N, N)))
        assert ref.DecomposeQRT(R, T, F(np.zeros((N, max(nb, 1)))), nb) == 0
        put(name, A=A, QR=R, T=T, nb=nb)
    for name, (M, N, nb) in {"qr_60x40_nb4": (60, 40, 4), "qr_60x40_unb": (60, 40, 0)}.items():
        A = F(rng.uniform(size=(M, N)))
        R, tau = F(A), np.zeros(N)
        assert ref.DecomposeQR(R, tau, F(np.zeros((N, max(nb, 1)))), nb) == 0
        T = F(np.zeros((N, N)))
        assert ref.BuildT(T, R, tau.copy()) == 0
        put(name, A=A, QR=R, tau=tau, T=T, nb=nb)
    # MultQT / SolveQRT on the 60 x 40 factorization of qrt_60x40_nb12 (qr_test.go:79-105,
    # 137-203)
    QR, T = F(out["qrt_60x40_nb12/QR"]), F(out["qrt_60x40_nb12/T"])
    for flags in (LEFT, LEFT | TRANS, RIGHT, RIGHT | TRANS):
        for nb in (0, 12):
            C = F(rng.uniform(size=(30, 60) if flags & RIGHT else (60, 30)))
            R = F(C)
            assert ref.MultQT(R, QR, T, F(np.zeros((60, 40))), flags, nb) == 0
            put(f"multqt_{flags}_{nb}", C=C, R=R, flags=flags, nb=nb)
    X0 = rng.uniform(size=(40, 30))
    A = F(out["qrt_60x40_nb12/A"])
    B = F(A @ X0)
    R = F(B)
    assert ref.SolveQRT(R, QR, T, F(np.zeros((30, 40))), 0, 12) == 0
    put("solveqrt_ls", B=B, R=R, flags=0, nb=12)
    As = F(rng.uniform(size=(40, 40)))
    QRs, Ts = F(As), F(np.zeros((40, 40)))
    assert ref.DecomposeQRT(QRs, Ts, F(np.zeros((40, 12))), 12) == 0
    B = F(rng.uniform(size=(40, 30)))
    R = F(B)
    assert ref.SolveQRT(R, QRs, Ts, F(np.zeros((30, 40))), TRANS, 12) == 0
    put("solveqrt_minnorm", B=B, R=R, flags=TRANS, nb=12, QR=QRs, T=Ts, A=As)
    # BuildQ / BuildQT (qrwyk.go:232, :278) on fresh 60 x 40 factorizations
    for nb in (0, 12):
        A = F(rng.uniform(size=(60, 40)))
        R, tau = F(A), np.zeros(40)
        assert ref.DecomposeQR(R, tau, None, 0) == 0
        Q = F(R)
        assert ref.BuildQ(Q, tau, F(np.zeros((40, max(nb, 1)))), nb) == 0
        put(f"buildq_{nb}", A=A, QR=R, tau=tau, Q=Q, nb=nb)
        R2, T2 = F(A), F(np.zeros((40, 40)))
        assert ref.DecomposeQRT(R2, T2, None, 0) == 0
        Q2 = F(R2)
        assert ref.BuildQT(Q2, T2, F(np.zeros((40, 40))), nb) == 0
        put(f"buildqt_{nb}", A=A, QR=R2, T=T2, Q=Q2, nb=nb)
    np.savez_compressed(os.path.join(HERE, "qr.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
