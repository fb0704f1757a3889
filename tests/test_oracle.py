"""CPU: the oracle (restated Go drivers + restated C kernels) against the reference.

1. golden.npz holds outputs of the reference's own C kernels (tests/golden/make_golden.py);
   the restatement must reproduce them (pivots exactly, values to rounding).
2. when oracle/_ref is built, port and reference are also compared on fresh inputs.
"""
import os

import numpy as np
import pytest

from util import EPS, colmajor, even_ld, fro, spd

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")
TA, TB, LO, UP, LEFT, RIGHT, UNIT = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40


@pytest.fixture(scope="module")
def golden():
    z = np.load(GOLDEN)
    cases = {}
    for k in z.files:
        name, field = k.split("/")
        cases.setdefault(name, {})[field] = z[k]
    return cases


def F(a):
    return colmajor(a, ld=even_ld(a.shape[0]))


def names(prefix):
    z = np.load(GOLDEN)
    return sorted({k.split("/")[0] for k in z.files if k.startswith(prefix)})


def rel(a, b):
    return fro(a - b) / max(fro(b), 1e-300)


@pytest.mark.parametrize("name", names("mult_"))
def test_golden_mult(oracle, golden, name):
    c = golden[name]
    R = F(c["C"])
    assert oracle.Mult(R, F(c["A"]), F(c["B"]), float(c["alpha"]), float(c["beta"]), int(c["flags"])) == 0
    assert rel(R, c["R"]) <= 1e-14


@pytest.mark.parametrize("name", names("syrk_"))
def test_golden_rank_update_sym(oracle, golden, name):
    c = golden[name]
    R = F(c["C"])
    assert oracle.RankUpdateSym(R, F(c["A"]), float(c["alpha"]), float(c["beta"]), int(c["flags"])) == 0
    assert rel(R, c["R"]) <= 1e-14


@pytest.mark.parametrize("name", names("trsm_") + names("ka_trsm_"))
def test_golden_solve_trm(oracle, golden, name):
    c = golden[name]
    X = F(c["B"])
    assert oracle.SolveTrm(X, F(c["A"]), float(c["alpha"]), int(c["flags"])) == 0
    assert rel(X, c["X"]) <= 1e-13


@pytest.mark.parametrize("name", names("chol_") + names("ka_chol"))
def test_golden_chol(oracle, golden, name):
    c = golden[name]
    L = F(c["A"])
    assert oracle.DecomposeCHOL(L, int(c["flags"]), int(c["nb"])) == 0
    assert rel(L, c["L"]) <= 1e-13
    if "Lexact" in c:  # decomp_test.go:150-163: chol(L L^T) recovers L
        assert np.allclose(np.tril(L), c["Lexact"], rtol=1e-5, atol=1e-8)
    if "B" in c:
        X = F(c["B"])
        oracle.SolveCHOL(X, L, int(c["flags"]))
        assert rel(X, c["X"]) <= 1e-12


@pytest.mark.parametrize("name", names("lu_") + names("ka_lu"))
def test_golden_lu(oracle, golden, name):
    c = golden[name]
    LU = F(c["A"])
    p = np.zeros(len(c["piv"]), np.int64)
    assert oracle.DecomposeLU(LU, p, int(c["nb"])) == 0
    assert np.array_equal(p, c["piv"])
    assert rel(LU, c["LU"]) <= 1e-12
    for tr in (0, TA):
        if f"B{tr}" in c:
            X = F(c[f"B{tr}"])
            assert oracle.SolveLU(X, LU, p, tr) == 0
            assert rel(X, c[f"X{tr}"]) <= 1e-11


@pytest.mark.parametrize("name", names("symm_"))
def test_golden_mult_sym(oracle, golden, name):
    c = golden[name]
    R = F(c["C"])
    assert oracle.MultSym(R, F(c["A"]), F(c["B"]), float(c["alpha"]), float(c["beta"]), int(c["flags"])) == 0
    assert rel(R, c["R"]) <= 1e-13


@pytest.mark.parametrize("name", names("trmm_"))
def test_golden_mult_trm(oracle, golden, name):
    c = golden[name]
    R = F(c["B"])
    assert oracle.MultTrm(R, F(c["A"]), float(c["alpha"]), int(c["flags"])) == 0
    assert rel(R, c["R"]) <= 1e-13


@pytest.mark.parametrize("name", names("syr2k_") + names("trmupd_"))
def test_golden_rank2_and_trm_update(oracle, golden, name):
    c = golden[name]
    R = F(c["C"])
    fn = oracle.RankUpdate2Sym if name.startswith("syr2k") else oracle.UpdateTrm
    assert fn(R, F(c["A"]), F(c["B"]), float(c["alpha"]), float(c["beta"]), int(c["flags"])) == 0
    assert rel(R, c["R"]) <= 1e-13
    # the opposite strict triangle is untouched
    n = R.shape[0]
    other = np.triu(np.ones((n, n), bool), 1) if int(c["flags"]) & LO else np.tril(np.ones((n, n), bool), -1)
    assert np.array_equal(R[other], c["C"][other])


@pytest.mark.parametrize("name", names("trinv_"))
def test_golden_inverse_trm(oracle, golden, name):
    c = golden[name]
    R = F(c["A"])
    assert oracle.InverseTrm(R, int(c["flags"]), int(c["nb"])) == 0
    assert rel(R, c["R"]) <= 1e-13


def test_golden_lu3x3_matches_lapack(golden):
    """decomp_test.go:85-108 compares against lapack.Getrf: pivots are LAPACK's minus one."""
    import scipy.linalg as sl
    c = golden["ka_lu3x3"]
    lu, piv = sl.lu_factor(c["A"])
    assert np.array_equal(piv, c["piv"])
    assert np.allclose(lu, c["LU"], rtol=1e-12, atol=1e-14)


# ---- port vs the reference's own kernels on fresh inputs ----

@pytest.mark.parametrize("seed", [1, 2])
def test_port_vs_ref_factorizations(oracle, ref_oracle, seed):
    rng = np.random.default_rng(seed)
    for n, nb in [(97, 16), (150, 68), (64, 0)]:
        A = F(spd(rng, n))
        a1, a2 = F(A), F(A)
        assert oracle.DecomposeCHOL(a1, LO, nb) == ref_oracle.DecomposeCHOL(a2, LO, nb) == 0
        assert rel(a1, a2) <= 1e-13
        G = F(rng.standard_normal((n, n)))
        g1, g2 = F(G), F(G)
        p1, p2 = np.zeros(n, np.int64), np.zeros(n, np.int64)
        oracle.DecomposeLU(g1, p1, nb)
        ref_oracle.DecomposeLU(g2, p2, nb)
        assert np.array_equal(p1, p2)
        assert rel(g1, g2) <= 1e-11


def test_port_vs_ref_mult_workers(oracle, ref_oracle):
    """Mult's goroutine split (mmult.go:137-255) restated with threads: same result."""
    rng = np.random.default_rng(7)
    m, n, k = 300, 260, 250
    A, B, C = F(rng.uniform(-1, 1, (m, k))), F(rng.uniform(-1, 1, (k, n))), F(rng.uniform(-1, 1, (m, n)))
    outs = []
    for o in (oracle, ref_oracle):
        for w in (1, 4, 6):
            old = o.NumWorkers(w)
            R = F(C)
            assert o.Mult(R, A, B, 1.5, -0.5, 0) == 0
            o.NumWorkers(old)
            outs.append(R)
    for R in outs[1:]:
        assert rel(R, outs[0]) <= 4 * k * EPS


def test_oracle_errors(oracle):
    assert oracle.Mult(F(np.zeros((3, 3))), F(np.zeros((3, 2))), F(np.zeros((3, 3))), 1, 1, 0) == -1
    assert oracle.DecomposeCHOL(F(np.zeros((3, 4))), LO, 0) == -2
    assert oracle.DecomposeLU(F(np.zeros((4, 4))), np.zeros(3, np.int64), 0) == -3
    assert oracle.RankUpdateSym(F(np.zeros((3, 4))), F(np.zeros((3, 2))), 1, 1, LO) == -4
    assert oracle.SolveTrm(F(np.zeros((3, 2))), F(np.eye(4)), 1, LEFT) == -5
    A = spd(np.random.default_rng(0), 50)
    A[20, 20] = -1.0
    assert oracle.DecomposeCHOL(F(A), LO, 16) == 21


def test_reference_gemv_unaligned_bug_is_real(ref_oracle, oracle):
    """calgo/dmvec_gemv.c:241 offsets Y by R*X->inc in the unaligned path.  With an odd
    leading dimension the reference's DecomposeLU writes outside the view at panel column
    1 (a 1x1 a01 has inc = ld); the restatement computes the intended result."""
    import scipy.linalg as sl
    rng = np.random.default_rng(5)
    n = 137
    A = colmajor(rng.standard_normal((n, n)), ld=n)   # odd ld -> unaligned path
    a1, a2 = colmajor(A, ld=n), colmajor(A, ld=n)
    p1, p2 = np.zeros(n, np.int64), np.zeros(n, np.int64)
    oracle.DecomposeLU(a1, p1, 0)
    ref_oracle.DecomposeLU(a2, p2, 0)
    lu, piv = sl.lu_factor(A)
    assert np.array_equal(p1, piv) and rel(a1, lu) <= 1e-12
    assert rel(a2, lu) > 1e-3


# ---------------- QR (qrwy.go, qrwym.go) ----------------

GOLDEN_QR = os.path.join(os.path.dirname(__file__), "golden", "qr.npz")


@pytest.fixture(scope="module")
def golden_qr():
    z = np.load(GOLDEN_QR)
    cases = {}
    for k in z.files:
        name, field = k.split("/")
        cases.setdefault(name, {})[field] = z[k]
    return cases


def qr_names(prefix):
    z = np.load(GOLDEN_QR)
    return sorted({k.split("/")[0] for k in z.files if k.startswith(prefix)})


@pytest.mark.parametrize("name", qr_names("qrt_"))
def test_golden_decompose_qrt(oracle, golden_qr, name):
    """the port in the reference's GEMV semantics reproduces the reference, the 200 x 120
    case (beta applied per 68-row block) included"""
    c = golden_qr[name]
    N = c["A"].shape[1]
    R, T = F(c["A"]), F(np.zeros((N, N)))
    assert oracle.DecomposeQRT(R, T, F(np.zeros((N, max(int(c["nb"]), 1)))), int(c["nb"])) == 0
    assert rel(R, c["QR"]) <= 1e-12
    assert rel(np.triu(T), np.triu(c["T"])) <= 1e-12


@pytest.mark.parametrize("name", qr_names("qr_"))
def test_golden_decompose_qr_build_t(oracle, golden_qr, name):
    c = golden_qr[name]
    N = c["A"].shape[1]
    R, tau = F(c["A"]), np.zeros(N)
    assert oracle.DecomposeQR(R, tau, F(np.zeros((N, max(int(c["nb"]), 1)))), int(c["nb"])) == 0
    assert rel(R, c["QR"]) <= 1e-12 and np.abs(tau - c["tau"]).max() <= 1e-13
    T = F(np.zeros((N, N)))
    assert oracle.BuildT(T, F(c["QR"]), c["tau"].copy()) == 0
    assert rel(np.triu(T), np.triu(c["T"])) <= 1e-12


@pytest.mark.parametrize("name", qr_names("multqt_") + qr_names("solveqrt_"))
def test_golden_mult_solve_qrt(oracle, golden_qr, name):
    c = golden_qr[name]
    if name == "solveqrt_minnorm":
        QR, T = F(c["QR"]), F(c["T"])
    else:
        QR, T = F(golden_qr["qrt_60x40_nb12"]["QR"]), F(golden_qr["qrt_60x40_nb12"]["T"])
    if name.startswith("multqt_"):
        R = F(c["C"])
        assert oracle.MultQT(R, QR, T, F(np.zeros((60, 40))), int(c["flags"]), int(c["nb"])) == 0
    else:
        R = F(c["B"])
        assert oracle.SolveQRT(R, QR, T, F(np.zeros((30, 40))), int(c["flags"]), int(c["nb"])) == 0
    assert rel(R, c["R"]) <= 1e-12


def test_reference_qrt_gemv_beta_quirk(oracle, golden_qr):
    """The reference's T recurrence goes through a transposed GEMV that scales y by beta
    once per 68-row block (calgo/dmvec_gemv.c:379-393), with beta = -tau (qrwy.go:66): its
    200 x 120 factorization is not A = Q R (golden, from its own kernels).  With one beta
    per product (BLAS semantics, what the device computes) the same drivers give A = Q R."""
    c = golden_qr["qrt_200x120_nb32"]
    A, QR, T = c["A"], c["QR"], c["T"]
    M, N = A.shape

    def recon(QR, T):
        Y = np.tril(QR, -1) + np.eye(M, N)
        R = np.vstack([np.triu(QR[:N]), np.zeros((M - N, N))])
        return R - Y @ (np.triu(T) @ (Y.T @ R))

    assert rel(recon(QR, T), A) > 1e-2  # the reference's own result
    old = oracle.GemvBetaOnce(True)
    try:
        R2, T2 = F(A), F(np.zeros((N, N)))
        assert oracle.DecomposeQRT(R2, T2, F(np.zeros((N, 32))), 32) == 0
    finally:
        oracle.GemvBetaOnce(old)
    assert rel(recon(R2, T2), A) <= 100 * M * EPS
    q, r = np.linalg.qr(A)
    assert rel(np.abs(np.triu(R2[:N])), np.abs(r)) <= 1e-12


@pytest.mark.parametrize("seed", [0, 1])
def test_port_vs_ref_qr(oracle, ref_oracle, seed):
    rng = np.random.default_rng(100 + seed)
    M, N, nb = 150, 90, 16
    A = colmajor(rng.uniform(-1, 1, (M, N)), ld=even_ld(M))
    outs = []
    for o in (oracle, ref_oracle):
        R, T = colmajor(A, ld=even_ld(M)), colmajor(np.zeros((N, N)))
        assert o.DecomposeQRT(R, T, colmajor(np.zeros((N, nb))), nb) == 0
        C = colmajor(rng.uniform(-1, 1, (M, 20)) if not outs else outs[0][2].copy())
        C0 = C.copy(order="F")
        assert o.MultQT(C, R, T, colmajor(np.zeros((20, N))), LEFT | 0x80, 0) == 0
        outs.append((R, T, C0, C))
    assert rel(outs[0][0], outs[1][0]) <= 1e-12
    assert rel(np.triu(outs[0][1]), np.triu(outs[1][1])) <= 1e-12
    assert rel(outs[0][3], outs[1][3]) <= 1e-12


def test_oracle_qr_errors(oracle):
    A = colmajor(np.ones((10, 8)))
    assert oracle.DecomposeQRT(A, colmajor(np.zeros((8, 8))), colmajor(np.zeros((7, 2))), 2) == -13
    C = colmajor(np.ones((10, 3)))
    T = colmajor(np.zeros((8, 8)))
    assert oracle.MultQT(C, A, T, None, LEFT, 0) == -14
    assert oracle.MultQT(colmajor(np.ones((3, 9))), A, T, colmajor(np.zeros((3, 8))), RIGHT, 0) == -15
    assert oracle.MultQT(C, A, T, colmajor(np.zeros((3, 4))), LEFT, 0) == -13
    assert oracle.BuildT(colmajor(np.zeros((7, 8))), A, np.zeros(8)) == -16


@pytest.mark.parametrize("name", qr_names("buildq_") + qr_names("buildqt_"))
def test_golden_build_q(oracle, golden_qr, name):
    c = golden_qr[name]
    Q = F(c["QR"])
    if name.startswith("buildqt_"):
        assert oracle.BuildQT(Q, F(c["T"]), F(np.zeros((40, 40))), int(c["nb"])) == 0
    else:
        assert oracle.BuildQ(Q, c["tau"].copy(), F(np.zeros((40, max(int(c["nb"]), 1)))),
                             int(c["nb"])) == 0
    assert rel(Q, c["Q"]) <= 1e-12
    assert fro(Q.T @ Q - np.eye(40)) <= 100 * 60 * EPS


# ---------------- symmetric indefinite LDL^T (ldlnp.go, ldl.go, ldlbk.go, ldlbks.go) ------

def _sym(rng, n):
    g = rng.uniform(-1, 1, (n, n))
    return g + g.T


@pytest.mark.parametrize("n", [1, 2, 5, 37, 120])
@pytest.mark.parametrize("flags", [LO, UP])
def test_port_vs_ref_ldl(oracle, ref_oracle, n, flags):
    """port and the reference's kernels: identical pivots, factors to rounding, and the
    solves satisfy A X = B"""
    rng = np.random.default_rng(300 + n)
    A0 = colmajor(_sym(rng, n), ld=even_ld(n))
    B0 = colmajor(rng.uniform(-1, 1, (n, 3)))
    res = []
    for o in (oracle, ref_oracle):
        Ad = colmajor(A0 + 2 * n * np.eye(n))
        assert o.DecomposeLDLnoPiv(Ad, flags) == 0
        A1, p1 = colmajor(A0), np.zeros(n, np.int64)
        assert o.DecomposeLDL(A1, p1, flags) == 0
        A2, p2 = colmajor(A0), np.zeros(n, np.int64)
        assert o.DecomposeBK(A2, p2, flags) == 0
        X = colmajor(B0)
        o.SolveBK(X, A2, p2, flags)
        res.append((Ad, A1, p1, A2, p2, X))
    (a, b) = res
    assert rel(a[0], b[0]) <= 1e-13
    assert np.array_equal(a[2], b[2]) and rel(a[1], b[1]) <= 1e-11
    assert np.array_equal(a[4], b[4]) and rel(a[3], b[3]) <= 1e-11
    S = np.tril(A0) if flags & LO else np.triu(A0)
    S = S + S.T - np.diag(np.diag(A0))
    for X in (a[5], b[5]):
        assert fro(S @ X - B0) <= 1e-9 * fro(S) * max(fro(X), 1.0)


def test_oracle_ldl_reference_cases(oracle):
    """ldl_test.go / ldlbkl_test.go style: the factors reproduce A (lower, 2 x 2 blocks
    included) and DecomposeLDL reports a zero pivot"""
    rng = np.random.default_rng(9)
    n = 40
    A0 = _sym(rng, n)
    A, p = colmajor(A0), np.zeros(n, np.int64)
    assert oracle.DecomposeBK(A, p, LO) == 0
    assert (p < 0).any() and (p > 0).any()
    Z, pz = colmajor(np.zeros((5, 5))), np.zeros(5, np.int64)
    assert oracle.DecomposeLDL(Z, pz, LO) == 1


GOLDEN_LDL = os.path.join(os.path.dirname(__file__), "golden", "ldl.npz")


def _ldl_cases():
    z = np.load(GOLDEN_LDL)
    cases = {}
    for k in z.files:
        name, field = k.split("/")
        cases.setdefault(name, {})[field] = z[k]
    return cases


@pytest.mark.parametrize("name", sorted(_ldl_cases()))
def test_golden_ldl(oracle, name):
    """the port reproduces the reference's kernels: pivots exactly, factors and solutions
    to rounding (the reference's Bunch-Kaufman test tables included)"""
    c = _ldl_cases()[name]
    fl = int(c["flags"])
    A = F(c["A"])
    n = A.shape[0]
    if name.startswith("np_"):
        assert oracle.DecomposeLDLnoPiv(A, fl) == 0
    else:
        p = np.zeros(n, np.int64)
        fn = oracle.DecomposeBK if ("bk" in name) else oracle.DecomposeLDL
        assert fn(A, p, fl) == 0
        assert np.array_equal(p, c["piv"])
    tri = np.tril if fl & LO else np.triu
    assert rel(tri(A), tri(c["LDL"])) <= 1e-12
    if "X" in c:
        X = F(c["B"])
        if name.startswith("np_"):
            oracle.SolveLDLnoPiv(X, A, fl)
        elif "bk" in name:
            oracle.SolveBK(X, A, c["piv"].copy(), fl)
        else:
            oracle.SolveLDL(X, A, c["piv"].copy(), fl)
        assert rel(X, c["X"]) <= 1e-10


@pytest.mark.parametrize("flags", [LEFT, LEFT | 0x80, RIGHT, RIGHT | 0x80])
def test_port_vs_ref_mult_q(oracle, ref_oracle, flags):
    """MultQ's unblocked path (qrwym.go:28-190): port and reference kernels agree and give
    the product of the reflectors"""
    rng = np.random.default_rng(77)
    m, n = 150, 90
    A = colmajor(rng.uniform(-1, 1, (m, n)))
    QR, tau = colmajor(A), np.zeros(n)
    assert oracle.DecomposeQR(QR, tau, None, 0) == 0
    Y = np.tril(QR, -1) + np.eye(m, n)
    Q = np.eye(m)
    for j in range(n):
        Q = Q - tau[j] * np.outer(Q @ Y[:, j], Y[:, j])
    C0 = rng.uniform(-1, 1, (5, m) if flags & RIGHT else (m, 5))
    outs = []
    for o in (oracle, ref_oracle):
        C = colmajor(C0)
        assert o.MultQ(C, QR, tau.copy(), None, flags, 0) == 0
        outs.append(C)
    exp = ((C0 @ Q.T if flags & 0x80 else C0 @ Q) if flags & RIGHT
           else (Q.T @ C0 if flags & 0x80 else Q @ C0))
    assert rel(outs[0], exp) <= 1e-13 and rel(outs[1], outs[0]) <= 1e-13
