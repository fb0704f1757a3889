"""GPU parity: DecomposeQRT / DecomposeQR / BuildT / MultQT / MultQ / SolveQRT / SolveQR
(qrwy.go, qrwym.go) against the oracle.

Where the computation is the reference's algorithm step for step, the oracle is the
reference's own calgo kernels (oracle/_ref) under the restated Go drivers when they were
built, else the port.  The reference's transposed GEMV scales its output by beta once per
68-row block (calgo/dmvec_gemv.c:379-393), which the factorization's and BuildT's T
recurrence call with beta = -tau (qrwy.go:66, :125): its T is the dlarft T only while at
most 68 rows lie below each column.  So the factorizations and BuildT are compared with the
reference's kernels for m <= 69 and, above that, with the oracle port switched to one beta
per product (GemvBetaOnce), the LAPACK definition the device computes; MultQT and SolveQRT
take A and T as inputs and use no GEMV, so they are compared with the reference's kernels
at every size.
"""
import numpy as np
import pytest

from util import EPS, colmajor, even_ld, fro

pytestmark = pytest.mark.gpu

LEFT, RIGHT, TRANS, UPPER, TRANSA = 0x10, 0x20, 0x80, 0x8, 0x1


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import Oracle, ref_available
    return Oracle("ref" if ref_available() else "port")


@pytest.fixture(scope="module")
def lapack():
    """the oracle port with BLAS-semantics transposed GEMV"""
    from oracle.oracle import Oracle
    o = Oracle("port")
    old = o.GemvBetaOnce(True)
    yield o
    o.GemvBetaOnce(old)


def dev(gpu, a):
    import torch
    if a.ndim != 2 or (a.shape[0] > 1 and a.strides[0] != 8):
        a = np.asfortranarray(a)
    ld = a.strides[1] // 8 if a.shape[1] > 1 else max(a.shape[0], 1)
    t = gpu.matrix(max(ld, 1), max(a.shape[1], 1))
    t.zero_()
    if a.size:
        t[: a.shape[0], : a.shape[1]].copy_(torch.from_numpy(np.asfortranarray(a)))
    return t[: a.shape[0], : a.shape[1]]


def host(t):
    return t.cpu().numpy()


def oracle_for(m, ref, lapack):
    return ref if m <= 69 else lapack


def qr_bound(m, n, A):
    return 8 * max(m, n) * EPS * max(fro(A), 1e-300)


@pytest.mark.parametrize("m,n,nb", [(1, 1, 0), (5, 3, 0), (60, 40, 12), (69, 69, 16), (69, 50, 0),
                                    (40, 60, 0), (200, 120, 32), (300, 300, 64), (1000, 700, 128),
                                    (2048, 2048, 64), (3000, 1000, 0), (1030, 1030, 32)])
def test_decompose_qrt(gpu, ref, lapack, rng, m, n, nb):
    A0 = colmajor(rng.uniform(-1, 1, (m, n)), ld=even_ld(m) + 2)
    k = min(m, n)
    # T exactly k x k: the reference partitions T by its own size, so a larger T puts its
    # last block out of step with A's.  Its upper triangle starts at zero, as in the
    # reference's tests: where a reflector is the identity (tau = 0, e.g. a square matrix's
    # last column) the reference leaves T's column above the diagonal as it was and its
    # blocked recurrence reads it; the device writes the zeros of the dlarft definition.
    # The strict lower part must stay untouched.
    T0 = colmajor(np.tril(rng.uniform(-1, 1, (k, k)), -1))
    Ag, Tg = dev(gpu, A0), dev(gpu, T0)
    Wg = gpu.matrix(max(n, 1), max(nb, 1))
    A_, err = gpu.DecomposeQRT(Ag, Tg, Wg, nb)
    assert err is None
    o = oracle_for(m, ref, lapack)
    Ar, Tr = A0.copy(order="F"), T0.copy(order="F")
    assert o.DecomposeQRT(Ar, Tr, np.zeros((max(n, 1), max(nb, 1)), order="F"), nb) == 0
    Ah, Th = host(Ag), host(Tg)
    bound = qr_bound(m, n, A0)
    assert fro(Ah - Ar) <= bound * max(1.0, np.sqrt(n)), fro(Ah - Ar)
    assert fro(np.triu(Th[:k, :k]) - np.triu(Tr[:k, :k])) <= bound * np.sqrt(k) + 1e-14
    assert np.array_equal(np.tril(Th, -1), np.tril(T0, -1))  # untouched
    # A = Q R with Q = I - Y T Y^T (properties of the device result alone)
    Y = np.tril(Ah[:, :k], -1) + np.eye(m, k)
    R = np.triu(Ah[:k, :])
    QR = R.copy()
    QR = np.vstack([R, np.zeros((m - k, n))]) if m > k else R[:m]
    QR = QR - Y @ (np.triu(Th[:k, :k]) @ (Y.T @ QR))
    assert fro(QR - A0) <= bound


@pytest.mark.parametrize("m,n,nb", [(60, 40, 12), (500, 300, 32), (257, 100, 0)])
def test_decompose_qr_and_build_t(gpu, ref, lapack, rng, m, n, nb):
    import torch
    A0 = colmajor(rng.uniform(-1, 1, (m, n)))
    k = min(m, n)
    Ag = dev(gpu, A0)
    tau = torch.zeros(k, dtype=torch.float64, device="cuda")
    _, err = gpu.DecomposeQR(Ag, tau, gpu.matrix(n, max(nb, 1)), nb)
    assert err is None
    o = oracle_for(m, ref, lapack)
    Ar, taur = A0.copy(order="F"), np.zeros(k)
    assert o.DecomposeQR(Ar, taur, np.zeros((n, max(nb, 1)), order="F"), nb) == 0
    bound = qr_bound(m, n, A0)
    assert fro(host(Ag) - Ar) <= bound * np.sqrt(n)
    assert np.abs(tau.cpu().numpy() - taur).max() <= 1e-12
    # BuildT on the same (device) reflectors and tau: reference kernels vs device
    T0 = colmajor(np.zeros((n, n)))
    Tg = dev(gpu, T0)
    _, err = gpu.BuildT(Tg, Ag, tau)
    assert err is None
    Tr = T0.copy(order="F")
    assert o.BuildT(Tr, host(Ag), tau.cpu().numpy().copy()) == 0
    assert fro(np.triu(host(Tg)) - np.triu(Tr)) <= bound * np.sqrt(k) + 1e-14


def factor(gpu, lapack, rng, m, n):
    """a device QR factorization (A, T) and the host copies"""
    A0 = colmajor(rng.uniform(-1, 1, (m, n)))
    k = min(m, n)
    Ag, Tg = dev(gpu, A0), dev(gpu, np.zeros((k, k)))
    _, err = gpu.DecomposeQRT(Ag, Tg, None, 0)
    assert err is None
    return A0, Ag, Tg, host(Ag), host(Tg)


@pytest.mark.parametrize("m,n", [(60, 40), (300, 200), (1100, 1000)])
@pytest.mark.parametrize("flags", [LEFT, LEFT | TRANS, RIGHT, RIGHT | TRANS, TRANS])
@pytest.mark.parametrize("nb", [0, 16, 64])
def test_mult_qt(gpu, ref, lapack, rng, m, n, flags, nb):
    A0, Ag, Tg, Ah, Th = factor(gpu, lapack, rng, m, n)
    p = 37
    C0 = colmajor(rng.uniform(-1, 1, (p, m) if flags & RIGHT else (m, p)), ld=even_ld(m) + 4)
    Cg = dev(gpu, C0)
    W = gpu.matrix(max(p, m), max(nb, n))
    assert gpu.MultQT(Cg, Ag, Tg, W, flags, nb) is None
    Cr = C0.copy(order="F")
    assert ref.MultQT(Cr, Ah, Th, np.zeros((max(p, m), max(nb, n)), order="F"), flags, nb) == 0
    err = fro(host(Cg) - Cr)
    assert err <= 16 * m * EPS * fro(C0), err


@pytest.mark.parametrize("m,n,p", [(60, 40, 30), (700, 500, 7), (2000, 1500, 64)])
@pytest.mark.parametrize("flags", [0, TRANS])
def test_solve_qrt(gpu, ref, lapack, rng, m, n, p, flags):
    A0, Ag, Tg, Ah, Th = factor(gpu, lapack, rng, m, n)
    if flags & TRANS:
        B0 = np.zeros((m, p))
        B0[:n] = rng.uniform(-1, 1, (n, p))
    else:
        B0 = A0 @ rng.uniform(-1, 1, (n, p)) + 1e-3 * rng.uniform(-1, 1, (m, p))
    B0 = colmajor(B0)
    Bg = dev(gpu, B0)
    W = gpu.matrix(p, n)
    assert gpu.SolveQRT(Bg, Ag, Tg, W, flags, 0) is None
    Br = B0.copy(order="F")
    assert ref.SolveQRT(Br, Ah, Th, np.zeros((p, n), order="F"), flags, 0) == 0
    Bh = host(Bg)
    cond = np.linalg.cond(A0)
    assert fro(Bh - Br) <= 64 * m * EPS * cond * max(fro(Br), 1.0), fro(Bh - Br)
    if flags & TRANS:
        assert fro(A0.T @ Bh - B0[:n]) <= 64 * m * EPS * cond * fro(B0)
    else:
        X = Bh[:n]
        # normal equations of the least-squares solution
        assert fro(A0.T @ (A0 @ X - B0)) <= 64 * m * EPS * cond * fro(A0) * fro(B0)


@pytest.mark.parametrize("m,n", [(90, 60), (700, 450)])
@pytest.mark.parametrize("flags", [LEFT, LEFT | TRANS, RIGHT, RIGHT | TRANS])
def test_mult_q_vs_reference(gpu, ref, rng, m, n, flags):
    """MultQ (tau form) against the reference kernels' unblocked MultQ (qrwym.go:28-190, no
    GEMV with beta != 1 on that path), the same reflectors on both sides"""
    import torch
    A0 = colmajor(rng.uniform(-1, 1, (m, n)))
    Ag = dev(gpu, A0)
    tau = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert gpu.DecomposeQR(Ag, tau, None, 0)[1] is None
    Ah, th = host(Ag), tau.cpu().numpy().copy()
    p = 21
    C0 = colmajor(rng.uniform(-1, 1, (p, m) if flags & RIGHT else (m, p)))
    Cg = dev(gpu, C0)
    assert gpu.MultQ(Cg, Ag, tau, None, flags, 0) is None
    Cr = C0.copy(order="F")
    assert ref.MultQ(Cr, Ah, th, None, flags, 0) == 0
    assert fro(host(Cg) - Cr) <= 16 * m * EPS * fro(C0)
    # SolveQR least squares on the same factorization
    B0 = colmajor(A0 @ rng.uniform(-1, 1, (n, 3)) + 1e-3 * rng.uniform(-1, 1, (m, 3)))
    Bg = dev(gpu, B0)
    assert gpu.SolveQR(Bg, Ag, tau, None, 0, 0) is None
    Br = B0.copy(order="F")
    assert ref.SolveQR(Br, Ah, th, None, 0, 0) == 0
    assert fro(host(Bg) - Br) <= 64 * m * EPS * np.linalg.cond(A0) * max(fro(Br), 1.0)


@pytest.mark.parametrize("flags", [LEFT | TRANS, RIGHT])
def test_mult_q_and_solve_qr(gpu, ref, lapack, rng, flags):
    import torch
    m, n, p = 400, 250, 20
    A0 = colmajor(rng.uniform(-1, 1, (m, n)))
    Ag = dev(gpu, A0)
    tau = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert gpu.DecomposeQR(Ag, tau, None, 0)[1] is None
    Ah, th = host(Ag), tau.cpu().numpy().copy()
    C0 = colmajor(rng.uniform(-1, 1, (p, m) if flags & RIGHT else (m, p)))
    Cg = dev(gpu, C0)
    assert gpu.MultQ(Cg, Ag, tau, gpu.matrix(max(m, p), 32), flags, 32) is None
    # unblocked reference MultQ (no GEMV with beta != 1 on this path)
    Cr = C0.copy(order="F")
    Tr = np.zeros((n, n), order="F")
    assert lapack.BuildT(Tr, Ah, th) == 0
    assert lapack.MultQT(Cr, Ah, Tr, np.zeros((max(m, p), n), order="F"), flags, 0) == 0
    assert fro(host(Cg) - Cr) <= 16 * m * EPS * fro(C0)
    B0 = colmajor(A0 @ rng.uniform(-1, 1, (n, p)))
    Bg = dev(gpu, B0)
    assert gpu.SolveQR(Bg, Ag, tau, None, 0, 0) is None
    X = host(Bg)[:n]
    assert fro(A0 @ X - B0) <= 64 * m * EPS * np.linalg.cond(A0) * fro(B0)


def test_errors(gpu, rng):
    import torch
    A = dev(gpu, colmajor(rng.uniform(-1, 1, (50, 40))))
    T = dev(gpu, np.zeros((40, 40)))
    small = gpu.matrix(39, 8)
    # blocked call (nb < cols) with a workspace below A.cols x nb
    _, err = gpu.DecomposeQRT(A, T, small, 16)
    assert err is not None and err.code == -13 and str(err) == "work space too small"
    _, err = gpu.DecomposeQRT(A, dev(gpu, np.zeros((39, 39))), None, 0)
    assert err is not None and err.code == -16
    assert gpu.DecomposeQRT(A, T, None, 0)[1] is None
    C = dev(gpu, colmajor(rng.uniform(-1, 1, (50, 5))))
    err = gpu.MultQT(C, A, T, None, LEFT, 0)
    assert err is not None and err.code == -14 and str(err) == "workspace not defined"
    err = gpu.MultQT(C, A, T, gpu.matrix(5, 10), LEFT, 0)  # nb = T.cols = 40 > 10
    assert err is not None and err.code == -13 and str(err) == "work space too small"
    Cr = dev(gpu, colmajor(rng.uniform(-1, 1, (5, 49))))
    err = gpu.MultQT(Cr, A, T, gpu.matrix(5, 40), RIGHT, 0)
    assert err is not None and err.code == -15 and str(err) == "C*Q: C.Cols != A.Rows"
    torch.cuda.synchronize()


@pytest.mark.parametrize("n", [8192])
def test_decompose_qrt_large_properties(gpu, rng, n):
    """full-size factorization: A = Q R and Q^T Q = I through MultQT (no host QR)"""
    import torch
    g = torch.Generator(device="cuda").manual_seed(6)
    A0 = gpu.matrix(n, n)
    A0.copy_(torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64))
    A = gpu.matrix(n, n)
    A.copy_(A0)
    T = gpu.matrix(n, n)
    T.zero_()
    assert gpu.DecomposeQRT(A, T, None, 0)[1] is None
    # Q R - A
    R = gpu.matrix(n, n)
    R.copy_(torch.triu(A))
    W = gpu.matrix(n, n)
    assert gpu.MultQT(R, A, T, W, LEFT, 0) is None
    rel = (torch.linalg.norm(R - A0) / torch.linalg.norm(A0)).item()
    assert rel <= 8 * n * EPS, rel
    # Q^T (Q E) = E for a block of unit columns
    E = gpu.matrix(n, 64)
    E.zero_()
    E[:64, :64] = torch.eye(64, dtype=torch.float64, device="cuda")
    E0 = E.clone()
    assert gpu.MultQT(E, A, T, W, LEFT, 0) is None
    assert gpu.MultQT(E, A, T, W, LEFT | TRANS, 0) is None
    assert (torch.linalg.norm(E - E0) / 8.0).item() <= 8 * n * EPS


@pytest.mark.parametrize("m,n,nb", [(60, 40, 0), (60, 40, 12), (500, 300, 32), (1024, 1024, 0)])
def test_build_q(gpu, ref, lapack, rng, m, n, nb):
    import torch
    A0 = colmajor(rng.uniform(-1, 1, (m, n)))
    o = oracle_for(m, ref, lapack) if nb else ref  # the unblocked BuildQ uses no beta != 1 GEMV
    # BuildQ from DecomposeQR's reflectors (the same device reflectors for both)
    Ag = dev(gpu, A0)
    tau = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert gpu.DecomposeQR(Ag, tau, None, 0)[1] is None
    Ah, th = host(Ag), tau.cpu().numpy().copy()
    _, err = gpu.BuildQ(Ag, tau, gpu.matrix(n, max(nb, 1)), nb)
    assert err is None
    Qr = Ah.copy(order="F")
    assert o.BuildQ(Qr, th, np.zeros((n, max(nb, 1)), order="F"), nb) == 0
    Qh = host(Ag)
    assert fro(Qh - Qr) <= 32 * m * EPS * np.sqrt(n)
    assert fro(Qh.T @ Qh - np.eye(n)) <= 32 * m * EPS * np.sqrt(n)
    assert fro(Qh @ np.triu(Ah[:n]) - A0) <= 32 * m * EPS * fro(A0)
    # BuildQT from DecomposeQRT
    Ag2, Tg = dev(gpu, A0), dev(gpu, np.zeros((n, n)))
    assert gpu.DecomposeQRT(Ag2, Tg, None, 0)[1] is None
    R2 = np.triu(host(Ag2)[:n])
    _, err = gpu.BuildQT(Ag2, Tg, gpu.matrix(n, n), nb)
    assert err is None
    Q2 = host(Ag2)
    assert fro(Q2 @ R2 - A0) <= 32 * m * EPS * fro(A0)
    _, err = gpu.BuildQ(dev(gpu, colmajor(np.ones((3, 5)))), tau[:5], None, 0)
    assert err is not None and err.code == -5
