"""GPU: mixed-precision Cholesky solve with FP64 refinement (mo_dsposv_ir) and the
split-product GEMM it is built on (mo_lp_gemm).

The reference has no mixed-precision path; the oracle for the solution is the FP64
solution of the same system (the C oracle's DecomposeCHOL + SolveCHOL), and every case
states its normwise backward error ||b - A x|| / (||A|| ||x|| + ||b||).  Test matrices
follow the mixed-precision benchmark's construction at smaller orders: A = Q diag(s) Q^T
with Q from the Householder QR of an iid N(0,1) matrix and s log-spaced from 1 to kappa.
"""
import numpy as np
import pytest
import torch

from util import EPS, colmajor, fro, spd

pytestmark = pytest.mark.gpu

LO, UP, TA, TB = 0x4, 0x8, 0x1, 0x2
BF16X3, TF32X3 = 1, 2
AUTO, CLASSIC, GMRES, NO_FALLBACK = 0, 1, 2, 0x100


def kappa_matrix(rng, n, kappa):
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    q *= np.sign(np.diag(r))
    s = np.logspace(0, np.log10(kappa), n)
    a = (q * s) @ q.T
    return (a + a.T) / 2


def berr_inf(A, X, B):
    """max over columns of |b - A x|_inf / (|A|_inf |x|_inf + |b|_inf), as mo_ir_info.berr"""
    R = B - A @ X
    an = np.abs(A).sum(axis=1).max()
    return max(np.abs(R[:, c]).max() / (an * np.abs(X[:, c]).max() + np.abs(B[:, c]).max())
               for c in range(B.shape[1]))


def fp64_solution(oracle, A, B):
    Ar, Br = colmajor(A), colmajor(B)
    assert oracle.DecomposeCHOL(Ar, LO, 64) == 0
    oracle.SolveCHOL(Br, Ar, LO)
    return Br


@pytest.mark.parametrize("prec", [TF32X3, BF16X3])
@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_mixed_solve_kappa(gpu, oracle, rng, prec, kappa):
    n, nrhs = 640, 16
    A = kappa_matrix(rng, n, kappa)
    B = rng.standard_normal((n, nrhs))
    Ag, Bg, Xg = gpu.to_device(A), gpu.to_device(B), gpu.matrix(n, nrhs)
    info, err = gpu.SolveCHOLMixed(Xg, Ag, Bg, LO, prec, AUTO, 1e-14, 40)
    assert err is None
    X = Xg.cpu().numpy()
    assert info.converged, info
    if info.abandoned:
        # MO_IR_AUTO judged that GMRES-IR would cost more than the FP64 path: a classic step
        # reduced berr less than 3x, or the projected GMRES steps exceed the FP64 cost (at
        # this small order the factor is cheap next to the latency of the inner iterations)
        assert info.fallback, info
    elif prec == BF16X3 and kappa > 1e9:
        # BF16x3 keeps about 16 bits (u ~ 1.5e-5): its factor breaks down, and MO_IR_AUTO
        # redoes it with the TF32x3 split
        assert info.prec == TF32X3, info
    else:
        assert not info.fallback, info
    assert info.berr <= 1e-14
    assert berr_inf(A, X, B) <= 1.5e-14
    # forward error against the FP64 factorization's solution: both are within about
    # kappa * u of the exact solution
    Xr = fp64_solution(oracle, A, B)
    assert fro(X - Xr) / fro(Xr) <= max(1e-12, 200 * kappa * EPS)
    # A is only read
    assert np.array_equal(Ag.cpu().numpy(), A)


def test_gmres_ir_converges_at_kappa_1e10(gpu, oracle, rng):
    """GMRES-IR preconditioned by the TF32x3 factor (shifted where FP32 rounding makes A
    numerically indefinite) reaches berr <= 1e-14 at kappa = 1e10 without the FP64 path."""
    n, nrhs = 640, 16
    A = kappa_matrix(rng, n, 1e10)
    B = rng.standard_normal((n, nrhs))
    Xg = gpu.matrix(n, nrhs)
    info, err = gpu.SolveCHOLMixed(Xg, gpu.to_device(A), gpu.to_device(B), LO, TF32X3,
                                   GMRES | NO_FALLBACK, 1e-14, 40)
    assert err is None and info.converged and not info.fallback, info
    assert info.method == GMRES and info.gmres_iters > 0
    X = Xg.cpu().numpy()
    assert berr_inf(A, X, B) <= 1.5e-14
    Xr = fp64_solution(oracle, A, B)
    assert fro(X - Xr) / fro(Xr) <= 200 * 1e10 * EPS


@pytest.mark.parametrize("method", [CLASSIC, GMRES])
def test_mixed_solve_methods(gpu, rng, method):
    n, nrhs = 500, 5
    A = spd(rng, n)
    B = rng.uniform(-1, 1, (n, nrhs))
    Xg = gpu.matrix(n, nrhs)
    info, err = gpu.SolveCHOLMixed(Xg, gpu.to_device(A), gpu.to_device(B), LO, TF32X3, method,
                                   1e-14, 30)
    assert err is None and info.converged and not info.fallback, info
    assert info.method == method
    if method == GMRES:
        assert info.gmres_iters >= info.iters >= 1
    assert berr_inf(A, Xg.cpu().numpy(), B) <= 1.5e-14


@pytest.mark.parametrize("n", [1, 7, 127, 128, 129, 300])
def test_mixed_solve_upper_reads_one_triangle(gpu, rng, n):
    A = spd(rng, n)
    B = rng.standard_normal((n, 3))
    Afill = A.copy()
    Afill[np.tril_indices(n, -1)] = 1e30  # the strict lower triangle must not be read
    Ag = gpu.to_device(Afill)
    Bg = gpu.to_device(B)
    info, err = gpu.SolveCHOLMixed(Bg, Ag, Bg, UP, BF16X3)  # X may be B
    assert err is None and info.converged, info
    assert berr_inf(A, Bg.cpu().numpy(), B) <= 1.5e-14
    assert np.array_equal(Ag.cpu().numpy(), Afill)


def test_mixed_solve_views_with_leading_dimension(gpu, rng):
    n, nrhs = 257, 4
    A = spd(rng, n)
    B = rng.standard_normal((n, nrhs))
    big = gpu.matrix(n + 9, n + 3, fill=7.0)
    Av = big[5:5 + n, 2:2 + n]
    Av.copy_(torch.as_tensor(A))
    bigB = gpu.matrix(n + 4, nrhs + 2, fill=3.0)
    Bv = bigB[1:1 + n, 1:1 + nrhs]
    Bv.copy_(torch.as_tensor(B))
    bigX = gpu.matrix(n + 6, nrhs, fill=-1.0)
    Xv = bigX[3:3 + n, :]
    info, err = gpu.SolveCHOLMixed(Xv, Av, Bv, LO, TF32X3)
    assert err is None and info.converged, info
    assert berr_inf(A, Xv.cpu().numpy(), B) <= 1.5e-14
    out = bigX.cpu().numpy()
    assert np.all(out[:3] == -1.0) and np.all(out[3 + n:] == -1.0)


def test_mixed_solve_not_spd_falls_back_and_panics(gpu, rng):
    n = 300
    A = spd(rng, n)
    A[200, 200] = -50.0
    Xg = gpu.matrix(n, 2)
    with pytest.raises(gpu.MatopsPanic, match="illegal value at 200"):
        gpu.SolveCHOLMixed(Xg, gpu.to_device(A), gpu.to_device(rng.standard_normal((n, 2))),
                           LO, TF32X3)


def test_mixed_solve_no_fallback_reports_failure(gpu, rng):
    # kappa 1e10 with classic refinement from a BF16x3 factor (u ~ 2^-16) diverges or stalls;
    # without the FP64 fallback the call reports what it reached
    n = 400
    A = kappa_matrix(rng, n, 1e10)
    B = rng.standard_normal((n, 2))
    Xg = gpu.matrix(n, 2)
    info, err = gpu.SolveCHOLMixed(Xg, gpu.to_device(A), gpu.to_device(B), LO, BF16X3,
                                   CLASSIC | NO_FALLBACK, 1e-14, 3)
    assert not info.fallback
    if info.converged:
        assert err is None and info.berr <= 1e-14
    else:
        assert info.iters <= 3


def test_mixed_solve_fallback_when_refinement_cannot_converge(gpu, rng):
    n = 400
    A = kappa_matrix(rng, n, 1e10)
    B = rng.standard_normal((n, 2))
    Xg = gpu.matrix(n, 2)
    info, err = gpu.SolveCHOLMixed(Xg, gpu.to_device(A), gpu.to_device(B), LO, BF16X3,
                                   CLASSIC, 1e-14, 1)
    assert err is None
    if not info.converged or info.fallback:
        assert info.fallback
    X = Xg.cpu().numpy()
    assert berr_inf(A, X, B) <= 1e-13


def test_mixed_solve_argument_errors(gpu):
    A, B, X = gpu.matrix(4, 5), gpu.matrix(4, 2), gpu.matrix(4, 2)
    _, err = gpu.SolveCHOLMixed(X, A, B)
    assert str(err) == "A not a square matrix"
    A = gpu.matrix(4, 4, fill=0.0)
    A.diagonal().fill_(1.0)
    _, err = gpu.SolveCHOLMixed(gpu.matrix(4, 3), A, B)
    assert str(err) == "Mult: size mismatch"
    _, err = gpu.SolveCHOLMixed(X, A, B, LO, 7)
    assert err is not None and err.code == -10
    info, err = gpu.SolveCHOLMixed(gpu.matrix(4, 0), A, gpu.matrix(4, 0))
    assert err is None and info.converged


def _split_bound(prec, k, A, B):
    u = 2.0 ** -16 if prec == BF16X3 else 2.0 ** -21
    return 4 * (u + k * 2.0 ** -24) * np.abs(A) @ np.abs(B)


@pytest.mark.parametrize("prec", [TF32X3, BF16X3])
@pytest.mark.parametrize("flags", [0, TA, TB, TA | TB])
@pytest.mark.parametrize("m,n,k", [(128, 128, 32), (300, 200, 100), (1000, 520, 260)])
def test_lp_gemm(gpu, rng, prec, flags, m, n, k):
    A = rng.uniform(-1, 1, (k, m) if flags & TA else (m, k)).astype(np.float32)
    B = rng.uniform(-1, 1, (n, k) if flags & TB else (k, n)).astype(np.float32)
    C0 = rng.uniform(-1, 1, (m, n)).astype(np.float32)

    def f32(a):
        t = torch.empty((a.shape[1], a.shape[0]), dtype=torch.float32, device="cuda").t()
        t.copy_(torch.as_tensor(a))
        return t
    Cg = f32(C0)
    assert gpu.LPGemm(Cg, f32(A), f32(B), 1.25, -0.5, flags, prec) is None
    opA = A.T.astype(np.float64) if flags & TA else A.astype(np.float64)
    opB = B.T.astype(np.float64) if flags & TB else B.astype(np.float64)
    ref = 1.25 * opA @ opB - 0.5 * C0.astype(np.float64)
    got = Cg.cpu().numpy().astype(np.float64)
    bound = _split_bound(prec, k, opA, opB) * 1.25 + 2.0 ** -23 * (np.abs(ref) + 0.5 * np.abs(C0))
    assert np.all(np.abs(got - ref) <= bound + 1e-30)


def test_lp_gemm_lower_leaves_upper(gpu, rng):
    m = k = 256
    A = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    C0 = rng.uniform(-1, 1, (m, m)).astype(np.float32)
    At = torch.empty((k, m), dtype=torch.float32, device="cuda").t()
    At.copy_(torch.as_tensor(A))
    Cg = torch.empty((m, m), dtype=torch.float32, device="cuda").t()
    Cg.copy_(torch.as_tensor(C0))
    assert gpu.LPGemm(Cg, At, At, -1.0, 1.0, TB | LO, TF32X3) is None
    got = Cg.cpu().numpy()
    iu = np.triu_indices(m, 1)
    assert np.array_equal(got[iu], C0[iu])
    A64 = A.astype(np.float64)
    ref = C0.astype(np.float64) - A64 @ A64.T
    bound = _split_bound(TF32X3, k, A64, A64.T) + 2.0 ** -23 * (np.abs(ref) + np.abs(C0))
    il = np.tril_indices(m)
    assert np.all(np.abs(got[il] - ref[il]) <= bound[il])


@pytest.mark.parametrize("flags", [LO, UP])
@pytest.mark.parametrize("n,nrhs", [(700, 64), (385, 37)])
def test_mixed_solve_many_rhs(gpu, oracle, rng, flags, n, nrhs):
    # above 32 right-hand sides the residual runs through the FP64 GEMM engine on a
    # symmetric copy of A and the triangular solves split the columns into groups of 16
    A = kappa_matrix(rng, n, 1e4)
    B = rng.standard_normal((n, nrhs))
    Afill = A.copy()
    if flags == LO:
        Afill[np.triu_indices(n, 1)] = 1e30
    else:
        Afill[np.tril_indices(n, -1)] = 1e30
    Xg = gpu.matrix(n, nrhs)
    info, err = gpu.SolveCHOLMixed(Xg, gpu.to_device(Afill), gpu.to_device(B), flags, TF32X3)
    assert err is None and info.converged and not info.fallback, info
    X = Xg.cpu().numpy()
    assert berr_inf(A, X, B) <= 1.5e-14
    Xr = fp64_solution(oracle, A, B)
    assert fro(X - Xr) / fro(Xr) <= 1e-9


@pytest.mark.parametrize("flags", [LO, UP])
@pytest.mark.parametrize("n", [1, 100, 128, 300])
def test_upload_triangle_then_solve(gpu, rng, flags, n):
    """mo_upload_tri moves the stored triangle in 128-column blocks (each block's
    diagonal square whole) and leaves the rest of the device matrix as it was; the
    mixed solve on that upload meets the refinement tolerance."""
    A = spd(rng, n)
    B = rng.standard_normal((n, 2))
    host_big = gpu.host_matrix(n + 5, n)
    Ah = host_big[2:2 + n, :]
    Ah.copy_(torch.as_tensor(A))
    Ad = gpu.matrix(n, n, fill=7.0)
    gpu.UploadTriangle(Ad, Ah, flags)
    gpu.Sync()
    out = Ad.cpu().numpy()
    i, j = np.indices((n, n))
    blk0 = (j // 128) * 128
    copied = (i >= blk0) if flags == LO else (i < np.minimum(blk0 + 128, n))
    assert np.array_equal(out[copied], A[copied])
    assert np.all(out[~copied] == 7.0)
    stored = (i >= j) if flags == LO else (i <= j)
    assert np.all(copied[stored])
    Xd = gpu.matrix(n, 2)
    info, err = gpu.SolveCHOLMixed(Xd, Ad, gpu.to_device(B), flags, TF32X3)
    assert err is None and info.converged, info
    assert berr_inf(A, Xd.cpu().numpy(), B) <= 1.5e-14
