"""GPU parity: Mult / RankUpdateSym / SolveTrm against the oracle on the same inputs."""
import os

import numpy as np
import pytest

from util import EPS, colmajor, even_ld, fro, gemm_bound

pytestmark = pytest.mark.gpu

TA, TB, LO, UP, LEFT, RIGHT, UNIT = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40


def dev(gpu, a):
    """device copy with the same leading dimension as the host view"""
    import torch
    ld = a.strides[1] // 8 if a.shape[1] > 1 else max(a.shape[0], 1)
    t = gpu.matrix(ld, a.shape[1])
    t.copy_(torch.from_numpy(np.asfortranarray(np.pad(a, ((0, ld - a.shape[0]), (0, 0))))))
    return t[: a.shape[0]]


def host(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("flags", [0, TA, TB, TA | TB])
@pytest.mark.parametrize("m,n,k", [(2048, 2048, 2048), (137, 91, 213), (1, 1, 1), (128, 128, 16),
                                   (129, 257, 65), (300, 5, 1000), (7, 300, 3),
                                   # few-wave shapes: K split over CTAs (stream-K partial sums)
                                   (1536, 1536, 256), (1280, 1408, 400), (1000, 700, 1333),
                                   # a few tiles with a long K: fewer CTAs of 4 slabs each
                                   (128, 128, 4096), (100, 250, 3000), (128, 384, 1100),
                                   # narrow C (N <= 64, M >= 2048): 256 x 64 tiles
                                   (2048, 64, 512), (2500, 33, 700), (4099, 1, 129), (3000, 64, 16)])
def test_mult(gpu, oracle, rng, flags, m, n, k):
    A = colmajor(rng.uniform(-1, 1, (k, m) if flags & TA else (m, k)))
    B = colmajor(rng.uniform(-1, 1, (n, k) if flags & TB else (k, n)))
    C0 = colmajor(rng.uniform(-1, 1, (m, n)))
    alpha, beta = 1.5, -0.5
    Cg = dev(gpu, C0)
    assert gpu.Mult(Cg, dev(gpu, A), dev(gpu, B), alpha, beta, flags) is None
    Cr = C0.copy(order="F")
    if m * n * k > 2e8:
        # the configured DGEMM (2048^3, alpha 1.5, beta -0.5): compared with the reference's
        # own calgo kernels (oracle/_ref) with NumWorkers = host cores when they were built,
        # else with the oracle port on all cores
        from oracle.oracle import Oracle, ref_available
        big = Oracle("ref" if ref_available() else "port")
        old = big.NumWorkers(os.cpu_count() or 1)
        try:
            assert big.Mult(Cr, A, B, alpha, beta, flags) == 0
        finally:
            big.NumWorkers(old)
    else:
        assert oracle.Mult(Cr, A, B, alpha, beta, flags) == 0
    err = fro(host(Cg) - Cr)
    assert err <= gemm_bound(k, alpha, beta, A, B, C0), err


@pytest.mark.parametrize("flags", [0, TA, TB])
def test_mult_narrow_unaligned_views(gpu, oracle, rng, flags):
    """Narrow C (256 x 64 tiles) on views at odd offsets and odd leading dimensions: the
    cp.async producer fills the 256-row A slab and the 64-row B slab."""
    m, n, k = 2305, 47, 333
    Abig = colmajor(rng.uniform(-1, 1, (k + 3, m + 2) if flags & TA else (m + 3, k + 2)), ld=None)
    Bbig = colmajor(rng.uniform(-1, 1, (n + 3, k + 2) if flags & TB else (k + 3, n + 2)))
    Cbig = colmajor(rng.uniform(-1, 1, (m + 3, n + 2)))
    Ag, Bg, Cg = dev(gpu, Abig), dev(gpu, Bbig), dev(gpu, Cbig)
    sa = (slice(1, 1 + k), slice(1, 1 + m)) if flags & TA else (slice(1, 1 + m), slice(1, 1 + k))
    sb = (slice(1, 1 + n), slice(1, 1 + k)) if flags & TB else (slice(1, 1 + k), slice(1, 1 + n))
    sc = (slice(1, 1 + m), slice(1, 1 + n))
    A, B, C0 = Abig[sa], Bbig[sb], Cbig[sc].copy()
    assert gpu.Mult(Cg[sc], Ag[sa], Bg[sb], 0.75, 1.25, flags) is None
    opA = A.T if flags & TA else A
    opB = B.T if flags & TB else B
    Cr = 1.25 * C0 + 0.75 * (opA @ opB)
    out = host(Cg)
    assert fro(out[sc] - Cr) <= gemm_bound(k, 0.75, 1.25, A, B, C0)
    keep = np.ones(out.shape, bool)
    keep[sc] = False
    assert np.array_equal(out[keep], Cbig[keep])


@pytest.mark.parametrize("off", [(0, 0), (1, 0), (0, 1), (1, 1), (3, 5)])
def test_mult_unaligned_views(gpu, oracle, rng, off):
    """Sub-views at odd offsets / odd leading dimensions take the cp.async producer."""
    r0, c0 = off
    big = [colmajor(rng.uniform(-1, 1, (301, 260)), ld=303) for _ in range(3)]
    m, n, k = 150, 130, 120
    A, B, C = big[0][r0:r0 + m, c0:c0 + k], big[1][r0:r0 + k, c0:c0 + n], big[2][r0:r0 + m, c0:c0 + n]
    import torch
    tg = [dev(gpu, b) for b in big]
    Ag, Bg, Cg = tg[0][r0:r0 + m, c0:c0 + k], tg[1][r0:r0 + k, c0:c0 + n], tg[2][r0:r0 + m, c0:c0 + n]
    C0 = C.copy()
    assert gpu.Mult(Cg, Ag, Bg, -1.0, 1.0, 0) is None
    Cr = np.asfortranarray(big[2]).copy(order="F")
    assert oracle.Mult(Cr[r0:r0 + m, c0:c0 + n], A, B, -1.0, 1.0, 0) == 0
    out = host(tg[2])
    assert fro(out - Cr) <= gemm_bound(k, 1, 1, A, B, C0)
    # nothing outside the view was touched
    mask = np.ones_like(out, dtype=bool)
    mask[r0:r0 + m, c0:c0 + n] = False
    assert np.array_equal(out[mask], big[2][mask])


def test_mult_beta_zero_ignores_nan(gpu, rng):
    A = colmajor(rng.uniform(-1, 1, (64, 32)))
    B = colmajor(rng.uniform(-1, 1, (32, 48)))
    C = colmajor(np.full((64, 48), np.nan))
    Cg = dev(gpu, C)
    assert gpu.Mult(Cg, dev(gpu, A), dev(gpu, B), 2.0, 0.0, 0) is None
    assert np.allclose(host(Cg), 2.0 * A @ B, rtol=1e-13, atol=1e-13)


def test_mult_k_zero_scales(gpu, rng):
    C = colmajor(rng.uniform(-1, 1, (33, 17)))
    Cg = dev(gpu, C)
    A = gpu.matrix(33, 0)
    B = gpu.matrix(0, 17)
    assert gpu.Mult(Cg, A, B, 1.0, 3.0, 0) is None
    assert np.allclose(host(Cg), 3.0 * C, rtol=0, atol=1e-15)


def test_mult_errors(gpu):
    C, A, B = gpu.matrix(4, 4), gpu.matrix(4, 3), gpu.matrix(2, 4)
    e = gpu.Mult(C, A, B, 1.0, 1.0, 0)
    assert e is not None and str(e) == "Mult: size mismatch"
    # empty operands are not an error (mmult.go:220-222)
    assert gpu.Mult(gpu.matrix(0, 4), gpu.matrix(0, 3), gpu.matrix(3, 4), 1.0, 1.0, 0) is None


@pytest.mark.parametrize("flags", [LO, UP | TA, UP, LO | TA])
@pytest.mark.parametrize("beta", [1.0, 0.0, 0.7])
@pytest.mark.parametrize("n,k", [(300, 37), (128, 128), (69, 200), (1, 5), (200, 1)])
def test_rank_update_sym(gpu, oracle, rng, flags, beta, n, k):
    A = colmajor(rng.standard_normal((k, n) if flags & TA else (n, k)))
    C0 = colmajor(rng.standard_normal((n, n)))
    Cg = dev(gpu, C0)
    assert gpu.RankUpdateSym(Cg, dev(gpu, A), -1.0, beta, flags) is None
    Cr = C0.copy(order="F")
    assert oracle.RankUpdateSym(Cr, A, -1.0, beta, flags) == 0
    out = host(Cg)
    tri = np.tril(np.ones((n, n), bool)) if flags & LO else np.triu(np.ones((n, n), bool))
    assert fro((out - Cr)[tri]) <= gemm_bound(k, 1.0, abs(beta), A, A, C0)
    # the other strict triangle is untouched
    assert np.array_equal(out[~tri], C0[~tri])


def test_rank_update_sym_errors(gpu):
    e = gpu.RankUpdateSym(gpu.matrix(4, 5), gpu.matrix(4, 2), 1.0, 1.0, LO)
    assert e is not None and str(e) == "C not a square matrix"
    gpu.SetPanicOnError(True)
    try:
        with pytest.raises(gpu.MatopsPanic):
            gpu.RankUpdateSym(gpu.matrix(4, 5), gpu.matrix(4, 2), 1.0, 1.0, LO)
    finally:
        gpu.SetPanicOnError(False)


def tri_matrix(rng, n, upper, unit):
    a = rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(max(n, 1))
    a += np.diag(rng.uniform(1.0, 2.0, n) * np.sign(rng.uniform(-1, 1, n)))
    return colmajor(a)


@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("trans", [0, TA])
@pytest.mark.parametrize("unit", [0, UNIT])
@pytest.mark.parametrize("n,nrhs", [(300, 37), (128, 64), (1, 3), (257, 1)])
def test_solve_trm(gpu, oracle, rng, side, uplo, trans, unit, n, nrhs):
    flags = side | uplo | trans | unit
    A = tri_matrix(rng, n, uplo == UP, unit)
    B0 = colmajor(rng.standard_normal((nrhs, n) if side == RIGHT else (n, nrhs)))
    Bg = dev(gpu, B0)
    assert gpu.SolveTrm(Bg, dev(gpu, A), 1.7, flags) is None
    Br = B0.copy(order="F")
    assert oracle.SolveTrm(Br, A, 1.7, flags) == 0
    err = fro(host(Bg) - Br) / max(fro(Br), 1e-300)
    assert err <= 100 * n * EPS, err
