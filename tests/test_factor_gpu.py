"""GPU parity: DecomposeCHOL / SolveCHOL / DecomposeLU / SolveLU against the oracle."""
import numpy as np
import pytest
import torch

from util import EPS, colmajor, even_ld, fro, spd

pytestmark = pytest.mark.gpu

LO, UP, TA = 0x4, 0x8, 0x1


def dev(gpu, a):
    return gpu.to_device(np.ascontiguousarray(a))


@pytest.mark.parametrize("flags", [LO, UP])
@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 127, 128, 129, 300, 700])
def test_decompose_chol(gpu, oracle, rng, flags, n):
    A = colmajor(spd(rng, n))
    Ag = dev(gpu, A)
    _, err = gpu.DecomposeCHOL(Ag, flags, 64)
    assert err is None
    out = Ag.cpu().numpy()
    L = np.tril(out) if flags == LO else np.triu(out).T
    assert fro(A - L @ L.T) / fro(A) <= 10 * n * EPS
    Ar = A.copy(order="F")
    assert oracle.DecomposeCHOL(Ar, flags, 64) == 0
    Lr = np.tril(Ar) if flags == LO else np.triu(Ar).T
    assert fro(L - Lr) / fro(Lr) <= 1e-12
    # the opposite strict triangle is not referenced
    other = np.triu(np.ones((n, n), bool), 1) if flags == LO else np.tril(np.ones((n, n), bool), -1)
    assert np.array_equal(out[other], A[other])


def test_decompose_chol_not_spd_panics(gpu, oracle, rng):
    n = 200
    A = spd(rng, n)
    A[150, 150] = -5.0
    A = colmajor(A)
    Ar = A.copy(order="F")
    info = oracle.DecomposeCHOL(Ar, LO, 64)
    assert info == 151
    with pytest.raises(gpu.MatopsPanic, match="illegal value at 150"):
        gpu.DecomposeCHOL(dev(gpu, A), LO, 64)


def test_decompose_chol_not_square(gpu):
    _, err = gpu.DecomposeCHOL(gpu.matrix(3, 4), LO, 0)
    assert str(err) == "A not a square matrix"


@pytest.mark.parametrize("flags", [LO, UP])
@pytest.mark.parametrize("n,nrhs", [(300, 64), (129, 1), (1000, 16)])
def test_solve_chol(gpu, oracle, rng, flags, n, nrhs):
    A = colmajor(spd(rng, n))
    B = colmajor(rng.uniform(-1, 1, (n, nrhs)))
    Ag, Bg = dev(gpu, A), dev(gpu, B)
    gpu.DecomposeCHOL(Ag, flags, 64)
    gpu.SolveCHOL(Bg, Ag, flags)
    X = Bg.cpu().numpy()
    berr = fro(B - A @ X) / (fro(A) * fro(X) + fro(B))
    assert berr <= 10 * n * EPS
    Ar, Br = A.copy(order="F"), B.copy(order="F")
    oracle.DecomposeCHOL(Ar, flags, 64)
    oracle.SolveCHOL(Br, Ar, flags)
    assert fro(X - Br) / fro(Br) <= 1e-10


@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (63, 63), (64, 64), (65, 65), (300, 300),
                                 (700, 700), (257, 100), (100, 257), (1030, 1030)])
@pytest.mark.parametrize("nb", [0, 64])
def test_decompose_lu(gpu, oracle, rng, m, n, nb):
    A = colmajor(rng.standard_normal((m, n)), ld=even_ld(m))
    mn = min(m, n)
    Ag = dev(gpu, A)
    piv = torch.zeros(mn, dtype=torch.int64, device="cuda")
    _, err = gpu.DecomposeLU(Ag, piv, nb)
    assert err is None
    out = Ag.cpu().numpy()
    p = piv.cpu().numpy()
    if m < n and 0 < nb < mn and m % nb != 0:
        # the reference's last diagonal block (repartition2x2to3x3 clips by columns only,
        # partition.go:252-254) runs past the last row and aliases the next column's
        # storage; compare with LAPACK's factorization instead
        import scipy.linalg as sl
        Ar, pr = sl.lu_factor(A)
    else:
        Ar = colmajor(A, ld=even_ld(m))
        pr = np.zeros(mn, np.int64)
        assert oracle.DecomposeLU(Ar, pr, nb) == 0
    assert np.array_equal(p, pr)
    L = np.tril(out[:, :mn], -1) + np.eye(m, mn)
    U = np.triu(out[:mn, :])
    PA = A.copy()
    for k in range(mn):
        PA[[k, p[k]]] = PA[[p[k], k]]
    assert fro(PA - L @ U) / fro(A) <= 10 * max(m, n) * EPS
    assert fro(out - Ar) / fro(Ar) <= 1e-11


def test_decompose_lu_short_pivots(gpu):
    _, err = gpu.DecomposeLU(gpu.matrix(5, 5), torch.zeros(4, dtype=torch.int64, device="cuda"), 0)
    assert str(err) == "pivot array < min(A.Rows(),A.Cols())"


@pytest.mark.parametrize("flags", [0, TA])
@pytest.mark.parametrize("n,nrhs", [(300, 64), (129, 1), (1000, 16)])
def test_solve_lu(gpu, oracle, rng, flags, n, nrhs):
    A = colmajor(rng.standard_normal((n, n)), ld=even_ld(n))
    B = colmajor(rng.uniform(-1, 1, (n, nrhs)))
    Ag, Bg = dev(gpu, A), dev(gpu, B)
    piv = torch.zeros(n, dtype=torch.int64, device="cuda")
    gpu.DecomposeLU(Ag, piv, 64)
    assert gpu.SolveLU(Bg, Ag, piv, flags) is None
    X = Bg.cpu().numpy()
    Ar, Br = A.copy(order="F"), B.copy(order="F")
    pr = np.zeros(n, np.int64)
    oracle.DecomposeLU(Ar, pr, 64)
    assert oracle.SolveLU(Br, Ar, pr, flags) == 0
    assert fro(X - Br) / fro(Br) <= 1e-9
    if flags == 0:
        assert fro(B - A @ X) / (fro(A) * fro(X) + fro(B)) <= 10 * n * EPS


@pytest.mark.parametrize("nrhs", [17, 48, 64])
def test_solve_chol_grouped_columns(gpu, oracle, rng, nrhs):
    # more than 16 right-hand sides: the few-column solve runs column groups side by side
    n = 1100
    A = colmajor(spd(rng, n))
    B = colmajor(rng.uniform(-1, 1, (n, nrhs)))
    Ag, Bg = dev(gpu, A), dev(gpu, B)
    gpu.DecomposeCHOL(Ag, LO, 64)
    gpu.SolveCHOL(Bg, Ag, LO)
    Ar, Br = A.copy(order="F"), B.copy(order="F")
    oracle.DecomposeCHOL(Ar, LO, 64)
    oracle.SolveCHOL(Br, Ar, LO)
    assert fro(Bg.cpu().numpy() - Br) / fro(Br) <= 1e-10
