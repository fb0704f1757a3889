"""GPU parity: MultSym / MultTrm / RankUpdate2Sym / UpdateTrm against the oracle.

The oracle is the reference's own calgo kernels (oracle/_ref) under the restated Go
wrappers when they were built, else the oracle port.  Inputs where the reference itself is
wrong (recorded, not reproduced) are checked against numpy instead: SYMM's blocked paths
for orders above its block size 68 with the right side or no side bit, and MultSym's
MO_TRANSB with the right side (the kernel reads B out of shape).
"""
import numpy as np
import pytest

from util import EPS, colmajor, even_ld, fro

pytestmark = pytest.mark.gpu

TA, TB, LO, UP, LEFT, RIGHT, UNIT = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import Oracle, ref_available
    return Oracle("ref" if ref_available() else "port")


def dev(gpu, a):
    import torch
    ld = a.strides[1] // 8 if a.shape[1] > 1 else max(a.shape[0], 1)
    t = gpu.matrix(ld, a.shape[1])
    t.copy_(torch.from_numpy(np.asfortranarray(np.pad(a, ((0, ld - a.shape[0]), (0, 0))))))
    return t[: a.shape[0]]


def sym(S, flags):
    T = np.triu(S) if flags & UP else np.tril(S)
    return T + T.T - np.diag(np.diag(S))


@pytest.mark.parametrize("n,p", [(1, 1), (37, 5), (68, 70), (200, 33), (700, 129)])
@pytest.mark.parametrize("flags", [LEFT | LO, LEFT | UP, LEFT | LO | TA, RIGHT | LO, RIGHT | UP, LO])
def test_mult_sym(gpu, ref, rng, n, p, flags):
    left = not flags & RIGHT
    if not left:
        p = n  # the reference's size check admits the right side only for square C
    A = colmajor(rng.uniform(-1, 1, (n, n)), ld=even_ld(n) + 2)
    B = colmajor(rng.uniform(-1, 1, (n, p) if left else (p, n)), ld=even_ld(n if left else p))
    C0 = colmajor(rng.uniform(-1, 1, (n, p) if left else (p, n)))
    Cg = dev(gpu, C0)
    assert gpu.MultSym(Cg, dev(gpu, A), dev(gpu, B), 1.5, -0.5, flags) is None
    S = sym(A, flags)
    if flags & LEFT or (flags & RIGHT and n <= 68):
        Cr = C0.copy(order="F")
        assert ref.MultSym(Cr, A, B, 1.5, -0.5, flags) == 0
    else:
        # the reference's right-side blocked path above its block size and its no-side-bit
        # mixture of the two branches are wrong (recorded in DESIGN): the documented product
        Cr = -0.5 * C0 + 1.5 * ((S @ B) if left else (B @ S))
    err = fro(Cg.cpu().numpy() - Cr)
    assert err <= 4 * n * EPS * (1.5 * fro(S) * fro(B) + 0.5 * fro(C0)) + 1e-300, err


def test_mult_sym_transb_and_errors(gpu, rng):
    n, p = 300, 40
    A = colmajor(rng.uniform(-1, 1, (n, n)))
    B = colmajor(rng.uniform(-1, 1, (p, n)))
    C0 = colmajor(rng.uniform(-1, 1, (p, n)))
    Cg = dev(gpu, C0)
    # right side, op(B) = B^T needs B n x p: the shapes here pass the reference's check
    # only when square; use a square case for the documented meaning
    Bs = colmajor(rng.uniform(-1, 1, (n, n)))
    Cs0 = colmajor(rng.uniform(-1, 1, (n, n)))
    Cs = dev(gpu, Cs0)
    assert gpu.MultSym(Cs, dev(gpu, A), dev(gpu, Bs), 1.0, 1.0, RIGHT | LO | TB) is None
    ref = Cs0 + Bs.T @ sym(A, LO)
    assert fro(Cs.cpu().numpy() - ref) <= 1e-12 * fro(ref)
    err = gpu.MultSym(Cg, dev(gpu, A), dev(gpu, B), 1.0, 1.0, LEFT | LO)
    assert str(err) == "MultSym: size mismatch"


@pytest.mark.parametrize("n,p", [(1, 3), (45, 7), (130, 64), (700, 300)])
@pytest.mark.parametrize("flags", [LEFT | LO, LEFT | UP, LEFT | LO | TA, LEFT | UP | TA | UNIT,
                                   RIGHT | LO, RIGHT | UP, RIGHT | LO | TA | UNIT, RIGHT | UP | TA,
                                   LO | UNIT])
def test_mult_trm(gpu, ref, rng, n, p, flags):
    A = colmajor(rng.uniform(-1, 1, (n, n)), ld=even_ld(n))
    right = bool(flags & RIGHT)
    B0 = colmajor(rng.uniform(-1, 1, (p, n) if right else (n, p)), ld=even_ld(p if right else n) + 2)
    Bg = dev(gpu, B0)
    assert gpu.MultTrm(Bg, dev(gpu, A), 0.75, flags) is None
    Br = B0.copy(order="F")
    assert ref.MultTrm(Br, A, 0.75, flags) == 0
    T = np.triu(A) if flags & UP else np.tril(A)
    err = fro(Bg.cpu().numpy() - Br)
    assert err <= 4 * n * EPS * 0.75 * fro(T) * fro(B0) + 1e-300, err


@pytest.mark.parametrize("n,k", [(1, 1), (70, 5), (200, 64), (513, 130)])
@pytest.mark.parametrize("flags", [LO, UP, LO | TA, UP | TA])
@pytest.mark.parametrize("beta", [1.0, 0.5, 0.0])
def test_rank_update2_sym(gpu, ref, rng, n, k, flags, beta):
    A = colmajor(rng.standard_normal((k, n) if flags & TA else (n, k)))
    B = colmajor(rng.standard_normal(A.shape))  # same leading dimension as A (see DESIGN)
    C0 = colmajor(rng.standard_normal((n, n)))
    Cg = dev(gpu, C0)
    assert gpu.RankUpdate2Sym(Cg, dev(gpu, A), dev(gpu, B), 1.5, beta, flags) is None
    Cr = C0.copy(order="F")
    assert ref.RankUpdate2Sym(Cr, A, B, 1.5, beta, flags) == 0
    out = Cg.cpu().numpy()
    err = fro(out - Cr)
    assert err <= 8 * k * EPS * (3 * fro(A) * fro(B) + fro(C0)) + 1e-300, err
    tri = np.tril(np.ones((n, n), bool)) if flags & LO else np.triu(np.ones((n, n), bool))
    assert np.array_equal(out[~tri], C0[~tri])


@pytest.mark.parametrize("n,k", [(1, 1), (70, 5), (200, 64), (513, 130)])
@pytest.mark.parametrize("flags", [LO, UP, LO | TA, UP | TB, LO | TA | TB])
@pytest.mark.parametrize("beta", [1.0, 0.5])
def test_update_trm(gpu, ref, rng, n, k, flags, beta):
    A = colmajor(rng.standard_normal((k, n) if flags & TA else (n, k)))
    B = colmajor(rng.standard_normal((n, k) if flags & TB else (k, n)))
    C0 = colmajor(rng.standard_normal((n, n)))
    Cg = dev(gpu, C0)
    assert gpu.UpdateTrm(Cg, dev(gpu, A), dev(gpu, B), 1.5, beta, flags) is None
    Cr = C0.copy(order="F")
    assert ref.UpdateTrm(Cr, A, B, 1.5, beta, flags) == 0
    out = Cg.cpu().numpy()
    assert fro(out - Cr) <= 4 * k * EPS * (1.5 * fro(A) * fro(B) + fro(C0)) + 1e-300
    tri = np.tril(np.ones((n, n), bool)) if flags & LO else np.triu(np.ones((n, n), bool))
    assert np.array_equal(out[~tri], C0[~tri])


def test_blas_beta_switch(gpu, rng):
    from matops_b200 import _lib
    n, k = 150, 9
    A = colmajor(rng.standard_normal((n, k)))
    B = colmajor(rng.standard_normal((n, k)))
    C0 = colmajor(rng.standard_normal((n, n)))
    ctx = gpu.context()
    old = _lib.lib().mo_set_syrk_blas_beta(ctx, 1)
    try:
        Cg = dev(gpu, C0)
        assert gpu.RankUpdate2Sym(Cg, dev(gpu, A), dev(gpu, B), 1.0, 0.5, LO) is None
        Cu = dev(gpu, C0)
        assert gpu.UpdateTrm(Cu, dev(gpu, A), dev(gpu, B.T.copy(order="F")), 1.0, 0.5, UP) is None
    finally:
        _lib.lib().mo_set_syrk_blas_beta(ctx, old)
    full = 0.5 * C0 + A @ B.T + B @ A.T
    lo = np.tril(np.ones((n, n), bool))
    assert fro((Cg.cpu().numpy() - full)[lo]) <= 1e-12 * fro(full)
    fu = 0.5 * C0 + A @ B.T
    up = np.triu(np.ones((n, n), bool))
    assert fro((Cu.cpu().numpy() - fu)[up]) <= 1e-12 * fro(fu)


@pytest.mark.parametrize("n", [1, 31, 128, 129, 300, 700, 1500])
@pytest.mark.parametrize("flags", [LO, UP, LO | UNIT, UP | UNIT])
def test_inverse_trm(gpu, ref, rng, n, flags):
    T = rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n) + np.diag(rng.uniform(1.0, 2.0, n))
    A = colmajor(T, ld=even_ld(n) + 2)
    Ag = dev(gpu, A)
    _, err = gpu.InverseTrm(Ag, flags, 64)
    assert err is None
    out = Ag.cpu().numpy()
    Ar = A.copy(order="F")
    assert ref.InverseTrm(Ar, flags, 64) == 0
    tri = np.tril(np.ones((n, n), bool)) if flags & LO else np.triu(np.ones((n, n), bool))
    if flags & UNIT:
        tri &= ~np.eye(n, dtype=bool)
    assert fro(out[tri] - Ar[tri]) <= 1e-12 * max(fro(Ar[tri]), 1.0)
    # the other triangle (and a unit diagonal) is not written
    assert np.array_equal(out[~tri], A[~tri])
