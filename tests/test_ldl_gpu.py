"""GPU parity: DecomposeLDLnoPiv / SolveLDLnoPiv, DecomposeLDL / SolveLDL, DecomposeBK /
SolveBK (ldlnp.go, ldl.go, ldlbk.go, ldlbks.go) against the oracle.

The oracle runs the restated Go sweeps over the reference's own calgo kernels (oracle/_ref)
when they were built, else over the port; the device runs the same unblocked sweeps, so
the pivot vectors must be identical and the factors agree to rounding.  SolveBK with UPPER
storage is checked by its residual and against the oracle's index-reversed solve (the
reference's own UPPER sweeps update empty and mismatched blocks of B).
"""
import numpy as np
import pytest

from util import EPS, colmajor, even_ld, fro

pytestmark = pytest.mark.gpu

LO, UP = 0x4, 0x8


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import Oracle, ref_available
    return Oracle("ref" if ref_available() else "port")


def dev(gpu, a):
    import torch
    a = np.asfortranarray(a) if (a.ndim != 2 or (a.shape[0] > 1 and a.strides[0] != 8)) else a
    ld = a.strides[1] // 8 if a.shape[1] > 1 else max(a.shape[0], 1)
    t = gpu.matrix(max(ld, 1), max(a.shape[1], 1))
    t.zero_()
    if a.size:
        t[: a.shape[0], : a.shape[1]].copy_(torch.from_numpy(np.asfortranarray(a)))
    return t[: a.shape[0], : a.shape[1]]


def sym(rng, n):
    g = rng.uniform(-1, 1, (n, n))
    return g + g.T


def tri(A, flags):
    return np.tril(A) if flags & LO else np.triu(A)


@pytest.mark.parametrize("n", [1, 2, 5, 37, 100, 257, 700])
@pytest.mark.parametrize("flags", [LO, UP])
def test_ldl_nopiv(gpu, ref, rng, n, flags):
    A0 = colmajor(sym(rng, n) + 2.0 * n * np.eye(n), ld=even_ld(n) + 2)
    Ag = dev(gpu, A0)
    _, err = gpu.DecomposeLDLnoPiv(Ag, None, flags, 0)
    assert err is None
    Ar = A0.copy(order="F")
    assert ref.DecomposeLDLnoPiv(Ar, flags) == 0
    Ah = Ag.cpu().numpy()
    assert fro(tri(Ah, flags) - tri(Ar, flags)) <= 64 * n * EPS * fro(A0)
    # the other triangle is not touched
    other = np.triu(A0, 1) if flags & LO else np.tril(A0, -1)
    assert np.array_equal(np.triu(Ah, 1) if flags & LO else np.tril(Ah, -1), other)
    B0 = colmajor(rng.uniform(-1, 1, (n, 5)))
    Bg = dev(gpu, B0)
    assert gpu.SolveLDLnoPiv(Bg, Ag, flags) is None
    Br = B0.copy(order="F")
    ref.SolveLDLnoPiv(Br, Ar, flags)
    assert fro(Bg.cpu().numpy() - Br) <= 64 * n * EPS * max(fro(Br), 1.0)


@pytest.mark.parametrize("n", [1, 2, 5, 37, 100, 257, 700])
@pytest.mark.parametrize("flags", [LO, UP])
def test_ldl_diag_pivoting(gpu, ref, rng, n, flags):
    import torch
    A0 = colmajor(sym(rng, n), ld=even_ld(n))
    Ag = dev(gpu, A0)
    piv = torch.full((n,), 77, dtype=torch.int64, device="cuda")
    _, err = gpu.DecomposeLDL(Ag, None, piv, flags, 0)
    assert err is None
    Ar, pr = A0.copy(order="F"), np.zeros(n, np.int64)
    assert ref.DecomposeLDL(Ar, pr, flags) == 0
    assert np.array_equal(piv.cpu().numpy(), pr)
    Ah = Ag.cpu().numpy()
    assert fro(tri(Ah, flags) - tri(Ar, flags)) <= 1e-9 * fro(A0)
    B0 = colmajor(rng.uniform(-1, 1, (n, 4)))
    Bg = dev(gpu, B0)
    assert gpu.SolveLDL(Bg, Ag, piv, flags) is None
    Br = B0.copy(order="F")
    ref.SolveLDL(Br, Ar, pr, flags)
    assert fro(Bg.cpu().numpy() - Br) <= 1e-8 * max(fro(Br), 1.0)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 37, 100, 257, 700, 1500])
@pytest.mark.parametrize("flags", [LO, UP])
def test_bunch_kaufman(gpu, ref, rng, n, flags):
    import torch
    A0 = colmajor(sym(rng, n), ld=even_ld(n) + 2)
    Ag = dev(gpu, A0)
    piv = torch.zeros(n, dtype=torch.int64, device="cuda")
    W = gpu.matrix(n, 2)
    _, err = gpu.DecomposeBK(Ag, W, piv, flags, 0)
    assert err is None
    Ar, pr = A0.copy(order="F"), np.zeros(n, np.int64)
    assert ref.DecomposeBK(Ar, pr, flags) == 0
    ph = piv.cpu().numpy()
    assert np.array_equal(ph, pr), np.flatnonzero(ph != pr)[:10]
    Ah = Ag.cpu().numpy()
    assert fro(tri(Ah, flags) - tri(Ar, flags)) <= 1e-9 * fro(A0)
    B0 = colmajor(rng.uniform(-1, 1, (n, 3)))
    Bg = dev(gpu, B0)
    assert gpu.SolveBK(Bg, Ag, piv, flags) is None
    Br = B0.copy(order="F")
    ref.SolveBK(Br, Ar, pr, flags)
    X = Bg.cpu().numpy()
    assert fro(X - Br) <= 1e-8 * max(fro(Br), 1.0)
    S = tri(A0, flags)
    S = S + S.T - np.diag(np.diag(A0))
    assert fro(S @ X - B0) <= 1e-8 * fro(S) * max(fro(X), 1.0)


def test_ldl_errors(gpu, rng):
    import torch
    A = dev(gpu, colmajor(sym(rng, 8)))
    piv = torch.zeros(8, dtype=torch.int64, device="cuda")
    _, err = gpu.DecomposeLDL(dev(gpu, colmajor(np.ones((4, 5)))), None, piv, LO, 0)
    assert err is not None and err.code == -2
    _, err = gpu.DecomposeLDL(A.clone(), None, piv[:7], LO, 0)
    assert err is not None and err.code == -3
    _, err = gpu.DecomposeLDL(dev(gpu, colmajor(np.zeros((6, 6)))), None, piv[:6], LO, 0)
    assert err is not None and err.code == -18 and str(err) == "zero value on diagonal"
    _, err = gpu.DecomposeBK(A.clone(), gpu.matrix(8, 1), piv, LO, 0)
    assert err is not None and err.code == -19 and str(err) == "Workspace too small"
    _, err = gpu.DecomposeLDLnoPiv(A.clone(), None, LO, 4)
    assert err is not None and err.code == -17
    torch.cuda.synchronize()


@pytest.mark.parametrize("seed", [1, 2])
def test_bunch_kaufman_2048_repeated(gpu, ref, seed):
    """back-to-back factorizations at n = 2048 (no synchronization between them): the same
    pivots each time and as the oracle's"""
    import torch
    n = 2048
    g = torch.Generator(device="cuda").manual_seed(seed)
    A0 = gpu.matrix(n, n)
    A0.uniform_(-1.0, 1.0, generator=g)
    A0.copy_(A0 + A0.t())
    A, W = gpu.matrix(n, n), gpu.matrix(n, 2)
    pivs = []
    for _ in range(3):
        A.copy_(A0)
        piv = torch.zeros(n, dtype=torch.int64, device="cuda")
        assert gpu.DecomposeBK(A, W, piv, LO, 0)[1] is None
        pivs.append(piv)
    assert gpu.Sync() == 0
    Ar, pr = colmajor(A0.cpu().numpy()), np.zeros(n, np.int64)
    assert ref.DecomposeBK(Ar, pr, LO) == 0
    for piv in pivs:
        assert np.array_equal(piv.cpu().numpy(), pr)
    assert fro(np.tril(A.cpu().numpy()) - np.tril(Ar)) <= 1e-8 * fro(Ar)


def _golden():
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "ldl.npz"))
    cases = {}
    for k in z.files:
        name, field = k.split("/")
        cases.setdefault(name, {})[field] = z[k]
    return cases


@pytest.mark.parametrize("name", sorted(_golden()))
def test_golden_ldl_device(gpu, name):
    """the device against the reference's kernels' outputs (tests/golden/ldl.npz): the
    reference's own Bunch-Kaufman test tables and seeded cases"""
    import torch
    c = _golden()[name]
    fl = int(c["flags"])
    A0 = c["A"]
    n = A0.shape[0]
    Ag = dev(gpu, A0)
    piv = torch.zeros(n, dtype=torch.int64, device="cuda")
    if name.startswith("np_"):
        assert gpu.DecomposeLDLnoPiv(Ag, None, fl, 0)[1] is None
    elif "bk" in name:
        assert gpu.DecomposeBK(Ag, gpu.matrix(n, 2), piv, fl, 0)[1] is None
    else:
        assert gpu.DecomposeLDL(Ag, None, piv, fl, 0)[1] is None
    if "piv" in c:
        assert np.array_equal(piv.cpu().numpy(), c["piv"])
    Ah = Ag.cpu().numpy()
    assert fro(tri(Ah, fl) - tri(c["LDL"], fl)) <= 1e-10 * max(fro(c["LDL"]), 1.0)
    if "X" in c:
        Bg = dev(gpu, c["B"])
        if name.startswith("np_"):
            assert gpu.SolveLDLnoPiv(Bg, Ag, fl) is None
        elif "bk" in name:
            assert gpu.SolveBK(Bg, Ag, piv, fl) is None
        else:
            assert gpu.SolveLDL(Bg, Ag, piv, fl) is None
        assert fro(Bg.cpu().numpy() - c["X"]) <= 1e-9 * max(fro(c["X"]), 1.0)
