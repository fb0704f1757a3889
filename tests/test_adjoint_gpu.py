"""GPU: Cholesky adjoint (mo_decompose_chol_adjoint, batched form) and solve adjoint
(mo_solve_chol_adjoint), wrapped as torch.autograd.Functions used only as a test harness.

Checks, all in FP64: the closed form Abar = sym(L^-T Phi(L^T Lbar) L^-1); the gradient of
torch.linalg.cholesky / torch.linalg.solve for the loss
    loss(A) = sum(W * L) + 2 sum(log diag L) + w^T x,   L = chol(A),  x = A^-1 b
with A = G G^T / n + I; and central finite differences (h = 1e-6, symmetric perturbation
of 64 random entries, relative error <= 1e-7)."""
import numpy as np
import pytest
import torch

from util import fro

pytestmark = pytest.mark.gpu

LO = 0x4


def _cm(t):
    """column-major CUDA float64 copy"""
    import matops_b200 as mo
    out = mo.matrix(t.shape[0], t.shape[1])
    out.copy_(t)
    return out


class CholeskyFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A):
        import matops_b200 as mo
        L = _cm(A)
        _, err = mo.DecomposeCHOL(L, LO, 64)
        assert err is None
        ctx.save_for_backward(L)
        return torch.tril(L)

    @staticmethod
    def backward(ctx, gL):
        import matops_b200 as mo
        (L,) = ctx.saved_tensors
        G = _cm(torch.tril(gL))
        assert mo.DecomposeCHOLAdjoint(L, G, LO) is None
        return G


class CholSolveFn(torch.autograd.Function):
    """x = A^-1 b with the factor L of A (L is not differentiated through: the solve's
    gradient with respect to A is returned directly)"""

    @staticmethod
    def forward(ctx, A, L, b):
        import matops_b200 as mo
        L = _cm(L)
        x = _cm(b)
        mo.SolveCHOL(x, L, LO)
        ctx.save_for_backward(L, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        import matops_b200 as mo
        L, x = ctx.saved_tensors
        xb = _cm(gx)
        Abar = _cm(torch.zeros(L.shape, dtype=torch.float64, device=L.device))
        assert mo.SolveCHOLAdjoint(L, x, xb, Abar, LO) is None
        return Abar, None, xb


def loss_ours(A, W, w, b):
    L = CholeskyFn.apply(A)
    x = CholSolveFn.apply(A, L.detach(), b)
    return (W * L).sum() + 2 * torch.log(torch.diagonal(L)).sum() + (w * x).sum()


def loss_torch(A, W, w, b):
    L = torch.linalg.cholesky(A)
    x = torch.cholesky_solve(b, L)
    return (W * L).sum() + 2 * torch.log(torch.diagonal(L)).sum() + (w * x).sum()


def _problem(rng, n):
    G = rng.standard_normal((n, n))
    A = G @ G.T / n + np.eye(n)
    W, w, b = (rng.standard_normal(s) for s in ((n, n), (n, 1), (n, 1)))
    return A, W, w, b


@pytest.mark.parametrize("n", [1, 5, 127, 128, 129, 300, 700])
def test_chol_adjoint_closed_form(gpu, rng, n):
    A, _, _, _ = _problem(rng, n)
    L = np.linalg.cholesky(A)
    Lbar = np.tril(rng.standard_normal((n, n)))
    Li = np.linalg.inv(L)
    P = np.tril(L.T @ Lbar)
    P[np.diag_indices(n)] *= 0.5
    S = Li.T @ P @ Li
    ref = 0.5 * (S + S.T)
    Ld = gpu.to_device(np.tril(L) + np.triu(A, 1))  # the factor as DecomposeCHOL leaves it
    G = gpu.to_device(Lbar + np.triu(np.full((n, n), 7.0), 1))  # upper part of Lbar ignored
    assert gpu.DecomposeCHOLAdjoint(Ld, G, LO) is None
    out = G.cpu().numpy()
    assert fro(out - ref) / fro(ref) <= 1e-10
    assert np.array_equal(out, out.T)


@pytest.mark.parametrize("n", [64, 256, 520])
def test_gradient_matches_torch(gpu, rng, n):
    A, W, w, b = _problem(rng, n)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
    A1 = t(A).requires_grad_(True)
    loss_ours(A1, t(W), t(w), t(b)).backward()
    A2 = torch.tensor(A, dtype=torch.float64).requires_grad_(True)
    loss_torch(A2, *(torch.tensor(a, dtype=torch.float64) for a in (W, w, b))).backward()
    g1, g2 = A1.grad.cpu().numpy(), A2.grad.numpy()
    # torch's gradient is the symmetric one as well (cholesky_backward symmetrizes)
    g2 = 0.5 * (g2 + g2.T)
    assert fro(g1 - g2) / fro(g2) <= 1e-10


def test_gradient_matches_finite_differences(gpu, rng):
    n = 256
    A, W, w, b = _problem(rng, n)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
    Wt, wt, bt = t(W), t(w), t(b)
    A1 = t(A).requires_grad_(True)
    loss_ours(A1, Wt, wt, bt).backward()
    g = A1.grad.cpu().numpy()
    h = 1e-6
    picks = [(int(i), int(j)) for i, j in rng.integers(0, n, (64, 2))]
    fd, an = [], []
    with torch.no_grad():
        for i, j in picks:
            E = np.zeros((n, n))
            E[i, j] += 1.0
            if i != j:
                E[j, i] += 1.0
            lp = float(loss_ours(t(A + h * E), Wt, wt, bt))
            lm = float(loss_ours(t(A - h * E), Wt, wt, bt))
            fd.append((lp - lm) / (2 * h))
            an.append(g[i, j] + (g[j, i] if i != j else 0.0))
    fd, an = np.array(fd), np.array(an)
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) <= 1e-7


def test_batched_adjoint_matches_single(gpu, rng):
    count, n = 24, 256
    # orders up to 512 take the one-kernel path, larger ones the per-matrix sweep
    others = {0: 1, 3: 33, 6: 600}
    Ls, Gs, refs = [], [], []
    for k in range(count):
        nk = others.get(k, n if k % 3 else 100 + k)  # a few other orders in the same call
        A, _, _, _ = _problem(rng, nk)
        L = gpu.to_device(A)
        gpu.DecomposeCHOL(L, LO, 64)
        Gb = np.tril(rng.standard_normal((nk, nk)))
        G1, G2 = gpu.to_device(Gb), gpu.to_device(Gb)
        assert gpu.DecomposeCHOLAdjoint(L, G1, LO) is None
        Ls.append(L)
        Gs.append(G2)
        refs.append(G1)
    assert gpu.DecomposeCHOLAdjointBatched(Ls, Gs, LO) is None
    torch.cuda.synchronize()
    for G2, G1 in zip(Gs, refs):
        assert fro(G2.cpu().numpy() - G1.cpu().numpy()) / fro(G1.cpu().numpy()) <= 1e-13


def test_solve_adjoint(gpu, rng):
    n, nrhs = 300, 3
    A, _, _, _ = _problem(rng, n)
    B = rng.standard_normal((n, nrhs))
    Xbar = rng.standard_normal((n, nrhs))
    X = np.linalg.solve(A, B)
    Bbar = np.linalg.solve(A, Xbar)
    ref = -0.5 * (Bbar @ X.T + X @ Bbar.T)
    L = gpu.to_device(A)
    gpu.DecomposeCHOL(L, LO, 64)
    Xd, XBd = gpu.to_device(X), gpu.to_device(Xbar)
    Ab = gpu.to_device(np.zeros((n, n)))
    assert gpu.SolveCHOLAdjoint(L, Xd, XBd, Ab, LO) is None
    assert fro(XBd.cpu().numpy() - Bbar) / fro(Bbar) <= 1e-10
    assert fro(Ab.cpu().numpy() - ref) / fro(ref) <= 1e-10


def test_adjoint_argument_errors(gpu):
    L, G = gpu.matrix(4, 4, fill=1.0), gpu.matrix(4, 5)
    assert str(gpu.DecomposeCHOLAdjoint(L, G, LO)) == "A not a square matrix"
    assert gpu.DecomposeCHOLAdjoint(L, gpu.matrix(3, 3), LO).code == -1
    assert gpu.DecomposeCHOLAdjoint(L, gpu.matrix(4, 4), 0x8).code == -10
    assert gpu.SolveCHOLAdjoint(L, gpu.matrix(4, 2), gpu.matrix(4, 3), gpu.matrix(4, 4)).code == -1
