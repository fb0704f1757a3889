"""GPU: batched Cholesky / LU factor + solve (mo_batch_*) against the oracle, matrix by
matrix: every factor equals the oracle's DecomposeCHOL / DecomposeLU result to rounding,
LU pivots are identical, and every solution equals SolveCHOL / SolveLU's."""
import numpy as np
import pytest
import torch

from util import EPS, colmajor, fro

pytestmark = pytest.mark.gpu

LO = 0x4
EDGE_SIZES = [1, 2, 15, 16, 17, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 200, 255, 256, 257,
              300, 511, 512]


def _spd(rng, n):
    g = rng.standard_normal((n, n))
    return g @ g.T / n + np.eye(n)


def _batch(gpu, mats, extra_ld=0):
    """device copies (views into taller buffers when extra_ld > 0)"""
    out = []
    for a in mats:
        n = a.shape[0]
        buf = gpu.matrix(n + extra_ld, n, fill=-7.0)
        v = buf[:n, :]
        v.copy_(torch.as_tensor(a))
        out.append(v)
    return out


@pytest.mark.parametrize("nrhs,extra_ld", [(1, 0), (3, 5)])
def test_batched_cholesky_matches_oracle(gpu, oracle, rng, nrhs, extra_ld):
    sizes = EDGE_SIZES + list(rng.integers(16, 513, 18))
    As = [_spd(rng, n) for n in sizes]
    Bs = [rng.uniform(-1, 1, (n, nrhs)) for n in sizes]
    dA = _batch(gpu, As, extra_ld)
    dB = [gpu.to_device(b) for b in Bs]
    plan = gpu.BatchPlan(gpu.BATCH_CHOL, sizes, nrhs)
    info = plan.run(dA, dB)
    assert info.cpu().numpy().tolist() == [0] * len(sizes)
    for n, A, B, a, b in zip(sizes, As, Bs, dA, dB):
        out = a.cpu().numpy()
        L = np.tril(out)
        assert fro(A - L @ L.T) / fro(A) <= 10 * n * EPS
        Ar, Br = colmajor(A), colmajor(B)
        assert oracle.DecomposeCHOL(Ar, LO, 64) == 0
        oracle.SolveCHOL(Br, Ar, LO)
        assert fro(L - np.tril(Ar)) / fro(np.tril(Ar)) <= 1e-12
        iu = np.triu_indices(n, 1)
        assert np.array_equal(out[iu], A[iu])  # strict upper part not touched
        X = b.cpu().numpy()
        assert fro(X - Br) / fro(Br) <= 1e-10


@pytest.mark.parametrize("nrhs,extra_ld", [(1, 0), (2, 3)])
def test_batched_lu_matches_oracle(gpu, oracle, rng, nrhs, extra_ld):
    sizes = EDGE_SIZES + list(rng.integers(16, 513, 18))
    As = [rng.standard_normal((n, n)) for n in sizes]
    Bs = [rng.uniform(-1, 1, (n, nrhs)) for n in sizes]
    dA = _batch(gpu, As, extra_ld)
    dB = [gpu.to_device(b) for b in Bs]
    pivs = [torch.full((n,), -1, dtype=torch.int64, device="cuda") for n in sizes]
    plan = gpu.BatchPlan(gpu.BATCH_LU, sizes, nrhs)
    info = plan.run(dA, dB, pivs)
    assert info.cpu().numpy().tolist() == [0] * len(sizes)
    for n, A, B, a, b, pv in zip(sizes, As, Bs, dA, dB, pivs):
        out = a.cpu().numpy()
        p = pv.cpu().numpy()
        Ar = colmajor(A, ld=n + (n % 2))
        pr = np.zeros(n, np.int64)
        assert oracle.DecomposeLU(Ar, pr, 64) == 0
        assert np.array_equal(p, pr), n
        L = np.tril(out, -1) + np.eye(n)
        U = np.triu(out)
        PA = A.copy()
        for k in range(n):
            PA[[k, p[k]]] = PA[[p[k], k]]
        assert fro(PA - L @ U) / fro(A) <= 10 * n * EPS
        assert fro(out - Ar) / fro(Ar) <= 1e-11
        Br = colmajor(B)
        assert oracle.SolveLU(Br, Ar, pr, 0) == 0
        assert fro(b.cpu().numpy() - Br) / fro(Br) <= 1e-9


def test_batched_failures_are_per_matrix(gpu, rng):
    sizes = [40, 300, 64, 129]
    As = [_spd(rng, n) for n in sizes]
    As[1][170, 170] = -3.0  # not positive definite at column 170 (or earlier)
    dA = _batch(gpu, As)
    dB = [gpu.to_device(np.ones((n, 1))) for n in sizes]
    info = gpu.BatchPlan(gpu.BATCH_CHOL, sizes, 1).run(dA, dB).cpu().numpy()
    assert info[0] == 0 and info[2] == 0 and info[3] == 0
    assert 1 <= info[1] <= 171
    for i in (0, 2, 3):
        X = dB[i].cpu().numpy()
        assert fro(As[i] @ X - 1.0) / fro(X) <= 1e-10
    # LU: an exactly zero column gives a zero pivot there
    G = [rng.standard_normal((n, n)) for n in sizes]
    G[2][:, 10] = 0.0
    pivs = [torch.zeros(n, dtype=torch.int64, device="cuda") for n in sizes]
    info = gpu.BatchPlan(gpu.BATCH_LU, sizes, 0).run(_batch(gpu, G), None, pivs).cpu().numpy()
    assert info.tolist() == [0, 0, 11, 0]


def test_batched_graph_replay_and_new_pointers(gpu, oracle, rng):
    sizes = [int(x) for x in rng.integers(16, 200, 30)]
    plan = gpu.BatchPlan(gpu.BATCH_CHOL, sizes, 1)
    for rep in range(3):  # replay, replay with the same lists, then new lists
        As = [_spd(rng, n) for n in sizes]
        dA = _batch(gpu, As)
        dB = [gpu.to_device(rng.standard_normal((n, 1))) for n in sizes]
        Bh = [b.cpu().numpy() for b in dB]
        assert plan.run(dA, dB).cpu().numpy().tolist() == [0] * len(sizes)
        for A, b, B in zip(As, dB, Bh):
            assert fro(A @ b.cpu().numpy() - B) / fro(B) <= 1e-12


@pytest.mark.parametrize("kind", [1, 2])
def test_batched_tuner_and_schedules(gpu, rng, kind):
    sizes = [int(x) for x in rng.integers(16, 513, 80)]
    plan = gpu.BatchPlan(kind, sizes, 1)
    times = plan.tune(1)
    assert times and all(t > 0 for v in times.values() for t in v)
    cfg = plan.schedule()
    assert all(c in (0, 1) for c in cfg)
    for forced in ([0, 0, 0, 0], [1, 1, 1, 1], [1, 0, 1, 0]):
        plan.schedule(forced)
        assert plan.schedule() == forced
        As = [_spd(rng, n) if kind == 1 else rng.standard_normal((n, n)) for n in sizes]
        dA = _batch(gpu, As)
        dB = [gpu.to_device(np.ones((n, 1))) for n in sizes]
        pivs = [torch.zeros(n, dtype=torch.int64, device="cuda") for n in sizes] if kind == 2 else None
        assert plan.run(dA, dB, pivs).cpu().numpy().tolist() == [0] * len(sizes)
        for A, b in zip(As, dB):
            X = b.cpu().numpy()
            assert fro(A @ X - 1.0) / (fro(A) * fro(X)) <= 1e-13


def test_batched_rejects_bad_orders(gpu):
    with pytest.raises(gpu.MatopsError, match="MO_BATCH_MAX_N"):
        gpu.BatchPlan(gpu.BATCH_CHOL, [4, 513], 1)
    with pytest.raises(gpu.MatopsError, match="MO_BATCH_MAX_N"):
        gpu.BatchPlan(gpu.BATCH_LU, [0], 1)
    plan = gpu.BatchPlan(gpu.BATCH_LU, [], 1)
    assert plan.run([], [], []).numel() == 0
