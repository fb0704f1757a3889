"""GPU: a bounded device-side wait that runs out reports MO_EDEVTIMEOUT and leaves the
context usable.

The triangular solve with at most 64 right-hand sides runs as one cooperative launch whose
CTAs wait on the step flags of earlier CTAs.  With the context's spin limit set to 0 polls a
CTA whose predecessor has not yet published gives up at once: it records the timeout, waits
for its own outstanding cp.async copies and returns (no bulk copy or TMEM is held).  The
next call on the same context, with the default limit, must succeed and match the oracle.
No GPU is faulted or hung: every wait ends by itself.
"""
import numpy as np
import pytest

from util import EPS, colmajor, fro

pytestmark = pytest.mark.gpu

LO, LEFT = 0x4, 0x10
MO_EDEVTIMEOUT = -21


def _tri(rng, n):
    a = np.tril(rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n))
    a += np.diag(rng.uniform(1.0, 2.0, n))
    return colmajor(a)


def test_step_flag_wait_times_out_then_context_recovers(gpu, oracle, rng):
    import torch
    n, nrhs = 4096, 16
    A = _tri(rng, n)
    B0 = colmajor(rng.standard_normal((n, nrhs)))
    Ag = gpu.to_device(A)
    assert gpu.Sync() == 0
    old = gpu.SetSpinLimit(0)
    try:
        Bg = gpu.to_device(B0)
        assert gpu.SolveTrm(Bg, Ag, 1.0, LEFT | LO) is None  # enqueued
        assert gpu.Sync() == MO_EDEVTIMEOUT
        assert gpu.Sync() == 0  # the status word was cleared by the first read
    finally:
        assert gpu.SetSpinLimit(old) == 0
    # the same context, default limit: a normal solve succeeds and matches the oracle
    Bg = gpu.to_device(B0)
    assert gpu.SolveTrm(Bg, Ag, 1.0, LEFT | LO) is None
    assert gpu.Sync() == 0
    torch.cuda.synchronize()
    Br = B0.copy(order="F")
    assert oracle.SolveTrm(Br, A, 1.0, LEFT | LO) == 0
    err = fro(Bg.cpu().numpy() - Br) / fro(Br)
    assert err <= 100 * n * EPS, err
