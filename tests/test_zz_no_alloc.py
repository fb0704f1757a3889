"""GPU: mo_solve_trm_static, the SolveTrm entry point that allocates no device memory.

It exists for programs that cannot let a library call cudaMalloc (their device memory is
owned by their own pool, or held to a fixed footprint).  Its results must equal those of
the regular entry point, mo_solve_trm, on two calls in a row (the calls share one fixed
scratch block), and a matrix above the fixed limit must be refused.  This file is collected
last so that a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from util import EPS, colmajor, fro

pytestmark = pytest.mark.gpu

TA, LO, UP, LEFT, RIGHT, UNIT = 0x1, 0x4, 0x8, 0x10, 0x20, 0x40


def _static_solve(gpu, B, A, alpha, flags):
    import torch

    from matops_b200 import _lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _lib.lib().mo_solve_trm_static(gpu.view(B), gpu.view(A), alpha, flags, stream)


def _tri(rng, n):
    a = rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n)
    a += np.diag(rng.uniform(1.0, 2.0, n) * np.sign(rng.uniform(-1, 1, n)))
    return colmajor(a)


@pytest.mark.parametrize("n,nrhs", [(300, 37), (1024, 16)])
def test_static_solve_matches_regular_entry_point(gpu, rng, n, nrhs):
    import torch
    cases = [LEFT | LO, LEFT | UP | TA, RIGHT | LO | TA, RIGHT | UP | UNIT]
    for call in range(2):  # two calls in a row: the second reuses the first one's scratch
        for flags in cases:
            A = gpu.to_device(_tri(rng, n))
            B0 = rng.standard_normal((nrhs, n) if flags & RIGHT else (n, nrhs))
            B_regular = gpu.to_device(B0)
            B_static = gpu.to_device(B0)
            assert gpu.SolveTrm(B_regular, A, 1.3, flags) is None
            assert _static_solve(gpu, B_static, A, 1.3, flags) == 0
            torch.cuda.synchronize()
            ref = B_regular.cpu().numpy()
            err = fro(B_static.cpu().numpy() - ref) / fro(ref)
            assert err <= 100 * n * EPS, (call, hex(flags), err)


def test_static_solve_matches_oracle(gpu, oracle, rng):
    """The static entry point against the oracle's SolveTrm (the reference's algorithm on the
    CPU), not only against the regular entry point."""
    import torch
    n, nrhs = 700, 96
    for flags in (LEFT | LO, RIGHT | UP | TA):
        A = _tri(rng, n)
        B0 = colmajor(rng.standard_normal((nrhs, n) if flags & RIGHT else (n, nrhs)))
        Bg = gpu.to_device(B0)
        assert _static_solve(gpu, Bg, gpu.to_device(A), -0.7, flags) == 0
        torch.cuda.synchronize()
        Br = B0.copy(order="F")
        assert oracle.SolveTrm(Br, A, -0.7, flags) == 0
        err = fro(Bg.cpu().numpy() - Br) / fro(Br)
        assert err <= 100 * n * EPS, (hex(flags), err)


def test_static_solve_allocates_nothing(gpu, rng):
    import torch
    n = 512
    A = gpu.to_device(_tri(rng, n))
    B = gpu.to_device(rng.standard_normal((n, 8)))
    assert _static_solve(gpu, B, A, 1.0, LEFT | LO) == 0  # first call: one-time symbol lookup
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert _static_solve(gpu, B, A, 1.0, LEFT | LO) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_static_solve_rejects_order_above_limit(gpu):
    from matops_b200 import _lib
    n = 1025
    A = gpu.matrix(n, n)
    B = gpu.matrix(n, 2)
    rc = _static_solve(gpu, B, A, 1.0, LEFT | LO)
    assert rc == -11
    assert b"fixed scratch" in _lib.lib().mo_strerror(rc)
