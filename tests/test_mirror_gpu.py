"""GPU: device mirrors of host arrays (mo_mirror_*), the residency layer of a Go shim.

A FloatMatrix view is a window into a host slice shared with its parent (the reference
works in place on such views, mmult.go:228-233, partition.go:210-340).  One mirror per
registered array must serve every view inside it: a chain of calls on overlapping views
runs on the device copy and the host sees the results after one download, equal to the
oracle run on the host array itself."""
import ctypes

import numpy as np
import pytest

from util import colmajor, fro, spd

pytestmark = pytest.mark.gpu

LO = 0x4


def test_chain_on_overlapping_views(gpu, oracle, rng):
    from matops_b200 import _lib
    L = _lib.lib()
    n, nrhs = 300, 5
    root = np.asfortranarray(rng.uniform(-1, 1, (n + 7, n + nrhs + 3)))
    A = root[2:2 + n, 1:1 + n]            # the system matrix, a view at an odd offset
    B = root[2:2 + n, 1 + n:1 + n + nrhs]  # right-hand sides: columns of the same array
    A[:] = spd(rng, n)
    host = root.copy(order="F")
    m = gpu.Mirror(root)
    ctx = gpu.context()
    Am = m.view(A, write=True)
    bad = ctypes.c_double()
    assert L.mo_decompose_chol(ctx, Am, LO, 64, ctypes.byref(bad)) == 0
    assert L.mo_solve_chol(ctx, m.view(B, write=True), m.view(A), LO) == 0
    # a sub-view of the factor, taken through the registry by address alone
    h, off = gpu.Mirror.find(A[10:, 10:])
    assert h == m._h.value and off == (2 + 10) + (1 + 10) * root.shape[0]
    assert m.state == 2  # device newer
    m.to_host()
    assert m.state == 0
    # the same chain on the host copy with the oracle
    hA = host[2:2 + n, 1:1 + n]
    hB = host[2:2 + n, 1 + n:1 + n + nrhs]
    assert oracle.DecomposeCHOL(hA, LO, 64) == 0
    oracle.SolveCHOL(hB, hA, LO)
    assert fro(np.tril(A) - np.tril(hA)) / fro(np.tril(hA)) <= 1e-12
    assert fro(B - hB) / fro(hB) <= 1e-10
    # everything outside the two views is untouched
    mask = np.ones(root.shape, bool)
    mask[2:2 + n, 1:1 + n + nrhs] = False
    assert np.array_equal(root[mask], host[mask])
    m.close()


def test_host_edits_and_refusals(gpu, rng):
    from matops_b200 import _lib
    L = _lib.lib()
    root = np.asfortranarray(rng.uniform(-1, 1, (64, 48)))
    m = gpu.Mirror(root)
    ctx = gpu.context()
    C = root[:32, :16]
    Am = root[:32, 16:24]
    Bm = root[:8, 24:40]
    assert L.mo_mult(ctx, m.view(C, True), m.view(Am), m.view(Bm), 1.0, 0.0, 0) == 0
    m.to_host()
    expect = root[:32, 16:24] @ root[:8, 24:40]
    assert fro(C - expect) <= 1e-13 * fro(expect)
    # host edit: marked, then the next view uploads it
    root[:32, 16:24] = 2.0
    assert m.host_modified() == 0 and m.state == 1
    assert L.mo_mult(ctx, m.view(C, True), m.view(Am), m.view(Bm), 1.0, 0.0, 0) == 0
    m.to_host()
    assert fro(C - 2.0 * np.ones((32, 8)) @ root[:8, 24:40]) <= 1e-12 * fro(C)
    # a device write not yet brought back plus a host edit: refused
    m.view(C, True)
    assert m.host_modified() == -10
    m.to_host()
    # an overlapping registration and a view outside the array are refused
    with pytest.raises(gpu.MatopsError):
        gpu.Mirror(root[:, 5:])
    out = _lib.MoMatrix()
    assert L.mo_mirror_view(m._h, ctypes.c_void_p(root[60:, 40:].ctypes.data), 10, 9, 64, 0,
                            ctypes.byref(out)) == -10
    m.close()
    # after destroy the range is free again
    m2 = gpu.Mirror(root)
    m2.close()
