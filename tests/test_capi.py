"""CPU: the C-ABI library loads without a GPU and exports every symbol the header declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "matops_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^MO_API\s+[\w\s\*]+?\b(mo_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared()
    for n in ["mo_mult", "mo_rank_update_sym", "mo_solve_trm", "mo_decompose_chol",
              "mo_solve_chol", "mo_decompose_lu", "mo_solve_lu", "mo_ctx_create", "mo_sync"]:
        assert n in names


def test_library_exports_all_declared_symbols():
    from matops_b200 import _lib
    L = _lib.lib()
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_strerror_matches_go_errors():
    from matops_b200 import _lib
    L = _lib.lib()
    assert L.mo_strerror(-1) == b"Mult: size mismatch"
    assert L.mo_strerror(-2) == b"A not a square matrix"
    assert L.mo_strerror(-3) == b"pivot array < min(A.Rows(),A.Cols())"
    assert L.mo_strerror(-4) == b"C not a square matrix"
    assert L.mo_strerror(-5) == b"A, B size mismatch"
    # QR (qrwy.go:526, qrwym.go:652, :656, qrwy.go:550) and LDL^T (ldlnp.go:224, ldl.go:62,
    # ldlbk.go:1121)
    assert L.mo_strerror(-13) == b"work space too small"
    assert L.mo_strerror(-14) == b"workspace not defined"
    assert L.mo_strerror(-15) == b"C*Q: C.Cols != A.Rows"
    assert L.mo_strerror(-16) == b"reflector matrix T too small"
    assert L.mo_strerror(-17) == b"No workspace for blocking invocation"
    assert L.mo_strerror(-18) == b"zero value on diagonal"
    assert L.mo_strerror(-19) == b"Workspace too small"


def test_null_context_is_rejected_without_gpu():
    from matops_b200 import _lib
    L = _lib.lib()
    assert L.mo_sync(None) == -10
    assert L.mo_ctx_destroy(None) == -10
