"""Oracle loader -- TEST INFRASTRUCTURE ONLY.

ctypes access to the CPU restatement of hrautila/matops's level-3 / Cholesky / LU path
(oracle/drivers.c over oracle/calgo_port.c) and, when it was built here, to the same
drivers over the reference's own C kernels (oracle/_ref/libmatops_ref.so).

Matrices are numpy float64 arrays in column-major (Fortran) layout; a slice of such an
array is a view with the parent's leading dimension, exactly like a FloatMatrix view
(hrautila/matrix SubMatrix).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liboracle_port.so")
REF_LIB = os.path.join(HERE, "_ref", "libmatops_ref.so")

# flag values, calgo/cmops.go:19-31
TRANSA, TRANSB, LOWER, UPPER, LEFT, RIGHT, UNIT, TRANS = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40, 0x80
NOTRANS = 0

ERRORS = {
    -1: "Mult: size mismatch",
    -2: "A not a square matrix",
    -3: "pivot array < min(A.Rows(),A.Cols())",
    -4: "C not a square matrix",
    -5: "A, B size mismatch",
    -6: "X not a vector.",
    -7: "MultSym: size mismatch",
    -13: "work space too small",
    -14: "workspace not defined",
    -15: "C*Q: C.Cols != A.Rows",
    -16: "reflector matrix T too small",
}


def build(ref: bool = False) -> None:
    """Compile the oracle (and, with ref=True, the reference's own kernels) via make."""
    targets = ["port"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def view(a: np.ndarray):
    """(pointer, rows, cols, ld) of a column-major float64 matrix view."""
    if a.ndim != 2 or a.dtype != np.float64:
        raise TypeError("expected a 2-D float64 array")
    r, c = a.shape
    if r > 1 and a.strides[0] != 8:
        raise TypeError("matrix view must be column-major (unit row stride)")
    ld = a.strides[1] // 8 if c > 1 or a.strides[1] // 8 >= r else max(r, 1)
    ld = max(ld, 1)
    return ctypes.c_void_p(a.ctypes.data), r, c, ld


class Oracle:
    """The restated Go API over one of the two kernel libraries."""

    def __init__(self, which: str = "port"):
        path = PORT_LIB if which == "port" else REF_LIB
        if not os.path.exists(path):
            if which == "port":
                build()
            else:
                raise FileNotFoundError(f"{path} not built (needs the reference sources)")
        self.which = which
        L = self.lib = ctypes.CDLL(path)
        d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        M = [p, i, i, i]
        L.or_mult.argtypes = M + M + M + [d, d, i]
        L.or_rank_update_sym.argtypes = M + M + [d, d, i]
        L.or_solve_trm.argtypes = M + M + [d, i]
        L.or_decompose_chol.argtypes = M + [i, i]
        L.or_decompose_lu.argtypes = M + [p, i, i]
        L.or_decompose_chol_steps.argtypes = M + [i, i, i, i]
        L.or_mult_sym.argtypes = M + M + M + [d, d, i]
        L.or_mult_trm.argtypes = M + M + [d, i]
        L.or_rank_update2_sym.argtypes = M + M + M + [d, d, i]
        L.or_update_trm.argtypes = M + M + M + [d, d, i]
        L.or_inverse_trm.argtypes = M + [i, i]
        L.or_solve_chol.argtypes = M + M + [i]
        L.or_solve_chol.restype = None
        L.or_solve_lu.argtypes = M + M + [p, i, i]
        L.or_num_workers.argtypes = [i]
        L.or_blocking_params.argtypes = [i, i, i]
        L.or_blocking_params.restype = None
        L.or_decompose_qrt.argtypes = M + M + M + [i]
        L.or_decompose_qr.argtypes = M + [p, i] + [p, i, i, i] + [i]
        L.or_build_t.argtypes = M + M + [p, i]
        L.or_mult_qt.argtypes = M + M + M + M + [i, i]
        L.or_solve_qrt.argtypes = M + M + M + M + [i, i]
        L.or_decompose_ldl_nopiv.argtypes = M + [i]
        L.or_solve_ldl_nopiv.argtypes = M + M + [i]
        L.or_solve_ldl_nopiv.restype = None
        L.or_decompose_ldl.argtypes = M + [p, i, i]
        L.or_solve_ldl.argtypes = M + M + [p, i]
        L.or_solve_ldl.restype = None
        L.or_decompose_bk.argtypes = M + [p, i, i]
        L.or_solve_bk.argtypes = M + M + [p, i]
        L.or_solve_bk.restype = None
        L.or_mult_q.argtypes = M + M + [p, i] + [p, i, i, i] + [i, i]
        L.or_solve_qr.argtypes = M + M + [p, i] + [p, i, i, i] + [i, i]
        L.or_build_q.argtypes = M + [p, i] + [p, i, i, i] + [i]
        L.or_build_qt.argtypes = M + M + M + [i]

    # each method returns the raw status code (0 = nil error)
    def Mult(self, C, A, B, alpha, beta, flags):
        return self.lib.or_mult(*view(C), *view(A), *view(B), alpha, beta, flags)

    def RankUpdateSym(self, C, A, alpha, beta, flags):
        return self.lib.or_rank_update_sym(*view(C), *view(A), alpha, beta, flags)

    def SolveTrm(self, B, A, alpha, flags):
        return self.lib.or_solve_trm(*view(B), *view(A), alpha, flags)

    def DecomposeCHOL(self, A, flags, nb):
        return self.lib.or_decompose_chol(*view(A), flags, nb)

    def MultSym(self, C, A, B, alpha, beta, flags):
        return self.lib.or_mult_sym(*view(C), *view(A), *view(B), alpha, beta, flags)

    def MultTrm(self, B, A, alpha, flags):
        return self.lib.or_mult_trm(*view(B), *view(A), alpha, flags)

    def RankUpdate2Sym(self, C, A, B, alpha, beta, flags):
        return self.lib.or_rank_update2_sym(*view(C), *view(A), *view(B), alpha, beta, flags)

    def UpdateTrm(self, C, A, B, alpha, beta, flags):
        return self.lib.or_update_trm(*view(C), *view(A), *view(B), alpha, beta, flags)

    def InverseTrm(self, A, flags, nb):
        """trinv.go:219: A := inverse of its LOWER (else upper) triangle, in place"""
        return self.lib.or_inverse_trm(*view(A), flags, nb)

    def DecomposeCHOLSteps(self, A, flags, nb, k0, k1):
        """blockedCHOL's block steps with first column in [k0, k1) (chol.go:58-94)"""
        return self.lib.or_decompose_chol_steps(*view(A), flags, nb, k0, k1)

    def DecomposeLU(self, A, pivots: np.ndarray, nb):
        assert pivots.dtype == np.int64 and pivots.flags.c_contiguous
        return self.lib.or_decompose_lu(*view(A), ctypes.c_void_p(pivots.ctypes.data), len(pivots), nb)

    def SolveCHOL(self, B, A, flags):
        self.lib.or_solve_chol(*view(B), *view(A), flags)

    def SolveLU(self, B, A, pivots: np.ndarray, flags):
        assert pivots.dtype == np.int64 and pivots.flags.c_contiguous
        return self.lib.or_solve_lu(*view(B), *view(A), ctypes.c_void_p(pivots.ctypes.data), len(pivots), flags)

    # QR (qrwy.go, qrwym.go); W=None is the reference's nil workspace
    @staticmethod
    def _wview(W):
        if W is None:
            return ctypes.c_void_p(0), 0, 0, 1
        return view(W)

    def DecomposeQRT(self, A, T, W, nb):
        """qrwy.go:517: A = Q R in place (R on and above the diagonal, the reflectors below),
        T the block reflector, Q = I - Y T Y^T"""
        return self.lib.or_decompose_qrt(*view(A), *view(T), *self._wview(W), nb)

    def DecomposeQR(self, A, tau: np.ndarray, W, nb):
        """qrwy.go:474: LAPACK DGEQRF form (tau, no T)"""
        assert tau.dtype == np.float64 and tau.flags.c_contiguous
        return self.lib.or_decompose_qr(*view(A), ctypes.c_void_p(tau.ctypes.data), len(tau),
                                        *self._wview(W), nb)

    def BuildT(self, T, A, tau: np.ndarray):
        """qrwy.go:546: block reflector T from the reflectors in A and tau"""
        assert tau.dtype == np.float64 and tau.flags.c_contiguous
        return self.lib.or_build_t(*view(T), *view(A), ctypes.c_void_p(tau.ctypes.data), len(tau))

    def MultQT(self, C, A, T, W, flags, nb):
        """qrwym.go:646: C = Q C, Q^T C (MO_TRANS), C Q, C Q^T (MO_RIGHT)"""
        return self.lib.or_mult_qt(*view(C), *view(A), *view(T), *self._wview(W), flags, nb)

    def SolveQRT(self, B, A, T, W, flags, nb):
        """qrwym.go:784: least squares min ||A X - B|| or (MO_TRANS) min-norm A^T X = B"""
        return self.lib.or_solve_qrt(*view(B), *view(A), *view(T), *self._wview(W), flags, nb)

    def MultQ(self, C, A, tau: np.ndarray, W, flags, nb):
        """qrwym.go:573 (the unblocked path): C = Q C, Q^T C, C Q, C Q^T from A and tau"""
        assert tau.dtype == np.float64 and tau.flags.c_contiguous
        return self.lib.or_mult_q(*view(C), *view(A), ctypes.c_void_p(tau.ctypes.data), len(tau),
                                  *self._wview(W), flags, nb)

    def SolveQR(self, B, A, tau: np.ndarray, W, flags, nb):
        """qrwym.go:717: least squares (or, TRANS, minimum norm) with Q from tau"""
        assert tau.dtype == np.float64 and tau.flags.c_contiguous
        return self.lib.or_solve_qr(*view(B), *view(A), ctypes.c_void_p(tau.ctypes.data), len(tau),
                                    *self._wview(W), flags, nb)

    def BuildQ(self, A, tau: np.ndarray, W, nb):
        """qrwyk.go:232: A := the first A.cols columns of Q = H(0)...H(k-1) (DORGQR)"""
        assert tau.dtype == np.float64 and tau.flags.c_contiguous
        return self.lib.or_build_q(*view(A), ctypes.c_void_p(tau.ctypes.data), len(tau),
                                   *self._wview(W), nb)

    def BuildQT(self, A, T, W, nb):
        """qrwyk.go:278: BuildQ with the reflector block T of DecomposeQRT"""
        return self.lib.or_build_qt(*view(A), *view(T), *self._wview(W), nb)

    # symmetric indefinite LDL^T (ldlnp.go, ldl.go, ldlbk.go, ldlbks.go); pivots are the
    # reference's 1-based ipiv (0 = no interchange for DecomposeLDL, negative = 2x2 block)
    def DecomposeLDLnoPiv(self, A, flags):
        return self.lib.or_decompose_ldl_nopiv(*view(A), flags)

    def SolveLDLnoPiv(self, B, A, flags):
        self.lib.or_solve_ldl_nopiv(*view(B), *view(A), flags)

    def DecomposeLDL(self, A, ipiv: np.ndarray, flags):
        assert ipiv.dtype == np.int64 and ipiv.flags.c_contiguous
        return self.lib.or_decompose_ldl(*view(A), ctypes.c_void_p(ipiv.ctypes.data), len(ipiv), flags)

    def SolveLDL(self, B, A, ipiv: np.ndarray, flags):
        self.lib.or_solve_ldl(*view(B), *view(A), ctypes.c_void_p(ipiv.ctypes.data), flags)

    def DecomposeBK(self, A, ipiv: np.ndarray, flags):
        assert ipiv.dtype == np.int64 and ipiv.flags.c_contiguous
        return self.lib.or_decompose_bk(*view(A), ctypes.c_void_p(ipiv.ctypes.data), len(ipiv), flags)

    def SolveBK(self, B, A, ipiv: np.ndarray, flags):
        self.lib.or_solve_bk(*view(B), *view(A), ctypes.c_void_p(ipiv.ctypes.data), flags)

    def GemvBetaOnce(self, on: bool) -> bool:
        """Port only: make the transposed GEMV apply beta once (BLAS semantics) instead of
        once per 68-row block as calgo/dmvec_gemv.c:379-393 does; returns the old mode"""
        if self.which != "port":
            raise RuntimeError("the reference's own kernels have no such switch")
        f = self.lib.or_gemv_beta_once
        f.argtypes = [ctypes.c_int]
        return bool(f(1 if on else 0))

    def NumWorkers(self, n: int) -> int:
        return self.lib.or_num_workers(n)

    def BlockingParams(self, mb: int, nb: int, kb: int) -> None:
        self.lib.or_blocking_params(mb, nb, kb)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)
