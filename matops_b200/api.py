"""Host-side mirror of the reference's Go API for the level-3 / Cholesky / LU path.

Names, argument order, flag values and error behaviour follow package matops
(mmult.go, chol.go, lu.go): functions return ``None`` for a nil error or a
:class:`MatopsError` carrying the Go error string; a Go ``panic`` (non-SPD Cholesky,
chol.go:33-36, or any error after ``SetPanicOnError(True)`` for the wrappers that use
``onError``, mmult.go:46-57) raises :class:`MatopsPanic`.

Matrices are CUDA float64 tensors in column-major layout (stride(0) == 1); slicing such
a tensor gives a view with the parent's leading dimension, like FloatMatrix.SubMatrix.
Every call goes through the C ABI of libmatops_b200.so on the current torch stream.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

# flags, calgo/cmops.go:19-31
TRANSA, TRANSB, LOWER, UPPER, LEFT, RIGHT, UNIT, TRANS = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40, 0x80
NOTRANS = NONE = 0


class MatopsError(Exception):
    """A Go error value returned by a matops function."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class MatopsPanic(RuntimeError):
    """A Go panic in the reference (raised, not returned)."""


_panic_on_error = False
_contexts: dict[int, ctypes.c_void_p] = {}
_settings = {"blocking": (68, 68, 196), "workers": 1}


def SetPanicOnError(newval: bool) -> None:
    """mmult.go:55-57"""
    global _panic_on_error
    _panic_on_error = bool(newval)


def BlockingParams(mb: int, nb: int, kb: int) -> None:
    """mmult.go:63-67 (nb sets RankUpdateSym's beta block; see mo_blocking_params)"""
    _settings["blocking"] = (mb, nb, kb)
    for c in _contexts.values():
        _lib.lib().mo_blocking_params(c, mb, nb, kb)


def NumWorkers(newWorkers: int) -> int:
    """mmult.go:69-73 -- kept for drop-in compatibility; the device does not use it."""
    old = _settings["workers"]
    _settings["workers"] = newWorkers
    return old


def DecomposeBlockSize(nb: int) -> None:
    """lu.go:35-37 -- sets a global that the reference never reads."""


def context(device: int | None = None) -> ctypes.c_void_p:
    dev = torch.cuda.current_device() if device is None else device
    c = _contexts.get(dev)
    if c is None:
        c = ctypes.c_void_p()
        rc = _lib.lib().mo_ctx_create(dev, ctypes.byref(c))
        if rc != 0:
            raise RuntimeError(f"mo_ctx_create({dev}) failed: {_lib.lib().mo_strerror(rc).decode()}")
        _lib.lib().mo_blocking_params(c, *_settings["blocking"])
        _contexts[dev] = c
    _lib.lib().mo_set_stream(c, ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    return c


def view(t: torch.Tensor) -> _lib.MoMatrix:
    """mo_matrix of a column-major CUDA float64 tensor view."""
    if t.dim() != 2 or t.dtype != torch.float64 or not t.is_cuda:
        raise TypeError("expected a 2-D float64 CUDA tensor")
    r, c = t.shape
    if r > 1 and t.stride(0) != 1:
        raise TypeError("matrix view must be column-major (stride(0) == 1)")
    ld = t.stride(1) if c > 1 else max(t.stride(1), r, 1)
    return _lib.MoMatrix(t.data_ptr(), r, c, max(ld, r, 1))


def matrix(rows: int, cols: int, device=None, fill=None) -> torch.Tensor:
    """Allocate a column-major float64 matrix on the device."""
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    t = torch.empty((cols, rows), dtype=torch.float64, device=dev).t()
    if fill is not None:
        t.fill_(fill)
    return t


def to_device(a, device=None) -> torch.Tensor:
    """Copy a 2-D host array (numpy or torch) into a new column-major device matrix."""
    src = torch.as_tensor(a, dtype=torch.float64)
    t = matrix(src.shape[0], src.shape[1], device)
    t.copy_(src)
    return t


def _err(rc: int, use_on_error: bool = False):
    if rc == 0:
        return None
    msg = _lib.lib().mo_strerror(rc).decode()
    if use_on_error and _panic_on_error:
        raise MatopsPanic(msg)
    if rc in (-20, -21, -22, -23):
        raise RuntimeError(f"matops_b200 device failure: {msg} ({rc})")
    return MatopsError(rc, msg)


def Mult(C, A, B, alpha: float, beta: float, flags: int = NOTRANS):
    """mmult.go:198 -- C = beta*C + alpha*op(A)*op(B)."""
    return _err(_lib.lib().mo_mult(context(), view(C), view(A), view(B), alpha, beta, flags))


def RankUpdateSym(C, A, alpha: float, beta: float, flags: int):
    """mmult.go:426 -- triangle(C) = beta*C + alpha*A*A^T (or A^T*A with TRANSA)."""
    return _err(_lib.lib().mo_rank_update_sym(context(), view(C), view(A), alpha, beta, flags), True)


def SolveTrm(B, A, alpha: float, flags: int):
    """mmult.go:388 -- B = alpha*op(A)^-1*B (LEFT) or alpha*B*op(A)^-1 (RIGHT)."""
    return _err(_lib.lib().mo_solve_trm(context(), view(B), view(A), alpha, flags), True)


def MultSym(C, A, B, alpha: float, beta: float, flags: int):
    """mmult.go:266: C = beta*C + alpha*S*op(B) (LEFT) or beta*C + alpha*op(B)*S, S the
    symmetric matrix of A's UPPER (else lower) triangle"""
    return _err(_lib.lib().mo_mult_sym(context(), view(C), view(A), view(B), alpha, beta, flags))


def MultTrm(B, A, alpha: float, flags: int):
    """mmult.go:338: B = alpha*op(T)*B (LEFT) or alpha*B*op(T) (RIGHT), T triangular"""
    return _err(_lib.lib().mo_mult_trm(context(), view(B), view(A), alpha, flags), True)


def RankUpdate2Sym(C, A, B, alpha: float, beta: float, flags: int):
    """mmult.go:453: triangle(C) = beta*C + alpha*(A*B^T + B*A^T) (TRANSA: A^T*B + B^T*A)"""
    return _err(_lib.lib().mo_rank_update2_sym(context(), view(C), view(A), view(B), alpha, beta,
                                               flags), True)


def UpdateTrm(C, A, B, alpha: float, beta: float, flags: int):
    """mmult.go:501: triangle(C) = beta*C + alpha*op(A)*op(B)"""
    return _err(_lib.lib().mo_update_trm(context(), view(C), view(A), view(B), alpha, beta,
                                         flags), True)


def InverseTrm(A, flags: int, nb: int):
    """trinv.go:219: A := inverse of its LOWER (else upper) triangle (UNIT: unit diagonal);
    returns (A, err)"""
    return A, _err(_lib.lib().mo_inverse_trm(context(), view(A), flags, nb))


def DecomposeCHOL(A, flags: int, nb: int):
    """chol.go:116 -- returns (A, err); a non-positive pivot panics like the reference."""
    bad = ctypes.c_double(0.0)
    rc = _lib.lib().mo_decompose_chol(context(), view(A), flags, nb, ctypes.byref(bad))
    if rc > 0:
        raise MatopsPanic(f"illegal value at {rc - 1}: {bad.value:e}")
    return A, _err(rc)


def SolveCHOL(B, A, flags: int) -> None:
    """chol.go:147 (no return value)."""
    rc = _lib.lib().mo_solve_chol(context(), view(B), view(A), flags)
    if rc != 0:
        e = _err(rc, True)
        if e is not None:
            raise MatopsPanic(str(e))


def DecomposeLU(A, pivots: torch.Tensor, nb: int):
    """lu.go:257 -- returns (A, err); pivots is a CUDA int64 tensor (0-based rows)."""
    if pivots.dtype != torch.int64 or not pivots.is_cuda or not pivots.is_contiguous():
        raise TypeError("pivots must be a contiguous CUDA int64 tensor")
    rc = _lib.lib().mo_decompose_lu(context(), view(A), ctypes.c_void_p(pivots.data_ptr()),
                                    pivots.numel(), nb)
    return A, _err(rc)


def SolveLU(B, A, pivots: torch.Tensor, flags: int):
    """lu.go:320 -- apply the interchanges, then the two triangular solves."""
    if pivots.dtype != torch.int64 or not pivots.is_cuda or not pivots.is_contiguous():
        raise TypeError("pivots must be a contiguous CUDA int64 tensor")
    rc = _lib.lib().mo_solve_lu(context(), view(B), view(A), ctypes.c_void_p(pivots.data_ptr()),
                                pivots.numel(), flags)
    return _err(rc)


# ---- symmetric indefinite LDL^T (ldlnp.go, ldl.go, ldlbk.go, ldlbks.go) ----

def _piv(ipiv):
    if ipiv.dtype != torch.int64 or not ipiv.is_cuda or not ipiv.is_contiguous():
        raise TypeError("ipiv must be a contiguous CUDA int64 tensor")
    return ctypes.c_void_p(ipiv.data_ptr()), ipiv.numel()


def DecomposeLDLnoPiv(A, W, flags: int, nb: int):
    """ldlnp.go:211 -- A = L D L^T (LOWER) or U D U^T without interchanges; (A, err)"""
    return A, _err(_lib.lib().mo_decompose_ldl_nopiv(context(), view(A), _wview(W), flags, nb))


def SolveLDLnoPiv(B, A, flags: int):
    """ldlnp.go:251 -- B = A^-1 B with DecomposeLDLnoPiv's factor"""
    return _err(_lib.lib().mo_solve_ldl_nopiv(context(), view(B), view(A), flags))


def DecomposeLDL(A, W, ipiv, flags: int, nb: int):
    """ldl.go:439 -- 1x1 diagonal pivoting; ipiv (CUDA int64) in the reference's encoding"""
    return A, _err(_lib.lib().mo_decompose_ldl(context(), view(A), _wview(W), *_piv(ipiv), flags,
                                               nb))


def SolveLDL(B, A, ipiv, flags: int):
    """ldl.go:486"""
    return _err(_lib.lib().mo_solve_ldl(context(), view(B), view(A), *_piv(ipiv), flags))


def DecomposeBK(A, W, ipiv, flags: int, nb: int):
    """ldlbk.go:1114 -- Bunch-Kaufman LDL^T; ipiv negative for 2x2 blocks"""
    return A, _err(_lib.lib().mo_decompose_bk(context(), view(A), _wview(W), *_piv(ipiv), flags,
                                              nb))


def SolveBK(B, A, ipiv, flags: int):
    """ldlbks.go:303"""
    return _err(_lib.lib().mo_solve_bk(context(), view(B), view(A), *_piv(ipiv), flags))


# ---- QR with the compact WY form (qrwy.go, qrwym.go) ----

def _wview(W):
    """the reference's optional workspace: None stands for a nil matrix"""
    return _lib.MoMatrix(None, 0, 0, 1) if W is None else view(W)


def _vec(tau):
    """a 1-D or (k x 1) CUDA float64 tensor as a column vector view"""
    if tau.dim() == 1:
        tau = tau.unsqueeze(1)
    return view(tau)


def DecomposeQRT(A, T, W, nb: int):
    """qrwy.go:517 -- A = Q R in place, T the block reflector (Q = I - Y T Y^T); returns
    (A, err)"""
    return A, _err(_lib.lib().mo_decompose_qrt(context(), view(A), view(T), _wview(W), nb))


def DecomposeQR(A, tau, W, nb: int):
    """qrwy.go:474 -- A = Q R in place, the reflectors' scalar factors in tau (DGEQRF);
    returns (A, err)"""
    return A, _err(_lib.lib().mo_decompose_qr(context(), view(A), _vec(tau), _wview(W), nb))


def BuildT(T, A, tau):
    """qrwy.go:546 -- T = the block reflector of A's reflectors and tau; returns (T, err)"""
    return T, _err(_lib.lib().mo_build_t(context(), view(T), view(A), _vec(tau)))


def BuildQ(A, tau, W, nb: int):
    """qrwyk.go:232 -- A := the first A.cols columns of Q (DORGQR); returns (A, err)"""
    return A, _err(_lib.lib().mo_build_q(context(), view(A), _vec(tau), _wview(W), nb))


def BuildQT(A, T, W, nb: int):
    """qrwyk.go:278 -- BuildQ with Q from DecomposeQRT's T; returns (A, err)"""
    return A, _err(_lib.lib().mo_build_qt(context(), view(A), view(T), _wview(W), nb))


def MultQT(C, A, T, W, flags: int, nb: int):
    """qrwym.go:646 -- C = Q C, Q^T C (TRANS), C Q (RIGHT), C Q^T (RIGHT|TRANS)"""
    return _err(_lib.lib().mo_mult_qt(context(), view(C), view(A), view(T), _wview(W), flags, nb))


def MultQ(C, A, tau, W, flags: int, nb: int):
    """qrwym.go:573 -- MultQT with Q from A and tau (DORMQR)"""
    return _err(_lib.lib().mo_mult_q(context(), view(C), view(A), _vec(tau), _wview(W), flags, nb))


def SolveQRT(B, A, T, W, flags: int, nb: int):
    """qrwym.go:784 -- least squares min ||A X - B|| (or, TRANS, min-norm A^T X = B) into B"""
    return _err(_lib.lib().mo_solve_qrt(context(), view(B), view(A), view(T), _wview(W), flags,
                                        nb))


def SolveQR(B, A, tau, W, flags: int, nb: int):
    """qrwym.go:717 -- SolveQRT with Q from A and tau"""
    return _err(_lib.lib().mo_solve_qr(context(), view(B), view(A), _vec(tau), _wview(W), flags,
                                       nb))


# ---- mixed precision (no counterpart in the reference; LAPACK dsposv is the model) ----

PREC_BF16X3, PREC_TF32X3 = 1, 2
IR_AUTO, IR_CLASSIC, IR_GMRES, IR_NO_FALLBACK = 0, 1, 2, 0x100


class IRInfo:
    """Outcome of SolveCHOLMixed (mo_ir_info)."""

    def __init__(self, raw):
        self.iters = raw.iters
        self.gmres_iters = raw.gmres_iters
        self.converged = bool(raw.converged)
        self.fallback = bool(raw.fallback)
        self.shifts = raw.shifts
        self.method = raw.method
        self.abandoned = bool(raw.abandoned)
        self.prec = raw.prec
        self.berr = raw.berr
        self.shift = raw.shift
        self.history = [raw.history[i] for i in range(min(32, raw.iters + 1))]

    def __repr__(self):
        return (f"IRInfo(iters={self.iters}, gmres_iters={self.gmres_iters}, "
                f"converged={self.converged}, fallback={self.fallback}, shifts={self.shifts}, "
                f"method={self.method}, abandoned={self.abandoned}, berr={self.berr:.3e}, "
                f"shift={self.shift:.3e})")


def SolveCHOLMixed(X, A, B, flags: int = LOWER, prec: int = PREC_TF32X3, method: int = IR_AUTO,
                   tol: float = 1e-14, maxit: int = 30):
    """X = A^-1 B for SPD A: low-precision Cholesky (BF16x3 or TF32x3 split products on the
    tensor cores) refined in FP64 (classic IR / GMRES-IR).  Only the triangle selected by
    flags (LOWER or UPPER) is read; A is not modified.  Returns (IRInfo, err); a matrix
    that is not positive definite in FP64 raises MatopsPanic like DecomposeCHOL."""
    info = _lib.MoIRInfo()
    rc = _lib.lib().mo_dsposv_ir(context(), view(X), view(A), view(B), flags, prec, method, tol,
                                 maxit, ctypes.byref(info))
    if rc > 0:
        raise MatopsPanic(f"illegal value at {rc - 1}")
    return IRInfo(info), _err(rc)


def _fview(t: torch.Tensor):
    if t.dim() != 2 or t.dtype != torch.float32 or not t.is_cuda:
        raise TypeError("expected a 2-D float32 CUDA tensor")
    r, c = t.shape
    if r > 1 and t.stride(0) != 1:
        raise TypeError("matrix view must be column-major (stride(0) == 1)")
    ld = t.stride(1) if c > 1 else max(t.stride(1), r, 1)
    return ctypes.c_void_p(t.data_ptr()), max(ld, r, 1)


def LPGemm(C, A, B, alpha: float, beta: float, flags: int = NOTRANS, prec: int = PREC_TF32X3):
    """C = beta*C + alpha*op(A)*op(B) on column-major float32 CUDA tensors with the
    split-product tensor-core arithmetic of the mixed-precision factorization; LOWER in
    flags updates only C(i, j) with i >= j."""
    m, n = C.shape
    k = A.shape[0] if flags & TRANSA else A.shape[1]
    (pa, lda), (pb, ldb), (pc, ldc) = _fview(A), _fview(B), _fview(C)
    return _err(_lib.lib().mo_lp_gemm(context(), prec, m, n, k, alpha, pa, lda, pb, ldb, beta, pc,
                                      ldc, flags))


def SetSpinLimit(polls: int) -> int:
    """Polls a device-side wait on another CTA's step flag makes before it gives up with
    MO_EDEVTIMEOUT (see mo_set_spin_limit); returns the previous value."""
    old = ctypes.c_uint32(0)
    rc = _lib.lib().mo_set_spin_limit(context(), polls, ctypes.byref(old))
    if rc:
        raise RuntimeError(_lib.lib().mo_strerror(rc).decode())
    return old.value


def Sync() -> int:
    """Wait for the context's stream; returns the first device-side status recorded."""
    return _lib.lib().mo_sync(context())


# ---- host <-> device transfers through the C ABI (what a shim holding host matrices uses) ----

def _host_view(h: torch.Tensor):
    if h.dim() != 2 or h.dtype != torch.float64 or h.is_cuda:
        raise TypeError("expected a 2-D float64 host tensor")
    r, c = h.shape
    if r > 1 and h.stride(0) != 1:
        raise TypeError("host matrix must be column-major (stride(0) == 1)")
    ld = h.stride(1) if c > 1 else max(h.stride(1), r, 1)
    return h.data_ptr(), max(ld, r, 1)


def Upload(dst: torch.Tensor, src: torch.Tensor) -> None:
    """Asynchronous host -> device copy of a column-major matrix (mo_upload)."""
    ptr, ld = _host_view(src)
    rc = _lib.lib().mo_upload(context(), view(dst), ctypes.c_void_p(ptr), ld)
    if rc:
        raise RuntimeError(_lib.lib().mo_strerror(rc).decode())


def UploadTriangle(dst: torch.Tensor, src: torch.Tensor, flags: int = LOWER) -> None:
    """Asynchronous host -> device copy of the stored triangle (LOWER or UPPER in flags) of
    a square column-major matrix, in 128-column blocks (mo_upload_tri): what the symmetric
    solvers read, about half the bytes of Upload."""
    ptr, ld = _host_view(src)
    rc = _lib.lib().mo_upload_tri(context(), view(dst), ctypes.c_void_p(ptr), ld, flags)
    if rc:
        raise RuntimeError(_lib.lib().mo_strerror(rc).decode())


def Download(dst: torch.Tensor, src: torch.Tensor) -> None:
    """Asynchronous device -> host copy of a column-major matrix (mo_download)."""
    ptr, ld = _host_view(dst)
    rc = _lib.lib().mo_download(context(), ctypes.c_void_p(ptr), ld, view(src))
    if rc:
        raise RuntimeError(_lib.lib().mo_strerror(rc).decode())


def host_matrix(rows: int, cols: int, pinned: bool = True) -> torch.Tensor:
    """Column-major float64 host matrix (page-locked by default)."""
    return torch.empty((cols, rows), dtype=torch.float64, pin_memory=pinned).t()


class Profile:
    """Per-kernel-class launches / device time / algorithmic work (mo_profile)."""
    CLASSES = ("gemm", "diag", "trtri", "panel", "laswp", "other", "lpgemm", "ir", "batch")

    def __init__(self, raw):
        self.launches = {k: int(raw.launches[i]) for i, k in enumerate(self.CLASSES)}
        self.ms = {k: float(raw.ms[i]) for i, k in enumerate(self.CLASSES)}
        self.flops = {k: float(raw.flops[i]) for i, k in enumerate(self.CLASSES)}
        self.bytes = {k: float(raw.bytes[i]) for i, k in enumerate(self.CLASSES)}


def ProfileEnable(on: bool) -> None:
    _lib.lib().mo_profile_enable(context(), 1 if on else 0)


def ProfileRead() -> Profile:
    raw = _lib.MoProfile()
    rc = _lib.lib().mo_profile_read(context(), ctypes.byref(raw))
    if rc:
        raise RuntimeError(_lib.lib().mo_strerror(rc).decode())
    return Profile(raw)


def MeasureFP64Peak(ms: float = 200.0) -> float:
    """FP64 tensor-pipe TFLOP/s of this device (register-resident DMMA loop)."""
    out = ctypes.c_double(0.0)
    rc = _lib.lib().mo_measure_fp64_peak(context(), ms, ctypes.byref(out))
    if rc:
        raise RuntimeError(_lib.lib().mo_strerror(rc).decode())
    return out.value


# ---- batched factor + solve (no counterpart in the reference; one DecomposeCHOL /
# SolveCHOL or DecomposeLU / SolveLU per matrix there) ----

BATCH_CHOL, BATCH_LU = 1, 2
BATCH_MAX_N, BATCH_BUCKETS = 512, 4


class BatchPlan:
    """A reusable plan (mo_batch) for factoring, and optionally solving, many small
    systems of the given orders in one CUDA-graph launch.  run() takes lists of column-major
    CUDA float64 matrices (views allowed); their pointer arrays are cached on the device
    while the same list objects are passed again."""

    def __init__(self, kind: int, orders, nrhs: int = 0):
        import numpy as np
        self.kind, self.nrhs = kind, nrhs
        self.orders = np.ascontiguousarray(orders, dtype=np.int32)
        self._h = ctypes.c_void_p()
        rc = _lib.lib().mo_batch_create(context(), kind, len(self.orders),
                                        ctypes.c_void_p(self.orders.ctypes.data), nrhs,
                                        ctypes.byref(self._h))
        if rc:
            raise MatopsError(rc, _lib.lib().mo_strerror(rc).decode())
        self._arrays = None
        self._key = None

    def close(self):
        if self._h:
            _lib.lib().mo_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _pack(self, As, Bs, pivs):
        key = (tuple(a.data_ptr() for a in As), tuple(b.data_ptr() for b in Bs) if Bs else None,
               tuple(p.data_ptr() for p in pivs) if pivs else None)
        if key == self._key:
            return self._arrays
        dev = As[0].device if As else torch.device("cuda", torch.cuda.current_device())

        def ptrs(ts):
            return torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device=dev)

        def lds(ts):
            return torch.tensor([view(t).ld for t in ts], dtype=torch.int64, device=dev)
        for a, n in zip(As, self.orders):
            if tuple(a.shape) != (int(n), int(n)):
                raise ValueError("matrix shape does not match the plan's order")
        arr = {"A": ptrs(As), "lda": lds(As),
               "B": ptrs(Bs) if Bs else None, "ldb": lds(Bs) if Bs else None,
               "piv": ptrs(pivs) if pivs else None,
               "info": torch.zeros(len(As), dtype=torch.int32, device=dev)}
        self._arrays, self._key = arr, key
        return arr

    def run(self, As, Bs=None, pivs=None):
        """Factor every A (and solve A X = B in place when Bs is given).  pivs: list of CUDA
        int64 tensors (LU).  Returns the device int32 info tensor (0 = success)."""
        if len(As) != len(self.orders):
            raise ValueError("number of matrices does not match the plan")
        for a in As:
            view(a)
        if Bs is not None:
            for b, n in zip(Bs, self.orders):
                if view(b).rows != n or b.shape[1] != self.nrhs:
                    raise ValueError("right-hand side shape does not match the plan")
        arr = self._pack(As, Bs, pivs)

        def p(t):
            return ctypes.c_void_p(t.data_ptr()) if t is not None else None
        rc = _lib.lib().mo_batch_run(self._h, p(arr["A"]), p(arr["lda"]), p(arr["B"]),
                                     p(arr["ldb"]), p(arr["piv"]), p(arr["info"]))
        if rc:
            raise MatopsError(rc, _lib.lib().mo_strerror(rc).decode())
        return arr["info"]

    def tune(self, reps: int = 3):
        """Autotune the per-bucket kernel configuration; returns {bucket: [ms cfg0, ms cfg1]}."""
        ms = (ctypes.c_double * (BATCH_BUCKETS * 2))()
        rc = _lib.lib().mo_batch_tune(self._h, reps, ms)
        if rc:
            raise MatopsError(rc, _lib.lib().mo_strerror(rc).decode())
        return {b: [ms[2 * b], ms[2 * b + 1]] for b in range(BATCH_BUCKETS) if ms[2 * b] >= 0}

    def schedule(self, cfg=None):
        """Read (cfg None) or set the per-bucket configuration table."""
        arr = (ctypes.c_int * BATCH_BUCKETS)(*(cfg or [0] * BATCH_BUCKETS))
        rc = _lib.lib().mo_batch_schedule(self._h, arr, 1 if cfg is not None else 0)
        if rc:
            raise MatopsError(rc, _lib.lib().mo_strerror(rc).decode())
        return list(arr)


# ---- reverse mode (no counterpart in the reference) ----

def DecomposeCHOLAdjoint(L, Lbar, flags: int = LOWER):
    """Lbar (adjoint of the lower factor L of A = L L^T) is overwritten with the symmetric
    gradient of A.  Returns None or a MatopsError."""
    return _err(_lib.lib().mo_decompose_chol_adjoint(context(), view(L), view(Lbar), flags))


def DecomposeCHOLAdjointBatched(Ls, Lbars, flags: int = LOWER):
    """DecomposeCHOLAdjoint for lists of independent matrices (one call, a pool of streams)."""
    n = len(Ls)
    arrL = (_lib.MoMatrix * max(n, 1))(*[view(t) for t in Ls])
    arrG = (_lib.MoMatrix * max(n, 1))(*[view(t) for t in Lbars])
    return _err(_lib.lib().mo_decompose_chol_adjoint_batched(context(), n, arrL, arrG, flags))


def SolveCHOLAdjoint(L, X, Xbar, Abar, flags: int = LOWER):
    """Adjoint of X = A^-1 B (A = L L^T): Xbar becomes Bbar = A^-1 Xbar and
    Abar -= (Bbar X^T + X Bbar^T) / 2."""
    return _err(_lib.lib().mo_solve_chol_adjoint(context(), view(L), view(X), view(Xbar),
                                                 view(Abar), flags))


# ---- residency: device mirrors of host arrays (what a cgo shim over FloatMatrix uses) ----

class Mirror:
    """A registered host backing array (a float64 numpy array) with a device copy.

    `view(sub, write)` maps any column-major view `sub` of the array (a numpy slice, as a
    FloatMatrix view shares its parent's storage) to a device mo_matrix over the same
    elements, uploading first if the host copy is newer; `to_host()` downloads if a device
    view was written; `host_modified()` marks host-side edits.  Overlapping views share one
    device copy, so a chain of calls on views of one array needs no host round trip."""

    def __init__(self, host):
        import numpy as np
        if not isinstance(host, np.ndarray) or host.dtype != np.float64:
            raise TypeError("expected a float64 numpy array")
        self.host = host
        base = host
        while base.base is not None and isinstance(base.base, np.ndarray):
            base = base.base
        self._root = base
        self._h = ctypes.c_void_p()
        rc = _lib.lib().mo_mirror_create(context(), ctypes.c_void_p(base.ctypes.data),
                                         base.size, ctypes.byref(self._h))
        if rc:
            raise MatopsError(rc, _lib.lib().mo_strerror(rc).decode())

    def view(self, sub, write: bool = False) -> _lib.MoMatrix:
        r, c = sub.shape
        if r > 1 and sub.strides[0] != 8:
            raise TypeError("view must be column-major")
        ld = sub.strides[1] // 8 if c > 1 else max(r, 1)
        out = _lib.MoMatrix()
        rc = _lib.lib().mo_mirror_view(self._h, ctypes.c_void_p(sub.ctypes.data), r, c, max(ld, 1),
                                       1 if write else 0, ctypes.byref(out))
        if rc:
            raise MatopsError(rc, _lib.lib().mo_strerror(rc).decode())
        return out

    def to_host(self) -> None:
        rc = _lib.lib().mo_mirror_to_host(self._h)
        if rc:
            raise MatopsError(rc, _lib.lib().mo_strerror(rc).decode())

    def host_modified(self) -> int:
        return _lib.lib().mo_mirror_host_modified(self._h)

    @property
    def state(self) -> int:
        return _lib.lib().mo_mirror_state(self._h)

    @staticmethod
    def find(p):
        """(mirror handle, element offset) of the registered array containing numpy view p"""
        h, off = ctypes.c_void_p(), ctypes.c_int64()
        rc = _lib.lib().mo_mirror_find(ctypes.c_void_p(p.ctypes.data), ctypes.byref(h),
                                       ctypes.byref(off))
        return (h.value, off.value) if rc == 0 else (None, None)

    def close(self) -> None:
        if self._h:
            _lib.lib().mo_mirror_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
