#!/usr/bin/env python
"""Benchmark: Cholesky solve at n = 16384 (64 RHS) on B200, mixed precision + FP64
refinement against the plain FP64 path on the same system.

System: A = G*G^T/n + 0.5*I (G iid N(0,1), seed 2), B iid U[-1,1] (seed 3), generated on
the device.  Through the C ABI (libmatops_b200.so):
  headline step  SolveCHOLMixed: BF16x3 split-product Cholesky on the tensor cores (FP32
                 accumulation and storage, FP64 diagonal blocks; --prec tf32x3 for the
                 TF32 split), FP64 residuals and updates until the normwise backward error
                 is <= 1e-14 (A is read, not modified; 2 GiB > L2 per step)
  fp64_path      DecomposeCHOL + SolveCHOL in FP64 on fresh copies of A

Reported on one JSON line (rank 0):
  value / ms_per_step   device time of one headline step (CUDA events, max over ranks)
  roofline              the dominant kernel of the step, the tcgen05 split-product GEMM:
                        its algorithmic bytes / summed event time vs measured HBM bandwidth
                        (with its tensor-pipe fraction beside)
  e2e                   the headline step through the public API with HOST buffers: upload
                        A's lower triangle and B (pinned), solve, download X
  cpu_baseline          the reference's own C kernels (oracle/_ref) on this host (FP64
                        DecomposeCHOL + SolveCHOL; the reference has no mixed precision), on a
                        bounded sample scaled to n = 16384
  extras                DGEMM 2048^3 (alpha 1.5, beta -0.5) as % of FP64 peak; LU + SolveLU;
                        the kappa sweep of the mixed solve; batched and adjoint workloads

--impl reference times the reference's CPU path alone (rank 0) and prints its line.
Multi-GPU (torchrun): independent replicas, one system per rank, no collective in the path.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Cholesky solve s at n=16384, mixed+IR vs FP64 at err≤1e-14; DGEMM % FP64 peak"
LOWER = 0x4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--nrhs", type=int, default=64)
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--prec", default="bf16x3", choices=["tf32x3", "bf16x3"],
                    help="split format of the headline's low-precision factor (BF16x3 measured "
                         "35.8 ms vs TF32x3 37.2 ms at n=16384, both 3 corrections)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--case", default=None,
                    help="profiling aid: run one operation instead of the benchmark, e.g. "
                         "dgemm:M:N:K:flags, dsyrk:N:K, dpotrf:N, dgetrf:N (W+K calls)")
    return ap.parse_args()


def run_case(args):
    """Run a single operation W+K times (for ncu captures); prints its mean device time."""
    import torch

    import matops_b200 as mo
    kind, *dims = args.case.split(":")
    dims = [int(x) for x in dims]
    g = torch.Generator(device="cuda").manual_seed(1)
    if kind == "dgemm":
        m, n, k, fl = dims
        A = mo.matrix(k, m) if fl & 1 else mo.matrix(m, k)
        B = mo.matrix(n, k) if fl & 2 else mo.matrix(k, n)
        C = mo.matrix(m, n)
        for t in (A, B, C):
            t.uniform_(-1.0, 1.0, generator=g)
        fn, flops = (lambda: mo.Mult(C, A, B, 1.5, -0.5, fl)), 2.0 * m * n * k
    elif kind == "dsyrk":
        n, k = dims
        A, C = mo.matrix(n, k), mo.matrix(n, n)
        A.uniform_(-1.0, 1.0, generator=g)
        C.uniform_(-1.0, 1.0, generator=g)
        fn, flops = (lambda: mo.RankUpdateSym(C, A, -1.0, 1.0, LOWER)), float(n) * n * k
    elif kind == "dpotrs":
        n, nrhs = dims
        G = mo.matrix(n, n)
        G.normal_(generator=g)
        A = mo.matrix(n, n)
        mo.Mult(A, G, G, 1.0 / n, 0.0, mo.TRANSB)
        A.diagonal().add_(0.5)
        del G
        mo.DecomposeCHOL(A, LOWER, 64)
        B0 = mo.matrix(n, nrhs)
        B0.uniform_(-1.0, 1.0, generator=g)
        B = mo.matrix(n, nrhs)

        def fn():
            B.copy_(B0)
            mo.SolveCHOL(B, A, LOWER)
        flops = 2.0 * 2.0 * n * n * nrhs
    elif kind == "dsposv":
        # dsposv:N:NRHS:KAPPA_EXP -- mixed vs FP64 Cholesky solve, both precisions
        n, nrhs, kexp = dims
        res = mixed_leg(mo, n, nrhs, [10.0 ** kexp], [mo.PREC_TF32X3, mo.PREC_BF16X3],
                        torch.device("cuda", torch.cuda.current_device()), reps=max(1, args.steps))
        print(json.dumps({"case": args.case, **res}), flush=True)
        return 0
    elif kind == "mixed":
        # mixed:N:NRHS[:PREC] -- SolveCHOLMixed on A = G G^T/n + 0.5 I (PREC 2 = TF32x3, 1 = BF16x3)
        n, nrhs = dims[0], dims[1]
        prec = dims[2] if len(dims) > 2 else mo.PREC_TF32X3
        G = mo.matrix(n, n)
        G.normal_(generator=g)
        A = mo.matrix(n, n)
        mo.Mult(A, G, G, 1.0 / n, 0.0, mo.TRANSB)
        A.diagonal().add_(0.5)
        del G
        B = mo.matrix(n, nrhs)
        B.uniform_(-1.0, 1.0, generator=g)
        X = mo.matrix(n, nrhs)

        def fn():
            info, err = mo.SolveCHOLMixed(X, A, B, LOWER, prec, mo.IR_AUTO, 1e-14, 40)
            assert err is None and info.converged
        flops = n ** 3 / 3.0
    elif kind == "adjoint":
        res = adjoint_leg(mo, torch.device("cuda", torch.cuda.current_device()),
                          reps=max(1, args.steps))
        print(json.dumps({"case": args.case, **res}), flush=True)
        return 0
    elif kind == "batched":
        # batched:KIND:COUNT[:TUNE] -- config 4 (KIND 1 = Cholesky, 2 = LU; TUNE 0 skips
        # the autotuner)
        bk, cnt = dims[0], dims[1]
        tune = dims[2] != 0 if len(dims) > 2 else True
        res, _ = batched_leg(mo, bk, cnt, 8 if bk == 1 else 9,
                             torch.device("cuda", torch.cuda.current_device()),
                             reps=max(1, args.steps), tune=tune)
        print(json.dumps({"case": args.case, **res}), flush=True)
        return 0
    elif kind == "dsytrf":
        # dsytrf:N -- DecomposeBK (Bunch-Kaufman, LOWER) of an N x N symmetric uniform matrix
        n = dims[0]
        A0 = mo.matrix(n, n)
        A0.uniform_(-1.0, 1.0, generator=g)
        A0.copy_(A0 + A0.t())
        A, W = mo.matrix(n, n), mo.matrix(n, 2)
        piv = torch.zeros(n, dtype=torch.int64, device="cuda")

        def fn():
            A.copy_(A0)
            assert mo.DecomposeBK(A, W, piv, LOWER, 0)[1] is None
        flops = n ** 3 / 3.0
    elif kind == "dgeqrt":
        # dgeqrt:N -- DecomposeQRT of an N x N iid N(0,1) matrix
        n = dims[0]
        A0 = mo.matrix(n, n)
        A0.normal_(generator=g)
        A, T = mo.matrix(n, n), mo.matrix(n, n)

        def fn():
            A.copy_(A0)
            assert mo.DecomposeQRT(A, T, None, 0)[1] is None
        flops = 4.0 * n ** 3 / 3.0
    elif kind in ("dpotrf", "dgetrf"):
        n = dims[0]
        A0 = mo.matrix(n, n)
        A0.normal_(generator=g)
        if kind == "dpotrf":
            G = A0.clone()
            mo.Mult(A0, G, G, 1.0 / n, 0.0, mo.TRANSB)
            A0.diagonal().add_(0.5)
            del G
        A = mo.matrix(n, n)
        piv = torch.zeros(n, dtype=torch.int64, device="cuda")

        def fn():
            A.copy_(A0)
            if kind == "dpotrf":
                mo.DecomposeCHOL(A, LOWER, 64)
            else:
                mo.DecomposeLU(A, piv, 64)
        flops = n ** 3 / 3.0 if kind == "dpotrf" else 2.0 * n ** 3 / 3.0
    else:
        raise SystemExit(f"unknown case {kind}")
    for _ in range(args.warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        fn()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    print(json.dumps({"case": args.case, "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}), flush=True)
    return 0


def kappa_spd(mo, n, kappa, seed, dev):
    """A = Q diag(s) Q^T, Q from the Householder QR of an iid N(0,1) matrix (seed) -- this
    package's DecomposeQRT + MultQT (qrwy.go:517, qrwym.go:646) applied to the identity --
    and s log-spaced from 1 to kappa; built on the device in FP64."""
    import torch
    g = torch.Generator(device=dev).manual_seed(seed)
    F = mo.matrix(n, n)
    F.copy_(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
    T = mo.matrix(n, n)
    assert mo.DecomposeQRT(F, T, None, 0)[1] is None
    Qc = mo.matrix(n, n)
    Qc.zero_()
    Qc.diagonal().fill_(1.0)
    assert mo.MultQT(Qc, F, T, mo.matrix(n, 128), mo.LEFT, 128) is None
    del F, T
    s = torch.logspace(0, float(torch.log10(torch.tensor(kappa))), n, dtype=torch.float64,
                       device=dev)
    QS = mo.matrix(n, n)
    QS.copy_(Qc * s.unsqueeze(0))
    A = mo.matrix(n, n)
    assert mo.Mult(A, QS, Qc, 1.0, 0.0, mo.TRANSB) is None
    del QS, Qc
    A.copy_((A + A.t()) * 0.5)
    return A


def qr_leg(mo, dev, n, fp64_peak, nrhs=64, reps=3):
    """DecomposeQRT (qrwy.go:517) of an n x n iid N(0,1) matrix and the least-squares
    SolveQRT (qrwym.go:784) of nrhs right-hand sides with it, FP64 on the device, timed with
    CUDA events; ||A - Q R|| / ||A|| from MultQT on R."""
    import torch
    g = torch.Generator(device=dev).manual_seed(6)
    A0 = mo.matrix(n, n)
    A0.copy_(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
    B0 = mo.matrix(n, nrhs)
    B0.uniform_(-1.0, 1.0, generator=g)
    A, T, B = mo.matrix(n, n), mo.matrix(n, n), mo.matrix(n, nrhs)
    W = mo.matrix(nrhs, n)  # the reference's workspace rule: B.cols x T.cols
    fts, sts = [], []
    for it in range(reps + 1):
        A.copy_(A0)
        T.zero_()
        B.copy_(B0)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        assert mo.DecomposeQRT(A, T, None, 0)[1] is None
        ev[1].record()
        assert mo.SolveQRT(B, A, T, W, 0, 0) is None
        ev[2].record()
        torch.cuda.synchronize()
        if it:
            fts.append(ev[0].elapsed_time(ev[1]))
            sts.append(ev[1].elapsed_time(ev[2]))
    f_ms, s_ms = min(fts), min(sts)
    R = mo.matrix(n, n)
    R.copy_(torch.triu(A))
    assert mo.MultQT(R, A, T, mo.matrix(n, 128), mo.LEFT, 128) is None
    residual = float(torch.linalg.norm(R - A0) / torch.linalg.norm(A0))
    del R
    Rb = B0.clone()
    assert mo.Mult(Rb, A0, B, -1.0, 1.0, 0) is None
    berr = float(torch.linalg.norm(Rb) / (torch.linalg.norm(A0) * torch.linalg.norm(B)
                                          + torch.linalg.norm(B0)))
    fp64 = fp64_peak
    geqrf, with_t = 4.0 * n ** 3 / 3.0, 2.0 * n ** 3
    return {"n": n, "factor_ms": f_ms, "factor_tflops": geqrf / (f_ms * 1e-3) / 1e12,
            "factor_tflops_incl_T": with_t / (f_ms * 1e-3) / 1e12,
            "frac_fp64_peak_incl_T": with_t / (f_ms * 1e-3) / 1e12 / fp64,
            "solve_ms": s_ms, "nrhs": nrhs, "residual_A_minus_QR": residual, "solve_berr": berr,
            "flops": "4n^3/3 (DGEQRF count); incl_T adds the n^3 x 2/3 of the full block "
                     "reflector T that DecomposeQRT returns"}


def ldl_leg(mo, dev, n=4096, nrhs=64, reps=2):
    """DecomposeLDLnoPiv / DecomposeLDL / DecomposeBK (ldlnp.go:211, ldl.go:439,
    ldlbk.go:1114) of an n x n symmetric matrix (uniform, + 2n I for the unpivoted form) and
    the matching solves of nrhs right-hand sides; CUDA events, residual checked with Mult."""
    import torch
    g = torch.Generator(device=dev).manual_seed(11)
    S = mo.matrix(n, n)
    S.uniform_(-1.0, 1.0, generator=g)
    S.copy_(S + S.t())
    B0 = mo.matrix(n, nrhs)
    B0.uniform_(-1.0, 1.0, generator=g)
    A, B = mo.matrix(n, n), mo.matrix(n, nrhs)
    piv = torch.zeros(n, dtype=torch.int64, device=dev)
    W = mo.matrix(n, 2)
    out = {"n": n, "nrhs": nrhs}
    for kind in ("nopiv", "ldl", "bk"):
        Sk = S.clone() if kind != "nopiv" else S + 2.0 * n * torch.eye(n, dtype=torch.float64, device=dev)
        Sc = mo.matrix(n, n)
        Sc.copy_(Sk)
        del Sk
        fts, sts = [], []
        for it in range(reps + 1):
            A.copy_(Sc)
            B.copy_(B0)
            torch.cuda.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record()
            if kind == "nopiv":
                assert mo.DecomposeLDLnoPiv(A, None, LOWER, 0)[1] is None
            elif kind == "ldl":
                assert mo.DecomposeLDL(A, None, piv, LOWER, 0)[1] is None
            else:
                assert mo.DecomposeBK(A, W, piv, LOWER, 0)[1] is None
            ev[1].record()
            if kind == "nopiv":
                assert mo.SolveLDLnoPiv(B, A, LOWER) is None
            elif kind == "ldl":
                assert mo.SolveLDL(B, A, piv, LOWER) is None
            else:
                assert mo.SolveBK(B, A, piv, LOWER) is None
            ev[2].record()
            torch.cuda.synchronize()
            if it:
                fts.append(ev[0].elapsed_time(ev[1]))
                sts.append(ev[1].elapsed_time(ev[2]))
        R = B0.clone()
        assert mo.Mult(R, Sc, B, -1.0, 1.0, 0) is None
        berr = float(torch.linalg.norm(R) / (torch.linalg.norm(Sc) * torch.linalg.norm(B)
                                             + torch.linalg.norm(B0)))
        out[kind] = {"factor_ms": min(fts), "solve_ms": min(sts),
                     "factor_tflops": n ** 3 / 3.0 / (min(fts) * 1e-3) / 1e12, "solve_berr": berr}
        if kind == "bk":
            out[kind]["two_by_two_blocks"] = int((piv < 0).sum().item()) // 2
        del Sc
    return out


def mixed_leg(mo, n, nrhs, kappas, precs, dev, reps=2):
    """Mixed-precision + FP64-refined Cholesky solve against the FP64 path on the same
    A = Q diag(s) Q^T (seed 6) and B ~ N(0,1) (seed 7): time, iterations, backward and
    forward error per (kappa, prec)."""
    import torch
    B = mo.matrix(n, nrhs)
    B.normal_(generator=torch.Generator(device=dev).manual_seed(7))
    out = {}
    for kappa in kappas:
        A = kappa_spd(mo, n, kappa, 6, dev)
        Af = mo.matrix(n, n)
        Xf = mo.matrix(n, nrhs)
        tf = []
        for _ in range(reps):
            Af.copy_(A)
            Xf.copy_(B)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            _, err = mo.DecomposeCHOL(Af, LOWER, 64)
            assert err is None
            mo.SolveCHOL(Xf, Af, LOWER)
            b.record()
            torch.cuda.synchronize()
            tf.append(a.elapsed_time(b))
        del Af
        an = float(A.abs().sum(1).max())

        def berr(X):
            R = B.clone()
            mo.Mult(R, A, X, -1.0, 1.0, 0)
            return max(float(R[:, c].abs().max() / (an * X[:, c].abs().max() + B[:, c].abs().max()))
                       for c in range(nrhs))
        row = {"fp64_ms": min(tf), "fp64_berr": berr(Xf)}
        for prec in precs:
            X = mo.matrix(n, nrhs)
            tm, info = [], None
            for _ in range(reps):
                torch.cuda.synchronize()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                info, err = mo.SolveCHOLMixed(X, A, B, LOWER, prec, mo.IR_AUTO, 1e-14, 40)
                b.record()
                torch.cuda.synchronize()
                assert err is None, err
                tm.append(a.elapsed_time(b))
            # one more solve with per-kernel-class tracing (not part of the timing above)
            mo.ProfileRead()
            mo.ProfileEnable(True)
            mo.SolveCHOLMixed(X, A, B, LOWER, prec, mo.IR_AUTO, 1e-14, 40)
            prof = mo.ProfileRead()
            mo.ProfileEnable(False)
            by_class = {k: {"ms": round(v, 3), "launches": prof.launches[k]}
                        for k, v in prof.ms.items() if prof.launches[k]}
            name = "tf32x3" if prec == mo.PREC_TF32X3 else "bf16x3"
            row[name] = {"ms": min(tm), "speedup_vs_fp64": min(tf) / min(tm),
                         "iters": info.iters, "gmres_iters": info.gmres_iters,
                         "method": "gmres" if info.method == mo.IR_GMRES else "classic",
                         "fallback": info.fallback, "abandoned": info.abandoned,
                         "converged": info.converged, "prec_used": info.prec,
                         "berr_history": info.history,
                         "shift": info.shift, "berr": info.berr, "berr_check": berr(X),
                         "ferr_vs_fp64": float((X - Xf).norm() / Xf.norm()),
                         "traced_ms_by_class": by_class}
            del X
        out[f"kappa={kappa:.0e}"] = row
        del A, Xf
        torch.cuda.empty_cache()
    return out


def batched_leg(mo, kind, count, seed, dev, reps=5, tune=True):
    """Config 4: `count` systems with n_i ~ U{16..512} (seed), 1 RHS each; SPD
    A_i = G_i G_i^T / n_i + I for Cholesky, iid N(0,1) for LU.  All matrices live in one
    flat device buffer; each timed run factors and solves a fresh copy (one D2D copy
    outside the timed region)."""
    import numpy as np
    import torch
    rng = np.random.default_rng(seed)
    sizes = rng.integers(16, 513, count).astype(np.int32)
    offs = np.concatenate([[0], np.cumsum(sizes.astype(np.int64) ** 2)])
    g = torch.Generator(device=dev).manual_seed(seed)
    flat0 = torch.empty(int(offs[-1]), dtype=torch.float64, device=dev)
    rhs0 = torch.empty(int(sizes.sum()), dtype=torch.float64, device=dev)
    roffs = np.concatenate([[0], np.cumsum(sizes.astype(np.int64))])

    def mats(flat):
        return [flat[offs[i]:offs[i + 1]].view(int(n), int(n)).t() for i, n in enumerate(sizes)]

    def vecs(flat):
        return [flat[roffs[i]:roffs[i + 1]].view(1, int(n)).t() for i, n in enumerate(sizes)]
    for a, n in zip(mats(flat0), sizes):
        G = torch.randn(int(n), int(n), dtype=torch.float64, device=dev, generator=g)
        if kind == mo.BATCH_CHOL:
            a.copy_(G @ G.t() / float(n))
            a.diagonal().add_(1.0)
        else:
            a.copy_(G)
    rhs0.normal_(generator=g)
    flat, rhs = flat0.clone(), rhs0.clone()
    As, Bs = mats(flat), vecs(rhs)
    pivs = [torch.zeros(int(n), dtype=torch.int64, device=dev) for n in sizes] \
        if kind == mo.BATCH_LU else None
    plan = mo.BatchPlan(kind, sizes, 1)
    tune_ms = plan.tune(2) if tune else None
    ts = []
    for r in range(reps + 1):
        flat.copy_(flat0)
        rhs.copy_(rhs0)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        info = plan.run(As, Bs, pivs)
        b.record()
        torch.cuda.synchronize()
        if r > 0:
            ts.append(a.elapsed_time(b))
    ok = int((info != 0).sum())
    # backward error of every 64th system against the untouched copy
    worst = 0.0
    A0s, B0s = mats(flat0), vecs(rhs0)
    for i in range(0, count, 64):
        r_ = B0s[i] - A0s[i] @ Bs[i]
        worst = max(worst, float(r_.norm() / (A0s[i].norm() * Bs[i].norm() + B0s[i].norm())))
    ms = min(ts)
    flops = float(np.sum(sizes.astype(np.float64) ** 3)) * (1 if kind == mo.BATCH_CHOL else 2) / 3 \
        + float(np.sum(2.0 * sizes.astype(np.float64) ** 2))
    byts = float(np.sum(16.0 * sizes.astype(np.float64) ** 2 + 16.0 * sizes))
    out = {"ms": ms, "gflops": flops / (ms * 1e-3) / 1e9, "tflops": flops / (ms * 1e-3) / 1e12,
           "gbs": byts / (ms * 1e-3) / 1e9, "failed": ok, "berr_sample_max": worst,
           "schedule": plan.schedule(), "tune_ms": tune_ms, "count": count,
           "sizes": "n_i ~ U{16..512}", "flops": flops, "bytes": byts}
    plan.close()
    return out, (sizes, mats(flat0), vecs(rhs0))


def adjoint_leg(mo, dev, n_single=8192, batch=512, n_batch=256, reps=3):
    """Config 5: forward (DecomposeCHOL + SolveCHOL) and reverse (Cholesky adjoint + solve
    adjoint) of loss = sum(W*L) + 2 sum(log diag L) + w^T x in FP64, A = G G^T / n + I;
    single n = 8192 and a batch of 512 x n = 256.  Device time of forward and backward."""
    import torch
    res = {}
    g = torch.Generator(device=dev).manual_seed(10)

    def problem(n):
        G = mo.matrix(n, n)
        G.normal_(generator=g)
        A = mo.matrix(n, n)
        assert mo.Mult(A, G, G, 1.0 / n, 0.0, mo.TRANSB) is None
        A.diagonal().add_(1.0)
        W = torch.randn(n, n, dtype=torch.float64, device=dev, generator=g)
        b = mo.matrix(n, 1)
        b.normal_(generator=g)
        w = mo.matrix(n, 1)
        w.normal_(generator=g)
        return A, W, b, w

    def ev():
        return torch.cuda.Event(enable_timing=True)
    # single
    n = n_single
    A, W, b, w = problem(n)
    L, x, G, xb, Ab = mo.matrix(n, n), mo.matrix(n, 1), mo.matrix(n, n), mo.matrix(n, 1), mo.matrix(n, n)
    tf, tb = [], []
    for r in range(reps + 1):
        L.copy_(A)
        x.copy_(b)
        torch.cuda.synchronize()
        e0, e1, e2 = ev(), ev(), ev()
        e0.record()
        _, err = mo.DecomposeCHOL(L, LOWER, 64)
        assert err is None
        mo.SolveCHOL(x, L, LOWER)
        e1.record()
        # Lbar = tril(W) + 2 diag(1/L_ii), xbar = w
        G.copy_(torch.tril(W))
        G.diagonal().add_(2.0 / L.diagonal())
        xb.copy_(w)
        Ab.zero_()
        assert mo.SolveCHOLAdjoint(L, x, xb, Ab, LOWER) is None
        assert mo.DecomposeCHOLAdjoint(L, G, LOWER) is None
        G.add_(Ab)
        e2.record()
        torch.cuda.synchronize()
        if r > 0:
            tf.append(e0.elapsed_time(e1))
            tb.append(e1.elapsed_time(e2))
    fl_f = n ** 3 / 3 + 2.0 * n * n
    fl_b = 2 * n ** 3 / 3 + 6.0 * n * n
    res["single_8192"] = {"forward_ms": min(tf), "backward_ms": min(tb),
                          "forward_tflops": fl_f / (min(tf) * 1e-3) / 1e12,
                          "backward_tflops": fl_b / (min(tb) * 1e-3) / 1e12,
                          "grad_symmetric": bool(torch.equal(G, G.t()))}
    del A, W, b, w, L, x, G, xb, Ab
    torch.cuda.empty_cache()
    # batch: forward by the batched factor + solve plan, reverse by the batched adjoint
    nb_ = n_batch
    probs = [problem(nb_) for _ in range(batch)]
    Ls = [mo.matrix(nb_, nb_) for _ in range(batch)]
    xs = [mo.matrix(nb_, 1) for _ in range(batch)]
    Gs = [mo.matrix(nb_, nb_) for _ in range(batch)]
    plan = mo.BatchPlan(mo.BATCH_CHOL, [nb_] * batch, 1)
    tf, tb = [], []
    for r in range(reps + 1):
        for (A, W, b, w), L, x in zip(probs, Ls, xs):
            L.copy_(A)
            x.copy_(b)
        torch.cuda.synchronize()
        e0, e1, e2 = ev(), ev(), ev()
        e0.record()
        info = plan.run(Ls, xs)
        e1.record()
        for (A, W, b, w), L, G in zip(probs, Ls, Gs):
            G.copy_(torch.tril(W))
        assert mo.DecomposeCHOLAdjointBatched(Ls, Gs, LOWER) is None
        e2.record()
        torch.cuda.synchronize()
        assert int(info.abs().sum()) == 0
        if r > 0:
            tf.append(e0.elapsed_time(e1))
            tb.append(e1.elapsed_time(e2))
    plan.close()
    res["batch_512x256"] = {"forward_ms": min(tf), "backward_ms_incl_Lbar_setup": min(tb),
                            "forward_tflops": batch * (nb_ ** 3 / 3) / (min(tf) * 1e-3) / 1e12,
                            "backward_tflops": batch * (2 * nb_ ** 3 / 3) / (min(tb) * 1e-3) / 1e12}
    return res


def workload(n, nrhs):
    return (f"Cholesky solve, n={n}, {nrhs} RHS, A=G*G^T/n+0.5I (G~N(0,1) seed 2), "
            f"B~U[-1,1] seed 3: mixed-precision factor + FP64 refinement to berr<=1e-14 "
            f"(value), DecomposeCHOL+SolveCHOL FP64 (fp64_path)")


def _measured_peak(key, fallback):
    """(value, source): the pool's measured peak from MEASURED_PEAKS.json, else the earlier
    measurement on this pool that stands in for it (6.65 TB/s, 1.59 PFLOP/s bf16)."""
    try:
        v = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))[key])
        return v, f"MEASURED_PEAKS.json {key} (measured)"
    except Exception:
        return fallback, f"fallback {fallback:g} (MEASURED_PEAKS.json absent)"


# --------------------------------------------------------------------------------------
# CPU side: the reference's kernels (oracle/_ref) or, if they were not built, the oracle
# --------------------------------------------------------------------------------------

def cpu_sample(n_s: int, nrhs: int, reps: int):
    """Time DecomposeCHOL + SolveCHOL at n_s on the host; returns (best factor s, best
    solve s, kind, threads)."""
    import numpy as np

    from oracle.oracle import Oracle, ref_available
    kind = "reference" if ref_available() else "port"
    orc = Oracle("ref" if kind == "reference" else "port")
    cores = os.cpu_count() or 1
    orc.NumWorkers(cores)  # the reference parallelizes only Mult (mmult.go:241-255)
    rng = np.random.default_rng(2)
    ld = n_s + (n_s % 2)
    g = rng.standard_normal((n_s, n_s))
    A0 = np.zeros((ld, n_s), order="F")
    A0[:n_s] = g @ g.T / n_s + 0.5 * np.eye(n_s)
    B0 = np.zeros((ld, nrhs), order="F")
    B0[:n_s] = np.random.default_rng(3).uniform(-1, 1, (n_s, nrhs))
    tf, ts = [], []
    for _ in range(reps):
        A = A0.copy(order="F")[:n_s]
        B = B0.copy(order="F")[:n_s]
        t0 = time.perf_counter()
        assert orc.DecomposeCHOL(A, LOWER, 64) == 0
        t1 = time.perf_counter()
        orc.SolveCHOL(B, A, LOWER)
        t2 = time.perf_counter()
        tf.append(t1 - t0)
        ts.append(t2 - t1)
    return min(tf), min(ts), kind, 1  # the Cholesky path runs on one thread


def scaled_cpu_seconds(n, n_s, tf, ts):
    return tf * (n / n_s) ** 3 + ts * (n / n_s) ** 2


def reference_inputs(n, nrhs):
    """The headline system for the CPU arm, column-major float64 host arrays: A = G G^T/n +
    0.5 I (G iid N(0,1), seed 2) and B iid U[-1,1] (seed 3).  G G^T is formed on the GPU
    when one is present (torch, input preparation only: nothing of this repository's engine
    runs on the reference arm), else by numpy."""
    import numpy as np
    g = np.random.default_rng(2).standard_normal((n, n))
    try:
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError
        gt = torch.from_numpy(g).cuda()
        a = (gt @ gt.T / n).cpu().numpy()
        del gt
        torch.cuda.empty_cache()
    except Exception:
        a = g @ g.T / n
    del g
    a[np.diag_indices(n)] += 0.5
    A = np.asfortranarray(a)
    del a
    B = np.asfortranarray(np.random.default_rng(3).uniform(-1, 1, (nrhs, n)).T)
    return A, B


def run_reference(args, rank):
    """The reference's own CPU path (oracle/_ref: its calgo C kernels under the Go driver
    bodies restated in C; NumWorkers = host cores, nb = 64): ONE full DecomposeCHOL +
    SolveCHOL at the configured n, timed in K slices.  Step k runs the block steps of
    blockedCHOL (chol.go:58-94) whose first column lies in slice k of [0, n); the last step
    also runs SolveCHOL (chol.go:147-158).  The K slices run in order on the same matrix, so
    together they are exactly one factor + solve; value = their summed wall time.  Warm-up
    steps factor a separate n = 1024 system."""
    if rank != 0:
        return 0
    import numpy as np

    from oracle.oracle import Oracle, ref_available
    kind = "reference" if ref_available() else "port"
    orc = Oracle("ref" if kind == "reference" else "port")
    cores = os.cpu_count() or 1
    orc.NumWorkers(cores)  # the reference parallelizes only Mult (mmult.go:241-255)
    n, nrhs, nb, K = args.n, args.nrhs, 64, args.steps
    for _ in range(args.warmup):
        Aw, Bw = reference_inputs(1024, nrhs)
        assert orc.DecomposeCHOL(Aw, LOWER, nb) == 0
        orc.SolveCHOL(Bw, Aw, LOWER)
    A, B = reference_inputs(n, nrhs)
    nblk = (n + nb - 1) // nb
    bounds = [nb * ((nblk * k) // K) for k in range(K)] + [n]
    times = []
    for k in range(K):
        t0 = time.perf_counter()
        if bounds[k] < bounds[k + 1]:
            assert orc.DecomposeCHOLSteps(A, LOWER, nb, bounds[k], bounds[k + 1]) == 0
        if k == K - 1:
            orc.SolveCHOL(B, A, LOWER)
        times.append(time.perf_counter() - t0)
    v = sum(times)
    X = B
    del A
    sample = (f"one full DecomposeCHOL+SolveCHOL at n={n}, nb={nb}, {nrhs} RHS, timed in "
              f"{K} consecutive slices of blockedCHOL's block steps (the last one with the "
              f"solve); value = the sum")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
        "steps": K, "warmup": args.warmup, "ms_per_step": v * 1e3 / K,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": workload(n, nrhs), "n": n, "nrhs": nrhs, "nb": nb,
                   "parallelism": "host cores (only Mult is threaded in the reference)"},
        "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": kind, "sample": sample,
                         "num_workers": cores},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_s": times,
        "x_norm": float(np.linalg.norm(X)),
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------------------
# replicas: one independent system per rank, no collective in the data path; the ranks
# only meet at barriers and for the max over ranks of the device time
# --------------------------------------------------------------------------------------

def rank_barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def rank_max(x: float, world: int, device) -> float:
    """Max over ranks of a per-rank time (the slowest replica sets the job's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------------------
# clocks during the timed region (NVML, read-only)
# --------------------------------------------------------------------------------------

class ClockSampler:
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, torch_dev):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            import torch
            bus = torch.cuda.get_device_properties(torch_dev).pci_bus_id
            dom = torch.cuda.get_device_properties(torch_dev).pci_domain_id
            dev = torch.cuda.get_device_properties(torch_dev).pci_device_id
            pci = f"{dom:08X}:{bus:02X}:{dev:02X}.0"
            try:
                self._h = pynvml.nvmlDeviceGetHandleByPciBusId(pci)
            except Exception:
                self._h = pynvml.nvmlDeviceGetHandleByIndex(0)
            self._nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._h = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.1)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._h is not None:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        s = sorted(self.samples)
        return {"sm_mhz": s[len(s) // 2], "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(s)}


# --------------------------------------------------------------------------------------
# GPU side
# --------------------------------------------------------------------------------------

def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.case:
        return run_case(args)

    import torch
    import torch.distributed as dist

    import matops_b200 as mo

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)

    def barrier():
        rank_barrier(world)

    def max_over_ranks(x: float) -> float:
        return rank_max(x, world, dev)

    n, nrhs, K, W = args.n, args.nrhs, args.steps, args.warmup
    fp64_peak = mo.MeasureFP64Peak(300.0)

    # inputs, generated on the device (G G^T costs 8.8 TFLOP)
    g = torch.Generator(device=dev).manual_seed(2)
    G = mo.matrix(n, n)
    G.normal_(generator=g)
    A0 = mo.matrix(n, n)
    assert mo.Mult(A0, G, G, 1.0 / n, 0.0, mo.TRANSB) is None
    A0.diagonal().add_(0.5)
    del G
    B0 = mo.matrix(n, nrhs)
    B0.uniform_(-1.0, 1.0, generator=torch.Generator(device=dev).manual_seed(3))
    nsteps = W + K
    copies_bytes = nsteps * n * n * 8
    free = torch.cuda.mem_get_info(dev)[0]
    fresh = copies_bytes < 0.6 * free
    As = [A0.clone() for _ in range(nsteps)] if fresh else [mo.matrix(n, n)]
    Bs = [B0.clone() for _ in range(nsteps)]

    # ---- the comparison arm: the plain FP64 path, DecomposeCHOL + SolveCHOL ----
    def step(i):
        A = As[i] if fresh else As[0]
        if not fresh:
            A.copy_(A0)
        _, err = mo.DecomposeCHOL(A, LOWER, 64)
        assert err is None, err
        mo.SolveCHOL(Bs[i], A, LOWER)

    for i in range(W):
        step(i)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    e0.record()
    for i in range(W, nsteps):
        step(i)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    fp64_ms = max_over_ranks(e0.elapsed_time(e1) / K)
    X = Bs[nsteps - 1]
    # parity at the configured order: ||A - L L^T||_F / ||A||_F of the FP64 factor (torch
    # matmul as the checker)
    Lf = torch.tril(As[nsteps - 1] if fresh else As[0])
    parity = {"chol_residual": float(torch.linalg.norm(A0 - Lf @ Lf.T) / torch.linalg.norm(A0)),
              "bound_10n_eps": 10 * n * 2.0 ** -52}
    del Lf
    R = B0.clone()
    assert mo.Mult(R, A0, X, -1.0, 1.0, 0) is None
    fp64_berr = float(R.norm() / (A0.norm() * X.norm() + B0.norm()))
    # one more step, untimed, with per-kernel-class tracing (CUDA events around each launch)
    As[0].copy_(A0)
    Bs[0].copy_(B0)
    torch.cuda.synchronize()
    mo.ProfileRead()
    mo.ProfileEnable(True)
    step(0)
    prof64 = mo.ProfileRead()
    mo.ProfileEnable(False)
    del As, Bs, R
    torch.cuda.empty_cache()
    g_ms, g_fl = prof64.ms["gemm"], prof64.flops["gemm"]
    fp64_path = {
        "ms": fp64_ms, "berr": fp64_berr, "tflops": n ** 3 / 3 / (fp64_ms * 1e-3) / 1e12,
        "frac_fp64_peak": n ** 3 / 3 / (fp64_ms * 1e-3) / 1e12 / fp64_peak,
        "gemm_engine_tflops": g_fl / (g_ms * 1e-3) / 1e12 if g_ms else None,
        "per_class_ms_traced_step": {k: v for k, v in prof64.ms.items() if prof64.launches[k]},
        "launches_per_step": sum(prof64.launches.values()),
    }

    # ---- the headline: split-product factor + FP64 refinement to berr <= 1e-14, same A, B ----
    hprec = mo.PREC_TF32X3 if args.prec == "tf32x3" else mo.PREC_BF16X3
    Xm = mo.matrix(n, nrhs)

    def mstep():
        info, err = mo.SolveCHOLMixed(Xm, A0, B0, LOWER, hprec, mo.IR_AUTO, 1e-14, 40)
        assert err is None and info.converged and not info.fallback, (err, info)
        return info

    for _ in range(W):
        mstep()
    torch.cuda.synchronize()
    barrier()
    mo.ProfileRead()  # resets the launch counters (tracing stays off while timing)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    infos = []
    with ClockSampler(dev) as clk:
        e0.record()
        for _ in range(K):
            infos.append(mstep())
        e1.record()
        torch.cuda.synchronize()
    barrier()
    timed_launches = mo.ProfileRead().launches
    ms = max_over_ranks(e0.elapsed_time(e1) / K)
    # per-kernel-class device time from extra, untimed steps with tracing on
    PT = 2
    mo.ProfileEnable(True)
    for _ in range(PT):
        mstep()
    prof = mo.ProfileRead()
    mo.ProfileEnable(False)
    R = B0.clone()
    assert mo.Mult(R, A0, Xm, -1.0, 1.0, 0) is None
    berr = float(R.norm() / (A0.norm() * Xm.norm() + B0.norm()))
    del R

    # roofline of the dominant kernel, the tcgen05 split-product GEMM (lp_gemm_tc_kernel):
    # bytes = its C tile read + write and operand reads, flops = the three products
    l_ms, l_fl, l_by = prof.ms["lpgemm"] / PT, prof.flops["lpgemm"] / PT, prof.bytes["lpgemm"] / PT
    l_n = prof.launches["lpgemm"] / PT
    hbm_peak, hbm_src = _measured_peak("hbm_gbs", 6650.0)
    bf16_peak, bf16_src = _measured_peak("bf16_tflops", 1590.0)
    achieved_gbs = l_by / (l_ms * 1e-3) / 1e9 if l_ms else 0.0
    achieved_tf = l_fl / (l_ms * 1e-3) / 1e12 if l_ms else 0.0
    # DRAM traffic per launch: the measured traffic / algorithmic-bytes ratio of the ncu
    # capture summarized in profiles/lp_gemm_tc_kernel_traffic.md, times this run's
    # algorithmic bytes per launch
    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"lp_gemm_tc_kernel_traffic_{args.prec}.md")
    if not os.path.exists(tpath):
        tpath = os.path.join(ROOT, "profiles", "lp_gemm_tc_kernel_traffic.md")
    if os.path.exists(tpath) and l_n:
        for ln in open(tpath):
            if ln.startswith("traffic_over_algorithmic:"):
                traffic = float(ln.split(":")[1]) * l_by / l_n
    roofline = {
        "bound": "hbm", "kernel": f"lp_gemm_tc_kernel ({args.prec.upper()} trailing updates and panels)",
        "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
        "frac": achieved_gbs / hbm_peak, "traffic": traffic,
        "traffic_source": os.path.relpath(tpath, ROOT) if traffic is not None else None,
        "peak_source": hbm_src,
        "algorithmic_bytes_per_launch": l_by / l_n if l_n else None,
        "avg_launch_ms": l_ms / l_n if l_n else None,
        "tensor": ({"achieved_tflops": achieved_tf, "tf32_dense_peak_tflops": bf16_peak / 2,
                    "frac": achieved_tf / (bf16_peak / 2),
                    "peak_source": f"half of {bf16_src} (TF32 runs at half the BF16 rate)"}
                   if args.prec == "tf32x3" else
                   {"achieved_tflops": achieved_tf, "bf16_dense_peak_tflops": bf16_peak,
                    "frac": achieved_tf / bf16_peak,
                    "peak_source": bf16_src}),
        "share_of_step": l_ms / ms if ms else None,
        "per_class_ms_per_traced_step": {k: v / PT for k, v in prof.ms.items() if prof.launches[k]},
        "note": "achieved and per-class times come from 2 extra steps traced with CUDA events "
                "around every launch; the headline value is timed with tracing off",
    }

    # ---- e2e: host buffers through the public API ----
    e2e = None
    if not args.no_e2e:
        Ah = mo.host_matrix(n, n)
        Bh = mo.host_matrix(n, nrhs)
        Ah.copy_(A0.cpu())
        Bh.copy_(B0.cpu())
        Ad = mo.matrix(n, n)
        Bd = mo.matrix(n, nrhs)
        Xd = mo.matrix(n, nrhs)
        Xh = mo.host_matrix(n, nrhs)

        # the solver reads A's lower triangle only: upload that (128-column blocks)
        tri_elems = sum((n - j0) * min(128, n - j0) for j0 in range(0, n, 128))

        def e2e_step():
            mo.UploadTriangle(Ad, Ah, LOWER)
            mo.Upload(Bd, Bh)
            info, err = mo.SolveCHOLMixed(Xd, Ad, Bd, LOWER, hprec, mo.IR_AUTO, 1e-14, 40)
            assert err is None and info.converged
            mo.Download(Xh, Xd)

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        ke = max(1, min(K, 3))
        for _ in range(ke):
            e2e_step()
        f1.record()
        torch.cuda.synchronize()
        barrier()
        e_ms = max_over_ranks(f0.elapsed_time(f1) / ke)
        e2e = {"value": e_ms * 1e-3, "unit": "s", "h2d_bytes_per_step": 8 * (tri_elems + n * nrhs),
               "d2h_bytes_per_step": 8 * n * nrhs, "steps": ke,
               "what": "pinned host A, B -> upload (A: its lower triangle, the part the solver "
                       f"reads), SolveCHOLMixed ({args.prec.upper()} + FP64 refinement), download X"}
        del Ah, Bh, Ad, Bd, Xd, Xh

    # ---- extras: DGEMM 2048^3 and LU at n ----
    extras = {"mixed_ir": None}
    if not args.no_extras:
        m = 2048
        ga = torch.Generator(device=dev).manual_seed(1)
        Ag, Bg, Cg = mo.matrix(m, m), mo.matrix(m, m), mo.matrix(m, m)
        for t in (Ag, Bg, Cg):
            t.uniform_(-1.0, 1.0, generator=ga)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
        ts = []
        for it in range(3 + 10):
            flush.fill_(float(it))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            mo.Mult(Cg, Ag, Bg, 1.5, -0.5, 0)
            b.record()
            torch.cuda.synchronize()
            if it >= 3:
                ts.append(a.elapsed_time(b))
        gm = sorted(ts)[len(ts) // 2]
        gtf = 2 * m ** 3 / (gm * 1e-3) / 1e12
        extras["dgemm_2048"] = {"ms": gm, "tflops": gtf, "frac_fp64_peak": gtf / fp64_peak,
                                "alpha": 1.5, "beta": -0.5, "l2": "flushed (256 MiB write) between calls"}
        del Ag, Bg, Cg, flush
        # LU + SolveLU at n on the reference's golden input (numpy PCG64 seed 4, column by
        # column; 64 RHS U[-1,1] seed 5): the pivot vector is compared with the reference's
        # own run (tests/golden/n16384.npz) and ||PA - LU|| is checked with torch matmul
        import numpy as np
        L0 = mo.to_device(np.random.default_rng(4).standard_normal((n, n)).T)
        Lb0 = mo.to_device(np.random.default_rng(5).uniform(-1, 1, (nrhs, n)).T)
        LA, LB = mo.matrix(n, n), mo.matrix(n, nrhs)
        piv = torch.zeros(n, dtype=torch.int64, device=dev)
        lts = []
        for it in range(3):
            LA.copy_(L0)
            LB.copy_(Lb0)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            _, err = mo.DecomposeLU(LA, piv, 64)
            assert err is None
            assert mo.SolveLU(LB, LA, piv, 0) is None
            b.record()
            torch.cuda.synchronize()
            lts.append(a.elapsed_time(b))
        R = Lb0.clone()
        mo.Mult(R, L0, LB, -1.0, 1.0, 0)
        lberr = float(R.norm() / (L0.norm() * LB.norm() + Lb0.norm()))
        lms = min(lts[1:])
        extras["lu_16384"] = {"s": lms * 1e-3, "factor_tflops": 2 * n ** 3 / 3 / (lms * 1e-3) / 1e12,
                              "berr": lberr}
        pv = piv.cpu().numpy()
        perm = np.arange(n)
        for k in range(n):  # row interchanges in order (pivot.go:55-61)
            j = int(pv[k])
            perm[k], perm[j] = perm[j], perm[k]
        del R
        Lu = torch.tril(LA, -1)
        Lu.diagonal().fill_(1.0)
        parity["lu_residual"] = float(torch.linalg.norm(L0[torch.from_numpy(perm).to(dev)] - Lu @ torch.triu(LA))
                                      / torch.linalg.norm(L0))
        del Lu
        gpath = os.path.join(ROOT, "tests", "golden", "n16384.npz")
        if os.path.exists(gpath):
            gold = np.load(gpath)
            if int(gold["n"]) == n:
                d = np.flatnonzero(pv != gold["lu_piv"])
                parity["lu_pivots_vs_reference"] = {
                    "identical": bool(d.size == 0), "differing": int(d.size),
                    "reference": "tests/golden/n16384.npz (oracle/_ref DecomposeLU, nb=64)"}
        del L0, Lb0, LA, LB
        torch.cuda.empty_cache()
        extras["ldl"] = ldl_leg(mo, dev)
        torch.cuda.empty_cache()
        extras["qr"] = {}
        for nq in sorted({min(8192, n), n}):
            extras["qr"][f"n={nq}"] = qr_leg(mo, dev, nq, fp64_peak)
            torch.cuda.empty_cache()
        # the mixed-precision configuration: n in {8192, 16384}, 16 RHS, kappa sweep, both
        # split formats (A = Q diag(s) Q^T, Q from Householder QR, s log-spaced 1..kappa)
        extras["mixed_ir"] = {}
        for nm in sorted({min(8192, n), n}):
            extras["mixed_ir"][f"n={nm}"] = mixed_leg(mo, nm, 16, [1e2, 1e6, 1e10],
                                                      [mo.PREC_TF32X3, mo.PREC_BF16X3], dev)
            torch.cuda.empty_cache()
        torch.cuda.empty_cache()
        extras["batched_chol_4096"], _ = batched_leg(mo, mo.BATCH_CHOL, 4096, 8, dev, reps=3)
        extras["batched_lu_4096"], _ = batched_leg(mo, mo.BATCH_LU, 4096, 9, dev, reps=3)
        torch.cuda.empty_cache()
        extras["adjoint"] = adjoint_leg(mo, dev)

    # ---- CPU baseline (rank 0, one GPU only) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        n_s = min(n, 4096)
        tf, ts_, kind, cores = cpu_sample(n_s, nrhs, 2)
        cpu = {"value": scaled_cpu_seconds(n, n_s, tf, ts_), "unit": "s", "cores": cores,
               "kind": kind, "num_workers": os.cpu_count(),
               "sample": f"DecomposeCHOL+SolveCHOL at n={n_s}, {nrhs} RHS, best of 2; factor "
                         f"scaled by (n/{n_s})^3 and solve by (n/{n_s})^2 to n={n} (a bounded "
                         f"sample; `bench.py --impl reference` times one full n={n} solve)",
               "sample_s": tf + ts_}

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms * 1e-3, "unit": "s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": f"{args.prec}+f64", "data": "synthetic",
            "config": {"workload": workload(n, nrhs), "n": n, "nrhs": nrhs,
                       "factor": f"{args.prec.upper()} split products, FP32 storage, FP32 128x128 diagonal blocks",
                       "refinement": "FP64 residual and update, classic IR / GMRES-IR (auto), tol 1e-14",
                       "l2": "A (2 GiB FP64) is re-read from HBM by every step (inputs > L2)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "berr": berr, "berr_inf": max(i.berr for i in infos),
            "ir_iters": [i.iters for i in infos], "gmres_iters": [i.gmres_iters for i in infos],
            "ir_berr_history": infos[0].history,
            "fp64_path": fp64_path, "speedup_vs_fp64": fp64_ms / ms, "parity": parity,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(sum(timed_launches.values())),
            "gpu_launches_by_class": timed_launches,
            "clocks": clk.summary(), "fp64_peak_tflops": fp64_peak, "extras": extras,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
