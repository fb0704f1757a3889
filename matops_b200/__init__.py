"""matops_b200: B200 (sm_100a) implementation of hrautila/matops's level-3 hot path.

GEMM / SYRK / TRSM and the blocked Cholesky / LU factorizations and solves in FP64 on
device-resident column-major matrices, behind a C ABI (include/matops_b200.h) and this
Go-API mirror (see matops_b200.api).
"""
from .api import (  # noqa: F401
    LEFT, LOWER, NONE, NOTRANS, RIGHT, TRANS, TRANSA, TRANSB, UNIT, UPPER,
    BlockingParams, DecomposeBlockSize, DecomposeCHOL, DecomposeLU, MatopsError, MatopsPanic,
    Mult, NumWorkers, RankUpdateSym, SetPanicOnError, SolveCHOL, SolveLU, SolveTrm, Sync,
    matrix, to_device, view, Upload, UploadTriangle, Download, host_matrix, Profile, ProfileEnable, ProfileRead,
    MeasureFP64Peak, PREC_BF16X3, PREC_TF32X3, IR_AUTO, IR_CLASSIC, IR_GMRES, IR_NO_FALLBACK,
    IRInfo, SolveCHOLMixed, LPGemm, BATCH_CHOL, BATCH_LU, BATCH_MAX_N, BatchPlan,
    DecomposeCHOLAdjoint, DecomposeCHOLAdjointBatched, SolveCHOLAdjoint, SetSpinLimit, Mirror,
    context, MultSym, MultTrm, RankUpdate2Sym, UpdateTrm, InverseTrm,
    DecomposeQRT, DecomposeQR, BuildT, MultQT, MultQ, SolveQRT, SolveQR, BuildQ, BuildQT,
    DecomposeLDLnoPiv, SolveLDLnoPiv, DecomposeLDL, SolveLDL, DecomposeBK, SolveBK,
)
