"""KraNS-B200: a B200-native engine for the matrix-free null-space solvers of
Deep-SANE/krans (cyclic Lanczos / Golub-Kahan and block LOBPCG), reached
through the reference's MatrixInterface / VectorInterface / VectorFactory API.

The compute path is libkrans_cuda.so (hand-written sm_100a CUDA kernels, C ABI
in include/krans_cuda.h); this package is its Python host mirror.
"""
from ._capi import KransError, KransInvalidArgument  # noqa: F401
from .api import (  # noqa: F401
    Context, CudaCsrMatrixAdapter, CudaVectorAdapter, CudaVectorFactory,
    CyclicLanczosOptions, CyclicLanczosResult, LOBPCGOptions, LOBPCGResult,
    Precision, Precond, ReorthMode, basis_to_numpy, block_combine, block_gemm_tn, block_gram, default_context,
    find_nullspace_cyclic_lanczos, find_nullspace_cyclic_lanczos_ex,
    find_nullspace_lobpcg, find_nullspace_lobpcg_ex, read_matrix,
)

__all__ = [
    "Context", "CudaCsrMatrixAdapter", "CudaVectorAdapter", "CudaVectorFactory",
    "CyclicLanczosOptions", "CyclicLanczosResult", "LOBPCGOptions", "LOBPCGResult",
    "Precision", "Precond", "ReorthMode", "KransError", "KransInvalidArgument", "basis_to_numpy",
    "block_combine", "block_gemm_tn", "block_gram",
    "default_context", "find_nullspace_cyclic_lanczos", "find_nullspace_cyclic_lanczos_ex",
    "find_nullspace_lobpcg", "find_nullspace_lobpcg_ex", "read_matrix",
]
