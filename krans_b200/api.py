"""Host-side mirror of the reference's plug-in API over the CUDA engine.

Same names, argument meanings and error behaviour as Deep-SANE/krans:
  MatrixInterface  include/krans/MatrixInterface.hpp:10-24   -> CudaCsrMatrixAdapter
  VectorInterface  include/krans/VectorInterface.hpp:8-34    -> CudaVectorAdapter
  VectorFactory    include/krans/VectorFactory.hpp:9-23      -> CudaVectorFactory
  CyclicLanczosOptions/Result, find_nullspace_cyclic_lanczos[_ex]
                   include/krans/Solvers/CyclicLanczosSolver.hpp:77-178
  LOBPCGOptions/Result, find_nullspace_lobpcg[_ex]
                   include/krans/Solvers/LOBPCGSolver.hpp:68-149
Size or backend mismatches raise ValueError (std::invalid_argument in the
reference); solver failures raise KransError (std::runtime_error).
Everything runs on the GPU through libkrans_cuda.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _capi as K
from ._capi import check, load


class Context:
    """A device, its stream and an optional HBM budget (krans_ctx)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, tuning: bool = True):
        """tuning: apply the autotuner's table for this device
        (krans_b200/tuning/<device>.json) when one exists."""
        lib = load()
        h = C.c_void_p()
        check(lib.krans_ctx_create(device, hbm_budget, C.byref(h)), "krans_ctx_create")
        self.h = h
        self.lib = lib
        self.device = device
        self.tuning_table = None
        if tuning:
            from . import autotune
            self.tuning_table = autotune.apply_cached(self)

    def synchronize(self):
        check(self.lib.krans_ctx_synchronize(self.h), "synchronize")

    def memory_in_use(self) -> int:
        b = C.c_size_t()
        check(self.lib.krans_ctx_memory_in_use(self.h, C.byref(b)))
        return b.value

    def sm_count(self) -> int:
        s = C.c_int()
        check(self.lib.krans_ctx_sm_count(self.h, C.byref(s)))
        return s.value

    def set_batch_tuning(self, cluster_min: int = 0, pair_max: int = 0, cluster_size: int = 0, lanes=None):
        """Knobs of batched launches (krans_ctx_set_batch_tuning); 0 keeps the
        built-in value. lanes: 6 threads-per-row entries for mean row lengths
        <= 3, 8, 16, 32, 64 and above."""
        t = K.BatchTuning(cluster_min, pair_max, cluster_size, (C.c_int32 * 6)(*(lanes or [0] * 6)))
        check(self.lib.krans_ctx_set_batch_tuning(self.h, C.byref(t)), "set_batch_tuning")

    def batch_tuning(self) -> dict:
        t = K.BatchTuning()
        check(self.lib.krans_ctx_get_batch_tuning(self.h, C.byref(t)), "batch_tuning")
        return {"cluster_min": int(t.cluster_min), "pair_max": int(t.pair_max),
                "cluster_size": int(t.cluster_size), "lanes": [int(x) for x in t.lanes]}

    def stream_ptr(self) -> int:
        """The context's cudaStream_t (for ordering or timing caller work)."""
        p = C.c_void_p()
        check(self.lib.krans_ctx_stream(self.h, C.byref(p)))
        return int(p.value or 0)

    def close(self):
        if getattr(self, "h", None):
            self.lib.krans_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class CudaVectorAdapter:
    """VectorInterface over a device FP64 vector (krans_vec)."""

    def __init__(self, ctx: Context, n: int = 0, handle=None):
        self.ctx = ctx
        lib = ctx.lib
        if handle is None:
            h = C.c_void_p()
            check(lib.krans_vec_create(ctx.h, int(n), C.byref(h)), "krans_vec_create")
            self.h = h
            self.n = int(n)
        else:
            self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
            s = C.c_int64()
            check(lib.krans_vec_size(self.h, C.byref(s)))
            self.n = s.value

    @classmethod
    def from_numpy(cls, ctx: Context, x) -> "CudaVectorAdapter":
        x = np.ascontiguousarray(x, np.float64)
        v = cls(ctx, x.shape[0])
        check(ctx.lib.krans_vec_upload(v.h, _p(x), x.shape[0]), "upload")
        return v

    def _other(self, other, what):
        if not isinstance(other, CudaVectorAdapter):
            raise ValueError(f"CudaVectorAdapter::{what} backend mismatch")
        if other.n != self.n:
            raise ValueError(f"CudaVectorAdapter::{what} size mismatch")
        return other

    # --- VectorInterface ---------------------------------------------------
    def dot(self, other) -> float:
        o = self._other(other, "dot")
        r = C.c_double()
        check(self.ctx.lib.krans_vec_dot(self.h, o.h, C.byref(r)), "dot")
        return r.value

    def add_scaled(self, other, alpha: float):
        o = self._other(other, "add_scaled")
        check(self.ctx.lib.krans_vec_axpy(self.h, float(alpha), o.h), "add_scaled")

    def scale(self, alpha: float):
        check(self.ctx.lib.krans_vec_scale(self.h, float(alpha)), "scale")

    def normalize(self):
        check(self.ctx.lib.krans_vec_normalize(self.h), "normalize")

    def norm(self) -> float:
        r = C.c_double()
        check(self.ctx.lib.krans_vec_nrm2(self.h, C.byref(r)), "norm")
        return r.value

    def size(self) -> int:
        return self.n

    def set_zero(self):
        check(self.ctx.lib.krans_vec_fill(self.h, 0.0), "set_zero")

    def copy_from(self, other):
        o = self._other(other, "copy_from")
        check(self.ctx.lib.krans_vec_copy(self.h, o.h), "copy_from")

    def clone(self) -> "CudaVectorAdapter":
        h = C.c_void_p()
        check(self.ctx.lib.krans_vec_clone(self.h, C.byref(h)), "clone")
        return CudaVectorAdapter(self.ctx, handle=h)

    def data(self) -> np.ndarray:
        """Host copy of the entries (the reference's data() pointer)."""
        out = np.empty(self.n, np.float64)
        check(self.ctx.lib.krans_vec_download(self.h, _p(out), self.n), "download")
        return out

    def device_ptr(self) -> int:
        p = C.c_void_p()
        check(self.ctx.lib.krans_vec_device_ptr(self.h, C.byref(p)))
        return p.value or 0

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.ctx.lib.krans_vec_destroy(self.h)
                self.h = None
        except Exception:
            pass


class CudaCsrMatrixAdapter:
    """MatrixInterface over a device CSR matrix with a stored transpose
    (replaces EigenSparseMatrixAdapter, which caches A^T the same way)."""

    def __init__(self, ctx: Context, m: int, n: int, indptr, indices, data, fp32: bool = False):
        self.ctx = ctx
        indptr = np.ascontiguousarray(indptr, np.int32)
        indices = np.ascontiguousarray(indices, np.int32)
        data = np.ascontiguousarray(data, np.float64)
        nnz = int(indptr[-1]) if indptr.size else 0
        if indptr.shape[0] != m + 1 or indices.shape[0] < nnz or data.shape[0] < nnz:
            raise ValueError("CudaCsrMatrixAdapter: inconsistent CSR arrays")
        flags = K.KRANS_CSR_FP64 | (K.KRANS_CSR_FP32 if fp32 else 0)
        h = C.c_void_p()
        check(ctx.lib.krans_csr_create(ctx.h, m, n, nnz, _p(indptr), _p(indices), _p(data), flags,
                                       C.byref(h)), "krans_csr_create")
        self.h = h
        self.m, self.n, self.nnz = int(m), int(n), nnz
        self.fp32 = fp32

    @classmethod
    def load(cls, ctx: Context, path: str, fmt: int = K.KRANS_FMT_AUTO, fp32: bool = False) -> "CudaCsrMatrixAdapter":
        """A .mtx / .ija file (load_matrix_market / load_ija_triplet_matrix,
        src/IO/MatrixLoader.cpp:12-56) straight into a device matrix."""
        flags = K.KRANS_CSR_FP64 | (K.KRANS_CSR_FP32 if fp32 else 0)
        h = C.c_void_p()
        check(ctx.lib.krans_csr_load(ctx.h, os.fsencode(path), fmt, flags, C.byref(h)), "krans_csr_load")
        self = cls.__new__(cls)
        self.ctx = ctx
        self.h = h
        m, n, z = C.c_int64(), C.c_int64(), C.c_int64()
        check(ctx.lib.krans_csr_dims(h, C.byref(m), C.byref(n), C.byref(z)), "krans_csr_dims")
        self.m, self.n, self.nnz = m.value, n.value, z.value
        self.fp32 = fp32
        return self

    @classmethod
    def from_scipy(cls, ctx: Context, A, fp32: bool = False) -> "CudaCsrMatrixAdapter":
        A = A.tocsr()
        return cls(ctx, A.shape[0], A.shape[1], A.indptr, A.indices, A.data, fp32=fp32)

    def rows(self) -> int:
        return self.m

    def cols(self) -> int:
        return self.n

    def _chk(self, x, y, xs, ys, what):
        if not isinstance(x, CudaVectorAdapter) or not isinstance(y, CudaVectorAdapter):
            raise ValueError(f"CudaCsrMatrixAdapter::{what} backend mismatch")
        if x.n != xs or y.n != ys:
            raise ValueError(f"CudaCsrMatrixAdapter::{what} size mismatch")

    def multiply(self, x, y, precision: int = K.KRANS_PREC_FP64):
        self._chk(x, y, self.n, self.m, "multiply")
        check(self.ctx.lib.krans_spmv_ex(self.h, 0, precision, x.h, y.h), "multiply")

    def multiply_transpose(self, x, y, precision: int = K.KRANS_PREC_FP64):
        self._chk(x, y, self.m, self.n, "multiply_transpose")
        check(self.ctx.lib.krans_spmv_ex(self.h, 1, precision, x.h, y.h), "multiply_transpose")

    def set_spmv_tuning(self, trans: bool, kernel: int = K.KRANS_SPMV_AUTO, rows_per_block: int = 0,
                        x_evict_last: bool = False):
        """Kernel of multiply (trans False) / multiply_transpose (trans True):
        KRANS_SPMV_AUTO, _ROWTILE (rows_per_block rows per block, 0 = from the
        mean row length), _UNIFORM (rows of 1, 2 or 4 entries) or _LANES;
        x_evict_last: gather x with the L2 evict-last policy."""
        t = K.SpmvTuning(kernel, rows_per_block, int(bool(x_evict_last)), 0)
        check(self.ctx.lib.krans_csr_set_spmv_tuning(self.h, int(bool(trans)), C.byref(t)), "set_spmv_tuning")

    def spmv_tuning(self, trans: bool):
        t = K.SpmvTuning()
        check(self.ctx.lib.krans_csr_get_spmv_tuning(self.h, int(bool(trans)), C.byref(t)), "spmv_tuning")
        return int(t.kernel), int(t.rows_per_block)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.ctx.lib.krans_csr_destroy(self.h)
                self.h = None
        except Exception:
            pass


class CudaVectorFactory:
    """VectorFactory whose random vectors come from a device RNG stream.

    mode "mt19937" (default) reproduces std::mt19937(seed) +
    std::normal_distribution<double>(0,1), i.e. the reference's
    StdVectorFactory/EigenVectorFactory sequence; "philox" is a parallel
    counter-based stream. seed 0 draws a random seed, as in the reference."""

    def __init__(self, ctx: Context, default_size: int, seed: int = 0, mode: str = "mt19937"):
        self.ctx = ctx
        self.default_size = int(default_size)
        m = {"mt19937": K.KRANS_RNG_MT19937, "philox": K.KRANS_RNG_PHILOX}[mode]
        h = C.c_void_p()
        check(ctx.lib.krans_rng_create(ctx.h, seed & 0xFFFFFFFF, m, C.byref(h)), "krans_rng_create")
        self.h = h
        self.mode = mode

    def seed(self) -> int:
        s = C.c_uint32()
        check(self.ctx.lib.krans_rng_seed(self.h, C.byref(s)))
        return s.value

    def create_zero(self) -> CudaVectorAdapter:
        return self.create_zero_of_size(self.default_size)

    def create_random(self) -> CudaVectorAdapter:
        return self.create_random_of_size(self.default_size)

    def create_zero_of_size(self, n: int) -> CudaVectorAdapter:
        return CudaVectorAdapter(self.ctx, n)

    def create_random_of_size(self, n: int) -> CudaVectorAdapter:
        v = CudaVectorAdapter(self.ctx, n)
        check(self.ctx.lib.krans_rng_normal(self.h, v.h), "create_random_of_size")
        return v

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.ctx.lib.krans_rng_destroy(self.h)
                self.h = None
        except Exception:
            pass


# ---------------------------------------------------------------------------
# options / results (CyclicLanczosSolver.hpp:77-167, LOBPCGSolver.hpp:68-139)
# ---------------------------------------------------------------------------
class ReorthMode(enum.IntEnum):
    None_ = 0
    Single = 1
    Double = 2


class Precision(enum.IntEnum):
    FP64 = K.KRANS_PREC_FP64
    MIXED = K.KRANS_PREC_MIXED


class Precond(enum.IntEnum):
    """Device preconditioners (the device form of precond_AAt / M_inv)."""
    NONE = K.KRANS_PRECOND_NONE
    JACOBI = K.KRANS_PRECOND_JACOBI
    SD = K.KRANS_PRECOND_SD


@dataclass
class CyclicLanczosOptions:
    k: int = 1
    ncv: int = 48
    max_restarts: int = 80
    tol_abs: float = 1e-12
    tol_rel: float = 1e-10
    reorth: ReorthMode = ReorthMode.Double
    use_harmonic: bool = True
    target_tau: float = 0.0
    nullity_known: int = -1
    rank_known: int = -1
    initial_right_space: List[CudaVectorAdapter] = field(default_factory=list)
    cg_maxit: int = 80
    cg_rel_tol: float = 1e-10
    cg_breakdown_tol: float = 1e-30
    projector_passes: int = 1
    grad_max_iters: int = 3000
    frob_samples: int = 4
    prescreen_factor: float = 0.8
    stagnation_restarts: int = 30
    return_left_space: bool = False
    verbose: bool = False
    # engine knobs (no reference counterpart)
    precision: Precision = Precision.FP64
    team: int = K.KRANS_TEAM_AUTO
    precond_aat: Precond = Precond.NONE  # device form of precond_AAt (Precond.JACOBI or Precond.SD)
    precond_steps: int = 8                   # steps of the SD preconditioner
    polish_block: int = 0  # 1: block CG polish of up to 8 candidates at once
    # MIXED only: continue in FP64 when the mixed run stops short of k with its
    # FP64 polish at cg_maxit (single solves; not the batched/served paths)
    mixed_fallback: bool = True

    def to_c(self) -> K.CyclicOpts:
        o = K.CyclicOpts()
        load().krans_cyclic_opts_init(C.byref(o))
        for name, _ in K.CyclicOpts._fields_:
            v = getattr(self, name)
            setattr(o, name, int(v) if isinstance(v, (bool, enum.IntEnum)) else v)
        return o


@dataclass
class CyclicLanczosResult:
    right_null: List[CudaVectorAdapter]
    left_null: List[CudaVectorAdapter]
    restarts: int = 0
    krylov_steps_total: int = 0
    frob_norm_est: float = 0.0
    converged_to_target: bool = False
    cg_solves: int = 0
    cg_maxit_hits: int = 0
    spmv: int = 0
    spmvT: int = 0
    algo_bytes: float = 0.0
    device_ms: float = 0.0
    phase_ms: tuple = (0.0, 0.0, 0.0, 0.0)
    fp64_fallback: bool = False  # the mixed solve continued in FP64
    fallback_from: int = 0       # vectors the mixed run had accepted before that


@dataclass
class LOBPCGOptions:
    nev: int = 1
    block_size: int = 0
    max_iters: int = 1000
    tol_abs: float = 1e-12
    tol_rel: float = 1e-10
    soft_locking: bool = True
    restart: float = 0.9
    gs_tol: float = 1e-14
    gs_reorth: bool = True
    initial_block: List[CudaVectorAdapter] = field(default_factory=list)
    frob_samples: int = 4
    max_tiny_dim: int = 0
    nullity_known: int = -1
    rank_known: int = -1
    verbose: bool = False
    progress_every: int = 100
    precision: Precision = Precision.FP64
    team: int = K.KRANS_TEAM_AUTO
    precond_normal: Precond = Precond.NONE  # device form of M_inv (Precond.JACOBI or Precond.SD)
    precond_steps: int = 6                      # steps of the SD preconditioner

    def to_c(self) -> K.LobpcgOpts:
        o = K.LobpcgOpts()
        load().krans_lobpcg_opts_init(C.byref(o))
        for name, _ in K.LobpcgOpts._fields_:
            v = getattr(self, name)
            setattr(o, name, int(v) if isinstance(v, (bool, enum.IntEnum)) else v)
        return o


@dataclass
class LOBPCGResult:
    right_null: List[CudaVectorAdapter]
    theta: List[float] = field(default_factory=list)
    residuals_Av: List[float] = field(default_factory=list)
    iters: int = 0
    locked: int = 0
    frob_norm_est: float = 0.0
    accept_threshold: float = 0.0
    best_unaccepted_residual: float = 0.0
    block_size: int = 0
    converged_to_target: bool = False
    spmv: int = 0
    spmvT: int = 0
    algo_bytes: float = 0.0
    gram_flops: float = 0.0
    device_ms: float = 0.0
    phase_ms: tuple = ()
    final_polish_ms: float = 0.0  # part of the last phase: closing polish, sharpening and MGS


def _require(A, vf):
    if not isinstance(A, CudaCsrMatrixAdapter) or not isinstance(vf, CudaVectorFactory):
        raise ValueError("the device engine needs a CudaCsrMatrixAdapter and a CudaVectorFactory")
    if A.ctx is not vf.ctx:
        raise ValueError("matrix and factory belong to different contexts")


def find_nullspace_cyclic_lanczos_ex(A: CudaCsrMatrixAdapter, vf: CudaVectorFactory,
                                     opt: CyclicLanczosOptions) -> CyclicLanczosResult:
    """find_nullspace_cyclic_lanczos_ex (CyclicLanczosSolver.cpp:618-660) on the GPU."""
    _require(A, vf)
    ctx = A.ctx
    o = opt.to_c()
    k_target = opt.nullity_known if opt.nullity_known >= 0 else opt.k
    cap = max(int(k_target), int(opt.k), 1)
    right = (C.c_void_p * cap)()
    left = (C.c_void_p * max(int(opt.k), 1))()
    res = K.CyclicResultC()
    y0 = opt.initial_right_space[0].h if opt.initial_right_space else None
    check(ctx.lib.krans_solve_cyclic(ctx.h, A.h, vf.h, C.byref(o), y0,
                                     C.cast(right, K.PP), C.cast(left, K.PP), C.byref(res)),
          "find_nullspace_cyclic_lanczos")
    R = CyclicLanczosResult(
        right_null=[CudaVectorAdapter(ctx, handle=right[i]) for i in range(res.n_right)],
        left_null=[CudaVectorAdapter(ctx, handle=left[i]) for i in range(res.n_left)],
        restarts=res.restarts, krylov_steps_total=res.krylov_steps_total,
        frob_norm_est=res.frob_norm_est, converged_to_target=bool(res.converged_to_target),
        cg_solves=res.cg_solves, cg_maxit_hits=res.cg_maxit_hits, spmv=res.spmv,
        spmvT=res.spmvT, algo_bytes=res.algo_bytes, device_ms=res.device_ms,
        phase_ms=tuple(res.phase_ms), fp64_fallback=bool(res.fp64_fallback),
        fallback_from=res.fallback_from)
    return R


def find_nullspace_cyclic_lanczos(A, vf, opt) -> List[CudaVectorAdapter]:
    return find_nullspace_cyclic_lanczos_ex(A, vf, opt).right_null


def lobpcg_k_target(opt: LOBPCGOptions, n: int) -> int:
    k = max(1, int(opt.nev))
    if opt.nullity_known >= 0:
        k = int(opt.nullity_known)
    elif opt.rank_known >= 0:
        k = max(0, n - int(opt.rank_known))
    return k


def find_nullspace_lobpcg_ex(A: CudaCsrMatrixAdapter, vf: CudaVectorFactory,
                             opt: LOBPCGOptions) -> LOBPCGResult:
    """find_nullspace_lobpcg_ex (LOBPCGSolver.cpp:443-834) on the GPU."""
    _require(A, vf)
    ctx = A.ctx
    o = opt.to_c()
    cap = max(lobpcg_k_target(opt, A.n), 1)
    right = (C.c_void_p * cap)()
    theta = np.zeros(cap)
    resid = np.zeros(cap)
    res = K.LobpcgResultC()
    nin = len(opt.initial_block)
    init = (C.c_void_p * max(nin, 1))(*[v.h.value for v in opt.initial_block]) if nin else None
    check(ctx.lib.krans_solve_lobpcg(ctx.h, A.h, vf.h, C.byref(o),
                                     C.cast(init, K.PP) if nin else None, nin,
                                     C.cast(right, K.PP), _p(theta), _p(resid), C.byref(res)),
          "find_nullspace_lobpcg")
    nr = res.n_right
    return LOBPCGResult(
        right_null=[CudaVectorAdapter(ctx, handle=right[i]) for i in range(nr)],
        theta=list(theta[:nr]), residuals_Av=list(resid[:nr]), iters=res.iters,
        locked=res.locked, frob_norm_est=res.frob_norm_est,
        accept_threshold=res.accept_threshold,
        best_unaccepted_residual=res.best_unaccepted_residual, block_size=res.block_size,
        converged_to_target=bool(res.converged_to_target), spmv=res.spmv, spmvT=res.spmvT,
        algo_bytes=res.algo_bytes, gram_flops=res.gram_flops, device_ms=res.device_ms,
        phase_ms=tuple(res.phase_ms), final_polish_ms=res.final_polish_ms)


def find_nullspace_lobpcg(A, vf, opt) -> List[CudaVectorAdapter]:
    return find_nullspace_lobpcg_ex(A, vf, opt).right_null


def read_matrix(path: str, fmt: int = K.KRANS_FMT_AUTO):
    """Parse a .mtx / .ija file on the host (no GPU): scipy CSR matrix with the
    reference loader's rules (duplicates summed)."""
    import scipy.sparse as sp
    lib = load()
    m, n, z = C.c_int64(), C.c_int64(), C.c_int64()
    rp, ci, va = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)(), C.POINTER(C.c_double)()
    check(lib.krans_csr_read_host(os.fsencode(path), fmt, C.byref(m), C.byref(n), C.byref(z), C.byref(rp),
                                  C.byref(ci), C.byref(va)), "krans_csr_read_host")
    try:
        M, N, Z = m.value, n.value, z.value
        indptr = np.ctypeslib.as_array(rp, shape=(M + 1,)).copy()
        indices = np.ctypeslib.as_array(ci, shape=(max(Z, 1),))[:Z].copy()
        data = np.ctypeslib.as_array(va, shape=(max(Z, 1),))[:Z].copy()
    finally:
        lib.krans_host_free(C.cast(rp, C.c_void_p))
        lib.krans_host_free(C.cast(ci, C.c_void_p))
        lib.krans_host_free(C.cast(va, C.c_void_p))
    return sp.csr_matrix((data, indices, indptr), shape=(M, N))


def block_gram(ctx: Context, n: int, p: int, Z: int, ld: int, S: int, W: int = 0, G: int = 0) -> float:
    """S = Z^T Z (and G = Z^T W) for column-major n x p device blocks given by
    their addresses (krans_block_gram); returns the kernel's device ms."""
    ms = C.c_double()
    check(ctx.lib.krans_block_gram(ctx.h, n, p, Z, W or None, ld, S, G or None, C.byref(ms)), "krans_block_gram")
    return ms.value


def block_gemm_tn(ctx: Context, n: int, a: int, A: int, b: int, B: int, ld: int, Cm: int) -> float:
    """C = A^T B (a x b, column-major) for column-major n x a and n x b device
    blocks given by their addresses (krans_block_gemm_tn); returns the
    kernel's device ms."""
    ms = C.c_double()
    check(ctx.lib.krans_block_gemm_tn(ctx.h, n, a, A, b, B, ld, Cm, C.byref(ms)), "krans_block_gemm_tn")
    return ms.value


def block_combine(ctx: Context, n: int, zc: int, q: int, Z: int, ld: int, Cm: int, ldc: int, out: int) -> float:
    """out = Z C for a column-major n x zc device block and zc x q C
    (krans_block_combine); returns the kernel's device ms."""
    ms = C.c_double()
    check(ctx.lib.krans_block_combine(ctx.h, n, zc, q, Z, ld, Cm, ldc, out, C.byref(ms)), "krans_block_combine")
    return ms.value


def basis_to_numpy(vs: Sequence[CudaVectorAdapter]) -> np.ndarray:
    if not vs:
        return np.zeros((0, 0))
    return np.stack([v.data() for v in vs])
