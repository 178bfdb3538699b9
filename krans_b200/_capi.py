"""ctypes binding of libkrans_cuda.so (the C ABI declared in include/krans_cuda.h)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkrans_cuda.so")

KRANS_OK = 0
KRANS_ERR_INVALID_ARGUMENT = -1
KRANS_ERR_RUNTIME = -2
KRANS_ERR_CUDA = -3
KRANS_ERR_OUT_OF_MEMORY = -4
KRANS_ERR_TIMEOUT = -5
KRANS_ERR_NOT_FOUND = -6
KRANS_ERR_CANCELLED = -7

KRANS_CSR_FP64 = 1
KRANS_CSR_FP32 = 2
KRANS_RNG_MT19937 = 0
KRANS_RNG_PHILOX = 1
KRANS_PREC_FP64 = 0
KRANS_PREC_MIXED = 1
KRANS_PRECOND_NONE = 0
KRANS_PRECOND_JACOBI = 1
KRANS_PRECOND_SD = 2
KRANS_FMT_AUTO = 0
KRANS_FMT_MTX = 1
KRANS_FMT_IJA = 2
KRANS_TEAM_AUTO = 0
KRANS_TEAM_CTA = 1
KRANS_TEAM_GRID = 2
KRANS_SOLVER_CYCLIC = 0
KRANS_SOLVER_LOBPCG = 1
KRANS_SPMV_AUTO = 0
KRANS_SPMV_ROWTILE = 1
KRANS_SPMV_UNIFORM = 2
KRANS_SPMV_LANES = 3


class KransError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class KransInvalidArgument(KransError, ValueError):
    """std::invalid_argument in the reference."""


class SpmvTuning(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("rows_per_block", C.c_int32), ("x_evict_last", C.c_int32),
                ("reserved", C.c_int32)]


class BatchTuning(C.Structure):
    _fields_ = [("cluster_min", C.c_int64), ("pair_max", C.c_int64), ("cluster_size", C.c_int32),
                ("lanes", C.c_int32 * 6)]


class CyclicOpts(C.Structure):
    _fields_ = [("k", C.c_int64), ("ncv", C.c_int64), ("max_restarts", C.c_int64),
                ("tol_abs", C.c_double), ("tol_rel", C.c_double),
                ("reorth", C.c_int32), ("use_harmonic", C.c_int32), ("target_tau", C.c_double),
                ("nullity_known", C.c_int32), ("rank_known", C.c_int32),
                ("cg_maxit", C.c_int64), ("cg_rel_tol", C.c_double), ("cg_breakdown_tol", C.c_double),
                ("projector_passes", C.c_int32), ("grad_max_iters", C.c_int32),
                ("frob_samples", C.c_int32), ("prescreen_factor", C.c_double),
                ("stagnation_restarts", C.c_int64), ("return_left_space", C.c_int32),
                ("verbose", C.c_int32), ("precision", C.c_int32), ("team", C.c_int32),
                ("precond_aat", C.c_int32), ("precond_steps", C.c_int32), ("polish_block", C.c_int32),
                ("mixed_fallback", C.c_int32)]


class CyclicResultC(C.Structure):
    _fields_ = [("n_right", C.c_int64), ("n_left", C.c_int64), ("restarts", C.c_int64),
                ("krylov_steps_total", C.c_int64), ("frob_norm_est", C.c_double),
                ("converged_to_target", C.c_int32), ("status", C.c_int32),
                ("cg_solves", C.c_int64), ("cg_maxit_hits", C.c_int64),
                ("spmv", C.c_int64), ("spmvT", C.c_int64), ("algo_bytes", C.c_double),
                ("device_ms", C.c_double), ("phase_ms", C.c_double * 4),
                ("fp64_fallback", C.c_int32), ("fallback_from", C.c_int32)]


class LobpcgOpts(C.Structure):
    _fields_ = [("nev", C.c_int64), ("block_size", C.c_int64), ("max_iters", C.c_int64),
                ("tol_abs", C.c_double), ("tol_rel", C.c_double), ("soft_locking", C.c_int32),
                ("restart", C.c_double), ("gs_tol", C.c_double), ("gs_reorth", C.c_int32),
                ("frob_samples", C.c_int32), ("max_tiny_dim", C.c_int64),
                ("nullity_known", C.c_int32), ("rank_known", C.c_int32), ("verbose", C.c_int32),
                ("progress_every", C.c_int64), ("precision", C.c_int32), ("team", C.c_int32),
                ("precond_normal", C.c_int32), ("precond_steps", C.c_int32)]


class LobpcgResultC(C.Structure):
    _fields_ = [("n_right", C.c_int64), ("iters", C.c_int64), ("locked", C.c_int64),
                ("frob_norm_est", C.c_double), ("accept_threshold", C.c_double),
                ("best_unaccepted_residual", C.c_double), ("block_size", C.c_int64),
                ("converged_to_target", C.c_int32), ("status", C.c_int32),
                ("spmv", C.c_int64), ("spmvT", C.c_int64), ("algo_bytes", C.c_double),
                ("gram_flops", C.c_double), ("device_ms", C.c_double), ("phase_ms", C.c_double * 5),
                ("final_polish_ms", C.c_double)]


class Request(C.Structure):
    _fields_ = [("A", C.c_void_p), ("opts", CyclicOpts), ("seed", C.c_uint32),
                ("rng_mode", C.c_int32), ("basis_out", C.c_void_p), ("basis_capacity", C.c_int64),
                ("solver", C.c_int32), ("reserved", C.c_int32), ("lobpcg", LobpcgOpts)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("converged_to_target", C.c_int32), ("n_right", C.c_int64),
                ("restarts", C.c_int64), ("krylov_steps_total", C.c_int64),
                ("cg_solves", C.c_int64), ("cg_maxit_hits", C.c_int64),
                ("spmv", C.c_int64), ("spmvT", C.c_int64), ("frob_norm_est", C.c_double),
                ("max_residual", C.c_double), ("algo_bytes", C.c_double),
                ("queue_ms", C.c_double), ("device_ms", C.c_double), ("latency_ms", C.c_double),
                ("phase_ms", C.c_double * 4), ("launch_id", C.c_int64)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_inflight_launches", C.c_int32),
                ("max_batch", C.c_int32), ("batch_window_ms", C.c_double)]


P = C.c_void_p
PP = C.POINTER(C.c_void_p)
I = C.c_int
I64 = C.c_int64
D = C.c_double

# name -> argtypes (restype int unless listed in _RESTYPE)
SIGNATURES = {
    "krans_last_error": [],
    "krans_version": [],
    "krans_abi_sizes": [C.POINTER(I64), C.c_int],
    "krans_ctx_create": [I, C.c_size_t, PP],
    "krans_ctx_destroy": [P],
    "krans_ctx_synchronize": [P],
    "krans_ctx_memory_in_use": [P, C.POINTER(C.c_size_t)],
    "krans_ctx_sm_count": [P, C.POINTER(I)],
    "krans_ctx_stream": [P, PP],
    "krans_ctx_set_batch_tuning": [P, C.POINTER(BatchTuning)],
    "krans_ctx_get_batch_tuning": [P, C.POINTER(BatchTuning)],
    "krans_csr_create": [P, I64, I64, I64, P, P, P, I, PP],
    "krans_csr_destroy": [P],
    "krans_selftest_barrier_timeout": [P, D, C.POINTER(I), C.POINTER(D)],
    "krans_csr_read_host": [C.c_char_p, I, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64),
                            C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_int32)),
                            C.POINTER(C.POINTER(C.c_double))],
    "krans_host_free": [P],
    "krans_csr_load": [P, C.c_char_p, I, I, PP],
    "krans_csr_dims": [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)],
    "krans_csr_device_arrays": [P, I, PP, PP, PP, PP],
    "krans_vec_create": [P, I64, PP],
    "krans_vec_destroy": [P],
    "krans_vec_size": [P, C.POINTER(I64)],
    "krans_vec_device_ptr": [P, PP],
    "krans_vec_upload": [P, P, I64],
    "krans_vec_download": [P, P, I64],
    "krans_vec_dot": [P, P, C.POINTER(D)],
    "krans_vec_axpy": [P, D, P],
    "krans_vec_scale": [P, D],
    "krans_vec_nrm2": [P, C.POINTER(D)],
    "krans_vec_normalize": [P],
    "krans_vec_fill": [P, D],
    "krans_vec_copy": [P, P],
    "krans_vec_clone": [P, PP],
    "krans_vec_dot_noalloc": [P, P, I64, P, P],
    "krans_spmv": [P, I, P, P],
    "krans_spmv_ex": [P, I, I, P, P],
    "krans_block_gram": [P, I64, I64, P, P, I64, P, P, C.POINTER(D)],
    "krans_block_gemm_tn": [P, I64, I64, P, I64, P, I64, P, C.POINTER(D)],
    "krans_block_combine": [P, I64, I64, I64, P, I64, P, I64, P, C.POINTER(D)],
    "krans_csr_set_spmv_tuning": [P, I, C.POINTER(SpmvTuning)],
    "krans_csr_get_spmv_tuning": [P, I, C.POINTER(SpmvTuning)],
    "krans_rng_create": [P, C.c_uint32, I, PP],
    "krans_rng_destroy": [P],
    "krans_rng_normal": [P, P],
    "krans_rng_seed": [P, C.POINTER(C.c_uint32)],
    "krans_cyclic_opts_init": [C.POINTER(CyclicOpts)],
    "krans_lobpcg_opts_init": [C.POINTER(LobpcgOpts)],
    "krans_solve_cyclic": [P, P, P, C.POINTER(CyclicOpts), P, PP, PP, C.POINTER(CyclicResultC)],
    "krans_solve_lobpcg": [P, P, P, C.POINTER(LobpcgOpts), PP, I64, PP, P, P,
                           C.POINTER(LobpcgResultC)],
    "krans_solve_batch": [P, I64, C.POINTER(Request), C.POINTER(RequestResult), C.POINTER(D)],
    "krans_server_opts_init": [C.POINTER(ServerOpts)],
    "krans_server_create": [P, C.POINTER(ServerOpts), PP],
    "krans_server_destroy": [P],
    "krans_submit": [P, C.POINTER(Request), C.POINTER(C.c_uint64)],
    "krans_poll": [P, C.c_uint64, C.POINTER(I), C.POINTER(RequestResult)],
    "krans_cancel": [P, C.c_uint64],
    "krans_server_drain": [P, D],
    "krans_server_stats": [P, C.POINTER(I64)],
    "krans_server_completed": [P, C.POINTER(C.c_uint64), I64, C.POINTER(I64)],
}
_RESTYPE = {"krans_last_error": C.c_char_p, "krans_version": C.c_char_p, "krans_host_free": None}

_lib = None


def load(path: str = None):
    """Load the CUDA library (KRANS_B200_LIB overrides the in-tree path).
    Fails loudly when it is missing: there is no CPU fallback behind this API."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("KRANS_B200_LIB", LIB_PATH)
    if not os.path.exists(path):
        raise ImportError(f"{path} not built; run `python -m krans_b200.build` "
                          "(the engine has no CPU fallback)")
    L = C.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(L, name, None)
        if f is None:
            continue
        f.argtypes = args
        f.restype = _RESTYPE.get(name, C.c_int)
    _lib = L
    return L


def exported_symbols(path: str = LIB_PATH):
    """Names of SIGNATURES that the shared library exports (no GPU needed)."""
    L = C.CDLL(path)
    return {name for name in SIGNATURES if hasattr(L, name)}


def check(rc: int, what: str = ""):
    if rc != KRANS_OK:
        msg = load().krans_last_error().decode(errors="replace")
        cls = KransInvalidArgument if rc == KRANS_ERR_INVALID_ARGUMENT else KransError
        raise cls(rc, f"{what}: {msg}" if what else msg)
