"""ctypes binding of the C oracle (oracle/krans_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py's CPU-baseline leg. The product (krans_b200) never
imports this module.

The oracle restates the reference solvers on the CPU, single-threaded, FP64:
  find_nullspace_cyclic_lanczos_ex  src/Solvers/CyclicLanczosSolver.cpp:291-660
  find_nullspace_lobpcg_ex          src/Solvers/LOBPCGSolver.cpp:443-834
with the StdVectorFactory RNG (std::mt19937 + std::normal_distribution).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libkrans_oracle.so")
_lib = None

PRECOND_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))


class KoRng(C.Structure):
    _fields_ = [("mt", C.c_uint32 * 624), ("idx", C.c_int32), ("has_saved", C.c_int32),
                ("saved", C.c_double)]


class KoCsr(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64),
                ("rp", C.c_void_p), ("ci", C.c_void_p), ("v", C.c_void_p),
                ("rpT", C.c_void_p), ("ciT", C.c_void_p), ("vT", C.c_void_p)]


class KoCyclicOpts(C.Structure):
    _fields_ = [("k", C.c_int64), ("ncv", C.c_int64), ("max_restarts", C.c_int64),
                ("tol_abs", C.c_double), ("tol_rel", C.c_double),
                ("reorth", C.c_int32), ("use_harmonic", C.c_int32),
                ("target_tau", C.c_double),
                ("nullity_known", C.c_int32), ("rank_known", C.c_int32),
                ("initial_right", C.c_void_p),
                ("precond_AAt", PRECOND_FN), ("precond_user", C.c_void_p),
                ("cg_maxit", C.c_int64), ("cg_rel_tol", C.c_double),
                ("cg_breakdown_tol", C.c_double),
                ("projector_passes", C.c_int32), ("grad_max_iters", C.c_int32),
                ("frob_samples", C.c_int32), ("prescreen_factor", C.c_double),
                ("stagnation_restarts", C.c_int64),
                ("return_left_space", C.c_int32), ("verbose", C.c_int32)]


class KoCyclicResult(C.Structure):
    _fields_ = [("n_right", C.c_int64), ("n_left", C.c_int64),
                ("restarts", C.c_int64), ("krylov_steps_total", C.c_int64),
                ("frob_norm_est", C.c_double), ("converged_to_target", C.c_int32),
                ("cg_solves", C.c_int64), ("cg_maxit_hits", C.c_int64),
                ("spmv", C.c_int64), ("spmvT", C.c_int64)]


class KoLobpcgOpts(C.Structure):
    _fields_ = [("nev", C.c_int64), ("block_size", C.c_int64), ("max_iters", C.c_int64),
                ("tol_abs", C.c_double), ("tol_rel", C.c_double),
                ("soft_locking", C.c_int32), ("restart", C.c_double),
                ("gs_tol", C.c_double), ("gs_reorth", C.c_int32),
                ("M_inv", PRECOND_FN), ("M_user", C.c_void_p),
                ("initial_block", C.c_void_p), ("n_initial", C.c_int64),
                ("frob_samples", C.c_int32), ("max_tiny_dim", C.c_int64),
                ("nullity_known", C.c_int32), ("rank_known", C.c_int32),
                ("verbose", C.c_int32)]


class KoLobpcgResult(C.Structure):
    _fields_ = [("n_right", C.c_int64), ("iters", C.c_int64), ("locked", C.c_int64),
                ("frob_norm_est", C.c_double), ("accept_threshold", C.c_double),
                ("best_unaccepted_residual", C.c_double), ("block_size", C.c_int64),
                ("converged_to_target", C.c_int32), ("spmv", C.c_int64),
                ("spmvT", C.c_int64)]


def build():
    """Compile the oracle with its Makefile (gcc only; no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.ko_rng_seed.argtypes = [C.POINTER(KoRng), C.c_uint32]
        L.ko_rng_u32.argtypes = [C.POINTER(KoRng)]
        L.ko_rng_u32.restype = C.c_uint32
        L.ko_rng_fill_normal.argtypes = [C.POINTER(KoRng), C.c_void_p, C.c_int64]
        L.ko_spmv.argtypes = [C.POINTER(KoCsr), C.c_int, C.c_void_p, C.c_void_p]
        L.ko_cyclic_opts_default.argtypes = [C.POINTER(KoCyclicOpts)]
        L.ko_cyclic.argtypes = [C.POINTER(KoCsr), C.POINTER(KoRng), C.POINTER(KoCyclicOpts),
                                C.c_void_p, C.c_void_p, C.POINTER(KoCyclicResult)]
        L.ko_lobpcg_opts_default.argtypes = [C.POINTER(KoLobpcgOpts)]
        L.ko_lobpcg.argtypes = [C.POINTER(KoCsr), C.POINTER(KoRng), C.POINTER(KoLobpcgOpts),
                                C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(KoLobpcgResult)]
        L.ko_last_error.restype = C.c_char_p
        L.ko_mgs.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_double, C.c_int]
        L.ko_max_pairwise_abs_dot.argtypes = [C.c_int64, C.c_int64, C.c_void_p]
        L.ko_max_pairwise_abs_dot.restype = C.c_double
        L.ko_subspace_diff_rref.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_void_p,
                                            C.c_void_p, C.c_double]
        L.ko_subspace_diff_rref.restype = C.c_double
        L.ko_subspace_dist.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]
        L.ko_subspace_dist.restype = C.c_double
        L.ko_svd_right.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ko_sym_eig.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Rng:
    """std::mt19937(seed) + std::normal_distribution<double>(0, 1)."""

    def __init__(self, seed: int):
        self.s = KoRng()
        lib().ko_rng_seed(C.byref(self.s), seed & 0xFFFFFFFF)

    def u32(self) -> int:
        return lib().ko_rng_u32(C.byref(self.s))

    def normal(self, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float64)
        lib().ko_rng_fill_normal(C.byref(self.s), _p(out), n)
        return out


class Csr:
    """A CSR matrix with its explicit transpose, as int32/float64 arrays."""

    def __init__(self, m, n, indptr, indices, data):
        import scipy.sparse as sp
        A = sp.csr_matrix((np.asarray(data, np.float64), np.asarray(indices, np.int32),
                           np.asarray(indptr, np.int32)), shape=(m, n))
        A.sort_indices()
        AT = A.T.tocsr()
        AT.sort_indices()
        self.m, self.n = m, n
        self.rp = A.indptr.astype(np.int32)
        self.ci = A.indices.astype(np.int32)
        self.v = A.data.astype(np.float64)
        self.rpT = AT.indptr.astype(np.int32)
        self.ciT = AT.indices.astype(np.int32)
        self.vT = AT.data.astype(np.float64)
        self.s = KoCsr(m, n, _p(self.rp), _p(self.ci), _p(self.v),
                       _p(self.rpT), _p(self.ciT), _p(self.vT))

    @classmethod
    def from_scipy(cls, A):
        A = A.tocsr()
        return cls(A.shape[0], A.shape[1], A.indptr, A.indices, A.data)

    def matvec(self, x, trans=False):
        y = np.empty(self.n if trans else self.m, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        lib().ko_spmv(C.byref(self.s), int(trans), _p(x), _p(y))
        return y


@dataclass
class CyclicResult:
    right_null: np.ndarray
    left_null: np.ndarray
    restarts: int
    krylov_steps_total: int
    frob_norm_est: float
    converged_to_target: bool
    cg_solves: int
    cg_maxit_hits: int
    spmv: int
    spmvT: int


@dataclass
class LobpcgResult:
    right_null: np.ndarray
    theta: np.ndarray
    residuals_Av: np.ndarray
    iters: int
    locked: int
    frob_norm_est: float
    accept_threshold: float
    best_unaccepted_residual: float
    block_size: int
    converged_to_target: bool
    spmv: int
    spmvT: int


class OracleError(RuntimeError):
    pass


def _wrap_precond(fn, size):
    if fn is None:
        return PRECOND_FN(), None

    def cb(_u, r, y):
        rr = np.ctypeslib.as_array(r, shape=(size,))
        yy = np.ctypeslib.as_array(y, shape=(size,))
        yy[:] = fn(rr.copy())
    return PRECOND_FN(cb), cb


def cyclic(A: Csr, rng: Rng, initial_right=None, precond_AAt=None, **kw) -> CyclicResult:
    o = KoCyclicOpts()
    lib().ko_cyclic_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown cyclic option {k}")
        setattr(o, k, v)
    keep = []
    if initial_right is not None:
        y0 = np.ascontiguousarray(initial_right, np.float64)
        keep.append(y0)
        o.initial_right = _p(y0)
    cb, pyfn = _wrap_precond(precond_AAt, A.m)
    o.precond_AAt = cb
    keep.append(pyfn)
    k_target = o.nullity_known if o.nullity_known >= 0 else o.k
    right = np.zeros((max(k_target, 1), A.n), np.float64)
    left = np.zeros((max(o.k, 1), A.m), np.float64)
    r = KoCyclicResult()
    rc = lib().ko_cyclic(C.byref(A.s), C.byref(rng.s), C.byref(o), _p(right), _p(left),
                         C.byref(r))
    if rc != 0:
        raise OracleError(lib().ko_last_error().decode())
    return CyclicResult(right[:r.n_right].copy(), left[:r.n_left].copy(), r.restarts,
                        r.krylov_steps_total, r.frob_norm_est, bool(r.converged_to_target),
                        r.cg_solves, r.cg_maxit_hits, r.spmv, r.spmvT)


def lobpcg(A: Csr, rng: Rng, initial_block=None, M_inv=None, **kw) -> LobpcgResult:
    o = KoLobpcgOpts()
    lib().ko_lobpcg_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown lobpcg option {k}")
        setattr(o, k, v)
    keep = []
    if initial_block is not None:
        ib = np.ascontiguousarray(np.atleast_2d(initial_block), np.float64)
        keep.append(ib)
        o.initial_block = _p(ib)
        o.n_initial = ib.shape[0]
    cb, pyfn = _wrap_precond(M_inv, A.n)
    o.M_inv = cb
    keep.append(pyfn)
    k_target = max(1, o.nev)
    if o.nullity_known >= 0:
        k_target = o.nullity_known
    elif o.rank_known >= 0:
        k_target = max(0, A.n - o.rank_known)
    cap = max(k_target, 1)
    right = np.zeros((cap, A.n), np.float64)
    theta = np.zeros(cap)
    resid = np.zeros(cap)
    r = KoLobpcgResult()
    rc = lib().ko_lobpcg(C.byref(A.s), C.byref(rng.s), C.byref(o), _p(right), _p(theta),
                         _p(resid), C.byref(r))
    if rc != 0:
        raise OracleError(lib().ko_last_error().decode())
    nr = r.n_right
    return LobpcgResult(right[:nr].copy(), theta[:nr].copy(), resid[:nr].copy(), r.iters,
                        r.locked, r.frob_norm_est, r.accept_threshold,
                        r.best_unaccepted_residual, r.block_size, bool(r.converged_to_target),
                        r.spmv, r.spmvT)


def subspace_dist(U, V) -> float:
    """Largest principal-angle sine ||V - U (U^T V)||_2 (orthonormal rows)."""
    U = np.ascontiguousarray(np.atleast_2d(U), np.float64)
    V = np.ascontiguousarray(np.atleast_2d(V), np.float64)
    return lib().ko_subspace_dist(U.shape[0], V.shape[0], U.shape[1], _p(U), _p(V))


def subspace_diff_rref(B1, B2, tol=1e-12) -> float:
    B1 = np.ascontiguousarray(np.atleast_2d(B1), np.float64)
    B2 = np.ascontiguousarray(np.atleast_2d(B2), np.float64)
    n = B1.shape[1] if B1.size else (B2.shape[1] if B2.size else 0)
    if B1.size and B2.size and B1.shape[1] != B2.shape[1]:
        return 1e9
    return lib().ko_subspace_diff_rref(B1.shape[0] if B1.size else 0,
                                       B2.shape[0] if B2.size else 0, n, _p(B1), _p(B2), tol)


def mgs(V, tol=1e-12, reorth=True):
    V = np.ascontiguousarray(np.atleast_2d(V), np.float64).copy()
    ok = lib().ko_mgs(V.shape[0], V.shape[1], _p(V), tol, int(reorth))
    return bool(ok), V


def max_pairwise_abs_dot(V) -> float:
    V = np.ascontiguousarray(np.atleast_2d(V), np.float64)
    return lib().ko_max_pairwise_abs_dot(V.shape[0], V.shape[1], _p(V))


def svd_right(M):
    M = np.asfortranarray(M, np.float64)
    r, c = M.shape
    sv = np.zeros(c)
    V = np.zeros((c, c), order="F")
    lib().ko_svd_right(r, c, M.ctypes.data_as(C.c_void_p), _p(sv), V.ctypes.data_as(C.c_void_p))
    return sv, V


def sym_eig(A):
    A = np.asfortranarray(A, np.float64)
    n = A.shape[0]
    w = np.zeros(n)
    Q = np.zeros((n, n), order="F")
    lib().ko_sym_eig(n, A.ctypes.data_as(C.c_void_p), _p(w), Q.ctypes.data_as(C.c_void_p))
    return w, Q


# ---------------------------------------------------------------------------
# The reference's own solver sources compiled against the Eigen-subset shim
# (oracle/_ref/libkrans_ref.so, built by `make -C oracle ref` from a
# Deep-SANE/krans checkout; see oracle/ref_driver.cpp). Same options and
# results as the C restatement above.
# ---------------------------------------------------------------------------
REF_LIB = os.path.join(_HERE, "_ref", "libkrans_ref.so")
_ref_lib = None


def build_ref(reference_root):
    """Compile oracle/_ref from the reference sources under reference_root."""
    subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={reference_root}"], check=True)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        if not ref_available():
            raise OracleError(f"{REF_LIB} is not built (make -C oracle ref REF=<reference root>)")
        L = C.CDLL(REF_LIB)
        L.kref_last_error.restype = C.c_char_p
        L.kref_factory_create.restype = C.c_void_p
        L.kref_factory_create.argtypes = [C.c_int64, C.c_uint32]
        L.kref_factory_destroy.argtypes = [C.c_void_p]
        L.kref_factory_destroy.restype = None
        L.kref_cyclic.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.kref_lobpcg.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]
        _ref_lib = L
    return _ref_lib


class RefFactory:
    """The reference's StdVectorFactory(default_size, seed): std::mt19937 +
    std::normal_distribution, state carried across solves."""

    def __init__(self, default_size: int, seed: int):
        self.h = ref_lib().kref_factory_create(default_size, seed & 0xFFFFFFFF)

    def __del__(self):
        try:
            if self.h:
                ref_lib().kref_factory_destroy(self.h)
        except Exception:
            pass


def _ref_check(rc):
    if rc == 1:
        raise ValueError(ref_lib().kref_last_error().decode())
    if rc != 0:
        raise OracleError(ref_lib().kref_last_error().decode())


def ref_cyclic(A: Csr, vf: RefFactory, initial_right=None, precond_AAt=None, **kw) -> CyclicResult:
    """find_nullspace_cyclic_lanczos_ex of the reference itself."""
    o = KoCyclicOpts()
    lib().ko_cyclic_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown cyclic option {k}")
        setattr(o, k, v)
    keep = []
    if initial_right is not None:
        y0 = np.ascontiguousarray(initial_right, np.float64)
        keep.append(y0)
        o.initial_right = _p(y0)
    cb, pyfn = _wrap_precond(precond_AAt, A.m)
    o.precond_AAt = cb
    keep.append(pyfn)
    k_target = o.nullity_known if o.nullity_known >= 0 else o.k
    right = np.zeros((max(k_target, 1), A.n), np.float64)
    left = np.zeros((max(o.k, 1), A.m), np.float64)
    r = KoCyclicResult()
    _ref_check(ref_lib().kref_cyclic(C.byref(A.s), C.c_void_p(vf.h), C.byref(o), _p(right), _p(left),
                                     C.byref(r)))
    return CyclicResult(right[:r.n_right].copy(), left[:r.n_left].copy(), r.restarts,
                        r.krylov_steps_total, r.frob_norm_est, bool(r.converged_to_target),
                        r.cg_solves, r.cg_maxit_hits, r.spmv, r.spmvT)


def ref_lobpcg(A: Csr, vf: RefFactory, initial_block=None, M_inv=None, **kw) -> LobpcgResult:
    """find_nullspace_lobpcg_ex of the reference itself."""
    o = KoLobpcgOpts()
    lib().ko_lobpcg_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown lobpcg option {k}")
        setattr(o, k, v)
    keep = []
    if initial_block is not None:
        ib = np.ascontiguousarray(np.atleast_2d(initial_block), np.float64)
        keep.append(ib)
        o.initial_block = _p(ib)
        o.n_initial = ib.shape[0]
    cb, pyfn = _wrap_precond(M_inv, A.n)
    o.M_inv = cb
    keep.append(pyfn)
    cap = max(1, o.nev, o.nullity_known, A.n - o.rank_known if o.rank_known >= 0 else 0)
    right = np.zeros((cap, A.n), np.float64)
    theta = np.zeros(cap)
    resid = np.zeros(cap)
    r = KoLobpcgResult()
    _ref_check(ref_lib().kref_lobpcg(C.byref(A.s), C.c_void_p(vf.h), C.byref(o), cap, _p(right), _p(theta),
                                     _p(resid), C.byref(r)))
    nr = r.n_right
    return LobpcgResult(right[:nr].copy(), theta[:nr].copy(), resid[:nr].copy(), r.iters,
                        r.locked, r.frob_norm_est, r.accept_threshold,
                        r.best_unaccepted_residual, r.block_size, bool(r.converged_to_target),
                        r.spmv, r.spmvT)
