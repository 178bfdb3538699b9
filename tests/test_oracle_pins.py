"""Pins the CPU oracle against the reference's own known answers and golden
vectors (CPU only). The oracle is the reference result of every GPU parity test.

Known answers used (reference paths):
  examples/quickstart.cpp:41-66, README.md:74-79   config-1 shift operator
  tests/test_cyclic_lanczos.cpp:145-542             2x3, mat1, identity, 2x2, scale
  tests/test_lobpcg.cpp:104-447                     same cases for LOBPCG
  tests/test_difference_operator.cpp:49-114         ill-conditioned D
  tests/test_universal_adapter.cpp:17-64            2x3 kernel ~ [-1,-1,1]
  tests/test_subspace_compare.cpp:12-99             RREF subspace_diff cases
  tests/test_gram_schmidt.cpp                        MGS orthonormality
  data/mat1-6.ija nullities                          5, 15, 10, 15, 20, 25
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, dense_kernel, load_golden_matrix
from krans_b200 import generators as G


def test_rng_matches_libstdcxx_bitwise(oracle):
    lines = open(os.path.join(GOLDEN, "rng_normals.txt")).read().split("\n")
    i, total = 0, 0
    r = None
    while i < len(lines):
        t = lines[i]
        if t.startswith("seed"):
            r = oracle.Rng(int(t.split()[1]))
            i += 1
        elif t.startswith("vec"):
            L = int(t.split()[1])
            want = np.array([float.fromhex(x) for x in lines[i + 1:i + 1 + L]])
            got = r.normal(L)
            assert np.array_equal(got, want)
            total += L
            i += 1 + L
        else:
            i += 1
    assert total == 6018


def _shift_check(inst, U):
    A = inst.A
    res = max(np.linalg.norm(A @ u) for u in U)
    K = inst.kernel
    dist = max(np.linalg.norm(u - K.T @ (K @ u)) for u in U)
    return res, dist


def test_quickstart_cyclic_then_lobpcg(oracle):
    # README.md:78-79: cyclic 3 vectors, 6.4e-16 / 7.6e-16; lobpcg 3, 3.5e-11 / 6.4e-11
    inst = G.shift_operator(1000, 3, 0.5)
    A = oracle.Csr.from_scipy(inst.A)
    rng = oracle.Rng(42)
    R = oracle.cyclic(A, rng, k=3)
    assert R.right_null.shape[0] == 3 and R.converged_to_target
    res, dist = _shift_check(inst, R.right_null)
    assert res < 1e-14 and dist < 1e-8
    L = oracle.lobpcg(A, rng, nev=3)
    assert L.right_null.shape[0] == 3 and L.converged_to_target
    res, dist = _shift_check(inst, L.right_null)
    assert res < 1e-9 and dist < 1e-8


def _small_2x3(scale=1.0):
    return sp.csr_matrix(np.array([[1.0, 0, 1], [0, 1, 1]]) * scale)


def test_cyclic_reference_cases(oracle):
    # tests/test_cyclic_lanczos.cpp: Test 1 (2x3), Test 3 (identity), Test 5 (2x2 rank 1), Test 6 (scale)
    A = oracle.Csr.from_scipy(_small_2x3())
    R = oracle.cyclic(A, oracle.Rng(1), k=1, ncv=20, max_restarts=50, nullity_known=1,
                      rank_known=2, cg_maxit=40)
    assert R.right_null.shape[0] == 1
    assert abs(np.linalg.norm(R.right_null[0]) - 1) < 1e-12
    assert np.linalg.norm(A.matvec(R.right_null[0])) <= 1e-10
    I = oracle.Csr.from_scipy(sp.identity(3, format="csr"))
    R = oracle.cyclic(I, oracle.Rng(1), k=1, ncv=20, max_restarts=30, nullity_known=0, rank_known=3)
    assert R.right_null.shape[0] == 0
    B = oracle.Csr.from_scipy(sp.csr_matrix(np.ones((2, 2))))
    R = oracle.cyclic(B, oracle.Rng(1), k=1, ncv=20, max_restarts=50, nullity_known=1,
                      rank_known=1, return_left_space=1)
    assert R.right_null.shape[0] == 1 and R.left_null.shape[0] == 1
    assert np.linalg.norm(B.matvec(R.right_null[0])) <= 1e-10
    assert np.linalg.norm(B.matvec(R.left_null[0], trans=True)) <= 1e-10
    S = oracle.Csr.from_scipy(_small_2x3(1e6))
    R = oracle.cyclic(S, oracle.Rng(1), k=1, ncv=20, max_restarts=50, nullity_known=1,
                      rank_known=2, cg_maxit=40)
    assert R.right_null.shape[0] == 1
    assert np.linalg.norm(S.matvec(R.right_null[0])) / max(1.0, R.frob_norm_est) <= 1e-8


def test_lobpcg_reference_cases(oracle):
    A = oracle.Csr.from_scipy(_small_2x3())
    R = oracle.lobpcg(A, oracle.Rng(1), nev=1, block_size=4, max_iters=200, nullity_known=1,
                      rank_known=2)
    assert R.right_null.shape[0] == 1
    assert np.linalg.norm(A.matvec(R.right_null[0])) <= 1e-10
    v = R.right_null[0]  # tests/test_universal_adapter.cpp: kernel ~ [-1,-1,1]
    assert abs(v[0] + v[2]) < 1e-8 and abs(v[1] + v[2]) < 1e-8
    I = oracle.Csr.from_scipy(sp.identity(3, format="csr"))
    R = oracle.lobpcg(I, oracle.Rng(1), nev=1, block_size=4, max_iters=100, nullity_known=0,
                      rank_known=3)
    assert R.right_null.shape[0] == 0
    S = oracle.Csr.from_scipy(_small_2x3(1e6))
    R = oracle.lobpcg(S, oracle.Rng(1), nev=1, block_size=6, max_iters=300, nullity_known=1,
                      rank_known=2)
    assert R.right_null.shape[0] == 1
    assert np.linalg.norm(S.matvec(R.right_null[0])) / max(1.0, R.frob_norm_est) <= 1e-8


def test_lobpcg_invalid_arguments(oracle):
    A = oracle.Csr.from_scipy(_small_2x3())
    with pytest.raises(oracle.OracleError):
        oracle.lobpcg(A, oracle.Rng(1), nullity_known=5)
    with pytest.raises(oracle.OracleError):
        oracle.lobpcg(A, oracle.Rng(1), rank_known=2, nullity_known=2)


def test_difference_operator(oracle):
    # tests/test_difference_operator.cpp:49-114
    d = G.difference_operator(100)
    A = oracle.Csr.from_scipy(d.A)
    rng = oracle.Rng(42)
    R = oracle.lobpcg(A, rng)
    assert R.block_size == 1
    assert R.converged_to_target == (R.right_null.shape[0] == 1)
    if not R.converged_to_target:
        assert R.iters == 1000 and R.best_unaccepted_residual > R.accept_threshold
    R = oracle.lobpcg(A, rng, block_size=16)
    assert R.block_size == 16 and R.converged_to_target and R.right_null.shape[0] == 1
    assert np.all(np.abs(np.abs(R.right_null[0]) - 1 / np.sqrt(100)) < 1e-8)
    d4 = G.difference_operator(4)
    R = oracle.lobpcg(oracle.Csr.from_scipy(d4.A), oracle.Rng(42), block_size=16)
    assert R.block_size == 4 and R.converged_to_target
    dc = G.difference_operator(1000)
    Ac = oracle.Csr.from_scipy(dc.A)
    rngc = oracle.Rng(42)
    R = oracle.cyclic(Ac, rngc)
    assert R.cg_solves > 0
    if not R.converged_to_target:
        assert R.cg_maxit_hits > 0
    R = oracle.cyclic(Ac, rngc, cg_maxit=1000)
    assert R.converged_to_target and R.right_null.shape[0] == 1
    assert np.all(np.abs(np.abs(R.right_null[0]) - 1 / np.sqrt(1000)) < 1e-8)


@pytest.mark.parametrize("k", [1, 3, 4, 5, 6])
def test_golden_matrices_full_nullspace(oracle, k):
    # README.md:221-224: the full null space of mat1, mat3-mat6 (cyclic defaults)
    As, nul = load_golden_matrix(k)
    A = oracle.Csr.from_scipy(As)
    R = oracle.cyclic(A, oracle.Rng(1), k=nul)
    assert R.right_null.shape[0] == nul
    thr = max(1e-12, 1e-10 * max(1.0, R.frob_norm_est))
    assert max(np.linalg.norm(As @ u) for u in R.right_null) <= thr
    assert oracle.max_pairwise_abs_dot(R.right_null) <= 1e-8
    K = dense_kernel(As, nul)
    assert oracle.subspace_dist(K, R.right_null) < 1e-6


def test_subspace_compare_cases(oracle):
    # tests/test_subspace_compare.cpp
    e = np.eye(3)
    assert oracle.subspace_diff_rref(e[:2], e[:2]) < 1e-12
    assert oracle.subspace_diff_rref(e[:2], np.array([[1, 1, 0], [1, -1, 0.0]])) < 1e-12
    assert oracle.subspace_diff_rref(e[:2], np.array([[1, 0, 0], [0, 0, 1.0]])) > 0.1
    assert oracle.subspace_diff_rref(np.array([[2, 0, 4, 0], [0, 5, 0, 1.0]]),
                                     np.array([[1, 0, 2, 0], [0, 10, 0, 2.0]])) < 1e-12
    assert oracle.subspace_diff_rref(np.array([[1, 0, 0], [0, 1, 0], [1, 1, 0.0]]),
                                     np.array([[2, 0, 0], [0, 2, 0], [2, 2, 0.0]])) < 1e-12
    assert oracle.subspace_diff_rref(e[:2], e[:1]) == 1e9
    # principal-angle distance: orthonormal bases of one subspace
    q, _ = np.linalg.qr(np.random.default_rng(0).standard_normal((50, 4)))
    rot, _ = np.linalg.qr(np.random.default_rng(1).standard_normal((4, 4)))
    assert oracle.subspace_dist(q.T, (q @ rot).T) < 1e-14


def test_mgs_and_dense_helpers(oracle):
    rng = np.random.default_rng(3)
    V = rng.standard_normal((6, 40))
    ok, Q = oracle.mgs(V)
    assert ok and np.allclose(Q @ Q.T, np.eye(6), atol=1e-14)
    M = rng.standard_normal((9, 7))
    sv, Vm = oracle.svd_right(M)
    assert np.allclose(np.sort(sv), np.sort(np.linalg.svd(M, compute_uv=False)), atol=1e-13)
    S = M.T @ M
    w, Qe = oracle.sym_eig(S)
    assert np.allclose(w, np.linalg.eigvalsh(S), atol=1e-12)
    assert np.allclose(Qe.T @ S @ Qe, np.diag(w), atol=1e-11)
