"""The C restatement (oracle/krans_oracle.c) against the reference's own
solver sources compiled unchanged against the project's Eigen-subset shim
(oracle/_ref/libkrans_ref.so: the reference's CyclicLanczosSolver.cpp,
LOBPCGSolver.cpp, GramSchmidt.cpp and Projection.cpp, with its
StdMatrixAdapter and StdVectorFactory). Same inputs, same options, same
MT19937 seeds: the two must take the same path (restarts, Krylov steps,
operator applications, LOBPCG iterations) and return the same subspace.
Skipped when oracle/_ref is not built (it needs a checkout of the reference)."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import load_golden_matrix
from krans_b200 import generators as G


@pytest.fixture(scope="module")
def O(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref is not built (make -C oracle ref REF=<reference checkout>)")
    return oracle


def same_cyclic(O, A, seed, **kw):
    Ao = O.Csr.from_scipy(A)
    R = O.ref_cyclic(Ao, O.RefFactory(A.shape[1], seed), **kw)
    C = O.cyclic(Ao, O.Rng(seed), **kw)
    assert (R.restarts, R.krylov_steps_total, R.spmv, R.spmvT, R.cg_solves, R.cg_maxit_hits) == \
           (C.restarts, C.krylov_steps_total, C.spmv, C.spmvT, C.cg_solves, C.cg_maxit_hits)
    assert R.converged_to_target == C.converged_to_target
    assert R.right_null.shape == C.right_null.shape and R.left_null.shape == C.left_null.shape
    if R.right_null.shape[0]:
        assert O.subspace_dist(R.right_null, C.right_null) <= 1e-12
    if R.left_null.shape[0]:
        assert O.subspace_dist(R.left_null, C.left_null) <= 1e-12
    return R, C


def test_quickstart_same_factory(O):
    # examples/quickstart.cpp: cyclic then LOBPCG on one factory (seed 42)
    inst = G.shift_operator(1000, 3, 0.5)
    Ao = O.Csr.from_scipy(inst.A)
    f = O.RefFactory(1000, 42)
    rc, rl = O.ref_cyclic(Ao, f, k=3), O.ref_lobpcg(Ao, f, nev=3)
    rng = O.Rng(42)
    cc, cl = O.cyclic(Ao, rng, k=3), O.lobpcg(Ao, rng, nev=3)
    assert (rc.restarts, rc.krylov_steps_total, rc.spmv) == (cc.restarts, cc.krylov_steps_total, cc.spmv)
    assert (rl.iters, rl.spmv, rl.spmvT, rl.block_size) == (cl.iters, cl.spmv, cl.spmvT, cl.block_size)
    assert O.subspace_dist(rc.right_null, cc.right_null) <= 1e-12
    # default LOBPCG tolerance (accept at 1e-10 ||A||_F): the bases agree to that level
    assert O.subspace_dist(rl.right_null, cl.right_null) <= 1e-9
    # README.md:78-79: 3 vectors, max ||Au|| 6.4e-16 / 3.5e-11, distance 7.6e-16 / 6.4e-11
    assert max(np.linalg.norm(inst.A @ u) for u in rc.right_null) < 1e-14
    assert O.subspace_dist(inst.kernel, rl.right_null) < 1e-9


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6])
def test_golden_matrices_cyclic(O, k):
    A, nul = load_golden_matrix(k)
    R, _ = same_cyclic(O, A, 1, k=nul)
    assert R.right_null.shape[0] == nul


@pytest.mark.parametrize("k", [1, 3, 4])
def test_golden_matrices_lobpcg(O, k):
    A, nul = load_golden_matrix(k)
    Ao = O.Csr.from_scipy(A)
    R = O.ref_lobpcg(Ao, O.RefFactory(A.shape[1], 1), nev=nul, block_size=nul + 4, max_iters=3000)
    C = O.lobpcg(Ao, O.Rng(1), nev=nul, block_size=nul + 4, max_iters=3000)
    # same main loop; the final polish sweeps stop at a residual near the
    # rounding floor, so their operator count may differ by a few sweeps
    assert (R.iters, R.locked) == (C.iters, C.locked)
    assert abs(R.spmv - C.spmv) <= 0.1 * C.spmv and abs(R.spmvT - C.spmvT) <= 0.1 * C.spmvT
    assert R.right_null.shape == C.right_null.shape == (nul, A.shape[1])
    assert O.subspace_dist(R.right_null, C.right_null) <= 1e-8


def test_reference_unit_cases(O):
    # tests/test_cyclic_lanczos.cpp: 2x3 (kernel [-1,-1,1]/sqrt3), identity (none),
    # rank-1 2x2 with the left space, difference operator at default cg_maxit
    same_cyclic(O, sp.csr_matrix(np.array([[1.0, 0, 1], [0, 1, 1]])), 7, k=1)
    R, _ = same_cyclic(O, sp.identity(4, format="csr"), 7, k=1, rank_known=4)
    assert R.right_null.shape[0] == 0
    R, _ = same_cyclic(O, sp.csr_matrix(np.array([[1.0, 2.0], [2.0, 4.0]])), 3, k=1, return_left_space=1)
    assert R.left_null.shape[0] == 1
    d = G.difference_operator(100)
    same_cyclic(O, d.A, 42, k=1)
    same_cyclic(O, d.A, 42, k=1, cg_maxit=1000)


def test_random_projector_fallback(O):
    inst = G.shift_operator(1000, 3, 0.5)
    for k in (3, 5):
        R, _ = same_cyclic(O, inst.A, 42, k=k, max_restarts=0)
        assert R.right_null.shape[0] == 3


def test_planted_kernel_at_bound(O):
    inst = G.planted_kernel(1500, 1000, 8, seed=2)
    A2 = inst.A.multiply(inst.A)
    L = float(np.sqrt(max(A2.sum(axis=0).max(), A2.sum(axis=1).max())))
    R, _ = same_cyclic(O, inst.A, 42, k=8, tol_abs=1e-12 * L, tol_rel=0.0, cg_maxit=1000)
    assert R.right_null.shape[0] == 8
    assert O.subspace_dist(inst.kernel, R.right_null) <= 1e-10


def test_invalid_arguments_match(O):
    # std::invalid_argument in the reference (ValueError here)
    A = O.Csr.from_scipy(sp.csr_matrix(np.array([[1.0, 0, 1], [0, 1, 1]])))
    with pytest.raises(ValueError):
        O.ref_lobpcg(A, O.RefFactory(3, 1), nullity_known=5)
