"""Device preconditioners of the CG projector (precond_AAt's device form):
Jacobi and the k-step steepest-descent callback of the reference's tests,
against the oracle running the same callbacks on the host, and the
reference's mat2 case (tests/test_cyclic_lanczos.cpp:300-420: SD with 8 steps,
ncv 128, projector_passes 2, cg_maxit 200, prescreen 4, nullity 15)."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import load_golden_matrix
from krans_b200 import generators as G

pytestmark = pytest.mark.gpu


def weighted_incidence(n, comps, seed):
    inst = G.graph_incidence(n, comps, 6.0, seed=seed)
    w = np.random.default_rng(seed).uniform(0.05, 20.0, inst.A.shape[0])
    return sp.diags(w) @ inst.A, inst.kernel


def jacobi_fn(A):
    d = np.asarray(A.multiply(A).sum(axis=1)).ravel()
    dinv = np.where(d > 0, 1.0 / np.where(d > 0, d, 1.0), 1.0)
    return lambda r: dinv * r


def sd_fn(A, k):
    AT = A.T.tocsr()

    def f(r):
        z = np.zeros_like(r)
        q = r.copy()
        for _ in range(k):
            Oq = A @ (AT @ q)
            qOq = q @ Oq
            if not abs(qOq) >= 1e-30:
                break
            a = (q @ q) / qOq
            z += a * q
            q = q - a * Oq
            if q @ q <= 1e-30:
                break
        return z
    return f


@pytest.mark.parametrize("kind", ["jacobi", "sd"])
def test_precond_matches_oracle(ctx, oracle, kind):
    import krans_b200 as kb
    A, K = weighted_incidence(3000, 3, 7)
    A = A.tocsr()
    pk = kb.Precond.JACOBI if kind == "jacobi" else kb.Precond.SD
    fn = jacobi_fn(A) if kind == "jacobi" else sd_fn(A, 8)
    opts = dict(k=3, cg_maxit=200)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A)
    R = kb.find_nullspace_cyclic_lanczos_ex(M, kb.CudaVectorFactory(ctx, A.shape[1], seed=5),
                                            kb.CyclicLanczosOptions(precond_aat=pk, precond_steps=8, **opts))
    U = kb.basis_to_numpy(R.right_null)
    O = oracle.cyclic(oracle.Csr.from_scipy(A), oracle.Rng(5), precond_AAt=fn, **opts)
    assert U.shape[0] == 3 and O.right_null.shape[0] == 3 and R.converged_to_target
    thr = max(1e-12, 1e-10 * max(1.0, R.frob_norm_est))
    assert max(np.linalg.norm(A @ u) for u in U) <= thr
    assert oracle.subspace_dist(K, U) < 1e-8
    assert oracle.subspace_dist(O.right_null, U) < 1e-8
    # the preconditioned projector needs no more CG solves than the oracle's
    assert R.cg_solves <= O.cg_solves + 8
    # without a preconditioner the same budget hits the CG cap more often
    R0 = kb.find_nullspace_cyclic_lanczos_ex(M, kb.CudaVectorFactory(ctx, A.shape[1], seed=5),
                                             kb.CyclicLanczosOptions(**opts))
    assert R0.cg_maxit_hits >= R.cg_maxit_hits


def test_reference_mat2_with_sd_preconditioner(ctx, oracle):
    import krans_b200 as kb
    A, nul = load_golden_matrix(2)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A)
    vf = kb.CudaVectorFactory(ctx, A.shape[1], seed=1)
    opt = kb.CyclicLanczosOptions(
        k=nul, ncv=max(nul + 80, 128), max_restarts=400, projector_passes=2, cg_maxit=200, cg_rel_tol=1e-10,
        prescreen_factor=4.0, stagnation_restarts=0, tol_abs=1e-12, tol_rel=1e-10, nullity_known=nul,
        rank_known=A.shape[1] - nul, initial_right_space=[vf.create_random_of_size(A.shape[1])],
        precond_aat=kb.Precond.SD, precond_steps=8)
    R = kb.find_nullspace_cyclic_lanczos_ex(M, vf, opt)
    U = kb.basis_to_numpy(R.right_null)
    # the reference test's checks: every ||A u|| within the acceptance
    # threshold, orthonormal, and a random vector projected onto the span
    # stays within sqrt(k) times the threshold
    assert U.shape[0] == nul
    thr = max(1e-12, 1e-10 * max(1.0, R.frob_norm_est))
    assert max(np.linalg.norm(A @ u) for u in U) <= thr
    assert oracle.max_pairwise_abs_dot(U) <= 1e-8
    v = np.random.default_rng(3).standard_normal(A.shape[1])
    v /= np.linalg.norm(v)
    assert np.linalg.norm(A @ (U.T @ (U @ v))) <= np.sqrt(nul) * thr


def sd_normal_fn(A, k):
    AT = A.T.tocsr()

    def f(r):
        y = np.zeros_like(r)
        q = r.copy()
        for _ in range(k):
            Nq = AT @ (A @ q)
            qNq = q @ Nq
            if not abs(qNq) >= 1e-30:
                break
            a = (q @ q) / qNq
            y += a * q
            q = q - a * Nq
            if q @ q <= 1e-30:
                break
        return y
    return f


def test_lobpcg_reference_mat1_with_sd_preconditioner(ctx, oracle):
    """tests/test_lobpcg.cpp:150-250: nev 5, block 12, max_iters 500, two
    random initial vectors, 6-step SD M_inv; the test's asserts: 5 unit
    vectors with ||A v|| <= 1e-8, orthonormal, and a projected random vector
    with ||A P v|| <= 1e-8."""
    import krans_b200 as kb
    A, nul = load_golden_matrix(1)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A)
    vf = kb.CudaVectorFactory(ctx, A.shape[1], seed=1)
    init = [vf.create_random_of_size(A.shape[1]) for _ in range(2)]
    R = kb.find_nullspace_lobpcg_ex(M, vf, kb.LOBPCGOptions(
        nev=5, block_size=12, max_iters=500, tol_abs=1e-12, tol_rel=1e-10, nullity_known=5, rank_known=100,
        initial_block=init, precond_normal=kb.Precond.SD, precond_steps=6))
    U = kb.basis_to_numpy(R.right_null)
    assert U.shape[0] == nul
    assert np.all(np.abs(np.linalg.norm(U, axis=1) - 1) <= 1e-10)
    assert max(np.linalg.norm(A @ u) for u in U) <= 1e-8
    assert oracle.max_pairwise_abs_dot(U) <= 1e-8
    v = np.random.default_rng(4).standard_normal(A.shape[1])
    assert np.linalg.norm(A @ (U.T @ (U @ v))) <= 1e-8


@pytest.mark.parametrize("kind", ["jacobi", "sd"])
def test_lobpcg_precond_matches_oracle(ctx, oracle, kind):
    import krans_b200 as kb
    A, K = weighted_incidence(1500, 4, 11)
    A = A.tocsr()
    if kind == "jacobi":
        d = np.asarray(A.multiply(A).sum(axis=0)).ravel()
        dinv = np.where(d > 0, 1.0 / np.where(d > 0, d, 1.0), 1.0)
        fn, pk = (lambda r: dinv * r), kb.Precond.JACOBI
    else:
        fn, pk = sd_normal_fn(A, 6), kb.Precond.SD
    opts = dict(nev=4, block_size=8, max_iters=800)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A)
    R = kb.find_nullspace_lobpcg_ex(M, kb.CudaVectorFactory(ctx, A.shape[1], seed=9),
                                    kb.LOBPCGOptions(precond_normal=pk, precond_steps=6, **opts))
    U = kb.basis_to_numpy(R.right_null)
    O = oracle.lobpcg(oracle.Csr.from_scipy(A), oracle.Rng(9), M_inv=fn, **opts)
    assert U.shape[0] == 4 and O.right_null.shape[0] == 4
    thr = max(1e-12, 1e-10 * max(1.0, R.frob_norm_est))
    assert max(np.linalg.norm(A @ u) for u in U) <= thr
    assert oracle.subspace_dist(K, U) < 1e-8
    assert oracle.subspace_dist(O.right_null, U) < 1e-8
