"""GPU parity of the device cyclic Lanczos engine against the CPU oracle and
the analytic kernels, on the reference's own test cases
(tests/test_cyclic_lanczos.cpp, tests/test_difference_operator.cpp,
examples/quickstart.cpp) and the golden matrices.

Tolerances: max ||A u|| within the reference's acceptance threshold
max(tol_abs, tol_rel * max(1, ||A||_F~)); subspace distance (largest
principal-angle sine) to the oracle's basis and to the exact kernel <= 1e-10
where the threshold is 1e-12-level, else <= 1e3 * threshold / sigma_min."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import dense_kernel, load_golden_matrix
from krans_b200 import generators as G

pytestmark = pytest.mark.gpu

TEAMS = [1, 2]  # KRANS_TEAM_CTA, KRANS_TEAM_GRID


def solve(ctx, A, seed, team=0, precision=0, **kw):
    import krans_b200 as kb
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A, fp32=(precision == 1))
    vf = kb.CudaVectorFactory(ctx, A.shape[1], seed=seed)
    opt = kb.CyclicLanczosOptions(team=team, precision=kb.Precision(precision), **kw)
    R = kb.find_nullspace_cyclic_lanczos_ex(M, vf, opt)
    return R, kb.basis_to_numpy(R.right_null), kb.basis_to_numpy(R.left_null)


@pytest.mark.parametrize("team", TEAMS)
def test_quickstart_shift_operator(ctx, oracle, team):
    inst = G.shift_operator(1000, 3, 0.5)
    R, U, _ = solve(ctx, inst.A, 42, team=team, k=3)
    assert U.shape[0] == 3 and R.converged_to_target
    res = max(np.linalg.norm(inst.A @ u) for u in U)
    assert res < 1e-13
    assert oracle.subspace_dist(inst.kernel, U) < 1e-10
    O = oracle.cyclic(oracle.Csr.from_scipy(inst.A), oracle.Rng(42), k=3)
    assert oracle.subspace_dist(O.right_null, U) < 1e-10
    # same seeded start vectors (the factory's MT19937 stream) -> the same
    # ||A||_F estimate; the Krylov trajectory may drift by rounding only
    assert R.frob_norm_est == pytest.approx(O.frob_norm_est, rel=1e-12)
    assert abs(R.restarts - O.restarts) <= 2


@pytest.mark.parametrize("team", TEAMS)
def test_reference_small_cases(ctx, oracle, team):
    A = sp.csr_matrix(np.array([[1.0, 0, 1], [0, 1, 1]]))
    R, U, _ = solve(ctx, A, 1, team=team, k=1, ncv=20, max_restarts=50, nullity_known=1,
                    rank_known=2, cg_maxit=40)
    assert U.shape[0] == 1 and abs(np.linalg.norm(U[0]) - 1) < 1e-12
    assert np.linalg.norm(A @ U[0]) <= 1e-10
    R, U, _ = solve(ctx, sp.identity(3, format="csr"), 1, team=team, nullity_known=0, rank_known=3)
    assert U.shape[0] == 0 and R.converged_to_target
    B = sp.csr_matrix(np.ones((2, 2)))
    R, U, L = solve(ctx, B, 1, team=team, k=1, ncv=20, max_restarts=50, nullity_known=1,
                    rank_known=1, return_left_space=True)
    assert U.shape[0] == 1 and L.shape[0] == 1
    assert np.linalg.norm(B @ U[0]) <= 1e-10 and np.linalg.norm(B.T @ L[0]) <= 1e-10
    S = sp.csr_matrix(np.array([[1.0, 0, 1], [0, 1, 1]]) * 1e6)
    R, U, _ = solve(ctx, S, 1, team=team, k=1, ncv=20, max_restarts=50, nullity_known=1,
                    rank_known=2, cg_maxit=40)
    assert U.shape[0] == 1
    assert np.linalg.norm(S @ U[0]) / max(1.0, R.frob_norm_est) <= 1e-8


@pytest.mark.parametrize("k", [1, 3, 4, 5, 6])
def test_golden_matrices(ctx, oracle, k):
    A, nul = load_golden_matrix(k)
    R, U, _ = solve(ctx, A, 1, k=nul)
    assert U.shape[0] == nul and R.converged_to_target
    thr = max(1e-12, 1e-10 * max(1.0, R.frob_norm_est))
    assert max(np.linalg.norm(A @ u) for u in U) <= thr
    assert oracle.max_pairwise_abs_dot(U) <= 1e-8
    K = dense_kernel(A, nul)
    O = oracle.cyclic(oracle.Csr.from_scipy(A), oracle.Rng(1), k=nul)
    assert oracle.subspace_dist(K, U) < 1e-6
    assert oracle.subspace_dist(O.right_null, U) < 1e-6


@pytest.mark.parametrize("team", TEAMS)
@pytest.mark.parametrize("k", [1, 5])
def test_golden_matrices_block_polish(ctx, oracle, k, team):
    """Block CG polish (up to 8 candidates per group): same acceptance bar and
    the same subspace as the one-by-one polish."""
    A, nul = load_golden_matrix(k)
    R, U, _ = solve(ctx, A, 1, team=team, k=nul, polish_block=1)
    assert U.shape[0] == nul and R.converged_to_target
    thr = max(1e-12, 1e-10 * max(1.0, R.frob_norm_est))
    assert max(np.linalg.norm(A @ u) for u in U) <= thr
    assert oracle.max_pairwise_abs_dot(U) <= 1e-8
    assert oracle.subspace_dist(dense_kernel(A, nul), U) < 1e-6


def test_difference_operator_cg_limits(ctx):
    d = G.difference_operator(1000)
    R, U, _ = solve(ctx, d.A, 42)
    assert R.cg_solves > 0
    if not R.converged_to_target:
        assert R.cg_maxit_hits > 0
    R, U, _ = solve(ctx, d.A, 42, cg_maxit=1000)
    assert R.converged_to_target and U.shape[0] == 1
    assert np.all(np.abs(np.abs(U[0]) - 1 / np.sqrt(1000)) < 1e-8)


@pytest.mark.parametrize("team", TEAMS)
def test_mixed_precision_reaches_fp64_accuracy(ctx, oracle, team):
    """FP32 SpMV + Lanczos recurrence, FP64 reorth / tiny SVD / CG polish:
    the accepted basis must still meet max ||Au|| / ||A||_2 <= 1e-12."""
    inst = G.graph_incidence(30000, 5, 6.0, seed=4)
    A = inst.A
    normA = np.sqrt(sp.linalg.eigsh((A.T @ A).tocsr(), k=1, which="LM", return_eigenvectors=False)[0])
    R, U, _ = solve(ctx, A, 3, team=team, precision=1, k=inst.k, tol_abs=1e-12 * normA, tol_rel=0.0,
                    cg_maxit=400)
    assert U.shape[0] == inst.k and R.converged_to_target
    assert max(np.linalg.norm(A @ u) for u in U) / normA <= 1e-12
    assert oracle.subspace_dist(inst.kernel, U) <= 1e-10


def test_shared_memory_cg_vectors_same_answers():
    """KRANS_SMEM_CG_KB puts the CG vectors of one-block solves in shared
    memory (read once per process, so checked in a child process)."""
    import os
    import subprocess
    import sys
    code = (
        "import numpy as np, krans_b200 as kb\n"
        "from krans_b200 import generators as G\n"
        "ctx = kb.Context(0)\n"
        "inst = G.shift_operator(1000, 3, 0.5)\n"
        "M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, inst.A)\n"
        "R = kb.find_nullspace_cyclic_lanczos_ex(M, kb.CudaVectorFactory(ctx, 1000, seed=42),"
        " kb.CyclicLanczosOptions(k=3, team=1))\n"
        "U = kb.basis_to_numpy(R.right_null)\n"
        "P = inst.kernel.T @ np.linalg.lstsq(inst.kernel.T, U.T, rcond=None)[0]\n"
        "print(U.shape[0], max(np.linalg.norm(inst.A @ u) for u in U), np.linalg.norm(P - U.T, 2))\n")
    env = dict(os.environ, KRANS_SMEM_CG_KB="160")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    k, res, dist = out.stdout.split()[-3:]
    assert int(k) == 3 and float(res) < 1e-13 and float(dist) < 1e-10
