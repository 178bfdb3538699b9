"""GPU parity of the device LOBPCG engine against the CPU oracle and the
analytic kernels, on the reference's LOBPCG cases (tests/test_lobpcg.cpp,
tests/test_universal_adapter.cpp, tests/test_difference_operator.cpp,
examples/quickstart.cpp) and the golden matrices. The reference's asserts in
tests/test_lobpcg.cpp are compiled out (NDEBUG); here they are enforced."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import dense_kernel, load_golden_matrix
from krans_b200 import generators as G

pytestmark = pytest.mark.gpu
TEAMS = [1, 2]


def solve(ctx, A, vf=None, seed=1, team=0, **kw):
    import krans_b200 as kb
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A)
    vf = vf or kb.CudaVectorFactory(ctx, A.shape[1], seed=seed)
    R = kb.find_nullspace_lobpcg_ex(M, vf, kb.LOBPCGOptions(team=team, **kw))
    return R, kb.basis_to_numpy(R.right_null)


@pytest.mark.parametrize("team", TEAMS)
def test_quickstart_cyclic_then_lobpcg_same_factory(ctx, oracle, team):
    # examples/quickstart.cpp: cyclic, then LOBPCG on the same factory (the
    # LOBPCG start block comes from the RNG state cyclic left behind); both at
    # the accuracy bound tol_abs = 1e-12 L, tol_rel = 0
    import krans_b200 as kb
    inst = G.shift_operator(1000, 3, 0.5)
    A2 = inst.A.multiply(inst.A)
    L = float(np.sqrt(max(A2.sum(axis=0).max(), A2.sum(axis=1).max())))
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, inst.A)
    vf = kb.CudaVectorFactory(ctx, 1000, seed=42)
    kb.find_nullspace_cyclic_lanczos(M, vf, kb.CyclicLanczosOptions(k=3, team=team, tol_abs=1e-12 * L, tol_rel=0.0))
    R = kb.find_nullspace_lobpcg_ex(M, vf, kb.LOBPCGOptions(nev=3, team=team, tol_abs=1e-12 * L, tol_rel=0.0))
    U = kb.basis_to_numpy(R.right_null)
    assert U.shape[0] == 3 and R.converged_to_target
    assert max(np.linalg.norm(inst.A @ u) for u in U) <= 1e-12 * L
    assert oracle.subspace_dist(inst.kernel, U) <= 1e-10
    Ao = oracle.Csr.from_scipy(inst.A)
    rng = oracle.Rng(42)
    oracle.cyclic(Ao, rng, k=3, tol_abs=1e-12 * L, tol_rel=0.0)
    O = oracle.lobpcg(Ao, rng, nev=3, tol_abs=1e-12 * L, tol_rel=0.0)
    assert oracle.subspace_dist(O.right_null, U) <= 1e-10
    assert oracle.subspace_diff_rref(O.right_null, U) <= 1e-8
    assert R.block_size == O.block_size == 3


@pytest.mark.parametrize("team", TEAMS)
def test_reference_small_cases(ctx, team):
    A = sp.csr_matrix(np.array([[1.0, 0, 1], [0, 1, 1]]))
    R, U = solve(ctx, A, team=team, nev=1, block_size=4, max_iters=200, nullity_known=1, rank_known=2)
    assert U.shape[0] == 1 and abs(np.linalg.norm(U[0]) - 1) < 1e-12
    assert np.linalg.norm(A @ U[0]) <= 1e-10
    v = U[0]  # kernel ~ [-1, -1, 1] (tests/test_universal_adapter.cpp)
    assert abs(v[0] + v[2]) < 1e-8 and abs(v[1] + v[2]) < 1e-8
    R, U = solve(ctx, sp.identity(3, format="csr"), team=team, nev=1, block_size=4, max_iters=100,
                 nullity_known=0, rank_known=3)
    assert U.shape[0] == 0
    S = sp.csr_matrix(np.array([[1.0, 0, 1], [0, 1, 1]]) * 1e6)
    R, U = solve(ctx, S, team=team, nev=1, block_size=6, max_iters=300, nullity_known=1, rank_known=2)
    assert U.shape[0] == 1
    assert np.linalg.norm(S @ U[0]) / max(1.0, R.frob_norm_est) <= 1e-8


def test_invalid_arguments(ctx):
    import krans_b200 as kb
    A = sp.csr_matrix(np.array([[1.0, 0, 1], [0, 1, 1]]))
    with pytest.raises(ValueError, match="nullity_known > n"):
        solve(ctx, A, nullity_known=5)
    with pytest.raises(ValueError, match="inconsistent"):
        solve(ctx, A, rank_known=2, nullity_known=2)
    with pytest.raises(ValueError, match="rank_known > n"):
        solve(ctx, A, rank_known=4)


def test_difference_operator(ctx):
    import krans_b200 as kb
    d = G.difference_operator(100)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, d.A)
    vf = kb.CudaVectorFactory(ctx, 100, seed=42)
    R = kb.find_nullspace_lobpcg_ex(M, vf, kb.LOBPCGOptions())
    assert R.block_size == 1
    assert R.converged_to_target == (len(R.right_null) == 1)
    if not R.converged_to_target:
        assert R.iters == 1000 and R.best_unaccepted_residual > R.accept_threshold
    R = kb.find_nullspace_lobpcg_ex(M, vf, kb.LOBPCGOptions(block_size=16))
    assert R.block_size == 16 and R.converged_to_target and len(R.right_null) == 1
    u = R.right_null[0].data()
    assert np.all(np.abs(np.abs(u) - 1 / np.sqrt(100)) < 1e-8)
    d4 = G.difference_operator(4)
    R, U = solve(ctx, d4.A, seed=42, block_size=16)
    assert R.block_size == 4 and R.converged_to_target


@pytest.mark.parametrize("k", [1, 3, 4])
def test_golden_matrices(ctx, oracle, k):
    A, nul = load_golden_matrix(k)
    R, U = solve(ctx, A, nev=nul, block_size=nul + 4, max_iters=3000)
    assert U.shape[0] == nul and R.converged_to_target
    thr = max(1e-12, 1e-10 * max(1.0, R.frob_norm_est))
    assert max(np.linalg.norm(A @ u) for u in U) <= thr
    assert oracle.max_pairwise_abs_dot(U) <= 1e-8
    assert oracle.subspace_dist(dense_kernel(A, nul), U) < 1e-6


@pytest.mark.parametrize("team", TEAMS)
def test_incidence_components(ctx, oracle, team):
    inst = G.graph_incidence(4000, 6, 8.0, seed=2)
    R, U = solve(ctx, inst.A, seed=5, team=team, nev=inst.k, block_size=inst.k + 4, max_iters=2000)
    assert U.shape[0] == inst.k and R.converged_to_target
    assert oracle.subspace_dist(inst.kernel, U) < 1e-8
