"""Batched-launch tuning through the C ABI (krans_ctx_set/get_batch_tuning):
round trip, argument checks, and solves that stay correct under a
non-default table (other team-size thresholds, other lanes per row)."""
import numpy as np
import pytest

from krans_b200 import generators as G

pytestmark = pytest.mark.gpu


def test_batch_tuning_round_trip_and_checks():
    import krans_b200 as kb
    ctx = kb.Context(0, tuning=False)
    assert ctx.batch_tuning() == {"cluster_min": 16384, "pair_max": 120000, "cluster_size": 8,
                                  "lanes": [1, 2, 4, 8, 16, 32]}
    ctx.set_batch_tuning(cluster_min=8192, lanes=[2, 4, 0, 0, 0, 0])
    assert ctx.batch_tuning() == {"cluster_min": 8192, "pair_max": 120000, "cluster_size": 8,
                                  "lanes": [2, 4, 4, 8, 16, 32]}
    for bad in (dict(lanes=[3, 0, 0, 0, 0, 0]), dict(cluster_size=1), dict(cluster_size=17), dict(pair_max=-1)):
        with pytest.raises(ValueError):
            ctx.set_batch_tuning(**bad)


def test_solves_under_other_tuning():
    import krans_b200 as kb
    from krans_b200.serving import SolveRequest, solve_batch
    from oracle import oracle as O
    ctx = kb.Context(0, tuning=False)
    ctx.set_batch_tuning(cluster_min=4096, pair_max=30000, cluster_size=4, lanes=[2, 4, 8, 8, 16, 32])
    insts = [G.shift_operator(20000, 3, 0.6), G.graph_incidence(12000, 5, 6.0, seed=4),
             G.shift_operator(3000, 2, 0.5), G.graph_incidence(50000, 3, 6.0, seed=5)]
    reqs = []
    for i, inst in enumerate(insts):
        A2 = inst.A.multiply(inst.A)
        L = float(np.sqrt(max(A2.sum(axis=0).max(), A2.sum(axis=1).max())))
        M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, inst.A, fp32=True)
        reqs.append(SolveRequest(M, kb.CyclicLanczosOptions(k=inst.k, tol_abs=1e-12 * L, tol_rel=0.0, cg_maxit=1000,
                                                            precision=kb.Precision.MIXED), seed=3 + i))
    solve_batch(ctx, reqs)
    for inst, rq in zip(insts, reqs):
        assert rq.result.status == 0 and rq.result.converged_to_target
        assert O.subspace_dist(inst.kernel, rq.basis()) <= 1e-10
