"""Batched persistent launches and the continuous-batching server.

Checks: every request of a mixed batch meets max ||A u|| <= 1e-12 * L, where
L <= ||A||_2 is the max row/column norm of A (so the criterion is at least as
strict as ||Au||/||A||_2 <= 1e-12), and spans the analytic kernel to 1e-10;
a request gives bit-identical results alone and inside a batch; failures of
one request (NaN values, over-budget, cancellation) are reported per request
while the others finish bit-identically."""
import numpy as np
import pytest
import scipy.sparse as sp

from krans_b200 import generators as G

pytestmark = pytest.mark.gpu


def norm_lower_bound(A):
    A2 = A.multiply(A)
    return float(np.sqrt(max(A2.sum(axis=0).max(), A2.sum(axis=1).max())))


def make_requests(ctx, insts, precision, seed0=11, **kw):
    import krans_b200 as kb
    from krans_b200.serving import SolveRequest
    reqs = []
    for i, inst in enumerate(insts):
        M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, inst.A, fp32=True)
        opts = kb.CyclicLanczosOptions(k=inst.k, tol_abs=1e-12 * norm_lower_bound(inst.A), tol_rel=0.0,
                                       cg_maxit=1000, precision=kb.Precision(precision), **kw)
        reqs.append(SolveRequest(M, opts, seed=seed0 + i, rng_mode="philox"))
    return reqs


def small_mix(count=24, seed=3):
    out = []
    for i in range(count):
        r = np.random.default_rng([seed, i])
        n = int(np.exp(r.uniform(np.log(800), np.log(6000))))
        if i % 2 == 0:
            out.append(G.shift_operator(n, int(r.integers(1, 6)), float(r.uniform(0.3, 0.8))))
        else:
            out.append(G.graph_incidence(n, int(r.integers(1, 6)), 6.0, seed=int(r.integers(1 << 30))))
    return out


@pytest.mark.parametrize("precision,polish_block", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_batch_accuracy(ctx, oracle, precision, polish_block):
    from krans_b200.serving import solve_batch
    insts = small_mix()
    reqs = make_requests(ctx, insts, precision, polish_block=polish_block)
    solve_batch(ctx, reqs)
    for inst, rq in zip(insts, reqs):
        r = rq.result
        assert r.status == 0 and r.converged_to_target and r.n_right == inst.k
        U = rq.basis()
        L = norm_lower_bound(inst.A)
        assert max(np.linalg.norm(inst.A @ u) for u in U) <= 1e-12 * L
        assert r.max_residual <= 1e-12 * L
        assert oracle.subspace_dist(inst.kernel, U) <= 1e-10


def test_alone_equals_in_the_mix(ctx):
    from krans_b200.serving import solve_batch
    insts = small_mix(16, seed=5)
    mix = make_requests(ctx, insts, 1)
    solve_batch(ctx, mix)
    for i in [0, 3, 10]:
        alone = make_requests(ctx, [insts[i]], 1, seed0=11 + i)
        solve_batch(ctx, alone)
        np.testing.assert_array_equal(alone[0].basis(), mix[i].basis())
        assert alone[0].result.restarts == mix[i].result.restarts


def test_fault_isolation_nan_request(ctx):
    import krans_b200 as kb
    from krans_b200.serving import solve_batch
    insts = small_mix(8, seed=7)
    bad = insts[2].A.copy()
    bad.data[::7] = np.nan
    reqs = make_requests(ctx, insts, 1)
    solve_batch(ctx, reqs)
    ref = [r.basis().copy() for r in reqs]
    reqs2 = make_requests(ctx, insts, 1)
    reqs2[2].A = kb.CudaCsrMatrixAdapter.from_scipy(ctx, bad, fp32=True)
    solve_batch(ctx, reqs2)
    assert not reqs2[2].result.converged_to_target
    for i in range(8):
        if i != 2:
            np.testing.assert_array_equal(reqs2[i].basis(), ref[i])


def test_server_continuous_batching(ctx):
    import time
    from krans_b200.serving import Server, solve_batch
    insts = small_mix(20, seed=9)
    ref = make_requests(ctx, insts, 1)
    solve_batch(ctx, ref)
    srv = Server(ctx, max_inflight=3, max_batch=4)
    reqs = make_requests(ctx, insts, 1)
    tickets = []
    for i, rq in enumerate(reqs):
        tickets.append(srv.submit(rq))
        if i % 5 == 4:
            time.sleep(0.01)  # later arrivals join while earlier launches run
    srv.drain(120)
    for rq, rr in zip(reqs, ref):
        st, res = srv.poll(rq.ticket)
        assert st == "done" and res.status == 0
        assert res.latency_ms >= res.queue_ms >= 0
        np.testing.assert_array_equal(rq.basis(), rr.basis())
    srv.close()


def test_server_cancel_and_budget(ctx):
    from krans_b200.serving import Server
    insts = small_mix(6, seed=13)
    srv = Server(ctx, max_inflight=1, max_batch=1)
    reqs = make_requests(ctx, insts, 1)
    ts = [srv.submit(r) for r in reqs]
    srv.cancel(ts[-1])  # still queued behind the others
    srv.drain(120)
    assert srv.poll(ts[-1])[0] == "cancelled"
    for t in ts[:-1]:
        assert srv.poll(t)[0] == "done"
    srv.close()
    tiny = Server(ctx, hbm_budget=1 << 20, max_inflight=1)
    r = make_requests(ctx, insts[:1], 1)[0]
    t = tiny.submit(r)
    tiny.drain(60)
    st, res = tiny.poll(t)
    assert st == "failed" and res.status == -4  # KRANS_ERR_OUT_OF_MEMORY
    tiny.close()


def test_size_classes_and_pair_launch(ctx, oracle):
    """A batch with single-block (m + n < 16384), 2-block-cluster (< 120000)
    and 8-block-cluster requests: all converge, and a mid-size request gives
    bit-identical results alone and in the mix (its team kind depends only on
    its size)."""
    from krans_b200.serving import solve_batch
    insts = [G.shift_operator(3000, 2, 0.5), G.graph_incidence(2500, 3, 6.0, seed=1),
             G.shift_operator(20000, 3, 0.6), G.graph_incidence(12000, 4, 6.0, seed=2),
             G.shift_operator(70000, 2, 0.7), G.graph_incidence(40000, 2, 6.0, seed=3)]
    mix = make_requests(ctx, insts, 1)
    solve_batch(ctx, mix)
    for inst, rq in zip(insts, mix):
        r = rq.result
        assert r.status == 0 and r.converged_to_target and r.n_right == inst.k
        assert r.max_residual <= 1e-12 * norm_lower_bound(inst.A)
        assert oracle.subspace_dist(inst.kernel, rq.basis()) <= 1e-10
    for i in (2, 3):
        alone = make_requests(ctx, [insts[i]], 1, seed0=11 + i)
        solve_batch(ctx, alone)
        np.testing.assert_array_equal(alone[0].basis(), mix[i].basis())
