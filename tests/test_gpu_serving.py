"""Serving (krans_server_*, krans_submit): continuous batching inside a
running persistent launch, and LOBPCG requests.

* A cyclic request submitted while the server's launch is running joins that
  launch (same launch_id as the requests it started with) and gives the same
  basis, bit for bit, as when it is solved alone (its team kind depends only
  on its size, and its RNG stream only on its seed).
* LOBPCG requests (one block below cluster_min, a thread-block cluster above)
  meet ||Au|| <= 1e-12 L and subspace distance <= 1e-10 to the oracle's FP64
  basis on the same MT19937 stream, and give the same basis alone and in a mix
  with cyclic requests."""
import time

import numpy as np
import pytest

from krans_b200 import generators as G

pytestmark = pytest.mark.gpu


def norm_bound(A):
    A2 = A.multiply(A)
    return float(np.sqrt(max(A2.sum(axis=0).max(), A2.sum(axis=1).max())))


def cyclic_req(kb, ctx, inst, seed, mats):
    from krans_b200.serving import SolveRequest
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, inst.A, fp32=True)
    mats.append(M)
    o = kb.CyclicLanczosOptions(k=inst.k, tol_abs=1e-12 * norm_bound(inst.A), tol_rel=0.0, cg_maxit=1000,
                                precision=kb.Precision.MIXED)
    return SolveRequest(M, o, seed=seed)


def wait_done(srv, t, seconds=120):
    t0 = time.time()
    while time.time() - t0 < seconds:
        st, res = srv.poll(t)
        if st in ("done", "failed", "cancelled"):
            return st, res
        time.sleep(0.002)
    raise AssertionError("request did not finish")


def test_request_joins_running_launch(ctx, oracle):
    import krans_b200 as kb
    from krans_b200.serving import Server, solve_batch
    mats = []
    # requests that keep the launch busy for a while (single-block class)
    early = [G.graph_incidence(6000 + 500 * i, 3, 6.0, seed=20 + i) for i in range(12)]
    late = G.shift_operator(9000, 3, 0.55)
    srv = Server(ctx, max_inflight=2, max_batch=64)
    ereqs = [cyclic_req(kb, ctx, inst, 100 + i, mats) for i, inst in enumerate(early)]
    for r in ereqs:
        srv.submit(r)
    # wait until the launch is running, then submit the late request
    t0 = time.time()
    while srv.poll(ereqs[0].ticket)[0] != "running" and time.time() - t0 < 60:
        time.sleep(0.001)
    assert srv.poll(ereqs[0].ticket)[0] == "running"
    lreq = cyclic_req(kb, ctx, late, 777, mats)
    srv.submit(lreq)
    st, res = wait_done(srv, lreq.ticket)
    assert st == "done" and res.converged_to_target
    srv.drain(120)
    launch_ids = {srv.poll(r.ticket)[1].launch_id for r in ereqs}
    assert res.launch_id in launch_ids  # admitted into the running launch
    assert oracle.subspace_dist(late.kernel, lreq.basis()) <= 1e-10
    alone = cyclic_req(kb, ctx, late, 777, mats)
    solve_batch(ctx, [alone])
    np.testing.assert_array_equal(alone.basis(), lreq.basis())
    for inst, r in zip(early, ereqs):
        st, rr = srv.poll(r.ticket)
        assert st == "done" and rr.converged_to_target
        assert oracle.subspace_dist(inst.kernel, r.basis()) <= 1e-10
    srv.close()


@pytest.mark.parametrize("which", ["block", "cluster"])
def test_lobpcg_requests(ctx, oracle, which):
    import krans_b200 as kb
    from krans_b200.serving import Server, SolveRequest
    if which == "block":
        inst = G.shift_operator(1000, 3, 0.5)              # m + n < 16384: one thread block
        kw = dict(nev=3)
    else:
        inst = G.graph_incidence(8000, 4, 8.0, seed=6)      # m + n = 40000: a thread-block cluster
        kw = dict(nev=4, block_size=8)
    L = norm_bound(inst.A)
    opt = kb.LOBPCGOptions(tol_abs=1e-12 * L, tol_rel=0.0, **kw)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, inst.A, fp32=True)
    srv = Server(ctx, max_inflight=3, max_batch=16)
    alone = SolveRequest(M, opt, seed=42, rng_mode="mt19937")
    srv.submit(alone)
    st, res = wait_done(srv, alone.ticket)
    assert st == "done" and res.status == 0 and res.converged_to_target and res.n_right == inst.k
    U = alone.basis()
    assert max(np.linalg.norm(inst.A @ u) for u in U) <= 1e-12 * L
    assert res.max_residual <= 1e-12 * L
    O = oracle.lobpcg(oracle.Csr.from_scipy(inst.A), oracle.Rng(42), tol_abs=1e-12 * L, tol_rel=0.0, **kw)
    assert oracle.subspace_dist(O.right_null, U) <= 1e-10
    assert oracle.subspace_dist(inst.kernel, U) <= 1e-10
    # the same request in a mix with cyclic requests
    mats = []
    mix = [cyclic_req(kb, ctx, G.shift_operator(4000 + 300 * i, 2, 0.6), 9 + i, mats) for i in range(6)]
    again = SolveRequest(M, opt, seed=42, rng_mode="mt19937")
    for r in mix[:3]:
        srv.submit(r)
    srv.submit(again)
    for r in mix[3:]:
        srv.submit(r)
    srv.drain(120)
    st, res2 = srv.poll(again.ticket)
    assert st == "done"
    np.testing.assert_array_equal(again.basis(), U)
    for r in mix:
        assert srv.poll(r.ticket)[0] == "done"
    srv.close()


def test_lobpcg_request_errors(ctx):
    import krans_b200 as kb
    from krans_b200.serving import Server, SolveRequest
    inst = G.shift_operator(500, 2, 0.5)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, inst.A)
    srv = Server(ctx, max_inflight=2)
    bad = SolveRequest(M, kb.LOBPCGOptions(nev=2, nullity_known=900), seed=1)  # nullity_known > n
    srv.submit(bad)
    st, res = wait_done(srv, bad.ticket)
    assert st == "failed" and res.status == -1
    mixed = SolveRequest(M, kb.LOBPCGOptions(nev=2, precision=kb.Precision.MIXED), seed=1)
    srv.submit(mixed)
    st, res = wait_done(srv, mixed.ticket)
    assert st == "failed" and res.status == -1  # LOBPCG requests run in FP64
    srv.close()


def test_cancel_running_request_and_completed_list(ctx):
    """A running request is stopped through its device status word (no wait
    for it to finish); krans_server_completed hands out each finished ticket
    once; a request without an output buffer still reports its residual."""
    import krans_b200 as kb
    from krans_b200.serving import Server, SolveRequest
    d = G.difference_operator(200000)  # LOBPCG with block size 1 needs very many iterations here
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, d.A)
    srv = Server(ctx, max_inflight=2)
    slow = SolveRequest(M, kb.LOBPCGOptions(nev=1, block_size=1, max_iters=10**9), seed=3)
    srv.submit(slow)
    t0 = time.time()
    while srv.poll(slow.ticket)[0] != "running" and time.time() - t0 < 60:
        time.sleep(0.001)
    time.sleep(0.2)
    assert srv.poll(slow.ticket)[0] == "running"
    t1 = time.time()
    srv.cancel(slow.ticket)
    st, res = wait_done(srv, slow.ticket, 60)
    assert st == "cancelled" and res.status == -7 and time.time() - t1 < 30
    inst = G.shift_operator(2000, 2, 0.5)
    quick = cyclic_req(kb, ctx, inst, 5, [])
    quick.keep_basis = False
    srv.submit(quick)
    st, res = wait_done(srv, quick.ticket)
    assert st == "done" and res.converged_to_target and res.max_residual <= 1e-12 * norm_bound(inst.A)
    assert quick.basis().shape == (0, inst.A.shape[1])
    seen = srv.completed() + srv.completed()
    assert sorted(seen) == sorted([slow.ticket, quick.ticket]) and srv.completed() == []
    srv.close()
