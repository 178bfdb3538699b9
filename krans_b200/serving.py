"""Batched solves and the continuous-batching server (Python mirror of
krans_solve_batch / krans_server_* in include/krans_cuda.h).

A request is one null-space solve of its own matrix with its own options
and RNG stream: cyclic Lanczos (batched launches and the server) or LOBPCG
(the server); its basis is written to a device buffer owned by the request
object.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import _capi as K
from ._capi import check
from .api import Context, CudaCsrMatrixAdapter, CudaVectorAdapter, CyclicLanczosOptions, LOBPCGOptions

STATUS = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


@dataclass
class SolveRequest:
    """opts: CyclicLanczosOptions (solver "cyclic") or LOBPCGOptions (solver
    "lobpcg", served requests only; FP64). For LOBPCG results, `restarts`
    counts LOBPCG iterations and `krylov_steps_total` the locked vectors."""
    A: CudaCsrMatrixAdapter
    opts: object
    seed: int = 1
    rng_mode: str = "philox"
    keep_basis: bool = True  # False: no output buffer; only the result (max_residual included)
    buf: Optional[CudaVectorAdapter] = None
    result: Optional[K.RequestResult] = None
    ticket: int = 0

    @property
    def solver(self) -> str:
        return "lobpcg" if isinstance(self.opts, LOBPCGOptions) else "cyclic"

    def k_target(self) -> int:
        o = self.opts
        if self.solver == "lobpcg":
            if o.nullity_known >= 0:
                return o.nullity_known
            if o.rank_known >= 0:
                return max(0, self.A.n - o.rank_known)
            return max(1, o.nev)
        return o.nullity_known if o.nullity_known >= 0 else o.k

    def to_c(self, ctx: Context) -> K.Request:
        kt = max(self.k_target(), 1)
        if self.buf is None and self.keep_basis:
            self.buf = CudaVectorAdapter(ctx, kt * self.A.n)
        r = K.Request()
        r.A = self.A.h
        if self.solver == "lobpcg":
            r.solver = K.KRANS_SOLVER_LOBPCG
            r.lobpcg = self.opts.to_c()
            K.load().krans_cyclic_opts_init(C.byref(r.opts))
        else:
            r.solver = K.KRANS_SOLVER_CYCLIC
            r.opts = self.opts.to_c()
        r.seed = self.seed & 0xFFFFFFFF
        r.rng_mode = {"mt19937": K.KRANS_RNG_MT19937, "philox": K.KRANS_RNG_PHILOX}[self.rng_mode]
        r.basis_out = self.buf.device_ptr() if self.buf is not None else None
        r.basis_capacity = kt if self.buf is not None else 0
        return r

    def basis(self) -> np.ndarray:
        """Accepted null vectors as rows (host copy)."""
        nr = int(self.result.n_right) if self.result is not None else 0
        if nr == 0 or self.buf is None:
            return np.zeros((0, self.A.n))
        return self.buf.data()[: nr * self.A.n].reshape(nr, self.A.n)


def solve_batch(ctx: Context, reqs: List[SolveRequest]) -> float:
    """Run all requests in one persistent launch. Returns device ms."""
    arr = (K.Request * max(len(reqs), 1))(*[r.to_c(ctx) for r in reqs])
    res = (K.RequestResult * max(len(reqs), 1))()
    ms = C.c_double()
    check(ctx.lib.krans_solve_batch(ctx.h, len(reqs), arr, res, C.byref(ms)), "krans_solve_batch")
    for i, r in enumerate(reqs):
        r.result = res[i]
    return ms.value


class Server:
    """Continuous batching: submit() returns at once; requests are admitted
    against the HBM budget into persistent launches on a pool of streams."""

    def __init__(self, ctx: Context, hbm_budget: int = 0, max_inflight: int = 4, max_batch: int = 1024):
        self.ctx = ctx
        o = K.ServerOpts()
        check(ctx.lib.krans_server_opts_init(C.byref(o)))
        if hbm_budget:
            o.hbm_budget_bytes = hbm_budget
        o.max_inflight_launches = max_inflight
        o.max_batch = max_batch
        h = C.c_void_p()
        check(ctx.lib.krans_server_create(ctx.h, C.byref(o), C.byref(h)), "krans_server_create")
        self.h = h
        self.live: Dict[int, SolveRequest] = {}

    def submit(self, req: SolveRequest) -> int:
        c = req.to_c(self.ctx)
        t = C.c_uint64()
        check(self.ctx.lib.krans_submit(self.h, C.byref(c), C.byref(t)), "krans_submit")
        req.ticket = t.value
        self.live[t.value] = req
        return t.value

    def poll(self, ticket: int):
        st = C.c_int()
        res = K.RequestResult()
        check(self.ctx.lib.krans_poll(self.h, ticket, C.byref(st), C.byref(res)), "krans_poll")
        if st.value >= 2 and ticket in self.live:
            self.live[ticket].result = res
        return STATUS[st.value], res

    def cancel(self, ticket: int):
        """Queued: dropped at once; running: stopped at its team's next status
        check (the ticket ends as cancelled, or done if it finished first)."""
        check(self.ctx.lib.krans_cancel(self.h, ticket), "krans_cancel")

    def completed(self, capacity: int = 4096):
        """Tickets finished since the last call (krans_server_completed)."""
        buf = (C.c_uint64 * capacity)()
        n = C.c_int64()
        check(self.ctx.lib.krans_server_completed(self.h, buf, capacity, C.byref(n)), "krans_server_completed")
        return [int(buf[i]) for i in range(n.value)]

    def stats(self):
        """(queued, launches in flight, LOBPCG launches, running cyclic
        requests), or None while the scheduler holds its lock."""
        out = (C.c_int64 * 4)()
        rc = self.ctx.lib.krans_server_stats(self.h, out)
        return tuple(int(x) for x in out) if rc == 0 else None

    def drain(self, timeout_s: float = 600.0):
        check(self.ctx.lib.krans_server_drain(self.h, timeout_s * 1e3), "krans_server_drain")
        for t in list(self.live):
            self.poll(t)

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.krans_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
