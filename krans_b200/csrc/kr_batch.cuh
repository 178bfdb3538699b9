// Batched cyclic solves: many independent requests in one persistent launch.
// Each block is a team that takes the next request from a device queue
// (largest first), lays out its slot of workspace on the device and runs the
// full restart/polish loop; results and max ||A u|| are written per request.
#pragma once

#include "kr_cyclic.cuh"

namespace kr {

template <class Team> KR_DEV double team_max_residual(Team &tm, const CsrView &F, const double *basis,
                                                      int64_t ldb, int64_t nf) {
  double mr = 0.0;
  for (int64_t i = 0; i < nf; i++) {
    const double *u = basis + i * ldb;
    double s2 = 0.0;
    team_spmv(tm, F.rows, F.rp, F.ci, F.v64, u, F.lanes, [&](int64_t, double s) { s2 += s * s; });
    mr = fmax(mr, sqrt(tm.sum1(s2)));
  }
  return mr;
}

template <class KT>
__global__ void __launch_bounds__(512) cyclic_batch_kernel(const CyclicRequestDev *reqs, int count, int *queue,
                                                           char *ws, size_t ws_stride) {
  __shared__ TeamShared sh;
  __shared__ CyclicDesc d;
  __shared__ int s_item;
  char *slot = ws + (size_t)blockIdx.x * ws_stride;
  for (;;) {
    if (threadIdx.x == 0)
      s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= count)
      break;
    const CyclicRequestDev &rq = reqs[item];
    if (threadIdx.x == 0) {
      memset(&d, 0, sizeof d);
      cyclic_carve(rq.plan, slot, &d);
      d.F = rq.F;
      d.B = rq.B;
      d.o = rq.o;
      d.k_target = rq.plan.k_target;
      d.ncv = rq.plan.ncv;
      d.trans_run = rq.trans_run;
      d.rng = rq.rng;
      d.initial_right = rq.initial_right;
      d.basis = rq.basis;
      d.ldb = rq.plan.ldb;
      d.status = rq.status;
      d.res = rq.res;
    }
    __syncthreads();
    if (threadIdx.x == 0)
      rq.res->t_begin = globaltimer_ns();
    if (!rq.trivial) {
      TeamCta tm{&sh, d.status, 0};
      CyclicSolver<TeamCta, KT> s(tm, d);
      s.run();
      __syncthreads();
      const int64_t nf = *(volatile int64_t *)&d.res->n_found;
      const double mr = team_max_residual(tm, d.F, d.basis, d.ldb, nf);
      if (threadIdx.x == 0)
        *rq.max_resid = mr;
    }
    if (threadIdx.x == 0)
      rq.res->t_end = globaltimer_ns();
    __syncthreads();
  }
}

// Same as cyclic_batch_kernel with a thread-block cluster per request: the
// cluster's rank 0 takes the next request; every block lays out the same
// slot descriptor; the solve runs on a TeamCluster.
template <class KT>
__global__ void __launch_bounds__(512) cyclic_batch_cluster_kernel(const CyclicRequestDev *reqs, int count,
                                                                   int *queue, char *ws, size_t ws_stride) {
  __shared__ TeamShared sh;
  __shared__ CyclicDesc d;
  __shared__ int s_item;
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  const unsigned rank = cl.block_rank(), csize = cl.num_blocks();
  char *slot = ws + (size_t)(blockIdx.x / csize) * ws_stride;
  int cbuf = 0;
  for (;;) {
    if (rank == 0 && threadIdx.x == 0)
      s_item = atomicAdd(queue, 1);
    cl.sync();
    const int item = *cl.map_shared_rank(&s_item, 0);
    cl.sync();
    if (item >= count)
      break;
    const CyclicRequestDev &rq = reqs[item];
    if (threadIdx.x == 0) {
      memset(&d, 0, sizeof d);
      cyclic_carve(rq.plan, slot, &d);
      d.F = rq.F;
      d.B = rq.B;
      d.o = rq.o;
      d.k_target = rq.plan.k_target;
      d.ncv = rq.plan.ncv;
      d.trans_run = rq.trans_run;
      d.rng = rq.rng;
      d.initial_right = rq.initial_right;
      d.basis = rq.basis;
      d.ldb = rq.plan.ldb;
      d.status = rq.status;
      d.res = rq.res;
    }
    __syncthreads();
    if (rank == 0 && threadIdx.x == 0)
      rq.res->t_begin = globaltimer_ns();
    if (!rq.trivial) {
      TeamCluster tm{&sh, d.status, 0, cbuf, rank, csize};
      CyclicSolver<TeamCluster, KT> s(tm, d);
      s.run();
      tm.sync();
      const int64_t nf = *(volatile int64_t *)&d.res->n_found;
      const double mr = team_max_residual(tm, d.F, d.basis, d.ldb, nf);
      if (tm.leader())
        *rq.max_resid = mr;
      cbuf = tm.cbuf;
    }
    if (rank == 0 && threadIdx.x == 0)
      rq.res->t_end = globaltimer_ns();
    cl.sync();
  }
}

} // namespace kr
