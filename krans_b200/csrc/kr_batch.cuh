// Batched cyclic solves: many independent requests in one persistent launch.
// Each block is a team that takes the next request from a device queue
// (largest first), lays out its slot of workspace on the device and runs the
// full restart/polish loop; results and max ||A u|| are written per request.
#pragma once

#include "kr_cyclic.cuh"

#ifndef KR_BATCH_MIN_BLOCKS
#define KR_BATCH_MIN_BLOCKS 1 // resident blocks per SM the register budget is sized for
#endif

namespace kr {

template <class Team> KR_DEV double team_max_residual(Team &tm, const CsrView &F, const double *basis,
                                                      int64_t ldb, int64_t nf) {
  double mr = 0.0;
  for (int64_t i = 0; i < nf; i++) {
    const double *u = basis + i * ldb;
    double s2 = 0.0;
    csr_mv(tm, F, F.v64, u, [&](int64_t, double s) { s2 += s * s; });
    mr = fmax(mr, sqrt(tm.sum1(s2)));
  }
  return mr;
}

extern __shared__ __align__(16) char kr_dyn_smem[];

// Index of the next request of queue `which` (0 large, 1 mid, 2 small) for
// this team, or -1 when there is none. A closed launch (feed == nullptr)
// hands out 0 .. count-1. An open launch hands out what the host has
// published so far, claiming an index only once it is published; a team that
// finds nothing sleeps between looks until the host publishes more, closes
// the launch, or feed->idle_ns pass, and then leaves. Every wait is bounded.
// Open launches only: a published request of queue `which` that no team has
// claimed yet.
KR_DEV bool work_pending(const int *queue, const LaunchFeed *feed, int which) {
  return *(volatile const int *)queue < *(volatile const int32_t *)&feed->published[which];
}

// In an open launch, -2 from take_request: no request of this queue, but the
// `yield` queue has one waiting (the caller serves that queue first).
constexpr int kTakeYield = -2;

KR_DEV int take_request(int *queue, int count, const LaunchFeed *feed, int which, const int *yield_queue = nullptr,
                        int yield_which = 0) {
  if (!feed) {
    const int it = atomicAdd(queue, 1);
    return it < count ? it : -1;
  }
  const uint64_t t0 = globaltimer_ns();
  unsigned nap = 256;
  for (;;) {
    const int closed = *(volatile const int32_t *)&feed->closed;
    const int pub = *(volatile const int32_t *)&feed->published[which];
    int q = *(volatile int *)queue;
    while (q < pub) {
      const int got = atomicCAS(queue, q, q + 1);
      if (got == q)
        return q;
      q = got;
    }
    if (closed) // read before `published`: nothing more can come
      return -1;
    if (yield_queue && work_pending(yield_queue, feed, yield_which))
      return kTakeYield;
    if (globaltimer_ns() - t0 > feed->idle_ns)
      return -1;
    __nanosleep(nap);
    if (nap < 16384)
      nap *= 2;
  }
}

// Copy of request descriptor `src` in this block's shared memory, read
// through L2 (an open launch's descriptors are written by the host after the
// launch started, so a line cached in L1 from a neighbouring descriptor may be
// stale). Called by every thread of the block.
KR_DEV void load_request(CyclicRequestDev *dst, const CyclicRequestDev *src) {
  static_assert(sizeof(CyclicRequestDev) % 8 == 0, "descriptor size");
  const unsigned long long *s8 = reinterpret_cast<const unsigned long long *>(src);
  unsigned long long *d8 = reinterpret_cast<unsigned long long *>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(CyclicRequestDev) / 8); i += blockDim.x)
    d8[i] = __ldcg(s8 + i);
  __syncthreads();
}

// Open launches: copy a finished request's result to its host-mapped
// completion record, then raise its flag (leader thread only).
KR_DEV void publish_done(const CyclicRequestDev &rq) {
  if (!rq.done)
    return;
  static_assert(sizeof(CyclicDevResult) % 8 == 0, "result size");
  HostDone *h = rq.done;
  const volatile unsigned long long *src = reinterpret_cast<const volatile unsigned long long *>(rq.res);
  volatile unsigned long long *dst = reinterpret_cast<volatile unsigned long long *>(&h->res);
  for (int i = 0; i < (int)(sizeof(CyclicDevResult) / 8); i++)
    dst[i] = src[i];
  h->max_resid = *(volatile double *)rq.max_resid;
  h->status = *(volatile int32_t *)rq.status;
  __threadfence_system();
  *(volatile int32_t *)&h->done = 1;
}

// One request on one thread block, with its workspace laid out in `slot`.
template <class KT>
__device__ __noinline__ void run_cta_request(TeamShared *sh, CyclicDesc *dp, const CyclicRequestDev &rq,
                                             char *slot) {
  CyclicDesc &d = *dp;
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
    d.nb_init = rq.nb_init;
    d.frob_init = rq.frob_init;
    if (rq.basis) // else the basis stays in the workspace (own_basis)
      d.basis = rq.basis;
    d.ldb = rq.plan.ldb;
    d.status = rq.status;
    d.res = rq.res;
    // CG vectors in dynamic shared memory when the launch gave enough of it
    // (the solver reaches them through generic pointers)
    uint32_t dyn;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (cta_cg_smem_bytes(rq.plan.ldm, rq.plan.ldn) <= (size_t)dyn) {
      d.rp = reinterpret_cast<double2 *>(kr_dyn_smem);
      d.Ap = reinterpret_cast<double *>(kr_dyn_smem + 16 * rq.plan.ldm);
      d.tn = reinterpret_cast<double *>(kr_dyn_smem + 24 * rq.plan.ldm);
    }
    rq.res->t_begin = globaltimer_ns();
  }
  __syncthreads();
  if (!rq.trivial) {
    TeamCta tm{sh, d.status, 0};
    CyclicSolver<TeamCta, KT> s(tm, d);
    s.run();
    __syncthreads();
    const int64_t nf = *(volatile int64_t *)&d.res->n_found;
    const double mr = team_max_residual(tm, d.F, d.basis, d.ldb, nf);
    if (threadIdx.x == 0)
      *rq.max_resid = mr;
  }
  if (threadIdx.x == 0) {
    rq.res->t_end = globaltimer_ns();
    publish_done(rq);
  }
  __syncthreads();
}

// Persistent kernel, one thread block per request: blocks take requests from
// the device queue until it is empty. Block b owns workspace slot b.
template <class KT>
__global__ void __launch_bounds__(512, KR_BATCH_MIN_BLOCKS) cyclic_batch_kernel(const CyclicRequestDev *reqs,
                                                                               int count, int *queue, char *ws,
                                                                               size_t ws_stride,
                                                                               const LaunchFeed *feed) {
  __shared__ TeamShared sh;
  __shared__ CyclicDesc d;
  __shared__ CyclicRequestDev rq;
  __shared__ int s_item;
  char *slot = ws + (size_t)blockIdx.x * ws_stride;
  for (;;) {
    if (threadIdx.x == 0)
      s_item = take_request(queue, count, feed, 2);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item < 0)
      break;
    load_request(&rq, reqs + item);
    run_cta_request<KT>(&sh, &d, rq, slot);
  }
}

// Persistent kernel over a batch with large and small requests. Each
// thread-block cluster first takes large requests (a TeamCluster per request,
// the cluster's rank 0 draws from the large queue); once that queue is empty,
// every block of every cluster keeps going on its own with small requests
// (one-block teams), so no SM idles while work of either kind remains.
// Cluster c owns large slot c; block b owns small slot b.
// One large request on this thread-block cluster, workspace in `slot`.
template <class KT>
__device__ __noinline__ void run_cluster_request(TeamShared *sh, CyclicDesc *dp, const CyclicRequestDev &rq,
                                                 char *slot, unsigned rank, unsigned csize, int &cbuf) {
  CyclicDesc &d = *dp;
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
    d.nb_init = rq.nb_init;
    d.frob_init = rq.frob_init;
    if (rq.basis) // else the basis stays in the workspace (own_basis)
      d.basis = rq.basis;
    d.ldb = rq.plan.ldb;
    d.status = rq.status;
    d.res = rq.res;
  }
  __syncthreads();
  if (rank == 0 && threadIdx.x == 0)
    rq.res->t_begin = globaltimer_ns();
  if (!rq.trivial) {
    TeamCluster tm{sh, d.status, 0, cbuf, rank, csize};
    CyclicSolver<TeamCluster, KT> s(tm, d);
    s.run();
    tm.sync();
    const int64_t nf = *(volatile int64_t *)&d.res->n_found;
    const double mr = team_max_residual(tm, d.F, d.basis, d.ldb, nf);
    if (tm.leader())
      *rq.max_resid = mr;
    cbuf = tm.cbuf;
  }
  if (rank == 0 && threadIdx.x == 0) {
    rq.res->t_end = globaltimer_ns();
    publish_done(rq);
  }
  cooperative_groups::this_cluster().sync();
}

// Persistent kernel over a batch with large and small requests. Each
// thread-block cluster takes large requests (a TeamCluster per request, the
// cluster's rank 0 draws from the large queue); when there is none, every
// block of every cluster goes on by itself with small requests (one-block
// teams), so no SM idles while work of either kind remains. In a closed launch
// (feed == nullptr) that happens once the large queue is empty. In an open
// launch (the server publishes requests while it runs) the cluster serves
// small requests while no large one is waiting and regroups as soon as one
// is (each block checks before taking its next small request), and leaves
// once neither queue has had work for the feed's idle time.
// Cluster c owns large slot c; block b owns small slot b.
template <class KT>
__global__ void __launch_bounds__(512, KR_BATCH_MIN_BLOCKS)
    cyclic_batch_cluster_kernel(const CyclicRequestDev *reqs_large, int n_large, int *queue_large, char *ws_large,
                                size_t stride_large, const CyclicRequestDev *reqs_small, int n_small,
                                int *queue_small, char *ws_small, size_t stride_small, const LaunchFeed *feed,
                                int feed_large) {
  __shared__ TeamShared sh;
  __shared__ CyclicDesc d;
  __shared__ CyclicRequestDev rq;
  __shared__ int s_item, s_back;
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  const unsigned rank = cl.block_rank(), csize = cl.num_blocks();
  char *slot = ws_large + (size_t)(blockIdx.x / csize) * stride_large;
  char *cslot = ws_small + (size_t)blockIdx.x * stride_small;
  int cbuf = 0;
  if (!feed) {
    for (;;) {
      if (rank == 0 && threadIdx.x == 0)
        s_item = take_request(queue_large, n_large, nullptr, feed_large);
      cl.sync();
      const int item = *cl.map_shared_rank(&s_item, 0);
      cl.sync();
      if (item < 0)
        break;
      load_request(&rq, reqs_large + item);
      run_cluster_request<KT>(&sh, &d, rq, slot, rank, csize, cbuf);
    }
    // small requests, block by block (no cluster-wide synchronisation below)
    for (;;) {
      if (threadIdx.x == 0)
        s_item = take_request(queue_small, n_small, nullptr, 2);
      __syncthreads();
      const int item = s_item;
      __syncthreads();
      if (item < 0)
        break;
      load_request(&rq, reqs_small + item);
      run_cta_request<KT>(&sh, &d, rq, cslot);
    }
    return;
  }
  for (;;) {
    // large requests while there are any; give way when only small ones wait
    int large_end;
    for (;;) {
      if (rank == 0 && threadIdx.x == 0)
        s_item = take_request(queue_large, n_large, feed, feed_large, queue_small, 2);
      cl.sync();
      const int item = *cl.map_shared_rank(&s_item, 0);
      cl.sync();
      if (item < 0) {
        large_end = item;
        break;
      }
      load_request(&rq, reqs_large + item);
      run_cluster_request<KT>(&sh, &d, rq, slot, rank, csize, cbuf);
    }
    // small requests block by block, until large work waits (back to the
    // cluster) or none comes for the idle time
    if (threadIdx.x == 0)
      s_back = 0;
    for (;;) {
      if (threadIdx.x == 0) {
        // large work first; a block waiting for small work also returns when some arrives
        int it = work_pending(queue_large, feed, feed_large)
                     ? kTakeYield
                     : take_request(queue_small, n_small, feed, 2, queue_large, feed_large);
        if (it == kTakeYield) {
          s_back = 1;
          it = -1;
        }
        s_item = it;
      }
      __syncthreads();
      const int item = s_item;
      __syncthreads();
      if (item < 0)
        break;
      load_request(&rq, reqs_small + item);
      run_cta_request<KT>(&sh, &d, rq, cslot);
    }
    // regroup; leave when the large phase ended (not yielded) and no block
    // came back for large work
    cl.sync();
    int back = 0;
    for (unsigned r = 0; r < csize; r++)
      back |= *cl.map_shared_rank(&s_back, r);
    cl.sync();
    if (!back && large_end != kTakeYield)
      break;
  }
}

} // namespace kr
