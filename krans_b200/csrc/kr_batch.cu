// Host side of batched solves (krans_solve_batch) and of the serving loop
// (krans_server_*): request admission against an HBM budget, persistent
// launches on a pool of streams, completion tracking and latencies.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <numeric>
#include <thread>
#include <vector>

#include "kr_internal.h"
#include "kr_types.cuh"

namespace kr {


static void mt_seed(RngState &s, uint32_t seed) {
  memset(&s, 0, sizeof s);
  s.mt[0] = seed;
  for (int i = 1; i < 624; i++)
    s.mt[i] = 1812433253u * (s.mt[i - 1] ^ (s.mt[i - 1] >> 30)) + (uint32_t)i;
  s.idx = 624;
}

using Clock = std::chrono::steady_clock;
static double ms_since(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Idle time after which a team of an open launch leaves (no request in sight).
constexpr uint64_t kOpenIdleNs = 20ull * 1000ull * 1000ull;
// SMs an open launch leaves free: matrix set-up kernels (transposes) and the
// server's LOBPCG launches run there while the open launch stays resident.
constexpr int kOpenReserveSms = 20;

// Result fields of a finished cyclic request.
static void fill_result(const CyclicDevResult &r, double max_resid, int32_t status, bool trivial, int64_t k_target,
                        krans_request_result *out) {
  out->status = status != 0 ? status : r.status;
  if (trivial) {
    out->converged_to_target = k_target == 0 ? 1 : 0;
    return;
  }
  out->converged_to_target = r.converged;
  out->n_right = r.n_found;
  out->restarts = r.restarts;
  out->krylov_steps_total = r.krylov_steps_total;
  out->cg_solves = r.cg_solves;
  out->cg_maxit_hits = r.cg_maxit_hits;
  out->spmv = r.spmv;
  out->spmvT = r.spmvT;
  out->frob_norm_est = r.frob;
  out->max_residual = max_resid;
  out->algo_bytes = r.bytes;
  for (int q = 0; q < 4; q++)
    out->phase_ms[q] = r.phase_ms[q];
}

// One persistent launch over a set of requests. A closed launch
// (krans_solve_batch) runs a fixed set. An open launch (the server) starts
// with a set and takes more while it runs: the host writes a new request into
// a free descriptor slot of its size class and raises that queue's count in a
// host-mapped feed; a team with nothing to do claims it (take_request); each
// finished request raises its host-mapped completion record. The teams of an
// open launch leave after kOpenIdleNs without work, or once the host closes
// the launch, so every wait ends.
struct BatchLaunch {
  krans_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  bool open = false;
  int count = 0; // initial requests
  int precision = 0;
  int grid = 0;        // blocks of the launch (CTA teams of small requests)
  int n_large = 0;     // initial requests on clusters of csize blocks
  int n_mid = 0;       // initial requests on 2-block clusters (pairs)
  int npairs = 0;      // pair clusters of the second launch (the SMs the big clusters leave free)
  size_t stride_M = 0; // workspace slot of one pair
  size_t dyn_smem = 0; // dynamic shared memory per block (CG vectors of one-block solves)
  int csize = 8;       // blocks per cluster
  int nclusters = 0;   // resident clusters of the cluster launch
  size_t stride_L = 0; // workspace slot of one cluster
  int64_t cluster_min = 0, pair_max = 0;
  cudaStream_t aux = nullptr;
  cudaEvent_t evj = nullptr;
  std::vector<int> order; // position in launch -> index in the caller's array
  // descriptor slots: queue q (0 large, 1 mid, 2 small) owns [base[q], base[q] + cap[q])
  int cap[3] = {0, 0, 0}, base[3] = {0, 0, 0}, npub[3] = {0, 0, 0};
  int slots = 0, max_total = 0, published_total = 0;
  CyclicRequestDev *d_reqs = nullptr;
  CyclicDevResult *d_res = nullptr;
  int32_t *d_status = nullptr;
  double *d_mr = nullptr;
  RngState *d_rng = nullptr;
  int *d_queue = nullptr;
  char *ws = nullptr, *meta = nullptr;
  size_t ws_bytes = 0, ws_stride = 0, meta_bytes = 0;
  CyclicDevResult *h_res = nullptr;
  int32_t *h_status = nullptr;
  double *h_mr = nullptr;
  int *h_queue = nullptr;                           // queue counters once the launch ended
  LaunchFeed *feed = nullptr, *feed_dev = nullptr;   // host-mapped (open launches)
  HostDone *hdone = nullptr, *hdone_dev = nullptr;   // host-mapped (open launches)
  std::vector<char> slot_trivial;                    // per slot: nothing to compute
  std::vector<int64_t> slot_kt;                      // per slot: k_target
  cudaStream_t cs = nullptr;                         // publishing copies
  cudaEvent_t evc = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  std::vector<CyclicRequestDev> hreq;
  std::vector<RngState> hrng;

  int classify(const krans_mat *A) const {
    const int64_t sz = A->m + A->n;
    if (cluster_min <= 0 || sz < cluster_min)
      return 2;
    return (npairs > 0 && sz < pair_max) ? 1 : 0;
  }

  // Descriptor and RNG stream of one request (no per-slot pointers yet);
  // *carve = its workspace bytes (0 if trivial).
  int describe(const krans_request &r, CyclicRequestDev &q, RngState &s, size_t *carve) const {
    KR_CHECK_ARG(r.A && r.A->ctx == ctx, "krans_solve_batch: request without a matrix of this context");
    KR_CHECK_ARG(r.solver == KRANS_SOLVER_CYCLIC, "krans_solve_batch: batched launches take cyclic requests");
    KR_CHECK_ARG(r.opts.precision == precision, "krans_solve_batch: one precision per batch");
    KR_CHECK_ARG(precision == KRANS_PREC_FP64 || r.A->v32,
                 "krans_solve_batch: mixed precision needs matrices created with KRANS_CSR_FP32");
    const krans_mat *A = r.A;
    memset(&q, 0, sizeof q);
    q.F = CsrView{A->m, A->n, A->nnz, A->rp, A->ci, A->v, A->v32, tuned_lanes(A->ctx, A->m, A->nnz), A->ulen};
    q.B = CsrView{A->n, A->m, A->nnz, A->rpT, A->ciT, A->vT, A->vT32, tuned_lanes(A->ctx, A->n, A->nnz), A->ulenT};
    q.o = r.opts;
    q.o.team = KRANS_TEAM_CTA;
    int64_t kt = (r.opts.nullity_known >= 0) ? (int64_t)r.opts.nullity_known : r.opts.k;
    int trivial = 0;
    if (A->m == 0 || A->n == 0 || kt == 0 || (r.opts.rank_known >= 0 && A->n <= r.opts.rank_known))
      trivial = 1;
    const int64_t ncv = std::max<int64_t>(std::max<int64_t>(2, r.opts.ncv), kt + 2);
    KR_CHECK_ARG(kt <= 128 && ncv <= 256, "krans_solve_batch: k <= 128 and ncv <= 256 per request");
    KR_CHECK_ARG(r.opts.precond_aat >= KRANS_PRECOND_NONE && r.opts.precond_aat <= KRANS_PRECOND_SD &&
                     r.opts.precond_steps >= 1 && r.opts.precond_steps <= 1000,
                 "krans_solve_batch: precond_aat must be a KRANS_PRECOND_* value, precond_steps in [1, 1000]");
    if (!trivial && r.basis_out)
      KR_CHECK_ARG(r.basis_capacity >= kt, "krans_solve_batch: basis_out too small");
    q.trivial = trivial;
    q.plan.m = A->m;
    q.plan.n = A->n;
    q.plan.k_target = kt;
    q.plan.ncv = ncv;
    q.plan.ldn = kr_round_up(std::max<int64_t>(A->n, 1), 32);
    q.plan.ldm = kr_round_up(std::max<int64_t>(A->m, 1), 32);
    q.plan.ldb = A->n;
    q.plan.cap = ncv / 2 + 2;
    q.plan.ksz = precision == KRANS_PREC_MIXED ? 4 : 8;
    q.plan.grid_blocks = 1;
    q.plan.own_basis = r.basis_out ? 0 : 1; // no output buffer: the basis stays in the workspace
    q.plan.block_polish = r.opts.polish_block ? 1 : 0;
    q.plan.precond = r.opts.precond_aat;
    q.basis = r.basis_out;
    *carve = trivial ? 0 : cyclic_carve(q.plan, nullptr, nullptr);
    uint32_t seed = r.seed ? r.seed : 0x9E3779B9u;
    mt_seed(s, seed);
    s.philox_key = ((uint64_t)seed << 32) ^ 0x9E3779B97F4A7C15ull;
    s.mode = r.rng_mode;
    return KRANS_OK;
  }

  // workspace of a plain request of m + n = sz (k 16, ncv 48): the slot size
  // an open launch gives its small and mid queues, so that later arrivals of
  // those classes fit
  size_t class_floor(int64_t sz) const {
    CyclicPlan p{};
    p.m = p.n = sz;
    p.k_target = 16;
    p.ncv = 48;
    p.ldn = p.ldm = p.ldb = kr_round_up(std::max<int64_t>(sz, 1), 32);
    p.cap = p.ncv / 2 + 2;
    p.ksz = precision == KRANS_PREC_MIXED ? 4 : 8;
    p.grid_blocks = 1;
    p.own_basis = 1;
    return cyclic_carve(p, nullptr, nullptr);
  }

  int slot_of(int pos) const {
    if (!open)
      return pos;
    if (pos < n_large)
      return base[0] + pos;
    if (pos < n_large + n_mid)
      return base[1] + (pos - n_large);
    return base[2] + (pos - n_large - n_mid);
  }

  // Size the launch (no allocation): returns bytes of device memory needed.
  // open: the launch keeps taking requests (at most max_total in all);
  // floors: size the small and mid slots for any request of those classes.
  int plan(krans_ctx *c, const krans_request *reqs, int n, size_t *need, bool open_ = false, int max_total_ = 0,
           bool floors = true) {
    ctx = c;
    open = open_;
    count = n;
    precision = n > 0 ? reqs[0].opts.precision : 0;
    order.resize(n);
    std::iota(order.begin(), order.end(), 0);
    cluster_min = ctx->tune.cluster_min;
    pair_max = ctx->tune.pair_max;
    csize = ctx->tune.cluster_size;
    // Size classes (by m + n only, so a request runs on the same kind of
    // team, with the same rounding, in any batch): big ones on clusters of
    // csize blocks; mid-size ones on 2-block clusters launched next to them
    // on the SMs the big clusters cannot tile (a GPC holds whole clusters
    // only); small ones on single blocks.
    const bool mixed = precision == KRANS_PREC_MIXED;
    const int reserve = open ? kOpenReserveSms : 0;
    {
      const int maxc = cyclic_batch_cluster_max(mixed, csize, ctx->sms, 0);
      npairs = csize > 2 && pair_max > cluster_min ? std::max(0, (ctx->sms - maxc * csize - reserve) / 2) : 0;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      const int ca = classify(reqs[a].A), cb = classify(reqs[b].A);
      if (ca != cb)
        return ca < cb;
      return reqs[a].A->nnz > reqs[b].A->nnz;
    });
    n_large = n_mid = 0;
    for (int pos = 0; pos < n; pos++) {
      KR_CHECK_ARG(reqs[order[pos]].A, "krans_solve_batch: request without a matrix");
      const int cl = classify(reqs[order[pos]].A);
      n_large += cl == 0;
      n_mid += cl == 1;
    }
    hreq.assign(n, CyclicRequestDev{});
    hrng.assign(n, RngState{});
    ws_stride = stride_L = stride_M = 256;
    for (int pos = 0; pos < n; pos++) {
      size_t cv = 0;
      const int rc = describe(reqs[order[pos]], hreq[pos], hrng[pos], &cv);
      if (rc != KRANS_OK)
        return rc;
      if (pos < n_large)
        stride_L = std::max(stride_L, cv);
      else if (pos < n_large + n_mid)
        stride_M = std::max(stride_M, cv);
      else
        ws_stride = std::max(ws_stride, cv);
    }
    if (open && floors) {
      ws_stride = std::max(ws_stride, class_floor(cluster_min));
      if (npairs > 0)
        stride_M = std::max(stride_M, class_floor(pair_max));
    }
    ws_stride = (size_t)kr_round_up((int64_t)ws_stride, 256);
    stride_L = (size_t)kr_round_up((int64_t)stride_L, 256);
    stride_M = (size_t)kr_round_up((int64_t)stride_M, 256);
    const int n_small = n - n_large - n_mid;
    // dynamic shared memory for the CG vectors of one-block solves: the
    // largest small request that fits under the cap
    dyn_smem = 0;
    for (int pos = n_large + n_mid; pos < n; pos++) {
      const size_t b = cta_cg_smem_bytes(hreq[pos].plan.ldm, hreq[pos].plan.ldn);
      if (b <= cta_smem_cap())
        dyn_smem = std::max(dyn_smem, b);
    }
    const int per_sm = cyclic_batch_cta_per_sm(mixed);
    grid = n_small > 0 ? std::max(1, std::min(n_small, ctx->sms * per_sm)) : 0;
    nclusters = 0;
    if (!open && n_mid == 0)
      npairs = 0;
    if (open || n_large > 0 || n_mid > 0) {
      // one cluster launch fills the GPC clusters; its blocks take the small
      // requests after the large queue is empty (one small-request slot per block)
      const int maxc = cyclic_batch_cluster_max(mixed, csize, ctx->sms, dyn_smem);
      nclusters = std::max(1, maxc);
      grid = nclusters * csize;
    }
    if (open) {
      max_total = std::max(max_total_, n);
      cap[0] = cap[2] = max_total;
      cap[1] = npairs > 0 ? max_total : 0;
      base[0] = 0;
      base[1] = cap[0];
      base[2] = cap[0] + cap[1];
      slots = cap[0] + cap[1] + cap[2];
      npub[0] = n_large;
      npub[1] = n_mid;
      npub[2] = n_small;
      published_total = n;
    } else {
      slots = n;
    }
    meta_bytes = (size_t)std::max(slots, 1) *
                     (sizeof(CyclicRequestDev) + sizeof(CyclicDevResult) + 4 + 8 + sizeof(RngState)) +
                 4096;
    ws_bytes = (size_t)(grid + 2 * npairs) * ws_stride + (size_t)nclusters * stride_L +
               (size_t)npairs * stride_M + 256;
    *need = ws_bytes + meta_bytes;
    return KRANS_OK;
  }

  int alloc_and_launch(cudaStream_t s) {
    stream = s;
    int rc = dev_alloc_async(ctx, (void **)&ws, ws_bytes, s);
    if (rc != KRANS_OK)
      return rc;
    rc = dev_alloc_async(ctx, (void **)&meta, meta_bytes, s);
    if (rc != KRANS_OK) {
      dev_free_async(ctx, ws, ws_bytes, s);
      ws = nullptr;
      return rc;
    }
    Carver c;
    c.base = meta;
    d_reqs = c.take<CyclicRequestDev>(slots);
    d_res = c.take<CyclicDevResult>(slots);
    d_status = c.take<int32_t>(slots);
    d_mr = c.take<double>(slots);
    d_rng = c.take<RngState>(slots);
    d_queue = c.take<int>(4);
    slot_trivial.assign((size_t)std::max(slots, 1), 0);
    slot_kt.assign((size_t)std::max(slots, 1), 0);
    cudaError_t e = cudaSuccess;
    if (open) {
      e = cudaHostAlloc(&feed, sizeof(LaunchFeed), cudaHostAllocMapped);
      if (e == cudaSuccess)
        e = cudaHostAlloc(&hdone, sizeof(HostDone) * (size_t)slots, cudaHostAllocMapped);
      if (e == cudaSuccess)
        e = cudaHostGetDevicePointer((void **)&feed_dev, feed, 0);
      if (e == cudaSuccess)
        e = cudaHostGetDevicePointer((void **)&hdone_dev, hdone, 0);
      if (e == cudaSuccess) {
        memset(hdone, 0, sizeof(HostDone) * (size_t)slots);
        memset(feed, 0, sizeof(LaunchFeed));
        for (int q = 0; q < 3; q++)
          feed->published[q] = npub[q];
        feed->idle_ns = kOpenIdleNs;
        e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
      }
      if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&evc, cudaEventDisableTiming);
    }
    for (int pos = 0; pos < count; pos++) {
      const int g = slot_of(pos);
      hreq[pos].res = d_res + g;
      hreq[pos].status = d_status + g;
      hreq[pos].max_resid = d_mr + g;
      hreq[pos].rng = d_rng + g;
      hreq[pos].done = open ? hdone_dev + g : nullptr;
      slot_trivial[(size_t)g] = (char)hreq[pos].trivial;
      slot_kt[(size_t)g] = hreq[pos].plan.k_target;
    }
    if (e == cudaSuccess)
      e = cudaMallocHost(&h_res, sizeof(CyclicDevResult) * (size_t)std::max(count, 1));
    if (e == cudaSuccess)
      e = cudaMallocHost(&h_status, 4 * (size_t)std::max(count, 1));
    if (e == cudaSuccess)
      e = cudaMallocHost(&h_mr, 8 * (size_t)std::max(count, 1));
    if (e == cudaSuccess)
      e = cudaMallocHost(&h_queue, 4 * sizeof(int));
    if (e == cudaSuccess)
      e = cudaEventCreate(&ev0);
    if (e == cudaSuccess)
      e = cudaEventCreate(&ev1);
    if (e == cudaSuccess)
      e = cudaEventCreateWithFlags(&ev2, cudaEventDisableTiming);
    // initial descriptors: positions are grouped by class, slots by queue
    const int runs[3][2] = {{0, n_large}, {n_large, n_mid}, {n_large + n_mid, count - n_large - n_mid}};
    for (int q = 0; q < 3 && e == cudaSuccess; q++) {
      const int p0 = runs[q][0], len = runs[q][1];
      if (len <= 0)
        continue;
      const int g0 = slot_of(p0);
      e = cudaMemcpyAsync(d_reqs + g0, hreq.data() + p0, sizeof(CyclicRequestDev) * (size_t)len,
                          cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_rng + g0, hrng.data() + p0, sizeof(RngState) * (size_t)len, cudaMemcpyHostToDevice,
                            s);
    }
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_res, 0, sizeof(CyclicDevResult) * (size_t)slots, s);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_status, 0, 4 * (size_t)slots, s);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_mr, 0, 8 * (size_t)slots, s);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_queue, 0, 4 * sizeof(int), s);
    if (e == cudaSuccess)
      e = cudaEventRecord(ev0, s);
    if (e == cudaSuccess && cs) // publishing copies land in the stream-ordered allocation: after its set-up
      e = cudaStreamWaitEvent(cs, ev0, 0);
    char *ws_small = ws, *ws_small_p = ws + (size_t)grid * ws_stride;
    char *ws_large = ws_small_p + (size_t)2 * npairs * ws_stride;
    char *ws_mid = ws_large + (size_t)nclusters * stride_L;
    const bool mixed = precision == KRANS_PREC_MIXED;
    const int first_small = open ? base[2] : n_large + n_mid;
    const int n_small_q = open ? cap[2] : count - first_small;
    const CyclicRequestDev *q_mid = d_reqs + (open ? base[1] : n_large);
    if (e == cudaSuccess && npairs > 0) {
      // the pair launch runs beside the big clusters on its own stream; the
      // launch's end event waits for both
      e = cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking);
      if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&evj, cudaEventDisableTiming);
    }
    if (e == cudaSuccess && npairs > 0)
      e = cudaStreamWaitEvent(aux, ev0, 0); // the pairs start after the set-up copies
    if (e == cudaSuccess) {
      if (nclusters > 0) {
        e = launch_cyclic_batch_cluster(mixed, nclusters, csize, dyn_smem, s, d_reqs, n_large, d_queue, ws_large,
                                        stride_L, d_reqs + first_small, n_small_q, d_queue + 1, ws_small,
                                        ws_stride, feed_dev, 0);
        if (e == cudaSuccess && npairs > 0) {
          e = launch_cyclic_batch_cluster(mixed, npairs, 2, dyn_smem, aux, q_mid, n_mid, d_queue + 2, ws_mid,
                                          stride_M, d_reqs + first_small, n_small_q, d_queue + 1, ws_small_p,
                                          ws_stride, feed_dev, 1);
          if (e == cudaSuccess)
            e = cudaEventRecord(evj, aux);
          if (e == cudaSuccess)
            e = cudaStreamWaitEvent(s, evj, 0);
        }
      } else
        e = launch_cyclic_batch_cta(mixed, grid, 512, dyn_smem, s, d_reqs, count, d_queue + 1, ws_small, ws_stride,
                                    nullptr);
    }
    if (e == cudaSuccess)
      e = cudaEventRecord(ev1, s);
    if (e == cudaSuccess && !open)
      e = cudaMemcpyAsync(h_res, d_res, sizeof(CyclicDevResult) * (size_t)count, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && !open)
      e = cudaMemcpyAsync(h_status, d_status, 4 * (size_t)count, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && !open)
      e = cudaMemcpyAsync(h_mr, d_mr, 8 * (size_t)count, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h_queue, d_queue, 4 * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaEventRecord(ev2, s);
    if (e != cudaSuccess)
      return cuda_fail(e, "batch launch", __FILE__, __LINE__);
    return KRANS_OK;
  }

  // Open launch: publish one more request. Returns 1 and its slot when
  // published, 0 when it does not fit this launch (its class is full, its
  // workspace exceeds the class's slot, the launch is closed or ended, or
  // its precision differs), or a negative code for an invalid request. The
  // caller has made sure the request's matrix is ready on the device.
  int try_publish(const krans_request &r, int *slot) {
    if (!open || !feed || feed->closed || published_total >= max_total || done())
      return 0;
    if (r.opts.precision != precision)
      return 0;
    CyclicRequestDev q;
    RngState s;
    size_t cv = 0;
    const int rc = describe(r, q, s, &cv);
    if (rc != KRANS_OK)
      return rc;
    const int cl = classify(r.A);
    const size_t stride = cl == 0 ? stride_L : cl == 1 ? stride_M : ws_stride;
    if (npub[cl] >= cap[cl] || cv > stride || (cl == 0 && nclusters == 0) || (cl == 1 && npairs == 0))
      return 0;
    const int g = base[cl] + npub[cl];
    q.res = d_res + g;
    q.status = d_status + g;
    q.max_resid = d_mr + g;
    q.rng = d_rng + g;
    q.done = hdone_dev + g;
    hdone[g].done = 0;
    slot_trivial[(size_t)g] = (char)q.trivial;
    slot_kt[(size_t)g] = q.plan.k_target;
    cudaError_t e = cudaMemcpyAsync(d_reqs + g, &q, sizeof q, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_rng + g, &s, sizeof s, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_res + g, 0, sizeof(CyclicDevResult), cs);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_status + g, 0, 4, cs);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_mr + g, 0, 8, cs);
    if (e == cudaSuccess)
      e = cudaEventRecord(evc, cs);
    if (e == cudaSuccess)
      e = cudaEventSynchronize(evc); // the copies (host stack buffers) are complete before the count moves
    if (e != cudaSuccess)
      return cuda_fail(e, "publish request", __FILE__, __LINE__);
    std::atomic_thread_fence(std::memory_order_seq_cst);
    ((volatile int32_t *)feed->published)[cl] = npub[cl] + 1;
    npub[cl]++;
    published_total++;
    *slot = g;
    return 1;
  }

  // stop a published request: its team sees the status word at its next
  // check and unwinds (copied on `ctl`, beside the running kernel)
  int cancel_slot(int g, cudaStream_t ctl) const {
    static const int32_t cancelled = KRANS_ERR_CANCELLED;
    cudaError_t e = cudaMemcpyAsync(d_status + g, &cancelled, 4, cudaMemcpyHostToDevice, ctl);
    return e == cudaSuccess ? KRANS_OK : cuda_fail(e, "cancel request", __FILE__, __LINE__);
  }

  void close() {
    if (open && feed) {
      std::atomic_thread_fence(std::memory_order_seq_cst);
      ((volatile LaunchFeed *)feed)->closed = 1;
    }
  }

  // queue of a slot, and whether a team claimed it (valid once done())
  int queue_of(int g) const { return g >= base[2] ? 2 : (g >= base[1] && cap[1] > 0) ? 1 : 0; }
  bool claimed(int g) const {
    const int q = queue_of(g);
    const int counter = h_queue[q == 0 ? 0 : q == 1 ? 2 : 1];
    return g - base[q] < counter;
  }
  bool slot_done(int g) const { return open && ((volatile HostDone *)hdone)[g].done != 0; }

  void fill_slot(int g, krans_request_result *out) const {
    const HostDone &h = hdone[g];
    memset(out, 0, sizeof *out);
    fill_result(h.res, h.max_resid, h.status, slot_trivial[(size_t)g] != 0, slot_kt[(size_t)g], out);
    if (h.res.t_end >= h.res.t_begin && h.res.t_begin)
      out->device_ms = (double)(h.res.t_end - h.res.t_begin) * 1e-6;
  }

  bool done() const { return cudaEventQuery(ev2) == cudaSuccess; }

  double device_ms() const {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    return ms;
  }

  // earliest device start of any request of this launch (globaltimer ns)
  uint64_t t0() const {
    uint64_t t = ~0ull;
    for (int i = 0; i < count; i++)
      if (h_res[i].t_begin && h_res[i].t_begin < t)
        t = h_res[i].t_begin;
    return t == ~0ull ? 0 : t;
  }

  // closed launches: result of launch position pos
  void fill(int pos, krans_request_result *out) const {
    const CyclicDevResult &r = h_res[pos];
    memset(out, 0, sizeof *out);
    const uint64_t z = t0();
    if (z && r.t_begin >= z && r.t_end >= r.t_begin) {
      out->queue_ms = (double)(r.t_begin - z) * 1e-6;   // wait for a free team inside the launch
      out->latency_ms = (double)(r.t_end - z) * 1e-6;   // launch start -> request done
    }
    fill_result(r, h_mr[pos], h_status[pos], hreq[pos].trivial != 0, hreq[pos].plan.k_target, out);
  }

  // Device memory is freed in the launch's stream order (cudaFreeAsync: no
  // wait for other launches still running); pinned host buffers go to
  // `graveyard` when one is given (cudaFreeHost waits for the whole device;
  // the server frees them once nothing runs), else are freed here.
  void release(std::vector<void *> *graveyard = nullptr) {
    if (ws)
      dev_free_async(ctx, ws, ws_bytes, stream);
    if (meta)
      dev_free_async(ctx, meta, meta_bytes, stream);
    ws = meta = nullptr;
    d_reqs = nullptr;
    for (void *h : {(void *)h_res, (void *)h_status, (void *)h_mr, (void *)h_queue, (void *)feed, (void *)hdone})
      if (h) {
        if (graveyard)
          graveyard->push_back(h);
        else
          cudaFreeHost(h);
      }
    h_res = nullptr;
    h_status = nullptr;
    h_mr = nullptr;
    h_queue = nullptr;
    feed = nullptr;
    hdone = nullptr;
    if (aux)
      cudaStreamDestroy(aux);
    aux = nullptr;
    if (cs)
      cudaStreamDestroy(cs);
    cs = nullptr;
    if (evc)
      cudaEventDestroy(evc);
    evc = nullptr;
    if (evj)
      cudaEventDestroy(evj);
    evj = nullptr;
    if (ev0)
      cudaEventDestroy(ev0);
    if (ev1)
      cudaEventDestroy(ev1);
    if (ev2)
      cudaEventDestroy(ev2);
    ev0 = ev1 = ev2 = nullptr;
  }
};

} // namespace kr

using namespace kr;

extern "C" int krans_solve_batch(krans_ctx *ctx, int64_t count, const krans_request *reqs,
                                 krans_request_result *results, double *device_ms) {
  KR_CHECK_ARG(ctx && (count == 0 || (reqs && results)), "krans_solve_batch: NULL argument");
  KR_CHECK_ARG(count >= 0 && count < (1 << 30), "krans_solve_batch: bad count");
  if (device_ms)
    *device_ms = 0.0;
  if (count == 0)
    return KRANS_OK;
  KR_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lk(ctx->mu);
  BatchLaunch L;
  size_t need = 0;
  int rc = L.plan(ctx, reqs, (int)count, &need);
  if (rc != KRANS_OK)
    return rc;
  rc = L.alloc_and_launch(ctx->stream);
  if (rc == KRANS_OK) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
      rc = cuda_fail(e, "batch", __FILE__, __LINE__);
  }
  if (rc == KRANS_OK) {
    for (int pos = 0; pos < (int)count; pos++)
      L.fill(pos, &results[L.order[pos]]);
    if (device_ms)
      *device_ms = L.device_ms();
    for (int64_t i = 0; i < count; i++)
      results[i].device_ms = L.device_ms();
  }
  L.release();
  return rc;
}

// ---------------------------------------------------------------------------
// Serving: continuous batching. A scheduler thread keeps one open persistent
// launch of cyclic requests resident and publishes arriving requests into it
// (its idle teams claim them), starts the next launch for requests that do
// not fit the open one, runs LOBPCG requests as launches of their own on the
// other streams, and completes tickets as the device raises their completion
// records. Admission is bounded by the HBM budget.
// ---------------------------------------------------------------------------
namespace kr {
struct LobpcgAsync;
int lobpcg_async_plan(krans_ctx *ctx, const krans_request &r, LobpcgAsync **out, size_t *need);
int lobpcg_async_launch(LobpcgAsync *a, cudaStream_t s);
bool lobpcg_async_done(const LobpcgAsync *a);
void lobpcg_async_finish(const LobpcgAsync *a, krans_request_result *out);
void lobpcg_async_release(LobpcgAsync *a, std::vector<void *> *graveyard = nullptr);
int lobpcg_async_cancel(LobpcgAsync *a, cudaStream_t ctl);
} // namespace kr

struct ServerTicket {
  krans_request req;
  int state = 0; // 0 queued, 1 running, 2 done, 3 failed, 4 cancelled
  bool cancel_requested = false; // krans_cancel while running
  krans_request_result res;
  Clock::time_point submit_t, start_t, done_t;
};

struct InFlight {
  BatchLaunch L;            // cyclic requests (an open launch)
  LobpcgAsync *lob = nullptr; // or one LOBPCG request
  uint64_t lob_ticket = 0;
  struct Running {
    uint64_t ticket;
    int slot;
    Clock::time_point published;
  };
  std::vector<Running> running; // published, not yet completed
  size_t bytes = 0;
  int stream_idx = -1;
  int64_t id = 0;
};

struct krans_server {
  krans_ctx *ctx = nullptr;
  krans_server_opts opts;
  std::mutex mu;
  std::condition_variable cv;
  std::map<uint64_t, ServerTicket> tickets;
  std::deque<uint64_t> queue;
  std::vector<cudaStream_t> streams;
  std::vector<bool> stream_busy;
  cudaEvent_t ctx_ready = nullptr; // orders launches after work queued on the context's stream
  cudaStream_t ctl = nullptr;      // cancellations of running requests
  std::vector<InFlight *> inflight;
  InFlight *open = nullptr; // the launch that takes new cyclic requests
  std::deque<uint64_t> completed; // finished tickets not yet handed out by krans_server_completed
  std::vector<void *> graveyard;  // pinned host buffers of finished launches, freed once nothing runs
  void bury_if_idle() {
    if (!inflight.empty())
      return;
    for (void *h : graveyard)
      cudaFreeHost(h);
    graveyard.clear();
  }
  size_t bytes_in_use = 0;
  uint64_t next_ticket = 1;
  int64_t next_launch = 1;
  bool stop = false;
  std::thread worker;

  void run();
  int free_stream() const {
    for (size_t s = 0; s < streams.size(); s++)
      if (!stream_busy[s])
        return (int)s;
    return -1;
  }
  void fail(uint64_t id, int rc, Clock::time_point now) {
    ServerTicket &t = tickets[id];
    memset(&t.res, 0, sizeof t.res);
    t.res.status = rc;
    t.state = 3;
    t.start_t = t.done_t = now;
    t.res.latency_ms = ms_since(t.submit_t, now);
    completed.push_back(id);
  }
  void finish(uint64_t id, Clock::time_point now, int64_t launch) {
    ServerTicket &t = tickets[id];
    t.done_t = now;
    t.res.queue_ms = ms_since(t.submit_t, t.start_t);
    t.res.latency_ms = ms_since(t.submit_t, now);
    t.res.launch_id = launch;
    t.state = t.res.status == KRANS_OK ? 2 : t.res.status == KRANS_ERR_CANCELLED ? 4 : 3;
    completed.push_back(id);
  }
  bool admit_lobpcg(uint64_t id, Clock::time_point now);
  bool admit_cyclic(Clock::time_point now);
};

// LOBPCG request at the head of the queue: its own launch on a free stream.
// Returns true when the queue moved.
bool krans_server::admit_lobpcg(uint64_t id, Clock::time_point now) {
  ServerTicket &t = tickets[id];
  LobpcgAsync *a = nullptr;
  size_t need = 0;
  int rc = lobpcg_async_plan(ctx, t.req, &a, &need);
  if (rc != KRANS_OK) {
    fail(id, rc, now);
    queue.pop_front();
    return true;
  }
  if (need > opts.hbm_budget_bytes) {
    lobpcg_async_release(a);
    fail(id, KRANS_ERR_OUT_OF_MEMORY, now);
    queue.pop_front();
    return true;
  }
  const int fs = free_stream();
  if (fs < 0 || (bytes_in_use + need > opts.hbm_budget_bytes && !inflight.empty())) {
    lobpcg_async_release(a);
    return false; // wait for a stream or for memory
  }
  cudaError_t ew = cudaEventRecord(ctx_ready, ctx->stream);
  if (ew == cudaSuccess)
    ew = cudaStreamWaitEvent(streams[fs], ctx_ready, 0);
  rc = ew == cudaSuccess ? lobpcg_async_launch(a, streams[fs]) : cuda_fail(ew, "server stream order", __FILE__, __LINE__);
  queue.pop_front();
  if (rc != KRANS_OK) {
    lobpcg_async_release(a, &graveyard);
    fail(id, rc, now);
    return true;
  }
  auto *f = new InFlight();
  f->lob = a;
  f->lob_ticket = id;
  f->bytes = need;
  f->stream_idx = fs;
  f->id = next_launch++;
  stream_busy[fs] = true;
  bytes_in_use += need;
  t.state = 1;
  t.start_t = now;
  inflight.push_back(f);
  return true;
}

// Cyclic request at the head of the queue: into the open launch if it fits,
// else a new open launch with the queued cyclic requests of its precision.
bool krans_server::admit_cyclic(Clock::time_point now) {
  const uint64_t id = queue.front();
  ServerTicket &head = tickets[id];
  if (open && !open->L.done()) {
    // the request's matrix finishes its device set-up on the context's stream
    cudaError_t ew = cudaEventRecord(ctx_ready, ctx->stream);
    if (ew == cudaSuccess)
      ew = cudaEventSynchronize(ctx_ready);
    int slot = -1;
    const int r = ew == cudaSuccess ? open->L.try_publish(head.req, &slot)
                                    : cuda_fail(ew, "server stream order", __FILE__, __LINE__);
    if (r == 1) {
      queue.pop_front();
      head.state = 1;
      head.start_t = now;
      open->running.push_back({id, slot, now});
      return true;
    }
    if (r < 0) {
      queue.pop_front();
      fail(id, r, now);
      return true;
    }
    open->L.close(); // it does not fit: let the open launch drain, start the next one
    open = nullptr;
  }
  const int fs = free_stream();
  if (fs < 0)
    return false;
  std::vector<uint64_t> take;
  std::vector<krans_request> rq;
  const int prec = head.req.opts.precision;
  for (auto it = queue.begin(); it != queue.end() && (int)take.size() < opts.max_batch; ++it) {
    ServerTicket &t = tickets[*it];
    if (t.state == 4)
      continue;
    if (t.req.solver != KRANS_SOLVER_CYCLIC || t.req.opts.precision != prec)
      break;
    take.push_back(*it);
    rq.push_back(t.req);
  }
  if (take.empty()) {
    queue.pop_front(); // a cancelled head
    return true;
  }
  const size_t budget = opts.hbm_budget_bytes;
  auto *f = new InFlight();
  size_t need = 0;
  bool floors = true;
  int rc = f->L.plan(ctx, rq.data(), (int)rq.size(), &need, true, opts.max_batch, floors);
  while (rc == KRANS_OK && bytes_in_use + need > budget) {
    // shrink: first drop the slot floors, then requests from the back (keep at least one)
    if (floors)
      floors = false;
    else if (take.size() > 1) {
      take.pop_back();
      rq.pop_back();
    } else
      break;
    f->L = BatchLaunch();
    rc = f->L.plan(ctx, rq.data(), (int)rq.size(), &need, true, opts.max_batch, floors);
  }
  // the requests taken leave the queue (those that stayed keep their places):
  // they are its first entries in order, with only cancelled ones between
  for (size_t ti = 0; ti < take.size() && !queue.empty();) {
    const uint64_t q0 = queue.front();
    if (q0 == take[ti]) {
      queue.pop_front();
      ti++;
    } else if (tickets[q0].state == 4) {
      queue.pop_front();
    } else {
      break;
    }
  }
  if (rc != KRANS_OK) {
    for (auto id2 : take)
      fail(id2, rc, now);
    delete f;
    return true;
  }
  if (need > budget) {
    // a request larger than the whole budget can never be admitted
    for (auto id2 : take)
      fail(id2, KRANS_ERR_OUT_OF_MEMORY, now);
    delete f;
    return true;
  }
  if (bytes_in_use + need > budget) {
    // wait for memory to free up
    for (auto it = take.rbegin(); it != take.rend(); ++it)
      queue.push_front(*it);
    delete f;
    return false;
  }
  cudaError_t ew = cudaEventRecord(ctx_ready, ctx->stream);
  if (ew == cudaSuccess)
    ew = cudaStreamWaitEvent(streams[fs], ctx_ready, 0);
  rc = ew == cudaSuccess ? f->L.alloc_and_launch(streams[fs]) : cuda_fail(ew, "server stream order", __FILE__, __LINE__);
  if (rc != KRANS_OK) {
    for (auto id2 : take)
      fail(id2, rc, now);
    f->L.release(&graveyard);
    delete f;
    return true;
  }
  f->bytes = need;
  f->stream_idx = fs;
  f->id = next_launch++;
  stream_busy[fs] = true;
  bytes_in_use += need;
  for (int pos = 0; pos < f->L.count; pos++) {
    const uint64_t id2 = take[f->L.order[pos]];
    tickets[id2].state = 1;
    tickets[id2].start_t = now;
    f->running.push_back({id2, f->L.slot_of(pos), now});
  }
  inflight.push_back(f);
  open = f;
  return true;
}

void krans_server::run() {
  cudaSetDevice(ctx->device);
  std::unique_lock<std::mutex> lk(mu);
  while (!stop) {
    auto now = Clock::now();
    bool moved = false;
    // 1) requests that finished inside running launches
    for (InFlight *f : inflight) {
      if (f->lob)
        continue;
      for (size_t i = 0; i < f->running.size();) {
        const auto &r = f->running[i];
        if (f->L.slot_done(r.slot)) {
          f->L.fill_slot(r.slot, &tickets[r.ticket].res);
          finish(r.ticket, now, f->id);
          f->running.erase(f->running.begin() + (long)i);
          moved = true;
        } else {
          i++;
        }
      }
    }
    // 2) launches that ended
    for (size_t i = 0; i < inflight.size();) {
      InFlight *f = inflight[i];
      const bool ended = f->lob ? lobpcg_async_done(f->lob) : f->L.done();
      if (!ended) {
        i++;
        continue;
      }
      if (f->lob) {
        lobpcg_async_finish(f->lob, &tickets[f->lob_ticket].res);
        finish(f->lob_ticket, now, f->id);
        lobpcg_async_release(f->lob, &graveyard);
      } else {
        for (auto it = f->running.rbegin(); it != f->running.rend(); ++it) {
          ServerTicket &t = tickets[it->ticket];
          if (f->L.slot_done(it->slot)) {
            f->L.fill_slot(it->slot, &t.res);
            finish(it->ticket, now, f->id);
          } else if (!f->L.claimed(it->slot)) {
            if (t.cancel_requested) { // cancelled before any team took it
              memset(&t.res, 0, sizeof t.res);
              t.res.status = KRANS_ERR_CANCELLED;
              t.state = 4;
              t.done_t = now;
              completed.push_back(it->ticket);
            } else {
              t.state = 0; // published after its launch's teams had left: queue it again
              queue.push_front(it->ticket);
            }
          } else {
            fail(it->ticket, KRANS_ERR_RUNTIME, now);
          }
        }
        if (open == f)
          open = nullptr;
        f->L.release(&graveyard);
      }
      stream_busy[(size_t)f->stream_idx] = false;
      bytes_in_use -= std::min(bytes_in_use, f->bytes);
      delete f;
      inflight.erase(inflight.begin() + (long)i);
      moved = true;
    }
    bury_if_idle();
    // 3) admission
    while (!queue.empty()) {
      const uint64_t id = queue.front();
      ServerTicket &t = tickets[id];
      if (t.state == 4) {
        queue.pop_front();
        continue;
      }
      const bool ok = t.req.solver == KRANS_SOLVER_LOBPCG ? admit_lobpcg(id, now) : admit_cyclic(now);
      if (!ok)
        break;
      moved = true;
    }
    if (moved)
      cv.notify_all();
    // 4) sleep briefly (polling device completion)
    cv.wait_for(lk, std::chrono::microseconds(inflight.empty() && queue.empty() ? 2000 : 100));
  }
}

extern "C" {

int krans_server_opts_init(krans_server_opts *o) {
  KR_CHECK_ARG(o, "NULL argument");
  o->hbm_budget_bytes = (size_t)150 * 1000 * 1000 * 1000;
  o->max_inflight_launches = 4;
  o->max_batch = 1024;
  o->batch_window_ms = 0.0;
  return KRANS_OK;
}

int krans_server_create(krans_ctx *ctx, const krans_server_opts *opts, krans_server **out) {
  KR_CHECK_ARG(ctx && out, "krans_server_create: NULL argument");
  *out = nullptr;
  auto *s = new krans_server();
  s->ctx = ctx;
  if (opts)
    s->opts = *opts;
  else
    krans_server_opts_init(&s->opts);
  if (s->opts.hbm_budget_bytes == 0)
    s->opts.hbm_budget_bytes = (size_t)150 * 1000 * 1000 * 1000;
  if (s->opts.max_inflight_launches < 1)
    s->opts.max_inflight_launches = 1;
  if (s->opts.max_batch < 1)
    s->opts.max_batch = 1;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) {
    // launch workspaces come from the device's stream-ordered pool; keep what
    // finished launches return there instead of giving it back to the driver
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  for (int i = 0; i < s->opts.max_inflight_launches && e == cudaSuccess; i++) {
    cudaStream_t st;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
      s->streams.push_back(st);
      s->stream_busy.push_back(false);
    }
  }
  if (e == cudaSuccess)
    e = cudaEventCreateWithFlags(&s->ctx_ready, cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaStreamCreateWithFlags(&s->ctl, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    if (s->ctl)
      cudaStreamDestroy(s->ctl);
    for (auto st : s->streams)
      cudaStreamDestroy(st);
    if (s->ctx_ready)
      cudaEventDestroy(s->ctx_ready);
    delete s;
    return cuda_fail(e, "server streams", __FILE__, __LINE__);
  }
  s->worker = std::thread([s] { s->run(); });
  *out = s;
  return KRANS_OK;
}

int krans_server_destroy(krans_server *s) {
  if (!s)
    return KRANS_OK;
  krans_server_drain(s, 600000.0);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (auto *f : s->inflight)
      if (!f->lob)
        f->L.close();
  }
  s->cv.notify_all();
  if (s->worker.joinable())
    s->worker.join();
  for (auto *f : s->inflight) {
    cudaStreamSynchronize(s->streams[(size_t)f->stream_idx]);
    if (f->lob)
      lobpcg_async_release(f->lob);
    else
      f->L.release();
    delete f;
  }
  s->inflight.clear();
  s->bury_if_idle();
  for (auto st : s->streams)
    cudaStreamSynchronize(st); // stream-ordered frees done before the streams go
  for (auto st : s->streams)
    cudaStreamDestroy(st);
  if (s->ctl)
    cudaStreamDestroy(s->ctl);
  if (s->ctx_ready)
    cudaEventDestroy(s->ctx_ready);
  delete s;
  return KRANS_OK;
}

int krans_submit(krans_server *s, const krans_request *req, uint64_t *ticket) {
  KR_CHECK_ARG(s && req && ticket, "krans_submit: NULL argument");
  KR_CHECK_ARG(req->A && req->A->ctx == s->ctx, "krans_submit: request without a matrix of this context");
  KR_CHECK_ARG(req->solver == KRANS_SOLVER_CYCLIC || req->solver == KRANS_SOLVER_LOBPCG,
               "krans_submit: solver must be KRANS_SOLVER_CYCLIC or KRANS_SOLVER_LOBPCG");
  std::lock_guard<std::mutex> lk(s->mu);
  const uint64_t id = s->next_ticket++;
  ServerTicket &t = s->tickets[id];
  t.req = *req;
  t.state = 0;
  memset(&t.res, 0, sizeof t.res);
  t.submit_t = Clock::now();
  s->queue.push_back(id);
  *ticket = id;
  s->cv.notify_all();
  return KRANS_OK;
}

int krans_poll(krans_server *s, uint64_t ticket, int *status, krans_request_result *result) {
  KR_CHECK_ARG(s && status, "krans_poll: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) {
    set_error("krans_poll: unknown ticket %llu", (unsigned long long)ticket);
    return KRANS_ERR_NOT_FOUND;
  }
  *status = it->second.state;
  if (result)
    *result = it->second.res;
  return KRANS_OK;
}

int krans_cancel(krans_server *s, uint64_t ticket) {
  KR_CHECK_ARG(s, "krans_cancel: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) {
    set_error("krans_cancel: unknown ticket %llu", (unsigned long long)ticket);
    return KRANS_ERR_NOT_FOUND;
  }
  if (it->second.state == 1) {
    // running: write the cancellation into the request's device status word
    // (remembered too: a published request that no team claimed before its
    // launch ended is not queued again)
    it->second.cancel_requested = true;
    for (InFlight *f : s->inflight) {
      if (f->lob && f->lob_ticket == ticket)
        return lobpcg_async_cancel(f->lob, s->ctl);
      if (!f->lob)
        for (const auto &r : f->running)
          if (r.ticket == ticket)
            return f->L.cancel_slot(r.slot, s->ctl);
    }
    return KRANS_OK; // it has just finished
  }
  if (it->second.state != 0) {
    set_error("krans_cancel: ticket %llu has finished", (unsigned long long)ticket);
    return KRANS_ERR_RUNTIME;
  }
  // queued: marked cancelled; the scheduler drops it when it reaches the
  // queue's head or a batch being formed (no search of the queue here, which
  // would make cancelling a long queue quadratic)
  it->second.state = 4;
  memset(&it->second.res, 0, sizeof it->second.res);
  it->second.res.status = KRANS_ERR_CANCELLED;
  s->completed.push_back(ticket);
  return KRANS_OK;
}

int krans_server_completed(krans_server *s, uint64_t *tickets, int64_t capacity, int64_t *count) {
  KR_CHECK_ARG(s && count && (capacity == 0 || tickets), "krans_server_completed: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  int64_t k = 0;
  while (k < capacity && !s->completed.empty()) {
    tickets[k++] = s->completed.front();
    s->completed.pop_front();
  }
  *count = k;
  return KRANS_OK;
}

int krans_server_stats(krans_server *s, int64_t out[4]) {
  KR_CHECK_ARG(s && out, "krans_server_stats: NULL argument");
  std::unique_lock<std::mutex> lk(s->mu, std::try_to_lock);
  if (!lk.owns_lock()) {
    set_error("krans_server_stats: the scheduler holds its lock");
    return KRANS_ERR_TIMEOUT;
  }
  out[0] = (int64_t)s->queue.size();
  out[1] = (int64_t)s->inflight.size();
  out[2] = 0;
  out[3] = 0;
  for (const InFlight *f : s->inflight) {
    if (f->lob)
      out[2]++;
    else
      out[3] += (int64_t)f->running.size();
  }
  return KRANS_OK;
}

int krans_server_drain(krans_server *s, double timeout_ms) {
  KR_CHECK_ARG(s, "krans_server_drain: NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  const auto t0 = Clock::now();
  while (!s->queue.empty() || !s->inflight.empty()) {
    if (ms_since(t0, Clock::now()) > timeout_ms) {
      set_error("krans_server_drain: timed out with %zu queued, %zu launches in flight", s->queue.size(),
                s->inflight.size());
      return KRANS_ERR_TIMEOUT;
    }
    s->cv.wait_for(lk, std::chrono::milliseconds(1));
  }
  return KRANS_OK;
}

} // extern "C"
