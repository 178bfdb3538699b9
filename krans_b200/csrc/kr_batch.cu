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

// One persistent launch over a set of requests.
struct BatchLaunch {
  krans_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  int count = 0;
  int precision = 0;
  int grid = 0;        // CTA-team blocks (small requests)
  int n_large = 0;     // requests [0, n_large) run on clusters of csize blocks
  int n_mid = 0;       // requests [n_large, n_large + n_mid) run on 2-block clusters (pairs)
  int npairs = 0;      // pair clusters of the second launch (the SMs the big clusters leave free)
  size_t stride_M = 0; // workspace slot of one pair
  size_t dyn_smem = 0; // dynamic shared memory per block (CG vectors of one-block solves)
  int csize = 8;       // blocks per cluster
  int nclusters = 0;   // resident clusters of the cluster launch
  size_t stride_L = 0; // workspace slot of one cluster
  cudaStream_t aux = nullptr;
  cudaEvent_t evj = nullptr;
  std::vector<int> order; // position in launch -> index in the caller's array
  CyclicRequestDev *d_reqs = nullptr;
  CyclicDevResult *d_res = nullptr;
  int32_t *d_status = nullptr;
  double *d_mr = nullptr;
  RngState *d_rng = nullptr;
  int *d_queue = nullptr;
  char *ws = nullptr;
  size_t ws_bytes = 0, ws_stride = 0, meta_bytes = 0;
  CyclicDevResult *h_res = nullptr;
  int32_t *h_status = nullptr;
  double *h_mr = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<CyclicRequestDev> hreq;
  std::vector<RngState> hrng;

  // Size the launch (no allocation): returns bytes of device memory needed.
  int plan(krans_ctx *c, const krans_request *reqs, int n, size_t *need) {
    ctx = c;
    count = n;
    precision = n > 0 ? reqs[0].opts.precision : 0;
    order.resize(n);
    std::iota(order.begin(), order.end(), 0);
    const int64_t cluster_min = ctx->tune.cluster_min;
    const int64_t pair_max = ctx->tune.pair_max;
    csize = ctx->tune.cluster_size;
    // Size classes (by m + n only, so a request runs on the same kind of
    // team, with the same rounding, in any batch): big ones on clusters of
    // csize blocks; mid-size ones on 2-block clusters launched next to them
    // on the SMs the big clusters cannot tile (a GPC holds whole clusters
    // only); small ones on single blocks.
    const bool mixed_p = precision == KRANS_PREC_MIXED;
    {
      const int maxc = cyclic_batch_cluster_max(mixed_p, csize, ctx->sms, 0);
      npairs = csize > 2 && pair_max > cluster_min ? std::max(0, (ctx->sms - maxc * csize) / 2) : 0;
    }
    auto cls = [&](int a) {
      const int64_t sz = reqs[a].A->m + reqs[a].A->n;
      if (cluster_min <= 0 || sz < cluster_min)
        return 2;
      return (npairs > 0 && sz < pair_max) ? 1 : 0;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      const int ca = cls(a), cb = cls(b);
      if (ca != cb)
        return ca < cb;
      return reqs[a].A->nnz > reqs[b].A->nnz;
    });
    n_large = n_mid = 0;
    for (int pos = 0; pos < n; pos++) {
      const int c = cls(order[pos]);
      n_large += c == 0;
      n_mid += c == 1;
    }
    hreq.assign(n, CyclicRequestDev{});
    hrng.assign(n, RngState{});
    ws_stride = 256;
    for (int pos = 0; pos < n; pos++) {
      const krans_request &r = reqs[order[pos]];
      KR_CHECK_ARG(r.A && r.A->ctx == ctx, "krans_solve_batch: request without a matrix of this context");
      KR_CHECK_ARG(r.opts.precision == precision, "krans_solve_batch: one precision per batch");
      KR_CHECK_ARG(precision == KRANS_PREC_FP64 || r.A->v32,
                   "krans_solve_batch: mixed precision needs matrices created with KRANS_CSR_FP32");
      const krans_mat *A = r.A;
      CyclicRequestDev &q = hreq[pos];
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
      if (!trivial)
        KR_CHECK_ARG(r.basis_out && r.basis_capacity >= kt, "krans_solve_batch: basis_out too small");
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
      q.plan.own_basis = 0;
      q.plan.block_polish = r.opts.polish_block ? 1 : 0;
      q.plan.precond = r.opts.precond_aat;
      q.basis = r.basis_out;
      if (!trivial) {
        if (pos < n_large)
          stride_L = std::max(stride_L, cyclic_carve(q.plan, nullptr, nullptr));
        else if (pos < n_large + n_mid)
          stride_M = std::max(stride_M, cyclic_carve(q.plan, nullptr, nullptr));
        else
          ws_stride = std::max(ws_stride, cyclic_carve(q.plan, nullptr, nullptr));
      }
      RngState &s = hrng[pos];
      uint32_t seed = r.seed ? r.seed : 0x9E3779B9u;
      mt_seed(s, seed);
      s.philox_key = ((uint64_t)seed << 32) ^ 0x9E3779B97F4A7C15ull;
      s.mode = r.rng_mode;
    }
    ws_stride = (size_t)kr_round_up((int64_t)ws_stride, 256);
    stride_L = (size_t)kr_round_up((int64_t)std::max<size_t>(stride_L, 256), 256);
    stride_M = (size_t)kr_round_up((int64_t)std::max<size_t>(stride_M, 256), 256);
    const int n_small = n - n_large - n_mid;
    const bool mixed = precision == KRANS_PREC_MIXED;
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
    if (n_mid == 0)
      npairs = 0;
    if (n_large > 0 || n_mid > 0) {
      // one cluster launch fills the GPU; its blocks take the small requests
      // after the large queue is empty (one small-request slot per block)
      const int maxc = cyclic_batch_cluster_max(mixed, csize, ctx->sms, dyn_smem);
      nclusters = std::max(1, maxc);
      grid = nclusters * csize;
    }
    meta_bytes = (size_t)n * (sizeof(CyclicRequestDev) + sizeof(CyclicDevResult) + 4 + 8 + sizeof(RngState)) +
                 4096;
    ws_bytes = (size_t)(grid + 2 * npairs) * ws_stride + (size_t)nclusters * stride_L +
               (size_t)npairs * stride_M + 256;
    *need = ws_bytes + meta_bytes;
    return KRANS_OK;
  }

  int alloc_and_launch(cudaStream_t s) {
    stream = s;
    int rc = dev_alloc(ctx, (void **)&ws, ws_bytes);
    if (rc != KRANS_OK)
      return rc;
    char *meta = nullptr;
    rc = dev_alloc(ctx, (void **)&meta, meta_bytes);
    if (rc != KRANS_OK) {
      dev_free(ctx, ws, ws_bytes);
      ws = nullptr;
      return rc;
    }
    Carver c;
    c.base = meta;
    d_reqs = c.take<CyclicRequestDev>(count);
    d_res = c.take<CyclicDevResult>(count);
    d_status = c.take<int32_t>(count);
    d_mr = c.take<double>(count);
    d_rng = c.take<RngState>(count);
    d_queue = c.take<int>(4);
    for (int pos = 0; pos < count; pos++) {
      hreq[pos].res = d_res + pos;
      hreq[pos].status = d_status + pos;
      hreq[pos].max_resid = d_mr + pos;
      hreq[pos].rng = d_rng + pos;
    }
    cudaError_t e = cudaMallocHost(&h_res, sizeof(CyclicDevResult) * (size_t)std::max(count, 1));
    if (e == cudaSuccess)
      e = cudaMallocHost(&h_status, 4 * (size_t)std::max(count, 1));
    if (e == cudaSuccess)
      e = cudaMallocHost(&h_mr, 8 * (size_t)std::max(count, 1));
    if (e == cudaSuccess)
      e = cudaEventCreate(&ev0);
    if (e == cudaSuccess)
      e = cudaEventCreate(&ev1);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_reqs, hreq.data(), sizeof(CyclicRequestDev) * (size_t)count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_rng, hrng.data(), sizeof(RngState) * (size_t)count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_res, 0, sizeof(CyclicDevResult) * (size_t)count, s);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_status, 0, 4 * (size_t)count, s);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_mr, 0, 8 * (size_t)count, s);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_queue, 0, 4 * sizeof(int), s);
    if (e == cudaSuccess)
      e = cudaEventRecord(ev0, s);
    char *ws_small = ws, *ws_small_p = ws + (size_t)grid * ws_stride;
    char *ws_large = ws_small_p + (size_t)2 * npairs * ws_stride;
    char *ws_mid = ws_large + (size_t)nclusters * stride_L;
    const bool mixed = precision == KRANS_PREC_MIXED;
    const int first_small = n_large + n_mid;
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
      if (n_large > 0 || n_mid > 0) {
        e = launch_cyclic_batch_cluster(mixed, nclusters, csize, dyn_smem, s, d_reqs, n_large, d_queue, ws_large,
                                        stride_L, d_reqs + first_small, count - first_small, d_queue + 1,
                                        ws_small, ws_stride);
        if (e == cudaSuccess && npairs > 0) {
          e = launch_cyclic_batch_cluster(mixed, npairs, 2, dyn_smem, aux, d_reqs + n_large, n_mid,
                                            d_queue + 2, ws_mid, stride_M, d_reqs + first_small,
                                            count - first_small, d_queue + 1, ws_small_p, ws_stride);
          if (e == cudaSuccess)
            e = cudaEventRecord(evj, aux);
          if (e == cudaSuccess)
            e = cudaStreamWaitEvent(s, evj, 0);
        }
      } else
        e = launch_cyclic_batch_cta(mixed, grid, 512, dyn_smem, s, d_reqs, count, d_queue + 1, ws_small, ws_stride);
    }
    if (e == cudaSuccess)
      e = cudaEventRecord(ev1, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h_res, d_res, sizeof(CyclicDevResult) * (size_t)count, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h_status, d_status, 4 * (size_t)count, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h_mr, d_mr, 8 * (size_t)count, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess)
      return cuda_fail(e, "batch launch", __FILE__, __LINE__);
    return KRANS_OK;
  }

  bool done() const { return cudaEventQuery(ev1) == cudaSuccess && cudaStreamQuery(stream) == cudaSuccess; }

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

  void fill(int pos, krans_request_result *out) const {
    const CyclicDevResult &r = h_res[pos];
    memset(out, 0, sizeof *out);
    const uint64_t z = t0();
    if (z && r.t_begin >= z && r.t_end >= r.t_begin) {
      out->queue_ms = (double)(r.t_begin - z) * 1e-6;   // wait for a free team inside the launch
      out->latency_ms = (double)(r.t_end - z) * 1e-6;   // launch start -> request done
    }
    out->status = h_status[pos] != 0 ? h_status[pos] : r.status;
    if (hreq[pos].trivial) {
      out->converged_to_target = hreq[pos].plan.k_target == 0 ? 1 : 0;
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
    out->max_residual = h_mr[pos];
    out->algo_bytes = r.bytes;
    for (int q = 0; q < 4; q++)
      out->phase_ms[q] = r.phase_ms[q];
  }

  void release() {
    if (ws)
      dev_free(ctx, ws, ws_bytes);
    if (d_reqs)
      dev_free(ctx, d_reqs, meta_bytes);
    ws = nullptr;
    d_reqs = nullptr;
    if (h_res)
      cudaFreeHost(h_res);
    if (h_status)
      cudaFreeHost(h_status);
    if (h_mr)
      cudaFreeHost(h_mr);
    h_res = nullptr;
    h_status = nullptr;
    h_mr = nullptr;
    if (aux)
      cudaStreamDestroy(aux);
    aux = nullptr;
    if (evj)
      cudaEventDestroy(evj);
    evj = nullptr;
    if (ev0)
      cudaEventDestroy(ev0);
    if (ev1)
      cudaEventDestroy(ev1);
    ev0 = ev1 = nullptr;
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
// Serving: continuous batching. A scheduler thread admits queued requests
// while the HBM budget allows, launches them as one persistent batch on a
// free stream (several launches overlap on the device), and completes the
// tickets of finished launches.
// ---------------------------------------------------------------------------
struct ServerTicket {
  krans_request req;
  int state = 0; // 0 queued, 1 running, 2 done, 3 failed, 4 cancelled
  krans_request_result res;
  Clock::time_point submit_t, start_t, done_t;
};

struct InFlight {
  BatchLaunch L;
  std::vector<uint64_t> tickets; // launch-order ticket ids (order = caller index)
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  Clock::time_point launch_t;
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
  std::vector<InFlight *> inflight;
  size_t bytes_in_use = 0;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread worker;
  int last_error = KRANS_OK;
  std::string last_msg;

  void run();
};

void krans_server::run() {
  cudaSetDevice(ctx->device);
  std::unique_lock<std::mutex> lk(mu);
  while (!stop) {
    // 1) retire finished launches
    for (size_t i = 0; i < inflight.size();) {
      InFlight *f = inflight[i];
      if (!f->L.done()) {
        i++;
        continue;
      }
      const auto now = Clock::now();
      const double dms = f->L.device_ms();
      for (int pos = 0; pos < f->L.count; pos++) {
        const uint64_t id = f->tickets[f->L.order[pos]];
        ServerTicket &t = tickets[id];
        f->L.fill(pos, &t.res);
        t.res.device_ms = dms;
        t.done_t = now;
        t.res.queue_ms = ms_since(t.submit_t, t.start_t);
        t.res.latency_ms = ms_since(t.submit_t, now);
        t.state = t.res.status == KRANS_OK ? 2 : 3;
      }
      for (size_t s = 0; s < streams.size(); s++)
        if (streams[s] == f->stream)
          stream_busy[s] = false;
      bytes_in_use -= std::min(bytes_in_use, f->bytes);
      f->L.release();
      delete f;
      inflight.erase(inflight.begin() + (long)i);
      cv.notify_all();
    }
    // 2) admit queued requests into a new launch on a free stream
    int free_s = -1;
    for (size_t s = 0; s < streams.size(); s++)
      if (!stream_busy[s]) {
        free_s = (int)s;
        break;
      }
    if (free_s >= 0 && !queue.empty()) {
      // wait a short window to let a batch accumulate when the GPU is busy
      std::vector<uint64_t> take;
      std::vector<krans_request> rq;
      int prec = -1;
      size_t budget = opts.hbm_budget_bytes;
      while (!queue.empty() && (int)take.size() < opts.max_batch) {
        const uint64_t id = queue.front();
        ServerTicket &t = tickets[id];
        if (t.state == 4) {
          queue.pop_front();
          continue;
        }
        if (prec >= 0 && t.req.opts.precision != prec)
          break;
        prec = t.req.opts.precision;
        take.push_back(id);
        rq.push_back(t.req);
        queue.pop_front();
      }
      if (!take.empty()) {
        // shrink the batch until it fits the budget (keep at least one)
        auto *f = new InFlight();
        size_t need = 0;
        int rc = f->L.plan(ctx, rq.data(), (int)rq.size(), &need);
        while (rc == KRANS_OK && take.size() > 1 && bytes_in_use + need > budget) {
          queue.push_front(take.back());
          take.pop_back();
          rq.pop_back();
          f->L = BatchLaunch();
          rc = f->L.plan(ctx, rq.data(), (int)rq.size(), &need);
        }
        if (rc == KRANS_OK && need > budget) {
          // a single request larger than the whole budget can never be admitted
          const auto now = Clock::now();
          for (auto id : take) {
            ServerTicket &t = tickets[id];
            memset(&t.res, 0, sizeof t.res);
            t.res.status = KRANS_ERR_OUT_OF_MEMORY;
            t.state = 3;
            t.start_t = now;
            t.done_t = now;
            t.res.latency_ms = ms_since(t.submit_t, now);
          }
          delete f;
          cv.notify_all();
        } else if (rc == KRANS_OK && bytes_in_use + need > budget && !inflight.empty()) {
          // wait for memory to free up
          for (auto it = take.rbegin(); it != take.rend(); ++it)
            queue.push_front(*it);
          delete f;
        } else {
          // matrices finish their device set-up (transpose) on the context's
          // stream: the launch's stream waits for it
          if (rc == KRANS_OK) {
            cudaError_t ew = cudaEventRecord(ctx_ready, ctx->stream);
            if (ew == cudaSuccess)
              ew = cudaStreamWaitEvent(streams[free_s], ctx_ready, 0);
            if (ew != cudaSuccess)
              rc = cuda_fail(ew, "server stream order", __FILE__, __LINE__);
          }
          if (rc == KRANS_OK)
            rc = f->L.alloc_and_launch(streams[free_s]);
          const auto now = Clock::now();
          if (rc != KRANS_OK) {
            for (auto id : take) {
              ServerTicket &t = tickets[id];
              memset(&t.res, 0, sizeof t.res);
              t.res.status = rc;
              t.state = 3;
              t.start_t = now;
              t.done_t = now;
            }
            last_error = rc;
            last_msg = krans_last_error();
            f->L.release();
            delete f;
            cv.notify_all();
          } else {
            f->tickets = take;
            f->bytes = need;
            f->stream = streams[free_s];
            f->launch_t = now;
            stream_busy[free_s] = true;
            bytes_in_use += need;
            for (auto id : take) {
              tickets[id].state = 1;
              tickets[id].start_t = now;
            }
            inflight.push_back(f);
          }
        }
      }
    }
    // 3) sleep briefly (polling device completion)
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
  if (e != cudaSuccess) {
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
  }
  s->cv.notify_all();
  if (s->worker.joinable())
    s->worker.join();
  for (auto *f : s->inflight) {
    cudaStreamSynchronize(f->stream);
    f->L.release();
    delete f;
  }
  for (auto st : s->streams)
    cudaStreamDestroy(st);
  if (s->ctx_ready)
    cudaEventDestroy(s->ctx_ready);
  delete s;
  return KRANS_OK;
}

int krans_submit(krans_server *s, const krans_request *req, uint64_t *ticket) {
  KR_CHECK_ARG(s && req && ticket, "krans_submit: NULL argument");
  KR_CHECK_ARG(req->A && req->A->ctx == s->ctx, "krans_submit: request without a matrix of this context");
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
  if (it->second.state != 0) {
    set_error("krans_cancel: ticket %llu is no longer queued", (unsigned long long)ticket);
    return KRANS_ERR_RUNTIME;
  }
  it->second.state = 4;
  memset(&it->second.res, 0, sizeof it->second.res);
  it->second.res.status = KRANS_ERR_CANCELLED;
  for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
    if (*q == ticket) {
      s->queue.erase(q);
      break;
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
