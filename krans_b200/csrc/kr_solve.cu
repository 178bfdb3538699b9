// Solver launches: one cyclic request on a thread block or on the whole GPU
// (cooperative launch), and many requests in one persistent launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "kr_internal.h"
#include "kr_types.cuh"

namespace kr {

static inline int64_t round_up(int64_t x, int64_t a) { return kr_round_up(x, a); }

// Lay out (or, with base == nullptr, size) the workspace of one run.
static size_t cyclic_layout(const CyclicPlan &p, char *base, CyclicDesc *d) { return cyclic_carve(p, base, d); }

static CsrView view_of(const krans_mat *A, bool trans) {
  CsrView v;
  if (!trans) {
    v = CsrView{A->m, A->n, A->nnz, A->rp, A->ci, A->v, A->v32, tuned_lanes(A->ctx, A->m, A->nnz), A->ulen};
  } else {
    v = CsrView{A->n, A->m, A->nnz, A->rpT, A->ciT, A->vT, A->vT32, tuned_lanes(A->ctx, A->n, A->nnz), A->ulenT};
  }
  return v;
}

// Reference k_target / early-exit rules (CyclicLanczosSolver.cpp:297-311).
// Returns 1 when the run has nothing to do.
static int cyclic_targets(const krans_cyclic_opts &o, int64_t m, int64_t n, int64_t *k_target,
                          int64_t *ncv, bool *converged_trivially) {
  *converged_trivially = false;
  if (n == 0 || m == 0)
    return 1;
  *k_target = (o.nullity_known >= 0) ? (int64_t)o.nullity_known : o.k;
  if (*k_target == 0) {
    *converged_trivially = true;
    return 1;
  }
  if (o.rank_known >= 0 && n <= (int64_t)o.rank_known)
    return 1;
  int64_t nc = std::max<int64_t>(std::max<int64_t>(2, o.ncv), *k_target + 2);
  *ncv = nc;
  return 0;
}

struct RunOut {
  CyclicDevResult r;
  double ms;
  int32_t fp64_fallback = 0; // the mixed run continued in FP64
  int64_t fallback_from = 0; // vectors the mixed run had accepted
};

// One find_right_nullspace run on the device (a grid team, or one thread
// block through the persistent batched kernel with a single request); the
// basis rows are copied into new vectors owned by the caller.
// `prefill` (nprefill rows, stride round_up(n, 32)) and `frob_init` continue
// an earlier run: its accepted vectors are copied into the basis first and
// its ||A||_F estimate is kept. A MIXED run that stops short of k_target with
// its FP64 polish at cg_maxit continues that way in FP64 (o.mixed_fallback):
// the FP32 recurrence's Ritz vectors were too far from the null space for
// the projector to finish, which an FP64 recurrence avoids.
static int run_cyclic(krans_ctx *ctx, const krans_mat *A, bool trans, krans_rng *rng,
                      const krans_cyclic_opts &o, const double *init_right, int64_t k_target,
                      int64_t ncv, std::vector<krans_vec *> &found, RunOut *out,
                      const double *prefill = nullptr, int64_t nprefill = 0, double frob_init = 0.0) {
  const CsrView F = view_of(A, trans), B = view_of(A, !trans);
  const bool mixed = o.precision == KRANS_PREC_MIXED;
  if (mixed && !A->v32) {
    set_error("mixed precision needs a matrix created with KRANS_CSR_FP32");
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  KR_CHECK_ARG(k_target <= 128, "cyclic: at most 128 null vectors per request");
  KR_CHECK_ARG(ncv <= 256, "cyclic: ncv must be <= 256");
  KR_CHECK_ARG(o.precond_aat >= KRANS_PRECOND_NONE && o.precond_aat <= KRANS_PRECOND_SD && o.precond_steps >= 1 &&
                   o.precond_steps <= 1000,
               "cyclic: precond_aat must be a KRANS_PRECOND_* value, precond_steps in [1, 1000]");
  int team = o.team;
  if (team == KRANS_TEAM_AUTO)
    team = (F.rows + F.cols) < 120000 ? KRANS_TEAM_CTA : KRANS_TEAM_GRID;
  const bool grid = team == KRANS_TEAM_GRID;
  const int threads = 512;
  CyclicPlan p;
  memset(&p, 0, sizeof p);
  p.m = F.rows;
  p.n = F.cols;
  p.k_target = k_target;
  p.ncv = ncv;
  p.ldn = round_up(p.n, 32);
  p.ldm = round_up(p.m, 32);
  p.ldb = p.ldn;
  p.cap = ncv / 2 + 2;
  p.ksz = mixed ? 4 : 8;
  p.grid_blocks = grid ? cyclic_grid_blocks(ctx, mixed, threads) : 1;
  p.own_basis = grid ? 1 : 0;
  p.block_polish = o.polish_block ? 1 : 0;
  p.precond = o.precond_aat;
  // one allocation: solver workspace, basis, request record and counters
  char *slot = nullptr;
  double *basis = nullptr, *d_mr = nullptr;
  CyclicRequestDev *d_req = nullptr;
  CyclicDevResult *d_res = nullptr;
  int32_t *d_status = nullptr;
  int *d_queue = nullptr;
  auto layout = [&](char *base) {
    Carver c;
    c.base = base;
    slot = c.take<char>((int64_t)cyclic_carve(p, nullptr, nullptr));
    basis = c.take<double>(std::max<int64_t>(k_target, 1) * p.ldb);
    d_req = c.take<CyclicRequestDev>(1);
    d_res = c.take<CyclicDevResult>(1);
    d_status = c.take<int32_t>(1);
    d_mr = c.take<double>(1);
    d_queue = c.take<int>(1);
    return c.off + 256;
  };
  const size_t bytes = layout(nullptr);
  char *ws = nullptr;
  int rc = dev_alloc(ctx, (void **)&ws, bytes);
  if (rc != KRANS_OK)
    return rc;
  layout(ws);
  cudaStream_t s = ctx->stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t e = cudaMemsetAsync(d_res, 0, sizeof(CyclicDevResult), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d_status, 0, 4, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d_queue, 0, 4, s);
  CyclicDesc d;
  CyclicRequestDev q;
  if (grid) {
    memset(&d, 0, sizeof d);
    cyclic_carve(p, slot, &d);
    d.F = F;
    d.B = B;
    d.o = o;
    d.k_target = k_target;
    d.ncv = ncv;
    d.trans_run = trans ? 1 : 0;
    d.rng = rng->d;
    d.initial_right = init_right;
    d.nb_init = nprefill;
    d.frob_init = frob_init;
    d.status = d_status;
    d.res = d_res;
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d.gb, 0, sizeof(GridBarrierState), s);
  } else {
    memset(&q, 0, sizeof q);
    q.F = F;
    q.B = B;
    q.o = o;
    q.plan = p;
    q.rng = rng->d;
    q.basis = basis;
    q.res = d_res;
    q.status = d_status;
    q.max_resid = d_mr;
    q.initial_right = init_right;
    q.nb_init = nprefill;
    q.frob_init = frob_init;
    q.trivial = 0;
    q.trans_run = trans ? 1 : 0;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_req, &q, sizeof q, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess && nprefill > 0)
    e = cudaMemcpy2DAsync(grid ? d.basis : basis, (size_t)p.ldb * 8, prefill, (size_t)p.ldb * 8, (size_t)p.n * 8,
                          (size_t)nprefill, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess)
    e = cudaEventRecord(e0, s);
  if (e == cudaSuccess)
    e = grid ? launch_cyclic_grid(mixed, d, p.grid_blocks, threads, s)
             : launch_cyclic_batch_cta(mixed, 1, threads,
                                       cta_cg_smem_bytes(p.ldm, p.ldn) <= cta_smem_cap()
                                           ? cta_cg_smem_bytes(p.ldm, p.ldn)
                                           : 0,
                                       s, d_req, 1, d_queue, slot, 0, nullptr);
  if (e == cudaSuccess)
    e = cudaEventRecord(e1, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&out->r, d_res, sizeof(CyclicDevResult), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess)
    cudaEventElapsedTime(&ms, e0, e1);
  out->ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) {
    dev_free(ctx, ws, bytes);
    return cuda_fail(e, "cyclic solve launch", __FILE__, __LINE__);
  }
  if (out->r.status != KRANS_OK) {
    dev_free(ctx, ws, bytes);
    set_error("cyclic solve: device status %d (a bounded device wait gave up)", out->r.status);
    return out->r.status;
  }
  const double *bsrc = grid ? d.basis : basis;
  if (mixed && o.mixed_fallback && !out->r.converged && out->r.n_found < k_target && out->r.cg_maxit_hits > 0) {
    krans_cyclic_opts o64 = o;
    o64.precision = KRANS_PREC_FP64;
    RunOut o2;
    rc = run_cyclic(ctx, A, trans, rng, o64, init_right, k_target, ncv, found, &o2, bsrc, out->r.n_found,
                    out->r.frob);
    dev_free(ctx, ws, bytes);
    if (rc != KRANS_OK)
      return rc;
    const CyclicDevResult r1 = out->r;
    out->fallback_from = r1.n_found;
    out->fp64_fallback = 1;
    out->r = o2.r;
    out->r.restarts += r1.restarts;
    out->r.krylov_steps_total += r1.krylov_steps_total;
    out->r.cg_solves += r1.cg_solves;
    out->r.cg_maxit_hits += r1.cg_maxit_hits;
    out->r.spmv += r1.spmv;
    out->r.spmvT += r1.spmvT;
    out->r.bytes += r1.bytes;
    for (int q2 = 0; q2 < 4; q2++)
      out->r.phase_ms[q2] += r1.phase_ms[q2];
    out->ms += o2.ms;
    return KRANS_OK;
  }
  rc = KRANS_OK;
  for (int64_t i = 0; i < out->r.n_found && rc == KRANS_OK; i++) {
    krans_vec *v = nullptr;
    rc = krans_vec_create(ctx, p.n, &v);
    if (rc == KRANS_OK) {
      e = cudaMemcpyAsync(v->d, bsrc + i * p.ldb, (size_t)p.n * 8, cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess)
        rc = cuda_fail(e, "basis copy", __FILE__, __LINE__);
      found.push_back(v);
    }
  }
  cudaStreamSynchronize(s);
  dev_free(ctx, ws, bytes);
  return rc;
}

} // namespace kr

using namespace kr;

extern "C" int krans_solve_cyclic(krans_ctx *ctx, const krans_mat *A, krans_rng *rng,
                                  const krans_cyclic_opts *opts, const krans_vec *initial_right,
                                  krans_vec **right_out, krans_vec **left_out,
                                  krans_cyclic_result *result) {
  KR_CHECK_ARG(ctx && A && rng && opts && result, "krans_solve_cyclic: NULL argument");
  KR_CHECK_ARG(A->ctx == ctx && rng->ctx == ctx, "krans_solve_cyclic: objects of another context");
  memset(result, 0, sizeof *result);
  const krans_cyclic_opts &o = *opts;
  KR_CHECK_ARG(o.precision == KRANS_PREC_FP64 || o.precision == KRANS_PREC_MIXED,
               "krans_solve_cyclic: bad precision");
  KR_CHECK_ARG(o.reorth >= 0 && o.reorth <= 2, "krans_solve_cyclic: bad reorth mode");
  if (initial_right)
    KR_CHECK_ARG(initial_right->n == A->n, "krans_solve_cyclic: initial_right size mismatch");
  KR_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lk(ctx->mu);
  int64_t k_target = 0, ncv = 0;
  bool conv = false;
  std::vector<krans_vec *> right, left;
  int rc = KRANS_OK;
  if (cyclic_targets(o, A->m, A->n, &k_target, &ncv, &conv)) {
    result->converged_to_target = conv ? 1 : 0;
  } else {
    KR_CHECK_ARG(right_out, "krans_solve_cyclic: right_out is NULL");
    RunOut ro;
    rc = run_cyclic(ctx, A, false, rng, o, initial_right ? initial_right->d : nullptr, k_target, ncv,
                    right, &ro);
    if (rc != KRANS_OK) {
      for (auto *v : right)
        krans_vec_destroy(v);
      return rc;
    }
    result->restarts = ro.r.restarts;
    result->krylov_steps_total = ro.r.krylov_steps_total;
    result->frob_norm_est = ro.r.frob;
    result->converged_to_target = ro.r.converged;
    result->cg_solves = ro.r.cg_solves;
    result->cg_maxit_hits = ro.r.cg_maxit_hits;
    result->spmv = ro.r.spmv;
    result->spmvT = ro.r.spmvT;
    result->algo_bytes = ro.r.bytes;
    result->device_ms = ro.ms;
    for (int q = 0; q < 4; q++)
      result->phase_ms[q] = ro.r.phase_ms[q];
    result->fp64_fallback = ro.fp64_fallback;
    result->fallback_from = (int32_t)ro.fallback_from;
  }
  for (size_t i = 0; i < right.size(); i++)
    right_out[i] = right[i];
  result->n_right = (int64_t)right.size();
  if (o.return_left_space && A->m > 0 && A->n > 0) {
    // left null space = right null space of A^T (CyclicLanczosSolver.cpp:618-660)
    krans_cyclic_opts lo;
    krans_cyclic_opts_init(&lo);
    lo.k = o.k;
    lo.ncv = o.ncv;
    lo.max_restarts = o.max_restarts;
    lo.tol_abs = o.tol_abs;
    lo.tol_rel = o.tol_rel;
    lo.reorth = o.reorth;
    lo.use_harmonic = o.use_harmonic;
    lo.target_tau = o.target_tau;
    lo.cg_maxit = o.cg_maxit;
    lo.cg_rel_tol = o.cg_rel_tol;
    lo.cg_breakdown_tol = o.cg_breakdown_tol;
    lo.projector_passes = o.projector_passes;
    lo.grad_max_iters = o.grad_max_iters;
    lo.frob_samples = o.frob_samples;
    lo.prescreen_factor = o.prescreen_factor;
    lo.stagnation_restarts = o.stagnation_restarts;
    lo.verbose = o.verbose;
    lo.rank_known = o.rank_known;
    lo.precision = o.precision;
    lo.team = o.team;
    lo.polish_block = o.polish_block;
    lo.precond_aat = o.precond_aat;
    lo.precond_steps = o.precond_steps;
    lo.mixed_fallback = o.mixed_fallback;
    if (o.rank_known >= 0) {
      const int left_nullity = (int)A->m - o.rank_known;
      lo.nullity_known = std::max(0, std::min(left_nullity, (int)o.k));
    }
    int64_t lk_target = 0, lncv = 0;
    bool lconv = false;
    if (!cyclic_targets(lo, A->n, A->m, &lk_target, &lncv, &lconv)) {
      KR_CHECK_ARG(left_out, "krans_solve_cyclic: left_out is NULL");
      RunOut ro;
      rc = run_cyclic(ctx, A, true, rng, lo, nullptr, lk_target, lncv, left, &ro);
      if (rc == KRANS_OK) {
        result->cg_solves += ro.r.cg_solves;
        result->cg_maxit_hits += ro.r.cg_maxit_hits;
        result->spmv += ro.r.spmv;
        result->spmvT += ro.r.spmvT;
        result->algo_bytes += ro.r.bytes;
        result->device_ms += ro.ms;
        result->fp64_fallback |= ro.fp64_fallback;
      }
    }
    for (size_t i = 0; i < left.size(); i++)
      left_out[i] = left[i];
    result->n_left = (int64_t)left.size();
  }
  return rc;
}

