// Solver launches: one cyclic request on a thread block or on the whole GPU
// (cooperative launch), and many requests in one persistent launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "kr_cyclic.cuh"
#include "kr_internal.h"

namespace kr {

static inline int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// Carves one device allocation into 256-byte aligned arrays.
struct Carver {
  size_t off = 0;
  char *base = nullptr;
  template <class T> T *take(int64_t count) {
    off = (size_t)round_up((int64_t)off, 256);
    T *p = base ? (T *)(base + off) : nullptr;
    off += (size_t)std::max<int64_t>(count, 1) * sizeof(T);
    return p;
  }
};

struct CyclicPlan {
  int64_t m, n, k_target, ncv, ldn, ldm, ldb, cap;
  int ksz; // bytes of the Krylov storage type
  int grid_blocks;
};

// Lay out (or, with base == nullptr, size) the workspace of one run.
static size_t cyclic_layout(const CyclicPlan &p, char *base, CyclicDesc *d) {
  Carver c;
  c.base = base;
  CyclicDesc t;
  memset(&t, 0, sizeof t);
  t.Y = c.take<char>(p.cap * p.ldn * p.ksz);
  t.X = c.take<char>(p.cap * p.ldm * p.ksz);
  t.wx = c.take<char>(p.ldm * p.ksz);
  t.wy = c.take<char>(p.ldn * p.ksz);
  t.basis = c.take<double>(std::max<int64_t>(p.k_target, 1) * p.ldb);
  t.y0 = c.take<double>(p.ldn);
  t.v = c.take<double>(p.ldn);
  t.vp = c.take<double>(p.ldn);
  t.best_v = c.take<double>(p.ldn);
  t.tn = c.take<double>(p.ldn);
  t.tmv = c.take<double>(p.ldm);
  t.wm = c.take<double>(p.ldm);
  t.r = c.take<double>(p.ldm);
  t.p = c.take<double>(p.ldm);
  t.Ap = c.take<double>(p.ldm);
  t.alpha = c.take<double>(p.ncv + 2);
  t.beta = c.take<double>(p.ncv + 2);
  t.Tb = c.take<double>((p.ncv + 1) * p.ncv);
  t.Vt = c.take<double>(p.ncv * p.ncv);
  t.sv = c.take<double>(p.ncv + 1);
  t.ord = c.take<int32_t>(p.ncv + 2);
  t.eig_cs = c.take<double>(p.ncv * p.ncv + 2 * p.ncv + 4);
  t.eig_pq = c.take<int32_t>(p.ncv + 4);
  t.eig_ord = c.take<int32_t>(p.ncv + 4);
  t.status = c.take<int32_t>(1);
  t.res = c.take<CyclicDevResult>(1);
  t.gb = c.take<GridBarrierState>(1);
  t.gpart = c.take<double>(2 * std::max(p.grid_blocks, 1) * KR_RED_K);
  if (d) {
    d->Y = t.Y;
    d->X = t.X;
    d->wx = t.wx;
    d->wy = t.wy;
    d->basis = t.basis;
    d->y0 = t.y0;
    d->v = t.v;
    d->vp = t.vp;
    d->best_v = t.best_v;
    d->tn = t.tn;
    d->tmv = t.tmv;
    d->wm = t.wm;
    d->r = t.r;
    d->p = t.p;
    d->Ap = t.Ap;
    d->alpha = t.alpha;
    d->beta = t.beta;
    d->Tb = t.Tb;
    d->Vt = t.Vt;
    d->sv = t.sv;
    d->ord = t.ord;
    d->eig_cs = t.eig_cs;
    d->eig_pq = t.eig_pq;
    d->eig_ord = t.eig_ord;
    d->status = t.status;
    d->res = t.res;
    d->gb = t.gb;
    d->gpart = t.gpart;
    d->ldn = p.ldn;
    d->ldm = p.ldm;
    d->ldb = p.ldb;
    d->cap = p.cap;
  }
  return c.off + 256;
}

static CsrView view_of(const krans_mat *A, bool trans) {
  CsrView v;
  if (!trans) {
    v = CsrView{A->m, A->n, A->nnz, A->rp, A->ci, A->v, A->v32, A->lanes};
  } else {
    v = CsrView{A->n, A->m, A->nnz, A->rpT, A->ciT, A->vT, A->vT32, A->lanesT};
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

int grid_blocks_for(krans_ctx *ctx, const void *kernel, int threads) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  per_sm = std::min(per_sm, 2);
  return ctx->sms * per_sm;
}

struct RunOut {
  CyclicDevResult r;
  double ms;
};

// One find_right_nullspace run on the device; basis rows land in `basis_dev`
// (stride ldb) owned by the workspace, copied into new vectors by the caller.
static int run_cyclic(krans_ctx *ctx, const krans_mat *A, bool trans, krans_rng *rng,
                      const krans_cyclic_opts &o, const double *init_right, int64_t k_target,
                      int64_t ncv, std::vector<krans_vec *> &found, RunOut *out) {
  const CsrView F = view_of(A, trans), B = view_of(A, !trans);
  const bool mixed = o.precision == KRANS_PREC_MIXED;
  if (mixed && !A->v32) {
    set_error("mixed precision needs a matrix created with KRANS_CSR_FP32");
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  KR_CHECK_ARG(k_target <= 128, "cyclic: at most 128 null vectors per request");
  KR_CHECK_ARG(ncv <= 256, "cyclic: ncv must be <= 256");
  int team = o.team;
  if (team == KRANS_TEAM_AUTO)
    team = (F.rows + F.cols) < 120000 ? KRANS_TEAM_CTA : KRANS_TEAM_GRID;
  const void *gk = mixed ? (const void *)cyclic_grid_kernel<float> : (const void *)cyclic_grid_kernel<double>;
  const int threads_grid = 512, threads_cta = 512;
  CyclicPlan p;
  p.m = F.rows;
  p.n = F.cols;
  p.k_target = k_target;
  p.ncv = ncv;
  p.ldn = round_up(p.n, 32);
  p.ldm = round_up(p.m, 32);
  p.ldb = p.ldn;
  p.cap = ncv / 2 + 2;
  p.ksz = mixed ? 4 : 8;
  p.grid_blocks = team == KRANS_TEAM_GRID ? grid_blocks_for(ctx, gk, threads_grid) : 1;
  const size_t bytes = cyclic_layout(p, nullptr, nullptr);
  char *ws = nullptr;
  int rc = dev_alloc(ctx, (void **)&ws, bytes);
  if (rc != KRANS_OK)
    return rc;
  CyclicDesc d;
  memset(&d, 0, sizeof d);
  cyclic_layout(p, ws, &d);
  d.F = F;
  d.B = B;
  d.o = o;
  d.k_target = k_target;
  d.ncv = ncv;
  d.trans_run = trans ? 1 : 0;
  d.rng = rng->d;
  d.initial_right = init_right;
  cudaStream_t s = ctx->stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  CyclicDesc *d_desc = nullptr;
  int *d_queue = nullptr;
  cudaError_t e = cudaMemsetAsync(d.status, 0, 4, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d.gb, 0, sizeof(GridBarrierState), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d.res, 0, sizeof(CyclicDevResult), s);
  if (e == cudaSuccess)
    e = cudaEventRecord(e0, s);
  if (e == cudaSuccess) {
    if (team == KRANS_TEAM_GRID) {
      void *args[] = {(void *)&d};
      e = cudaLaunchCooperativeKernel(gk, dim3(p.grid_blocks), dim3(threads_grid), args, 0, s);
    } else {
      e = cudaMalloc(&d_desc, sizeof(CyclicDesc));
      if (e == cudaSuccess)
        e = cudaMalloc(&d_queue, sizeof(int));
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_desc, &d, sizeof d, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess)
        e = cudaMemsetAsync(d_queue, 0, sizeof(int), s);
      if (e == cudaSuccess) {
        if (mixed)
          cyclic_cta_kernel<float><<<1, threads_cta, 0, s>>>(d_desc, 1, d_queue);
        else
          cyclic_cta_kernel<double><<<1, threads_cta, 0, s>>>(d_desc, 1, d_queue);
        e = cudaGetLastError();
      }
    }
  }
  if (e == cudaSuccess)
    e = cudaEventRecord(e1, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&out->r, d.res, sizeof(CyclicDevResult), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess)
    cudaEventElapsedTime(&ms, e0, e1);
  out->ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (d_desc)
    cudaFree(d_desc);
  if (d_queue)
    cudaFree(d_queue);
  if (e != cudaSuccess) {
    dev_free(ctx, ws, bytes);
    return cuda_fail(e, "cyclic solve launch", __FILE__, __LINE__);
  }
  if (out->r.status != KRANS_OK) {
    dev_free(ctx, ws, bytes);
    set_error("cyclic solve: device status %d (a bounded device wait gave up)", out->r.status);
    return out->r.status;
  }
  rc = KRANS_OK;
  for (int64_t i = 0; i < out->r.n_found && rc == KRANS_OK; i++) {
    krans_vec *v = nullptr;
    rc = krans_vec_create(ctx, p.n, &v);
    if (rc == KRANS_OK) {
      e = cudaMemcpyAsync(v->d, d.basis + i * p.ldb, (size_t)p.n * 8, cudaMemcpyDeviceToDevice, s);
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
      }
    }
    for (size_t i = 0; i < left.size(); i++)
      left_out[i] = left[i];
    result->n_left = (int64_t)left.size();
  }
  return rc;
}

