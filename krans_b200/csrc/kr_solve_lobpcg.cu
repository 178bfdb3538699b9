// LOBPCG launch: argument rules of the reference, workspace, team choice.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "kr_internal.h"
#include "kr_types.cuh"

namespace kr {

static inline int64_t rup(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

struct LCarver {
  size_t off = 0;
  char *base = nullptr;
  template <class T> T *take(int64_t count) {
    off = (size_t)rup((int64_t)off, 256);
    T *p = base ? (T *)(base + off) : nullptr;
    off += (size_t)std::max<int64_t>(count, 1) * sizeof(T);
    return p;
  }
};

static size_t lobpcg_layout(int64_t m, int64_t n, int64_t bs, int64_t k, int64_t pmax, int ncta, char *base,
                            LobpcgDesc *d) {
  LCarver c;
  c.base = base;
  const int64_t ldn = rup(std::max<int64_t>(n, 1), 32), ldm = rup(std::max<int64_t>(m, 1), 32);
  LobpcgDesc t;
  memset(&t, 0, sizeof t);
  t.X = c.take<double>(bs * ldn);
  t.AX = c.take<double>(bs * ldn);
  t.Rb = c.take<double>(bs * ldn);
  t.W = c.take<double>(bs * ldn);
  t.P = c.take<double>(bs * ldn);
  t.T1 = c.take<double>(bs * ldn);
  t.T2 = c.take<double>(bs * ldn);
  t.Z = c.take<double>(3 * bs * ldn);
  t.AZ = c.take<double>(3 * bs * ldn);
  t.Yl = c.take<double>(std::max<int64_t>(k, 1) * ldn);
  t.RN = c.take<double>(std::max<int64_t>(k, 1) * ldn);
  t.tmv = c.take<double>(ldm);
  t.vacc = c.take<double>(ldn);
  t.Zi = c.take<double>(KR_NBP * ldn);
  t.Ti = c.take<double>(KR_NBP * ldm);
  t.avn = c.take<double>(bs);
  t.theta = c.take<double>(bs);
  t.th = c.take<double>(pmax);
  t.S = c.take<double>(pmax * pmax);
  t.G = c.take<double>(pmax * pmax);
  t.Ym = c.take<double>(pmax * pmax);
  t.Sj = c.take<double>(pmax * pmax);
  t.Li = c.take<double>(pmax * pmax);
  t.Tm = c.take<double>(pmax * pmax);
  t.Cm = c.take<double>(pmax * pmax);
  t.Q = c.take<double>(pmax * pmax);
  t.eig_cs = c.take<double>(2 * (pmax / 2 + 2));
  t.eig_pq = c.take<int32_t>(2 * (pmax / 2 + 2));
  t.eig_ord = c.take<int32_t>(pmax + 4);
  {
    // partials of the tiled products: up to (2 ncta + tiles) items of one
    // 64 x 64 tile (A^T B) or two (S and G of the Gram)
    const int64_t tiles = ((pmax + 63) / 64) * ((pmax + 63) / 64);
    t.gram_part = c.take<double>(std::max<int64_t>((int64_t)ncta * 2 * pmax * pmax, (2 * (int64_t)ncta + tiles) * 8192));
  }
  t.theta_out = c.take<double>(std::max<int64_t>(k, 1));
  t.resid_out = c.take<double>(std::max<int64_t>(k, 1));
  t.pr = c.take<double>(ldm);
  t.pg = c.take<double>(ldn);
  t.ptmp = c.take<double>(ldm);
  t.Vb = c.take<double>(std::max<int64_t>(k, 1) * ldn);
  t.D = c.take<double>((k + 2) * ldn);
  t.Vn = c.take<double>((k + 2) * ldn);
  t.Zp = c.take<double>((2 * k + 2) * ldn);
  t.AZp = c.take<double>((2 * k + 2) * ldn);
  t.sv_av = c.take<double>(ldm);
  t.sv_t = c.take<double>(ldn);
  t.sv_d = c.take<double>(ldn);
  t.sv_ad = c.take<double>(ldm);
  t.sv_nd = c.take<double>(ldn);
  t.sv_vn = c.take<double>(ldn);
  t.pc_q = c.take<double>(ldn);
  t.pc_nq = c.take<double>(ldn);
  t.pc_dinv = c.take<double>(ldn);
  t.pc_tm = c.take<double>(ldm);
  t.status = c.take<int32_t>(1);
  t.res = c.take<LobpcgDevResult>(1);
  t.gb = c.take<GridBarrierState>(1);
  t.gpart = c.take<double>(2 * std::max(ncta, 1) * KR_RED_K);
  t.flag = c.take<int32_t>(4);
  t.dflag = c.take<double>(4);
  if (d) {
    LobpcgDesc keep = *d;
    *d = t;
    d->F = keep.F;
    d->B = keep.B;
    d->o = keep.o;
    d->k_target = keep.k_target;
    d->bs = keep.bs;
    d->guards = keep.guards;
    d->rng = keep.rng;
    d->initial = keep.initial;
    d->n_initial = keep.n_initial;
    d->ldn = ldn;
    d->ldm = ldm;
    d->pmax = pmax;
  }
  return c.off + 256;
}

static const char *lobpcg_err_msg(int code) {
  switch (code) {
  case kLobErrInitialDependent:
    return "LOBPCG: initial block is dependent";
  case kLobErrRestartOrth:
    return "LOBPCG: restart orthogonalization failed";
  case kLobErrXSlice:
    return "LOBPCG: X slice orthonormalization failed";
  case kLobErrGep:
    return "LOBPCG tiny GEP: S not SPD (after jitter)";
  case kLobErrTinyDim:
    return "LOBPCG: tiny problem too large (nv cap)";
  default:
    return "LOBPCG: unknown device error";
  }
}

} // namespace kr

using namespace kr;

extern "C" int krans_solve_lobpcg(krans_ctx *ctx, const krans_mat *A, krans_rng *rng,
                                  const krans_lobpcg_opts *opts, const krans_vec *const *initial_block,
                                  int64_t n_initial, krans_vec **right_out, double *theta_out,
                                  double *resid_out, krans_lobpcg_result *result) {
  KR_CHECK_ARG(ctx && A && rng && opts && result, "krans_solve_lobpcg: NULL argument");
  KR_CHECK_ARG(A->ctx == ctx && rng->ctx == ctx, "krans_solve_lobpcg: objects of another context");
  memset(result, 0, sizeof *result);
  const krans_lobpcg_opts &o = *opts;
  const int64_t m = A->m, n = A->n;
  if (n == 0 || m == 0)
    return KRANS_OK;
  // k_target rules and argument checks (LOBPCGSolver.cpp:453-476)
  int64_t k_target = std::max<int64_t>(1, o.nev);
  if (o.nullity_known >= 0) {
    KR_CHECK_ARG((int64_t)o.nullity_known <= n, "LOBPCG: nullity_known > n");
    k_target = o.nullity_known;
  }
  if (o.rank_known >= 0) {
    const int64_t rk = o.rank_known;
    KR_CHECK_ARG(rk <= n, "LOBPCG: rank_known > n");
    const int64_t implied = n - rk;
    KR_CHECK_ARG(!(o.nullity_known >= 0 && implied != k_target),
                 "LOBPCG: inconsistent rank_known vs nullity_known");
    if (o.nullity_known < 0)
      k_target = implied;
    if (n <= rk) {
      result->frob_norm_est = 0.0;
      result->converged_to_target = (k_target == 0);
      return KRANS_OK;
    }
  }
  int64_t bs = o.block_size > 0 ? o.block_size : std::min<int64_t>(16, std::max<int64_t>(1, k_target));
  bs = std::min<int64_t>(bs, n);
  result->block_size = bs;
  const int64_t guards =
      (bs == 1) ? 0 : std::min<int64_t>((int64_t)((1.0 - o.restart) * (double)bs + 0.45), bs - 1);
  KR_CHECK_ARG(bs <= 128, "krans_solve_lobpcg: block_size above 128 is not supported");
  KR_CHECK_ARG(o.precond_normal >= KRANS_PRECOND_NONE && o.precond_normal <= KRANS_PRECOND_SD &&
                   o.precond_steps >= 1 && o.precond_steps <= 1000,
               "krans_solve_lobpcg: precond_normal must be a KRANS_PRECOND_* value, precond_steps in [1, 1000]");
  KR_CHECK_ARG(k_target <= 512, "krans_solve_lobpcg: more than 512 null vectors");
  if (n_initial > 0)
    KR_CHECK_ARG(initial_block != nullptr, "krans_solve_lobpcg: initial_block is NULL");
  for (int64_t i = 0; i < n_initial; i++)
    KR_CHECK_ARG(initial_block[i] && initial_block[i]->n == n, "krans_solve_lobpcg: initial vector size mismatch");
  KR_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lk(ctx->mu);

  const int64_t pmax = std::max<int64_t>(3 * bs, 2 * k_target + 2);
  int team = o.team;
  if (team == KRANS_TEAM_AUTO)
    team = (m + n) < 120000 ? KRANS_TEAM_CTA : KRANS_TEAM_GRID;
  const int threads = 512;
  const int ncta = team == KRANS_TEAM_GRID ? lobpcg_grid_blocks(ctx, threads) : 1;

  LobpcgDesc d;
  memset(&d, 0, sizeof d);
  d.F = CsrView{A->m, A->n, A->nnz, A->rp, A->ci, A->v, A->v32, tuned_lanes(A->ctx, A->m, A->nnz), A->ulen};
  d.B = CsrView{A->n, A->m, A->nnz, A->rpT, A->ciT, A->vT, A->vT32, tuned_lanes(A->ctx, A->n, A->nnz), A->ulenT};
  d.o = o;
  d.k_target = k_target;
  d.bs = bs;
  d.guards = guards;
  d.rng = rng->d;
  d.n_initial = n_initial;
  const size_t bytes = lobpcg_layout(m, n, bs, k_target, pmax, ncta, nullptr, nullptr);
  char *ws = nullptr;
  int rc = dev_alloc(ctx, (void **)&ws, bytes);
  if (rc != KRANS_OK)
    return rc;
  double **d_init = nullptr;
  std::vector<double *> hinit;
  for (int64_t i = 0; i < n_initial; i++)
    hinit.push_back(initial_block[i]->d);
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (n_initial > 0) {
    e = cudaMalloc(&d_init, sizeof(double *) * (size_t)n_initial);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_init, hinit.data(), sizeof(double *) * (size_t)n_initial, cudaMemcpyHostToDevice, s);
  }
  d.initial = d_init;
  lobpcg_layout(m, n, bs, k_target, pmax, ncta, ws, &d);
  LobpcgDesc *d_desc = nullptr;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d.status, 0, 4, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d.gb, 0, sizeof(GridBarrierState), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d.res, 0, sizeof(LobpcgDevResult), s);
  if (e == cudaSuccess)
    e = cudaEventRecord(e0, s);
  if (e == cudaSuccess && team != KRANS_TEAM_GRID) {
    e = cudaMalloc(&d_desc, sizeof(LobpcgDesc));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_desc, &d, sizeof d, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess)
    e = launch_lobpcg(team == KRANS_TEAM_GRID, d, d_desc, ncta, threads, s);
  if (e == cudaSuccess)
    e = cudaEventRecord(e1, s);
  LobpcgDevResult R;
  memset(&R, 0, sizeof R);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&R, d.res, sizeof R, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess)
    cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (d_desc)
    cudaFree(d_desc);
  if (d_init)
    cudaFree(d_init);
  if (e != cudaSuccess) {
    dev_free(ctx, ws, bytes);
    return cuda_fail(e, "lobpcg launch", __FILE__, __LINE__);
  }
  if (R.status != KRANS_OK) {
    dev_free(ctx, ws, bytes);
    set_error("LOBPCG: device status %d (a bounded device wait gave up)", R.status);
    return R.status;
  }
  result->iters = R.iters;
  result->locked = R.locked;
  result->frob_norm_est = R.frob;
  result->accept_threshold = R.accept;
  result->best_unaccepted_residual = R.best_unaccepted;
  result->converged_to_target = R.converged;
  result->spmv = R.spmv;
  result->spmvT = R.spmvT;
  result->algo_bytes = R.bytes;
  result->gram_flops = R.gram_flops;
  result->device_ms = ms;
  for (int i = 0; i < 5; i++)
    result->phase_ms[i] = R.phase_ms[i];
  result->final_polish_ms = R.final_polish_ms;
  if (R.err_code != kLobErrNone) {
    dev_free(ctx, ws, bytes);
    set_error("%s", lobpcg_err_msg(R.err_code));
    return KRANS_ERR_RUNTIME;
  }
  KR_CHECK_ARG(right_out || R.n_right == 0, "krans_solve_lobpcg: right_out is NULL");
  std::vector<double> th((size_t)std::max<int64_t>(R.n_right, 1)), rs((size_t)std::max<int64_t>(R.n_right, 1));
  if (R.n_right > 0) {
    e = cudaMemcpyAsync(th.data(), d.theta_out, 8 * (size_t)R.n_right, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(rs.data(), d.resid_out, 8 * (size_t)R.n_right, cudaMemcpyDeviceToHost, s);
  }
  for (int64_t i = 0; i < R.n_right && e == cudaSuccess && rc == KRANS_OK; i++) {
    krans_vec *v = nullptr;
    rc = krans_vec_create(ctx, n, &v);
    if (rc == KRANS_OK) {
      e = cudaMemcpyAsync(v->d, d.RN + i * d.ldn, (size_t)n * 8, cudaMemcpyDeviceToDevice, s);
      right_out[i] = v;
      result->n_right = i + 1;
    }
  }
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  dev_free(ctx, ws, bytes);
  if (e != cudaSuccess)
    return cuda_fail(e, "lobpcg results", __FILE__, __LINE__);
  if (theta_out)
    for (int64_t i = 0; i < R.n_right; i++)
      theta_out[i] = th[i];
  if (resid_out)
    for (int64_t i = 0; i < R.n_right; i++)
      resid_out[i] = rs[i];
  return rc;
}

// ---------------------------------------------------------------------------
// Served LOBPCG requests (krans_submit with KRANS_SOLVER_LOBPCG): planned,
// launched on one of the server's streams and polled, without blocking the
// server's scheduler. One thread block solves requests with m + n below the
// context's cluster_min, a thread-block cluster the larger ones (the whole-GPU
// cooperative team would stall every other launch). After the solve, one
// block computes max ||A u|| of the returned basis.
// ---------------------------------------------------------------------------
namespace kr {

cudaError_t launch_lobpcg_cluster(const LobpcgDesc *d_dev, int csize, cudaStream_t s);
cudaError_t launch_lobpcg_cta(const LobpcgDesc *d_dev, int threads, cudaStream_t s);
cudaError_t launch_basis_max_residual(const CsrView &F, const double *basis, int64_t ldb, const int64_t *nf,
                                      double *out, cudaStream_t s);

struct LobpcgAsync {
  krans_ctx *ctx = nullptr;
  krans_request req;
  LobpcgDesc d;
  int64_t m = 0, n = 0, k_target = 0, bs = 0, pmax = 0;
  int ncta = 1;
  bool trivial = false, converged_trivial = false;
  char *ws = nullptr;
  size_t bytes = 0, layout_bytes = 0;
  LobpcgDesc *d_desc = nullptr;
  RngState *d_rng = nullptr;
  double *d_mr = nullptr;
  LobpcgDevResult *h_res = nullptr;
  double *h_mr = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evd = nullptr;
  cudaStream_t stream = nullptr; // the launch's stream (stream-ordered workspace)
};

static void seed_state(RngState &s, uint32_t seed, int mode) {
  memset(&s, 0, sizeof s);
  s.mt[0] = seed;
  for (int i = 1; i < 624; i++)
    s.mt[i] = 1812433253u * (s.mt[i - 1] ^ (s.mt[i - 1] >> 30)) + (uint32_t)i;
  s.idx = 624;
  s.philox_key = ((uint64_t)seed << 32) ^ 0x9E3779B97F4A7C15ull;
  s.mode = mode;
}

int lobpcg_async_plan(krans_ctx *ctx, const krans_request &r, LobpcgAsync **out, size_t *need) {
  *out = nullptr;
  *need = 0;
  KR_CHECK_ARG(r.A && r.A->ctx == ctx, "krans_submit: request without a matrix of this context");
  const krans_lobpcg_opts &o = r.lobpcg;
  KR_CHECK_ARG(o.precision == KRANS_PREC_FP64, "krans_submit: LOBPCG requests run in FP64");
  auto *a = new LobpcgAsync();
  a->ctx = ctx;
  a->req = r;
  const krans_mat *A = r.A;
  a->m = A->m;
  a->n = A->n;
  const int64_t m = A->m, n = A->n;
  // k_target rules and argument checks (LOBPCGSolver.cpp:453-476)
  int64_t k_target = std::max<int64_t>(1, o.nev);
  if (o.nullity_known >= 0) {
    if ((int64_t)o.nullity_known > n) {
      delete a;
      set_error("LOBPCG: nullity_known > n");
      return KRANS_ERR_INVALID_ARGUMENT;
    }
    k_target = o.nullity_known;
  }
  if (o.rank_known >= 0) {
    const int64_t rk = o.rank_known, implied = n - rk;
    if (rk > n || (o.nullity_known >= 0 && implied != k_target)) {
      delete a;
      set_error(rk > n ? "LOBPCG: rank_known > n" : "LOBPCG: inconsistent rank_known vs nullity_known");
      return KRANS_ERR_INVALID_ARGUMENT;
    }
    if (o.nullity_known < 0)
      k_target = implied;
    if (n <= rk) {
      a->trivial = true;
      a->converged_trivial = k_target == 0;
    }
  }
  if (n == 0 || m == 0)
    a->trivial = true;
  a->k_target = k_target;
  if (a->trivial) {
    *out = a;
    return KRANS_OK;
  }
  int64_t bs = o.block_size > 0 ? o.block_size : std::min<int64_t>(16, std::max<int64_t>(1, k_target));
  bs = std::min<int64_t>(bs, n);
  if (bs > 128 || k_target > 512 || (r.basis_out && r.basis_capacity < k_target) ||
      o.precond_normal < KRANS_PRECOND_NONE || o.precond_normal > KRANS_PRECOND_SD || o.precond_steps < 1 ||
      o.precond_steps > 1000) {
    delete a;
    set_error("krans_submit: LOBPCG request needs block_size <= 128, at most 512 vectors, basis_out of "
              "capacity >= its target and a KRANS_PRECOND_* preconditioner");
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  a->bs = bs;
  a->pmax = std::max<int64_t>(3 * bs, 2 * k_target + 2);
  const bool cluster = (m + n) >= ctx->tune.cluster_min;
  a->ncta = cluster ? std::min(4, std::max(2, ctx->tune.cluster_size)) : 1;
  LobpcgDesc &d = a->d;
  memset(&d, 0, sizeof d);
  d.F = CsrView{A->m, A->n, A->nnz, A->rp, A->ci, A->v, A->v32, tuned_lanes(ctx, A->m, A->nnz), A->ulen};
  d.B = CsrView{A->n, A->m, A->nnz, A->rpT, A->ciT, A->vT, A->vT32, tuned_lanes(ctx, A->n, A->nnz), A->ulenT};
  d.o = o;
  d.o.team = cluster ? KRANS_TEAM_GRID : KRANS_TEAM_CTA; // informational only
  d.k_target = k_target;
  d.bs = bs;
  d.guards = (bs == 1) ? 0 : std::min<int64_t>((int64_t)((1.0 - o.restart) * (double)bs + 0.45), bs - 1);
  d.n_initial = 0;
  a->layout_bytes = lobpcg_layout(m, n, bs, k_target, a->pmax, a->ncta, nullptr, nullptr);
  a->bytes = kr_round_up((int64_t)a->layout_bytes, 256) + kr_round_up(sizeof(LobpcgDesc), 256) +
             kr_round_up(sizeof(RngState), 256) + 256;
  *need = a->bytes;
  *out = a;
  return KRANS_OK;
}

int lobpcg_async_launch(LobpcgAsync *a, cudaStream_t s) {
  if (a->trivial)
    return KRANS_OK;
  int rc = dev_alloc_async(a->ctx, (void **)&a->ws, a->bytes, s);
  if (rc != KRANS_OK)
    return rc;
  a->stream = s;
  char *p = a->ws;
  LobpcgDesc &d = a->d;
  d.rng = nullptr;
  lobpcg_layout(a->m, a->n, a->bs, a->k_target, a->pmax, a->ncta, p, &d);
  p += kr_round_up((int64_t)a->layout_bytes, 256);
  a->d_desc = reinterpret_cast<LobpcgDesc *>(p);
  p += kr_round_up(sizeof(LobpcgDesc), 256);
  a->d_rng = reinterpret_cast<RngState *>(p);
  d.rng = a->d_rng;
  a->d_mr = d.dflag + 3; // a spare slot of the workspace's scalar flags
  RngState st;
  seed_state(st, a->req.seed ? a->req.seed : 0x9E3779B9u, a->req.rng_mode);
  cudaError_t e = cudaMallocHost(&a->h_res, sizeof(LobpcgDevResult));
  if (e == cudaSuccess)
    e = cudaMallocHost(&a->h_mr, sizeof(double));
  if (e == cudaSuccess)
    e = cudaEventCreate(&a->ev0);
  if (e == cudaSuccess)
    e = cudaEventCreate(&a->ev1);
  if (e == cudaSuccess)
    e = cudaEventCreateWithFlags(&a->evd, cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->d_rng, &st, sizeof st, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->d_desc, &d, sizeof d, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d.status, 0, 4, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d.gb, 0, sizeof(GridBarrierState), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d.res, 0, sizeof(LobpcgDevResult), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(a->d_mr, 0, sizeof(double), s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s); // the host copies above came from this stack frame
  if (e == cudaSuccess)
    e = cudaEventRecord(a->ev0, s);
  if (e == cudaSuccess)
    e = a->ncta > 1 ? launch_lobpcg_cluster(a->d_desc, a->ncta, s) : launch_lobpcg_cta(a->d_desc, 512, s);
  if (e == cudaSuccess)
    e = cudaEventRecord(a->ev1, s);
  if (e == cudaSuccess)
    e = launch_basis_max_residual(d.F, d.RN, d.ldn, &d.res->n_right, a->d_mr, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->h_res, d.res, sizeof(LobpcgDevResult), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->h_mr, a->d_mr, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && a->k_target > 0 && a->req.basis_out)
    e = cudaMemcpy2DAsync(a->req.basis_out, (size_t)a->n * 8, d.RN, (size_t)d.ldn * 8, (size_t)a->n * 8,
                          (size_t)a->k_target, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess)
    e = cudaEventRecord(a->evd, s);
  if (e != cudaSuccess)
    return cuda_fail(e, "served LOBPCG launch", __FILE__, __LINE__);
  return KRANS_OK;
}

bool lobpcg_async_done(const LobpcgAsync *a) { return a->trivial || cudaEventQuery(a->evd) == cudaSuccess; }

void lobpcg_async_finish(const LobpcgAsync *a, krans_request_result *out) {
  memset(out, 0, sizeof *out);
  if (a->trivial) {
    out->converged_to_target = a->converged_trivial ? 1 : 0;
    return;
  }
  const LobpcgDevResult &R = *a->h_res;
  out->status = R.status;
  if (out->status == KRANS_OK && R.err_code != kLobErrNone) {
    out->status = KRANS_ERR_RUNTIME;
    set_error("%s", lobpcg_err_msg(R.err_code));
  }
  out->converged_to_target = R.converged;
  out->n_right = R.n_right;
  out->restarts = R.iters;
  out->krylov_steps_total = R.locked;
  out->spmv = R.spmv;
  out->spmvT = R.spmvT;
  out->frob_norm_est = R.frob;
  out->max_residual = *a->h_mr;
  out->algo_bytes = R.bytes;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a->ev0, a->ev1);
  out->device_ms = ms;
  out->phase_ms[0] = R.phase_ms[0];
  out->phase_ms[1] = R.phase_ms[1] + R.phase_ms[2];
  out->phase_ms[2] = R.phase_ms[3];
  out->phase_ms[3] = R.phase_ms[4];
}

int lobpcg_async_cancel(LobpcgAsync *a, cudaStream_t ctl) {
  static const int32_t cancelled = KRANS_ERR_CANCELLED;
  if (a->trivial || !a->ws)
    return KRANS_OK;
  cudaError_t e = cudaMemcpyAsync(a->d.status, &cancelled, 4, cudaMemcpyHostToDevice, ctl);
  return e == cudaSuccess ? KRANS_OK : cuda_fail(e, "cancel request", __FILE__, __LINE__);
}

// Pinned host buffers go to `graveyard` when one is given (cudaFreeHost
// waits for the whole device; the server frees them once nothing runs).
void lobpcg_async_release(LobpcgAsync *a, std::vector<void *> *graveyard) {
  if (!a)
    return;
  if (a->ws)
    dev_free_async(a->ctx, a->ws, a->bytes, a->stream);
  for (void *h : {(void *)a->h_res, (void *)a->h_mr})
    if (h) {
      if (graveyard)
        graveyard->push_back(h);
      else
        cudaFreeHost(h);
    }
  if (a->ev0)
    cudaEventDestroy(a->ev0);
  if (a->ev1)
    cudaEventDestroy(a->ev1);
  if (a->evd)
    cudaEventDestroy(a->evd);
  delete a;
}

} // namespace kr
