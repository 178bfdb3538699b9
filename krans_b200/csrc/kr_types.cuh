// Plain data shared by the host launchers and the device solvers: matrix
// views, solve descriptors, workspace layout and result records. Host
// translation units include only this header (fast to compile); the solver
// templates live in kr_cyclic.cuh / kr_lobpcg.cuh / kr_batch.cuh.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/krans_cuda.h"

#ifndef KR_RED_K
#define KR_RED_K 8 // values per fused team reduction
#endif
#define KR_NBP 8 // right-hand sides of the block CG polish (one fused reduction)

namespace kr {

struct GridBarrierState {
  unsigned int count;
  unsigned int gen;
  int error; // sticky: once set, barriers return at once and solvers unwind
  int pad;
  uint64_t timeout_ns; // longest wait at one barrier; 0 = the default (kBarrierTimeoutNs)
};

// State of one factory stream. Layout of the MT part equals the CPU oracle's.
struct RngState {
  uint32_t mt[624];
  int32_t idx;
  int32_t has_saved;
  double saved;
  uint64_t philox_key;
  uint64_t philox_ctr;
  int32_t mode;
  int32_t pad;
};

struct CsrView {
  int64_t rows, cols, nnz;
  const int32_t *rp, *ci;
  const double *v64;
  const float *v32;
  int lanes;    // threads per row in the SpMV
  int32_t ulen; // every row has exactly ulen entries (rp[i] = i*ulen), 0 if not
};

struct CyclicDevResult {
  int64_t n_found;
  int64_t restarts, krylov_steps_total, cg_solves, cg_maxit_hits, spmv, spmvT;
  double frob, bytes;
  int32_t converged;
  int32_t status;
  uint64_t t_begin, t_end; // device globaltimer (ns) when the request started / finished
  double phase_ms[4];      // device time in: Golub-Kahan + reorth, tiny SVD, CG polish, the rest
};

struct CyclicDesc {
  CsrView F, B; // F: the run's operator (rows m, cols n); B: its transpose
  krans_cyclic_opts o;
  int64_t k_target, ncv;
  int32_t trans_run; // 1 for the left-space run (counts swap)
  RngState *rng;
  const double *initial_right; // n doubles or nullptr
  double *basis;               // k_target x ldn (output, row i = vector i)
  int64_t nb_init;             // rows of basis already accepted (a continued run), else 0
  double frob_init;            // ||A||_F estimate of the run being continued, else 0 (estimate it)
  void *Y, *X, *wx, *wy;       // KT storage
  double *y0, *v, *vp, *best_v, *tn; // n-vectors
  double *Vc;                        // KR_NBP candidate n-vectors (block polish)
  double *Hb, *Wb, *Rk, *Pk, *Ak, *Tk; // interleaved CG blocks: m x KR_NBP (Tk: n x KR_NBP)
  double *tmv, *wm, *Ap;             // m-vectors
  double2 *rp;                       // CG residual and direction, interleaved (m)
  double *r_pre, *dinv, *sd_q, *sd_Oq; // preconditioned CG: residual, Jacobi weights, SD vectors (m)
  double *alpha, *beta;              // ncv + 2
  double *Tb, *Vt, *sv;              // tiny problem
  int32_t *ord;
  double *eig_cs;
  int32_t *eig_pq, *eig_ord;
  int64_t ldn, ldm, ldb, cap; // ldb: stride of the basis rows
  int32_t *status;
  CyclicDevResult *res;
  GridBarrierState *gb;
  double *gpart;
};

// Workspace plan of one cyclic run and the carving of one allocation into its
// arrays (256-byte aligned). Shared by the single-request launch (host) and
// the persistent batched kernel, which lays out a slot per block on device.
struct CyclicPlan {
  int64_t m, n, k_target, ncv, ldn, ldm, ldb, cap;
  int32_t ksz;         // bytes of the Krylov storage type
  int32_t grid_blocks; // blocks of a grid team (reduction partials)
  int32_t own_basis;   // basis lives in the workspace (else in the request)
  int32_t block_polish; // workspace for the block CG polish (KR_NBP candidates at once)
  int32_t precond;      // KRANS_PRECOND_* of the CG projector (workspace for it)
};

__host__ __device__ inline int64_t kr_round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// Shared-memory bytes that hold the CG vectors of a one-block solve (residual
// and direction interleaved, F F^T p, F^T p): 16 ldm + 8 ldm + 8 ldn.
__host__ __device__ inline size_t cta_cg_smem_bytes(int64_t ldm, int64_t ldn) {
  return (size_t)(24 * ldm + 8 * ldn);
}

struct Carver {
  size_t off = 0;
  char *base = nullptr;
  template <class T> __host__ __device__ T *take(int64_t count) {
    off = (size_t)kr_round_up((int64_t)off, 256);
    T *p = base ? (T *)(base + off) : nullptr;
    off += (size_t)(count > 1 ? count : 1) * sizeof(T);
    return p;
  }
};

__host__ __device__ inline size_t cyclic_carve(const CyclicPlan &p, char *base, CyclicDesc *d) {
  Carver c;
  c.base = base;
  void *Y = c.take<char>(p.cap * p.ldn * p.ksz);
  void *X = c.take<char>(p.cap * p.ldm * p.ksz);
  void *wx = c.take<char>(p.ldm * p.ksz);
  void *wy = c.take<char>(p.ldn * p.ksz);
  double *basis = p.own_basis ? c.take<double>((p.k_target > 1 ? p.k_target : 1) * p.ldb) : nullptr;
  double *y0 = c.take<double>(p.ldn), *v = c.take<double>(p.ldn), *vp = c.take<double>(p.ldn);
  double *best_v = c.take<double>(p.ldn), *tn = c.take<double>(p.ldn);
  double *tmv = c.take<double>(p.ldm), *wm = c.take<double>(p.ldm);
  double2 *rp = c.take<double2>(p.ldm);
  double *Ap = c.take<double>(p.ldm);
  double *alpha = c.take<double>(p.ncv + 2), *beta = c.take<double>(p.ncv + 2);
  double *Tb = c.take<double>((p.ncv + 1) * p.ncv), *Vt = c.take<double>(p.ncv * p.ncv);
  double *sv = c.take<double>(p.ncv + 1);
  int32_t *ord = c.take<int32_t>(p.ncv + 2);
  double *eig_cs = c.take<double>(p.ncv * p.ncv + 2 * p.ncv + 4);
  int32_t *eig_pq = c.take<int32_t>(p.ncv + 4), *eig_ord = c.take<int32_t>(p.ncv + 4);
  int32_t *status = c.take<int32_t>(1);
  CyclicDevResult *res = c.take<CyclicDevResult>(1);
  GridBarrierState *gb = c.take<GridBarrierState>(1);
  double *gpart = c.take<double>(2 * (p.grid_blocks > 1 ? p.grid_blocks : 1) * KR_RED_K);
  double *r_pre = nullptr, *dinv = nullptr, *sd_q = nullptr, *sd_Oq = nullptr;
  if (p.precond) {
    r_pre = c.take<double>(p.ldm);
    dinv = c.take<double>(p.ldm);
    sd_q = c.take<double>(p.ldm);
    sd_Oq = c.take<double>(p.ldm);
  }
  double *Vc = nullptr, *Hb = nullptr, *Wb = nullptr, *Rk = nullptr, *Pk = nullptr, *Ak = nullptr, *Tk = nullptr;
  if (p.block_polish) {
    Vc = c.take<double>(KR_NBP * p.ldn);
    Hb = c.take<double>(KR_NBP * p.ldm);
    Wb = c.take<double>(KR_NBP * p.ldm);
    Rk = c.take<double>(KR_NBP * p.ldm);
    Pk = c.take<double>(KR_NBP * p.ldm);
    Ak = c.take<double>(KR_NBP * p.ldm);
    Tk = c.take<double>(KR_NBP * p.ldn);
  }
  if (d) {
    d->Y = Y; d->X = X; d->wx = wx; d->wy = wy;
    if (p.own_basis) d->basis = basis;
    d->y0 = y0; d->v = v; d->vp = vp; d->best_v = best_v; d->tn = tn;
    d->tmv = tmv; d->wm = wm; d->rp = rp; d->Ap = Ap;
    d->alpha = alpha; d->beta = beta; d->Tb = Tb; d->Vt = Vt; d->sv = sv; d->ord = ord;
    d->eig_cs = eig_cs; d->eig_pq = eig_pq; d->eig_ord = eig_ord;
    if (p.own_basis) { d->status = status; d->res = res; }
    d->gb = gb; d->gpart = gpart;
    d->Vc = Vc; d->Hb = Hb; d->Wb = Wb; d->Rk = Rk; d->Pk = Pk; d->Ak = Ak; d->Tk = Tk;
    d->r_pre = r_pre; d->dinv = dinv; d->sd_q = sd_q; d->sd_Oq = sd_Oq;
    d->ldn = p.ldn; d->ldm = p.ldm; d->ldb = p.ldb; d->cap = p.cap;
  }
  return c.off + 256;
}

// Completion record of one request of an open launch, in host-mapped pinned
// memory: the team copies its result here and then sets `done`, which the
// host polls while the launch keeps running.
struct HostDone {
  CyclicDevResult res;
  double max_resid;
  int32_t status;
  int32_t done;
};

// The requests an open launch may take, published by the host while it runs
// (host-mapped pinned memory: the host writes, the device only reads).
struct LaunchFeed {
  int32_t published[3]; // requests published to the large, mid and small queues
  int32_t closed;       // nonzero: the host publishes no more requests to this launch
  uint64_t idle_ns;     // a team that finds no request for this long leaves the launch
};

struct CyclicRequestDev {
  CsrView F, B;
  krans_cyclic_opts o;
  CyclicPlan plan;
  RngState *rng;
  double *basis; // request output, row i = vector i, stride plan.ldb
  CyclicDevResult *res;
  int32_t *status;
  double *max_resid;
  const double *initial_right; // start vector y0 or nullptr
  int64_t nb_init;             // basis rows already accepted (continued run), else 0
  double frob_init;            // ||A||_F estimate to reuse (continued run), else 0
  HostDone *done;              // open launches: completion record (else nullptr)
  int32_t trivial;   // reference early exit: nothing to compute
  int32_t trans_run; // 1: the run is on A^T (left null space)
};

struct LobpcgDevResult {
  int64_t n_right, iters, locked, block_size;
  double frob, accept, best_unaccepted;
  int32_t converged, status;
  int32_t err_code, pad;
  int64_t spmv, spmvT;
  double bytes, gram_flops;
  double phase_ms[5]; // device time in: apply_normal, Gram, tiny GEP, orthonormalisation, the rest
  double final_polish_ms; // part of the rest: the closing polish, sharpening and MGS
};

// error codes of the reference's throws (reported as KRANS_ERR_RUNTIME)
enum LobpcgErr {
  kLobErrNone = 0,
  kLobErrInitialDependent = 1, // "LOBPCG: initial block is dependent"
  kLobErrRestartOrth = 2,      // "LOBPCG: restart orthogonalization failed"
  kLobErrXSlice = 3,           // "LOBPCG: X slice orthonormalization failed"
  kLobErrGep = 4,              // "LOBPCG tiny GEP: S not SPD (after jitter)"
  kLobErrTinyDim = 5,          // "LOBPCG: tiny problem too large (nv cap)"
};

struct LobpcgDesc {
  CsrView F, B; // A (m x n) and A^T
  krans_lobpcg_opts o;
  int64_t k_target, bs, guards;
  RngState *rng;
  double *const *initial; // n_initial device vectors (or nullptr)
  int64_t n_initial;
  // blocks (column-major, ld = ldn)
  double *X, *AX, *Rb, *W, *P, *T1, *T2, *Z, *AZ;
  double *Yl, *RN; // locked set and output basis (k_target columns)
  double *tmv, *vacc;
  double *Zi, *Ti, *avn; // interleaved groups of KR_NBP columns (n and m rows), ||A x_j|| of the block
  double *theta, *th;
  // small dense matrices (pmax x pmax)
  double *S, *G, *Ym, *Sj, *Li, *Tm, *Cm, *Q;
  double *eig_cs;
  int32_t *eig_pq, *eig_ord;
  double *gram_part;
  double *theta_out, *resid_out; // k_target
  // polish scratch
  double *pr, *pg, *ptmp;              // m, n, m
  double *Vb, *D, *Vn, *Zp, *AZp;      // k, k+2, k, 2k+2, 2k+2 columns
  double *sv_av, *sv_t, *sv_d, *sv_ad, *sv_nd, *sv_vn; // sharpen scratch
  double *pc_q, *pc_nq, *pc_dinv, *pc_tm;              // M_inv scratch (n, n, n, m)
  int64_t ldn, ldm, pmax;
  int32_t *status;
  LobpcgDevResult *res;
  GridBarrierState *gb;
  double *gpart;
  int32_t *flag; // uniform scalar broadcast slot (leader writes, all read)
  double *dflag;
};


// ---- host-side launchers (one translation unit per kernel family) ----------
int cyclic_grid_blocks(krans_ctx *ctx, bool mixed, int threads);
cudaError_t launch_cyclic_grid(bool mixed, const CyclicDesc &d, int blocks, int threads, cudaStream_t s);
int cyclic_batch_cta_per_sm(bool mixed);
cudaError_t launch_cyclic_batch_cta(bool mixed, int grid, int block, size_t dyn_smem, cudaStream_t s, const CyclicRequestDev *reqs, int count,
                                    int *queue, char *ws, size_t stride, const LaunchFeed *feed);
int cyclic_batch_cluster_max(bool mixed, int csize, int sms, size_t dyn_smem);
cudaError_t launch_cyclic_batch_cluster(bool mixed, int nclusters, int csize, size_t dyn_smem, cudaStream_t s,
                                        const CyclicRequestDev *reqs_large, int n_large, int *queue_large,
                                        char *ws_large, size_t stride_large, const CyclicRequestDev *reqs_small,
                                        int n_small, int *queue_small, char *ws_small, size_t stride_small,
                                        const LaunchFeed *feed, int feed_large);
int lobpcg_grid_blocks(krans_ctx *ctx, int threads);
cudaError_t launch_lobpcg(bool grid, const LobpcgDesc &d, const LobpcgDesc *d_dev, int blocks, int threads,
                          cudaStream_t s);

} // namespace kr
