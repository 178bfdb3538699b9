// Host-side internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/krans_cuda.h"

#include <cstdlib>

// Cap on the dynamic shared memory a one-block solve uses for its CG vectors
// (KRANS_SMEM_CG_KB, default 0: global memory). Measured on B200: 160 KiB
// gave 8% less CG time on a 1000-unknown solve and cost 16% of a batch of
// uneven solves, whose cluster teams lose L1 capacity to the carve-out. Larger
// carve-outs leave less of the SM's 256 KiB to the L1 cache.
inline size_t cta_smem_cap() {
  static const size_t cap = [] {
    const char *e = getenv("KRANS_SMEM_CG_KB");
    return (size_t)(e ? atoll(e) : 0) * 1024;
  }();
  return cap;
}

namespace kr {

void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define KR_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return ::kr::cuda_fail(e_, #call, __FILE__, __LINE__);                               \
  } while (0)

#define KR_CHECK_ARG(cond, msg)                                                             \
  do {                                                                                      \
    if (!(cond)) {                                                                          \
      ::kr::set_error("%s", msg);                                                           \
      return KRANS_ERR_INVALID_ARGUMENT;                                                    \
    }                                                                                       \
  } while (0)

struct RngState;
struct GridBarrierState;

} // namespace kr

struct krans_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t budget = 0;
  std::atomic<size_t> in_use{0}; // device bytes allocated through dev_alloc* (the server thread allocates too)
  int sms = 0;
  int cc_major = 0, cc_minor = 0;
  double *h_scalar = nullptr; // pinned scalars for D2H reads
  double *d_scalar = nullptr; // device scalars (reductions)
  double *d_partials = nullptr;
  int partial_blocks = 0;
  krans_batch_tuning tune{16384, 120000, 8, {1, 2, 4, 8, 16, 32}}; // batched-launch knobs in effect
  std::mutex mu;
};

struct krans_mat {
  krans_ctx *ctx = nullptr;
  int64_t m = 0, n = 0, nnz = 0;
  int32_t *rp = nullptr, *ci = nullptr, *rpT = nullptr, *ciT = nullptr;
  double *v = nullptr, *vT = nullptr;
  float *v32 = nullptr, *vT32 = nullptr;
  int lanes = 1, lanesT = 1;
  int32_t ulen = 0, ulenT = 0; // uniform row length of A / A^T (0 = not uniform)
  krans_spmv_tuning tune{}, tuneT{}; // standalone SpMV kernel of A / A^T (zero: automatic)
  char *base = nullptr;         // one device allocation holding every stored array
  size_t bytes = 0;
};

struct krans_vec {
  krans_ctx *ctx = nullptr;
  int64_t n = 0;
  double *d = nullptr;
};

struct krans_rng {
  krans_ctx *ctx = nullptr;
  kr::RngState *d = nullptr;
  uint32_t seed = 0;
  int mode = 0;
};

namespace kr {
// One stored operand (A or its transpose) as the standalone SpMV sees it.
struct SpmvOperand {
  int64_t rows, cols, nnz;
  const int32_t *rp, *ci;
  const double *v64;
  const float *v32;
  int lanes;
  int32_t ulen;
  krans_spmv_tuning tune;
};
inline SpmvOperand spmv_operand(const krans_mat *A, int trans) {
  return trans ? SpmvOperand{A->n, A->m, A->nnz, A->rpT, A->ciT, A->vT, A->vT32, A->lanesT, A->ulenT, A->tuneT}
               : SpmvOperand{A->m, A->n, A->nnz, A->rp, A->ci, A->v, A->v32, A->lanes, A->ulen, A->tune};
}
// y = op x on `s` (kr_spmv.cu); fp32: FP32 values and sums
cudaError_t spmv_launch(const SpmvOperand &A, bool fp32, const double *x, double *y, int sms, cudaStream_t s);
int spmv_rows_per_block(int64_t rows, int64_t nnz);
// allocation with budget accounting
int dev_alloc(krans_ctx *ctx, void **p, size_t bytes);
void dev_free(krans_ctx *ctx, void *p, size_t bytes);
// Stream-ordered forms (cudaMallocAsync / cudaFreeAsync on `s`): neither
// waits for kernels running on other streams, unlike cudaFree, which waits
// for the whole device. The served paths use them so that releasing one
// finished launch never waits for a persistent launch still resident.
int dev_alloc_async(krans_ctx *ctx, void **p, size_t bytes, cudaStream_t s);
// Loads every kernel of the library into the context when it is created.
// With CUDA's lazy module loading (the default), the first launch of a kernel
// loads it, and loading may wait for the kernels already running: a first
// launch beside a resident persistent launch (a new precision or solver in
// the server, a standalone SpMV) would wait until that launch ends. Each
// kernel translation unit lists its kernels in a preload_* function.
void preload(const void *kernel);
void preload_capi_kernels();
void preload_spmv_kernels();
void preload_gram_kernels();
void preload_batch_cta_kernels();
void preload_batch_cluster_kernels();
void preload_cyclic_grid_kernels();
void preload_lobpcg_kernels();
void preload_lobpcg_cta_kernels();
void preload_lobpcg_cluster_kernels();
void dev_free_async(krans_ctx *ctx, void *p, size_t bytes, cudaStream_t s);
int pick_lanes(int64_t rows, int64_t nnz);
// threads per row of the solvers' SpMV from the context's tuning table
inline int tuned_lanes(const krans_ctx *ctx, int64_t rows, int64_t nnz) {
  const double mean = rows > 0 ? (double)nnz / (double)rows : 0.0;
  const double bound[5] = {3.0, 8.0, 16.0, 32.0, 64.0};
  int b = 0;
  while (b < 5 && mean > bound[b])
    b++;
  return ctx->tune.lanes[b];
}
} // namespace kr
