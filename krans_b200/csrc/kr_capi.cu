// C ABI of the KraNS B200 engine: context, CSR matrices, vectors, SpMV,
// random vectors and the single-request solver launches.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "kr_device.cuh"
#include "kr_internal.h"

namespace kr {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
  set_error("CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e), what,
            file, line);
  if (e == cudaErrorMemoryAllocation)
    return KRANS_ERR_OUT_OF_MEMORY;
  return KRANS_ERR_CUDA;
}

static void release_bytes(krans_ctx *ctx, size_t bytes) {
  size_t cur = ctx->in_use.load();
  while (!ctx->in_use.compare_exchange_weak(cur, cur - std::min(cur, bytes))) {
  }
}

int dev_alloc(krans_ctx *ctx, void **p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0)
    bytes = 256;
  const size_t cur = ctx->in_use.load();
  if (ctx->budget && cur + bytes > ctx->budget) {
    set_error("HBM budget exceeded: %zu + %zu > %zu bytes", cur, bytes, ctx->budget);
    return KRANS_ERR_OUT_OF_MEMORY;
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
  ctx->in_use.fetch_add(bytes);
  return KRANS_OK;
}

void dev_free(krans_ctx *ctx, void *p, size_t bytes) {
  if (!p)
    return;
  if (bytes == 0)
    bytes = 256;
  cudaFree(p);
  release_bytes(ctx, bytes);
}

int dev_alloc_async(krans_ctx *ctx, void **p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  if (bytes == 0)
    bytes = 256;
  const size_t cur = ctx->in_use.load();
  if (ctx->budget && cur + bytes > ctx->budget) {
    set_error("HBM budget exceeded: %zu + %zu > %zu bytes", cur, bytes, ctx->budget);
    return KRANS_ERR_OUT_OF_MEMORY;
  }
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
  ctx->in_use.fetch_add(bytes);
  return KRANS_OK;
}

void dev_free_async(krans_ctx *ctx, void *p, size_t bytes, cudaStream_t s) {
  if (!p)
    return;
  if (bytes == 0)
    bytes = 256;
  cudaFreeAsync(p, s);
  release_bytes(ctx, bytes);
}

// Threads per row of the SpMV. Short rows go one per thread: the gathers of
// these operators are random sectors, and a thread walking a short row keeps
// the most of them in flight per instruction (measured on B200: the F^T of a
// shift operator, 2 entries per row, runs 1.5x faster with 1 lane than with 2;
// an incidence matrix's F^T, 6 entries per row on average, is fastest with 2).
int pick_lanes(int64_t rows, int64_t nnz) {
  const double mean = rows > 0 ? (double)nnz / (double)rows : 0.0;
  if (mean <= 3.0)
    return 1;
  if (mean <= 8.0)
    return 2;
  if (mean <= 16.0)
    return 4;
  if (mean <= 32.0)
    return 8;
  if (mean <= 64.0)
    return 16;
  return 32;
}

// two-stage deterministic reduction: partial per block, then one block sums
__global__ void __launch_bounds__(256) dot_partial_kernel(int64_t n, const double *x, const double *y,
                                                          double *part) {
  __shared__ TeamShared sh;
  int buf = 0;
  double v[1] = {0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[0] += x[i] * y[i];
  block_sum<1>(&sh, buf, v);
  if (threadIdx.x == 0)
    part[blockIdx.x] = v[0];
}
__global__ void __launch_bounds__(256) sum_partials_kernel(int nb, const double *part, double *out,
                                                           int take_sqrt) {
  __shared__ TeamShared sh;
  int buf = 0;
  double v[1] = {0.0};
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    v[0] += part[i];
  block_sum<1>(&sh, buf, v);
  if (threadIdx.x == 0)
    out[0] = take_sqrt ? sqrt(v[0]) : v[0];
}
__global__ void axpy_kernel(int64_t n, double a, const double *x, double *y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}
__global__ void scale_kernel(int64_t n, double a, double *x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void scale_by_inv_norm_kernel(int64_t n, const double *nrm, double *x) {
  const double s = nrm[0];
  if (!(s > 0.0))
    return;
  const double a = 1.0 / s;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void fill_kernel(int64_t n, double a, double *x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = a;
}
__global__ void to_f32_kernel(int64_t n, const double *x, float *y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

// ---- deterministic transpose: count, scan, scatter, per-row sort, gather ----
__global__ void col_count_kernel(int64_t nnz, const int32_t *ci, int32_t *cnt) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(cnt + ci[k], 1);
}
// exclusive scan of cnt[0..n) into out[0..n]; single block, chunked
__global__ void __launch_bounds__(1024) scan_kernel(int64_t n, const int32_t *cnt, int32_t *out) {
  __shared__ int32_t s[1024];
  __shared__ int32_t carry;
  if (threadIdx.x == 0)
    carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < n; base += 1024) {
    const int64_t i = base + threadIdx.x;
    const int32_t v = i < n ? cnt[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const int32_t t = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < n)
      out[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023)
      carry += s[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    out[n] = carry;
}
__global__ void scatter_kernel(int64_t nnz, const int32_t *ci, int32_t *cursor, int32_t *perm) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t pos = atomicAdd(cursor + ci[k], 1);
    perm[pos] = (int32_t)k;
  }
}
// sort each transposed row's source positions ascending (warp per row):
// rows up to 32 entries in registers (bitonic), longer rows by ranking.
__global__ void row_sort_kernel(int64_t rows, const int32_t *rp, int32_t *perm, int32_t *tmp) {
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = w; r < rows; r += nw) {
    const int32_t b = rp[r], e = rp[r + 1], L = e - b;
    if (L <= 1)
      continue;
    if (L <= 32) {
      int32_t v = lane < L ? perm[b + lane] : INT32_MAX;
      for (int k = 2; k <= 32; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
          const int32_t o = __shfl_xor_sync(0xffffffffu, v, j);
          const bool up = ((lane & k) == 0);
          const bool lower = ((lane & j) == 0);
          v = (lower == up) ? min(v, o) : max(v, o);
        }
      if (lane < L)
        perm[b + lane] = v;
    } else {
      for (int32_t i = lane; i < L; i += 32) {
        const int32_t key = perm[b + i];
        int32_t rank = 0;
        for (int32_t j = 0; j < L; j++)
          rank += perm[b + j] < key;
        tmp[b + rank] = key;
      }
      __syncwarp();
      for (int32_t i = lane; i < L; i += 32)
        perm[b + i] = tmp[b + i];
    }
  }
}
__global__ void row_of_kernel(int64_t m, const int32_t *rp, int32_t *rowof) {
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = w; r < m; r += nw)
    for (int32_t k = rp[r] + lane; k < rp[r + 1]; k += 32)
      rowof[k] = (int32_t)r;
}
__global__ void gather_t_kernel(int64_t nnz, const int32_t *perm, const int32_t *rowof, const double *v,
                                int32_t *ciT, double *vT) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = perm[p];
    ciT[p] = rowof[k];
    vT[p] = v[k];
  }
}

__global__ void rng_mt_kernel(RngState *st, double *out, int64_t n) { block_mt_normals(st, out, n); }
__global__ void rng_philox_kernel(RngState *st, double *out, int64_t n) {
  const uint64_t key = st->philox_key, base = st->philox_ctr;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = philox_normal(key, base + (uint64_t)i);
}
__global__ void rng_philox_advance(RngState *st, int64_t n) { st->philox_ctr += (uint64_t)n; }

void preload(const void *kernel) {
  cudaFuncAttributes a;
  if (cudaFuncGetAttributes(&a, kernel) != cudaSuccess)
    cudaGetLastError();
}

void preload_capi_kernels() {
  const void *ks[] = {(const void *)dot_partial_kernel, (const void *)sum_partials_kernel,
                      (const void *)axpy_kernel,        (const void *)scale_kernel,
                      (const void *)scale_by_inv_norm_kernel, (const void *)fill_kernel,
                      (const void *)to_f32_kernel,      (const void *)col_count_kernel,
                      (const void *)scan_kernel,        (const void *)scatter_kernel,
                      (const void *)row_sort_kernel,    (const void *)row_of_kernel,
                      (const void *)gather_t_kernel,    (const void *)rng_mt_kernel,
                      (const void *)rng_philox_kernel,  (const void *)rng_philox_advance};
  for (const void *k : ks)
    preload(k);
}

static int grid_for(krans_ctx *ctx, int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)ctx->sms * 8;
  if (b > cap)
    b = cap;
  if (b < 1)
    b = 1;
  return (int)b;
}

} // namespace kr

using namespace kr;

extern "C" {

const char *krans_last_error(void) { return kr::g_last_error.c_str(); }
const char *krans_version(void) { return "krans_b200 0.1 (sm_100a)"; }

int krans_abi_sizes(int64_t *out, int capacity) {
  const int64_t sz[9] = {(int64_t)sizeof(krans_cyclic_opts),    (int64_t)sizeof(krans_cyclic_result),
                         (int64_t)sizeof(krans_lobpcg_opts),    (int64_t)sizeof(krans_lobpcg_result),
                         (int64_t)sizeof(krans_request),        (int64_t)sizeof(krans_request_result),
                         (int64_t)sizeof(krans_server_opts),    (int64_t)sizeof(krans_spmv_tuning),
                         (int64_t)sizeof(krans_batch_tuning)};
  for (int i = 0; i < 9 && i < capacity && out; i++)
    out[i] = sz[i];
  return 9;
}

int krans_ctx_create(int device, size_t hbm_budget_bytes, krans_ctx **out) {
  KR_CHECK_ARG(out, "krans_ctx_create: out is NULL");
  *out = nullptr;
  int ndev = 0;
  KR_CUDA(cudaGetDeviceCount(&ndev));
  KR_CHECK_ARG(device >= 0 && device < ndev, "krans_ctx_create: no such device");
  KR_CUDA(cudaSetDevice(device));
  auto *c = new krans_ctx();
  c->device = device;
  c->budget = hbm_budget_bytes;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "cudaGetDeviceProperties", __FILE__, __LINE__);
  }
  c->sms = prop.multiProcessorCount;
  c->cc_major = prop.major;
  c->cc_minor = prop.minor;
  if (prop.major != 10) {
    delete c;
    set_error("krans_ctx_create: device %d is sm_%d%d; this library targets sm_100a (B200)", device,
              prop.major, prop.minor);
    return KRANS_ERR_RUNTIME;
  }
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess)
    e = cudaMallocHost(&c->h_scalar, 64 * sizeof(double));
  c->partial_blocks = c->sms * 8;
  if (e == cudaSuccess)
    e = cudaMalloc(&c->d_scalar, 64 * sizeof(double));
  if (e == cudaSuccess)
    e = cudaMalloc(&c->d_partials, (size_t)c->partial_blocks * sizeof(double));
  if (e != cudaSuccess) {
    int rc = cuda_fail(e, "context setup", __FILE__, __LINE__);
    krans_ctx_destroy(c);
    return rc;
  }
  preload_capi_kernels();
  preload_spmv_kernels();
  preload_gram_kernels();
  preload_batch_cta_kernels();
  preload_batch_cluster_kernels();
  preload_cyclic_grid_kernels();
  preload_lobpcg_kernels();
  preload_lobpcg_cta_kernels();
  preload_lobpcg_cluster_kernels();
  *out = c;
  return KRANS_OK;
}

int krans_ctx_destroy(krans_ctx *ctx) {
  if (!ctx)
    return KRANS_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream)
    cudaStreamSynchronize(ctx->stream);
  if (ctx->h_scalar)
    cudaFreeHost(ctx->h_scalar);
  if (ctx->d_scalar)
    cudaFree(ctx->d_scalar);
  if (ctx->d_partials)
    cudaFree(ctx->d_partials);
  if (ctx->stream)
    cudaStreamDestroy(ctx->stream);
  delete ctx;
  return KRANS_OK;
}

int krans_ctx_synchronize(krans_ctx *ctx) {
  KR_CHECK_ARG(ctx, "NULL context");
  KR_CUDA(cudaStreamSynchronize(ctx->stream));
  return KRANS_OK;
}

int krans_ctx_memory_in_use(const krans_ctx *ctx, size_t *bytes) {
  KR_CHECK_ARG(ctx && bytes, "NULL argument");
  *bytes = ctx->in_use.load();
  return KRANS_OK;
}

int krans_ctx_sm_count(const krans_ctx *ctx, int *sms) {
  KR_CHECK_ARG(ctx && sms, "NULL argument");
  *sms = ctx->sms;
  return KRANS_OK;
}

int krans_ctx_set_batch_tuning(krans_ctx *ctx, const krans_batch_tuning *t) {
  KR_CHECK_ARG(ctx && t, "krans_ctx_set_batch_tuning: NULL argument");
  KR_CHECK_ARG(t->cluster_min >= 0 && t->pair_max >= 0, "krans_ctx_set_batch_tuning: negative size threshold");
  KR_CHECK_ARG(t->cluster_size == 0 || (t->cluster_size >= 2 && t->cluster_size <= 16),
               "krans_ctx_set_batch_tuning: cluster_size must be 0 or 2..16");
  for (int b = 0; b < 6; b++)
    KR_CHECK_ARG(t->lanes[b] == 0 || (t->lanes[b] >= 1 && t->lanes[b] <= 32 && (t->lanes[b] & (t->lanes[b] - 1)) == 0),
                 "krans_ctx_set_batch_tuning: lanes must be 0 or a power of two up to 32");
  const krans_batch_tuning def{16384, 120000, 8, {1, 2, 4, 8, 16, 32}};
  std::lock_guard<std::mutex> lk(ctx->mu);
  krans_batch_tuning &u = ctx->tune;
  u.cluster_min = t->cluster_min ? t->cluster_min : def.cluster_min;
  u.pair_max = t->pair_max ? t->pair_max : def.pair_max;
  u.cluster_size = t->cluster_size ? t->cluster_size : def.cluster_size;
  for (int b = 0; b < 6; b++)
    u.lanes[b] = t->lanes[b] ? t->lanes[b] : def.lanes[b];
  return KRANS_OK;
}

int krans_ctx_get_batch_tuning(const krans_ctx *ctx, krans_batch_tuning *t) {
  KR_CHECK_ARG(ctx && t, "krans_ctx_get_batch_tuning: NULL argument");
  *t = ctx->tune;
  return KRANS_OK;
}

int krans_ctx_stream(const krans_ctx *ctx, void **stream) {
  KR_CHECK_ARG(ctx && stream, "NULL argument");
  *stream = (void *)ctx->stream;
  return KRANS_OK;
}

// ---------------------------------------------------------------------------
// CSR
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Self-test of the bounded grid barrier: block 0 waits at a barrier that
// block 1 never reaches (it returns at once), so the wait must run out after
// the state's timeout and leave KRANS_ERR_TIMEOUT in the status word.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(64) barrier_timeout_probe_kernel(GridBarrierState *gb, int *status,
                                                                   double *gpart) {
  __shared__ TeamShared sh;
  if (blockIdx.x != 0)
    return;
  TeamGrid tm{&sh, status, gb, gpart, 0, 0};
  tm.sync();
}

extern "C" int krans_selftest_barrier_timeout(krans_ctx *ctx, double timeout_ms, int *status_out,
                                              double *elapsed_ms) {
  KR_CHECK_ARG(ctx && status_out, "krans_selftest_barrier_timeout: NULL argument");
  KR_CHECK_ARG(timeout_ms > 0.0 && timeout_ms <= 10000.0,
               "krans_selftest_barrier_timeout: timeout_ms must be in (0, 10000]");
  KR_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lk(ctx->mu);
  struct Probe {
    GridBarrierState gb;
    int status;
    int pad;
    double gpart[2 * 2 * KR_RED_K];
  };
  Probe *d = nullptr;
  int rc = dev_alloc(ctx, (void **)&d, sizeof(Probe));
  if (rc != KRANS_OK)
    return rc;
  Probe h;
  memset(&h, 0, sizeof h);
  h.gb.timeout_ns = (uint64_t)(timeout_ms * 1e6);
  cudaStream_t s = ctx->stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMemcpyAsync(d, &h, sizeof h, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaEventCreate(&e0);
  if (e == cudaSuccess)
    e = cudaEventCreate(&e1);
  if (e == cudaSuccess)
    e = cudaEventRecord(e0, s);
  if (e == cudaSuccess) {
    GridBarrierState *gb = &d->gb;
    int *st = &d->status;
    double *gp = d->gpart;
    void *args[] = {(void *)&gb, (void *)&st, (void *)&gp};
    e = cudaLaunchCooperativeKernel((const void *)barrier_timeout_probe_kernel, dim3(2), dim3(64), args, 0, s);
  }
  if (e == cudaSuccess)
    e = cudaEventRecord(e1, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess)
    e = cudaEventElapsedTime(&ms, e0, e1);
  if (e0)
    cudaEventDestroy(e0);
  if (e1)
    cudaEventDestroy(e1);
  dev_free(ctx, d, sizeof(Probe));
  if (e != cudaSuccess)
    return cuda_fail(e, "krans_selftest_barrier_timeout", __FILE__, __LINE__);
  *status_out = h.status;
  if (elapsed_ms)
    *elapsed_ms = ms;
  return KRANS_OK;
}

int krans_csr_create(krans_ctx *ctx, int64_t m, int64_t n, int64_t nnz, const int32_t *row_ptr,
                     const int32_t *col_idx, const double *values, int flags, krans_mat **out) {
  KR_CHECK_ARG(ctx && out, "krans_csr_create: NULL argument");
  *out = nullptr;
  KR_CHECK_ARG(m >= 0 && n >= 0 && nnz >= 0, "krans_csr_create: negative size");
  KR_CHECK_ARG(m < INT32_MAX && n < INT32_MAX && nnz < INT32_MAX,
               "krans_csr_create: sizes must fit 32-bit indices");
  KR_CHECK_ARG(row_ptr && (nnz == 0 || (col_idx && values)), "krans_csr_create: NULL array");
  KR_CHECK_ARG(row_ptr[0] == 0 && row_ptr[m] == nnz, "krans_csr_create: row_ptr[0] != 0 or row_ptr[m] != nnz");
  // one pass over the rows (monotone, uniform length) and one over the
  // columns (range, per-column counts for the transpose's uniform length)
  const int64_t L = m > 0 ? (int64_t)(row_ptr[1] - row_ptr[0]) : 0;
  bool uni = m > 0 && L > 0 && L <= 8;
  for (int64_t i = 0; i < m; i++) {
    const int32_t len = row_ptr[i + 1] - row_ptr[i];
    KR_CHECK_ARG(len >= 0, "krans_csr_create: row_ptr not monotone");
    uni = uni && len == L;
  }
  std::vector<int32_t> cc((size_t)n, 0);
  for (int64_t k = 0; k < nnz; k++) {
    const int32_t c = col_idx[k];
    KR_CHECK_ARG(c >= 0 && c < n, "krans_csr_create: column index out of range");
    cc[(size_t)c]++;
  }
  const int32_t LT = n > 0 ? cc[0] : 0;
  bool uniT = n > 0 && LT > 0 && LT <= 8;
  for (int64_t j = 0; uniT && j < n; j++)
    uniT = cc[(size_t)j] == LT;
  if (!(flags & (KRANS_CSR_FP64 | KRANS_CSR_FP32)))
    flags |= KRANS_CSR_FP64;
  flags |= KRANS_CSR_FP64; // FP64 values are kept for every path (polish, residuals)
  KR_CUDA(cudaSetDevice(ctx->device));
  const bool f32 = (flags & KRANS_CSR_FP32) != 0;
  const size_t sz_rp = (size_t)(m + 1) * 4, sz_rpT = (size_t)(n + 1) * 4, sz_ci = (size_t)std::max<int64_t>(nnz, 1) * 4;
  const size_t sz_v = (size_t)std::max<int64_t>(nnz, 1) * 8, sz_v32 = (size_t)std::max<int64_t>(nnz, 1) * 4;
  // the stored arrays share one allocation (carved at 256-byte offsets)
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t total = up(sz_rp) + 2 * up(sz_ci) + 2 * up(sz_v) + up(sz_rpT) + (f32 ? 2 * up(sz_v32) : 0);
  char *base = nullptr;
  int rc = dev_alloc(ctx, (void **)&base, total);
  if (rc != KRANS_OK)
    return rc;
  auto *A = new krans_mat();
  A->ctx = ctx;
  A->m = m;
  A->n = n;
  A->nnz = nnz;
  A->base = base;
  A->bytes = total;
  size_t off = 0;
  auto take = [&](size_t b) {
    char *p = base + off;
    off += up(b);
    return p;
  };
  A->rp = (int32_t *)take(sz_rp);
  A->ci = (int32_t *)take(sz_ci);
  A->v = (double *)take(sz_v);
  A->rpT = (int32_t *)take(sz_rpT);
  A->ciT = (int32_t *)take(sz_ci);
  A->vT = (double *)take(sz_v);
  if (f32) {
    A->v32 = (float *)take(sz_v32);
    A->vT32 = (float *)take(sz_v32);
  }
  // scratch of the device transpose: stream-ordered, so releasing it does not
  // wait for the device, and the next matrix's host work overlaps this
  // matrix's transpose kernels
  cudaStream_t s = ctx->stream;
  int32_t *scratch = nullptr;
  const size_t sz_scr = up(sz_rpT) + 3 * up(sz_ci);
  cudaError_t e = cudaMallocAsync((void **)&scratch, sz_scr, s);
  int32_t *cnt = scratch, *perm = (int32_t *)((char *)scratch + up(sz_rpT));
  int32_t *tmp = (int32_t *)((char *)perm + up(sz_ci)), *rowof = (int32_t *)((char *)tmp + up(sz_ci));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(A->rp, row_ptr, sz_rp, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(A->ci, col_idx, (size_t)nnz * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(A->v, values, (size_t)nnz * 8, cudaMemcpyHostToDevice, s);
  // the host arrays may be reused once this returns: wait for the copies only
  cudaEvent_t copied = nullptr;
  if (e == cudaSuccess)
    e = cudaEventCreateWithFlags(&copied, cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaEventRecord(copied, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(cnt, 0, sz_rpT, s);
  if (e == cudaSuccess && nnz) {
    const int g = grid_for(ctx, nnz);
    col_count_kernel<<<g, 256, 0, s>>>(nnz, A->ci, cnt);
    scan_kernel<<<1, 1024, 0, s>>>(n, cnt, A->rpT);
    e = cudaMemcpyAsync(cnt, A->rpT, (size_t)n * 4, cudaMemcpyDeviceToDevice, s);
    scatter_kernel<<<g, 256, 0, s>>>(nnz, A->ci, cnt, perm);
    row_sort_kernel<<<grid_for(ctx, n * 32), 256, 0, s>>>(n, A->rpT, perm, tmp);
    row_of_kernel<<<grid_for(ctx, m * 32), 256, 0, s>>>(m, A->rp, rowof);
    gather_t_kernel<<<g, 256, 0, s>>>(nnz, perm, rowof, A->v, A->ciT, A->vT);
    if (f32) {
      to_f32_kernel<<<g, 256, 0, s>>>(nnz, A->v, A->v32);
      to_f32_kernel<<<g, 256, 0, s>>>(nnz, A->vT, A->vT32);
    }
  } else if (e == cudaSuccess) {
    e = cudaMemsetAsync(A->rpT, 0, sz_rpT, s);
  }
  if (e == cudaSuccess)
    e = cudaGetLastError();
  if (scratch) {
    const cudaError_t ef = cudaFreeAsync(scratch, s);
    if (e == cudaSuccess)
      e = ef;
  }
  if (copied) {
    const cudaError_t es = cudaEventSynchronize(copied);
    if (e == cudaSuccess)
      e = es;
    cudaEventDestroy(copied);
  }
  if (e != cudaSuccess) {
    cudaStreamSynchronize(s);
    rc = cuda_fail(e, "krans_csr_create", __FILE__, __LINE__);
    krans_csr_destroy(A);
    return rc;
  }
  A->lanes = pick_lanes(m, nnz);
  A->lanesT = pick_lanes(n, nnz);
  // uniform row lengths (e.g. incidence and difference operators) let the
  // SpMV skip the row pointers and use vector loads
  A->ulen = uni ? (int32_t)L : 0;
  A->ulenT = uniT ? LT : 0;
  *out = A;
  return KRANS_OK;
}

int krans_csr_destroy(krans_mat *A) {
  if (!A)
    return KRANS_OK;
  dev_free(A->ctx, A->base, A->bytes);
  delete A;
  return KRANS_OK;
}

int krans_csr_dims(const krans_mat *A, int64_t *m, int64_t *n, int64_t *nnz) {
  KR_CHECK_ARG(A, "NULL matrix");
  if (m)
    *m = A->m;
  if (n)
    *n = A->n;
  if (nnz)
    *nnz = A->nnz;
  return KRANS_OK;
}

int krans_csr_device_arrays(const krans_mat *A, int trans, const int32_t **row_ptr,
                            const int32_t **col_idx, const double **values, const float **values32) {
  KR_CHECK_ARG(A, "NULL matrix");
  if (row_ptr)
    *row_ptr = trans ? A->rpT : A->rp;
  if (col_idx)
    *col_idx = trans ? A->ciT : A->ci;
  if (values)
    *values = trans ? A->vT : A->v;
  if (values32)
    *values32 = trans ? A->vT32 : A->v32;
  return KRANS_OK;
}

// ---------------------------------------------------------------------------
// vectors
// ---------------------------------------------------------------------------
int krans_vec_create(krans_ctx *ctx, int64_t n, krans_vec **out) {
  KR_CHECK_ARG(ctx && out, "krans_vec_create: NULL argument");
  KR_CHECK_ARG(n >= 0, "krans_vec_create: negative size");
  *out = nullptr;
  auto *v = new krans_vec();
  v->ctx = ctx;
  v->n = n;
  int rc = dev_alloc(ctx, (void **)&v->d, (size_t)std::max<int64_t>(n, 1) * 8);
  if (rc != KRANS_OK) {
    delete v;
    return rc;
  }
  cudaError_t e = cudaMemsetAsync(v->d, 0, (size_t)std::max<int64_t>(n, 1) * 8, ctx->stream);
  if (e != cudaSuccess) {
    dev_free(ctx, v->d, (size_t)std::max<int64_t>(n, 1) * 8);
    delete v;
    return cuda_fail(e, "cudaMemsetAsync", __FILE__, __LINE__);
  }
  *out = v;
  return KRANS_OK;
}

int krans_vec_destroy(krans_vec *v) {
  if (!v)
    return KRANS_OK;
  dev_free(v->ctx, v->d, (size_t)std::max<int64_t>(v->n, 1) * 8);
  delete v;
  return KRANS_OK;
}

int krans_vec_size(const krans_vec *v, int64_t *n) {
  KR_CHECK_ARG(v && n, "NULL argument");
  *n = v->n;
  return KRANS_OK;
}

int krans_vec_device_ptr(krans_vec *v, double **dptr) {
  KR_CHECK_ARG(v && dptr, "NULL argument");
  *dptr = v->d;
  return KRANS_OK;
}

int krans_vec_upload(krans_vec *v, const double *host, int64_t n) {
  KR_CHECK_ARG(v && (host || n == 0), "NULL argument");
  KR_CHECK_ARG(n == v->n, "krans_vec_upload: size mismatch");
  if (n)
    KR_CUDA(cudaMemcpyAsync(v->d, host, (size_t)n * 8, cudaMemcpyHostToDevice, v->ctx->stream));
  KR_CUDA(cudaStreamSynchronize(v->ctx->stream));
  return KRANS_OK;
}

int krans_vec_download(const krans_vec *v, double *host, int64_t n) {
  KR_CHECK_ARG(v && (host || n == 0), "NULL argument");
  KR_CHECK_ARG(n == v->n, "krans_vec_download: size mismatch");
  if (n)
    KR_CUDA(cudaMemcpyAsync(host, v->d, (size_t)n * 8, cudaMemcpyDeviceToHost, v->ctx->stream));
  KR_CUDA(cudaStreamSynchronize(v->ctx->stream));
  return KRANS_OK;
}

static int reduce_to_host(krans_ctx *c, int64_t n, const double *x, const double *y, int take_sqrt,
                          double *out) {
  const int g = std::min<int>(grid_for(c, n), c->partial_blocks);
  dot_partial_kernel<<<g, 256, 0, c->stream>>>(n, x, y, c->d_partials);
  sum_partials_kernel<<<1, 256, 0, c->stream>>>(g, c->d_partials, c->d_scalar, take_sqrt);
  KR_CUDA(cudaGetLastError());
  KR_CUDA(cudaMemcpyAsync(c->h_scalar, c->d_scalar, 8, cudaMemcpyDeviceToHost, c->stream));
  KR_CUDA(cudaStreamSynchronize(c->stream));
  *out = c->h_scalar[0];
  return KRANS_OK;
}

int krans_vec_dot(const krans_vec *x, const krans_vec *y, double *out) {
  KR_CHECK_ARG(x && y && out, "NULL argument");
  KR_CHECK_ARG(x->n == y->n, "krans_vec_dot: size mismatch");
  return reduce_to_host(x->ctx, x->n, x->d, y->d, 0, out);
}

int krans_vec_nrm2(const krans_vec *v, double *out) {
  KR_CHECK_ARG(v && out, "NULL argument");
  return reduce_to_host(v->ctx, v->n, v->d, v->d, 1, out);
}

int krans_vec_axpy(krans_vec *y, double alpha, const krans_vec *x) {
  KR_CHECK_ARG(x && y, "NULL argument");
  KR_CHECK_ARG(x->n == y->n, "krans_vec_axpy: size mismatch");
  axpy_kernel<<<grid_for(y->ctx, y->n), 256, 0, y->ctx->stream>>>(y->n, alpha, x->d, y->d);
  KR_CUDA(cudaGetLastError());
  return KRANS_OK;
}

int krans_vec_scale(krans_vec *v, double alpha) {
  KR_CHECK_ARG(v, "NULL argument");
  scale_kernel<<<grid_for(v->ctx, v->n), 256, 0, v->ctx->stream>>>(v->n, alpha, v->d);
  KR_CUDA(cudaGetLastError());
  return KRANS_OK;
}

int krans_vec_normalize(krans_vec *v) {
  KR_CHECK_ARG(v, "NULL argument");
  krans_ctx *c = v->ctx;
  const int g = std::min<int>(grid_for(c, v->n), c->partial_blocks);
  dot_partial_kernel<<<g, 256, 0, c->stream>>>(v->n, v->d, v->d, c->d_partials);
  sum_partials_kernel<<<1, 256, 0, c->stream>>>(g, c->d_partials, c->d_scalar, 1);
  scale_by_inv_norm_kernel<<<grid_for(c, v->n), 256, 0, c->stream>>>(v->n, c->d_scalar, v->d);
  KR_CUDA(cudaGetLastError());
  return KRANS_OK;
}

int krans_vec_fill(krans_vec *v, double value) {
  KR_CHECK_ARG(v, "NULL argument");
  fill_kernel<<<grid_for(v->ctx, v->n), 256, 0, v->ctx->stream>>>(v->n, value, v->d);
  KR_CUDA(cudaGetLastError());
  return KRANS_OK;
}

int krans_vec_copy(krans_vec *dst, const krans_vec *src) {
  KR_CHECK_ARG(dst && src, "NULL argument");
  KR_CHECK_ARG(dst->n == src->n, "krans_vec_copy: size mismatch");
  if (dst->n)
    KR_CUDA(cudaMemcpyAsync(dst->d, src->d, (size_t)dst->n * 8, cudaMemcpyDeviceToDevice, dst->ctx->stream));
  return KRANS_OK;
}

int krans_vec_clone(const krans_vec *src, krans_vec **out) {
  KR_CHECK_ARG(src && out, "NULL argument");
  int rc = krans_vec_create(src->ctx, src->n, out);
  if (rc != KRANS_OK)
    return rc;
  return krans_vec_copy(*out, src);
}

int krans_spmv_ex(const krans_mat *A, int trans, int precision, const krans_vec *x, krans_vec *y) {
  KR_CHECK_ARG(A && x && y, "krans_spmv: NULL argument");
  const int64_t rows = trans ? A->n : A->m, cols = trans ? A->m : A->n;
  KR_CHECK_ARG(x->n == cols && y->n == rows, "krans_spmv: size mismatch");
  KR_CHECK_ARG(precision == KRANS_PREC_FP64 || precision == KRANS_PREC_MIXED, "krans_spmv: unknown precision");
  KR_CHECK_ARG(precision != KRANS_PREC_MIXED || A->v32,
               "krans_spmv: matrix has no FP32 values (create with KRANS_CSR_FP32)");
  krans_ctx *c = A->ctx;
  KR_CUDA(spmv_launch(spmv_operand(A, trans), precision == KRANS_PREC_MIXED, x->d, y->d, c->sms, c->stream));
  return KRANS_OK;
}

int krans_csr_set_spmv_tuning(krans_mat *A, int trans, const krans_spmv_tuning *t) {
  KR_CHECK_ARG(A && t, "krans_csr_set_spmv_tuning: NULL argument");
  KR_CHECK_ARG(t->kernel >= KRANS_SPMV_AUTO && t->kernel <= KRANS_SPMV_LANES,
               "krans_csr_set_spmv_tuning: unknown kernel");
  KR_CHECK_ARG(t->rows_per_block >= 0 && t->rows_per_block <= 2048,
               "krans_csr_set_spmv_tuning: rows_per_block outside 0..2048");
  KR_CHECK_ARG(t->x_evict_last == 0 || t->x_evict_last == 1, "krans_csr_set_spmv_tuning: x_evict_last must be 0 or 1");
  const int32_t ulen = trans ? A->ulenT : A->ulen;
  KR_CHECK_ARG(t->kernel != KRANS_SPMV_UNIFORM || ulen == 1 || ulen == 2 || ulen == 4,
               "krans_csr_set_spmv_tuning: UNIFORM needs every row to hold exactly 1, 2 or 4 entries");
  (trans ? A->tuneT : A->tune) = *t;
  return KRANS_OK;
}

int krans_csr_get_spmv_tuning(const krans_mat *A, int trans, krans_spmv_tuning *t) {
  KR_CHECK_ARG(A && t, "krans_csr_get_spmv_tuning: NULL argument");
  *t = trans ? A->tuneT : A->tune;
  return KRANS_OK;
}

int krans_spmv(const krans_mat *A, int trans, const krans_vec *x, krans_vec *y) {
  return krans_spmv_ex(A, trans, KRANS_PREC_FP64, x, y);
}

// ---------------------------------------------------------------------------
// RNG
// ---------------------------------------------------------------------------
static void mt_seed_host(RngState &s, uint32_t seed) {
  s.mt[0] = seed;
  for (int i = 1; i < 624; i++)
    s.mt[i] = 1812433253u * (s.mt[i - 1] ^ (s.mt[i - 1] >> 30)) + (uint32_t)i;
  s.idx = 624;
  s.has_saved = 0;
  s.saved = 0.0;
}

int krans_rng_create(krans_ctx *ctx, uint32_t seed, int mode, krans_rng **out) {
  KR_CHECK_ARG(ctx && out, "krans_rng_create: NULL argument");
  KR_CHECK_ARG(mode == KRANS_RNG_MT19937 || mode == KRANS_RNG_PHILOX, "krans_rng_create: bad mode");
  *out = nullptr;
  if (seed == 0)
    seed = std::random_device{}();
  RngState h;
  memset(&h, 0, sizeof h);
  mt_seed_host(h, seed);
  h.philox_key = ((uint64_t)seed << 32) ^ 0x9E3779B97F4A7C15ull;
  h.philox_ctr = 0;
  h.mode = mode;
  auto *r = new krans_rng();
  r->ctx = ctx;
  r->seed = seed;
  r->mode = mode;
  int rc = dev_alloc(ctx, (void **)&r->d, sizeof(RngState));
  if (rc != KRANS_OK) {
    delete r;
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(r->d, &h, sizeof h, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    krans_rng_destroy(r);
    return cuda_fail(e, "rng upload", __FILE__, __LINE__);
  }
  *out = r;
  return KRANS_OK;
}

int krans_rng_destroy(krans_rng *r) {
  if (!r)
    return KRANS_OK;
  dev_free(r->ctx, r->d, sizeof(RngState));
  delete r;
  return KRANS_OK;
}

int krans_rng_seed(const krans_rng *r, uint32_t *seed) {
  KR_CHECK_ARG(r && seed, "NULL argument");
  *seed = r->seed;
  return KRANS_OK;
}

int krans_rng_normal(krans_rng *r, krans_vec *out) {
  KR_CHECK_ARG(r && out, "krans_rng_normal: NULL argument");
  krans_ctx *c = r->ctx;
  if (r->mode == KRANS_RNG_PHILOX) {
    rng_philox_kernel<<<grid_for(c, out->n), 256, 0, c->stream>>>(r->d, out->d, out->n);
    rng_philox_advance<<<1, 1, 0, c->stream>>>(r->d, out->n);
  } else {
    rng_mt_kernel<<<1, 256, 0, c->stream>>>(r->d, out->d, out->n);
  }
  KR_CUDA(cudaGetLastError());
  return KRANS_OK;
}

int krans_cyclic_opts_init(krans_cyclic_opts *o) {
  KR_CHECK_ARG(o, "NULL argument");
  memset(o, 0, sizeof *o);
  o->k = 1;
  o->ncv = 48;
  o->max_restarts = 80;
  o->tol_abs = 1e-12;
  o->tol_rel = 1e-10;
  o->reorth = 2;
  o->use_harmonic = 1;
  o->target_tau = 0.0;
  o->nullity_known = -1;
  o->rank_known = -1;
  o->cg_maxit = 80;
  o->cg_rel_tol = 1e-10;
  o->cg_breakdown_tol = 1e-30;
  o->projector_passes = 1;
  o->grad_max_iters = 3000;
  o->frob_samples = 4;
  o->prescreen_factor = 0.8;
  o->stagnation_restarts = 30;
  o->return_left_space = 0;
  o->verbose = 0;
  o->precision = KRANS_PREC_FP64;
  o->team = KRANS_TEAM_AUTO;
  o->precond_aat = KRANS_PRECOND_NONE;
  o->precond_steps = 8;
  o->polish_block = 0;
  o->mixed_fallback = 1;
  return KRANS_OK;
}

int krans_lobpcg_opts_init(krans_lobpcg_opts *o) {
  KR_CHECK_ARG(o, "NULL argument");
  memset(o, 0, sizeof *o);
  o->nev = 1;
  o->block_size = 0;
  o->max_iters = 1000;
  o->tol_abs = 1e-12;
  o->tol_rel = 1e-10;
  o->soft_locking = 1;
  o->restart = 0.9;
  o->gs_tol = 1e-14;
  o->gs_reorth = 1;
  o->frob_samples = 4;
  o->max_tiny_dim = 0;
  o->nullity_known = -1;
  o->rank_known = -1;
  o->progress_every = 100;
  o->precision = KRANS_PREC_FP64;
  o->team = KRANS_TEAM_AUTO;
  o->precond_normal = KRANS_PRECOND_NONE;
  o->precond_steps = 6;
  return KRANS_OK;
}

} // extern "C"
