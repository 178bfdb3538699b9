// Kernel TU: the block solver's dense products on raw device arrays
// (krans_block_gram, krans_block_gemm_tn, krans_block_combine): the same
// device code as inside the LOBPCG kernel (team_gram_sym_tiled, team_gemm_tn,
// team_gemm_nn), run by every block of a cooperative launch, so that they can
// be tested and timed on their own.
#include <algorithm>

#include "kr_gram.cuh"
#include "kr_internal.h"

namespace kr {

__global__ void __launch_bounds__(512) block_gram_kernel(int64_t n, const double *Z, const double *W, int64_t ld,
                                                         int p, double *S, double *G, double *part,
                                                         GridBarrierState *gb, double *gpart, int *status) {
  __shared__ TeamShared sh;
  TeamGrid tm{&sh, status, gb, gpart, 0, 0};
  team_gram_sym_tiled(tm, n, Z, W, ld, p, S, G, part);
}

__global__ void __launch_bounds__(512) block_gemm_tn_kernel(int64_t n, const double *A, int a, const double *B,
                                                            int b, int64_t ld, double *C, double *part,
                                                            GridBarrierState *gb, double *gpart, int *status) {
  __shared__ TeamShared sh;
  TeamGrid tm{&sh, status, gb, gpart, 0, 0};
  team_gemm_tn(tm, n, A, a, B, b, ld, C, part);
}

__global__ void __launch_bounds__(512) block_combine_kernel(int64_t n, const double *Z, int64_t ld, int zc,
                                                            const double *C, int ldc, int q, double *out,
                                                            GridBarrierState *gb, double *gpart, int *status) {
  __shared__ TeamShared sh;
  TeamGrid tm{&sh, status, gb, gpart, 0, 0};
  team_gemm_nn(tm, n, Z, ld, zc, C, ldc, 0, q, out, false);
}

static int coop_blocks(const void *k, krans_ctx *ctx, size_t smem) {
  int per_sm = 0;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 512, smem) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return ctx->sms * std::min(per_sm, 2);
}

// workspace: grid barrier, reduction partials, status, Gram partials
static int coop_scratch(krans_ctx *ctx, int blocks, size_t part_doubles, char **ws, size_t *bytes,
                        GridBarrierState **gb, double **gpart, int **status, double **part) {
  Carver c;
  c.take<GridBarrierState>(1);
  c.take<double>(2 * (size_t)blocks * KR_RED_K);
  c.take<int>(1);
  c.take<double>((int64_t)std::max<size_t>(part_doubles, 1));
  *bytes = c.off + 256;
  int rc = dev_alloc(ctx, (void **)ws, *bytes);
  if (rc != KRANS_OK)
    return rc;
  Carver d;
  d.base = *ws;
  *gb = d.take<GridBarrierState>(1);
  *gpart = d.take<double>(2 * (size_t)blocks * KR_RED_K);
  *status = d.take<int>(1);
  *part = d.take<double>((int64_t)std::max<size_t>(part_doubles, 1));
  return KRANS_OK;
}

void preload_gram_kernels() {
  preload((const void *)block_gram_kernel);
  preload((const void *)block_gemm_tn_kernel);
  preload((const void *)block_combine_kernel);
}

} // namespace kr

using namespace kr;

// device time of one cooperative launch of `k` on `s` (events around it)
static cudaError_t timed_coop(const void *k, int blocks, void **args, size_t smem, cudaStream_t s, double *device_ms) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaSuccess;
  if (device_ms) {
    e = cudaEventCreate(&e0);
    if (e == cudaSuccess)
      e = cudaEventCreate(&e1);
    if (e == cudaSuccess)
      e = cudaEventRecord(e0, s);
  }
  if (e == cudaSuccess)
    e = cudaLaunchCooperativeKernel(k, dim3(blocks), dim3(512), args, smem, s);
  if (e == cudaSuccess && device_ms)
    e = cudaEventRecord(e1, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && device_ms) {
    float ms = 0.f;
    e = cudaEventElapsedTime(&ms, e0, e1);
    *device_ms = ms;
  }
  if (e0)
    cudaEventDestroy(e0);
  if (e1)
    cudaEventDestroy(e1);
  return e;
}

extern "C" int krans_block_gram(krans_ctx *ctx, int64_t n, int64_t p, const double *Z, const double *W, int64_t ld,
                                double *S, double *G, double *device_ms) {
  KR_CHECK_ARG(ctx && Z && S, "krans_block_gram: NULL argument");
  KR_CHECK_ARG(n >= 0 && p >= 1 && p <= 4096 && ld >= n, "krans_block_gram: need n >= 0, 1 <= p <= 4096, ld >= n");
  KR_CHECK_ARG(!W == !G, "krans_block_gram: W and G go together");
  KR_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lk(ctx->mu);
  const void *k = (const void *)block_gram_kernel;
  const int blocks = coop_blocks(k, ctx, gram_tiled_smem_bytes());
  const int64_t tp = (p + KR_GT - 1) / KR_GT;
  const size_t part = (size_t)(2 * blocks + tp * (tp + 1) / 2) * 2 * KR_GT * KR_GT;
  char *ws = nullptr;
  size_t bytes = 0;
  GridBarrierState *gb;
  double *gpart, *pt;
  int *status;
  int rc = coop_scratch(ctx, blocks, part, &ws, &bytes, &gb, &gpart, &status, &pt);
  if (rc != KRANS_OK)
    return rc;
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemsetAsync(gb, 0, sizeof(GridBarrierState), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(status, 0, sizeof(int), s);
  int pi = (int)p;
  void *args[] = {(void *)&n, (void *)&Z, (void *)&W, (void *)&ld, (void *)&pi, (void *)&S, (void *)&G,
                  (void *)&pt, (void *)&gb, (void *)&gpart, (void *)&status};
  if (e == cudaSuccess)
    e = timed_coop(k, blocks, args, gram_tiled_smem_bytes(), s, device_ms);
  int h_status = 0;
  if (e == cudaSuccess)
    e = cudaMemcpy(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost);
  dev_free(ctx, ws, bytes);
  if (e != cudaSuccess)
    return cuda_fail(e, "krans_block_gram", __FILE__, __LINE__);
  if (h_status != 0) {
    set_error("krans_block_gram: device status %d (a bounded grid barrier gave up)", h_status);
    return h_status;
  }
  return KRANS_OK;
}

extern "C" int krans_block_gemm_tn(krans_ctx *ctx, int64_t n, int64_t a, const double *A, int64_t b,
                                   const double *B, int64_t ld, double *C, double *device_ms) {
  KR_CHECK_ARG(ctx && A && B && C, "krans_block_gemm_tn: NULL argument");
  KR_CHECK_ARG(n >= 0 && a >= 1 && b >= 1 && a <= 4096 && b <= 4096 && ld >= n,
               "krans_block_gemm_tn: need n >= 0, 1 <= a, b <= 4096, ld >= n");
  KR_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lk(ctx->mu);
  const void *k = (const void *)block_gemm_tn_kernel;
  const int blocks = coop_blocks(k, ctx, gram_tiled_smem_bytes());
  // partials of both forms: the panel form's (2 blocks + tiles) 64 x 64 tiles,
  // the direct form's a x b per block
  const int64_t tiles = ((a + KR_GT - 1) / KR_GT) * ((b + KR_GT - 1) / KR_GT);
  const size_t part = std::max<size_t>((size_t)(2 * blocks + tiles) * KR_GT * KR_GT, (size_t)blocks * a * b);
  char *ws = nullptr;
  size_t bytes = 0;
  GridBarrierState *gb;
  double *gpart, *pt;
  int *status;
  int rc = coop_scratch(ctx, blocks, part, &ws, &bytes, &gb, &gpart, &status, &pt);
  if (rc != KRANS_OK)
    return rc;
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemsetAsync(gb, 0, sizeof(GridBarrierState), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(status, 0, sizeof(int), s);
  int ai = (int)a, bi = (int)b;
  void *args[] = {(void *)&n, (void *)&A, (void *)&ai, (void *)&B, (void *)&bi, (void *)&ld, (void *)&C,
                  (void *)&pt, (void *)&gb, (void *)&gpart, (void *)&status};
  if (e == cudaSuccess)
    e = timed_coop(k, blocks, args, gram_tiled_smem_bytes(), s, device_ms);
  int h_status = 0;
  if (e == cudaSuccess)
    e = cudaMemcpy(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost);
  dev_free(ctx, ws, bytes);
  if (e != cudaSuccess)
    return cuda_fail(e, "krans_block_gemm_tn", __FILE__, __LINE__);
  if (h_status != 0) {
    set_error("krans_block_gemm_tn: device status %d (a bounded grid barrier gave up)", h_status);
    return h_status;
  }
  return KRANS_OK;
}

extern "C" int krans_block_combine(krans_ctx *ctx, int64_t n, int64_t zc, int64_t q, const double *Z, int64_t ld,
                                   const double *C, int64_t ldc, double *out, double *device_ms) {
  KR_CHECK_ARG(ctx && Z && C && out, "krans_block_combine: NULL argument");
  KR_CHECK_ARG(n >= 0 && zc >= 1 && q >= 1 && zc <= 4096 && q <= 4096 && ld >= n && ldc >= zc,
               "krans_block_combine: need n >= 0, 1 <= zc, q <= 4096, ld >= n, ldc >= zc");
  KR_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lk(ctx->mu);
  const void *k = (const void *)block_combine_kernel;
  const int blocks = coop_blocks(k, ctx, gemm_nn_smem_bytes());
  char *ws = nullptr;
  size_t bytes = 0;
  GridBarrierState *gb;
  double *gpart, *pt;
  int *status;
  int rc = coop_scratch(ctx, blocks, 0, &ws, &bytes, &gb, &gpart, &status, &pt);
  if (rc != KRANS_OK)
    return rc;
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemsetAsync(gb, 0, sizeof(GridBarrierState), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(status, 0, sizeof(int), s);
  int zci = (int)zc, qi = (int)q, ldci = (int)ldc;
  void *args[] = {(void *)&n, (void *)&Z, (void *)&ld, (void *)&zci, (void *)&C, (void *)&ldci, (void *)&qi,
                  (void *)&out, (void *)&gb, (void *)&gpart, (void *)&status};
  if (e == cudaSuccess)
    e = timed_coop(k, blocks, args, gemm_nn_smem_bytes(), s, device_ms);
  dev_free(ctx, ws, bytes);
  if (e != cudaSuccess)
    return cuda_fail(e, "krans_block_combine", __FILE__, __LINE__);
  return KRANS_OK;
}
