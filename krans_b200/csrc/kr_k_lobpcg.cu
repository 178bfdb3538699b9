// Kernel TU: block LOBPCG on a grid team (one solve on the whole GPU).
#include <algorithm>

#define KR_LOBPCG_GRID_KERNEL
#include "kr_internal.h"
#include "kr_lobpcg.cuh"

namespace kr {

int lobpcg_grid_blocks(krans_ctx *ctx, int threads) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)lobpcg_grid_kernel, threads, 0) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return ctx->sms * std::min(per_sm, 2);
}

cudaError_t launch_lobpcg_cta(const LobpcgDesc *d_dev, int threads, cudaStream_t s);

cudaError_t launch_lobpcg(bool grid, const LobpcgDesc &d, const LobpcgDesc *d_dev, int blocks, int threads,
                          cudaStream_t s) {
  if (grid) {
    void *args[] = {(void *)&d};
    return cudaLaunchCooperativeKernel((const void *)lobpcg_grid_kernel, dim3(blocks), dim3(threads), args, 0, s);
  }
  return launch_lobpcg_cta(d_dev, threads, s);
}

} // namespace kr
