// Kernel TU: block LOBPCG on a grid team (one solve on the whole GPU).
#include <algorithm>

#define KR_LOBPCG_GRID_KERNEL
#include "kr_internal.h"
#include "kr_lobpcg.cuh"

namespace kr {

// dynamic shared memory of the LOBPCG kernels: the tiles of the Gram and Z * Y products
static cudaError_t lobpcg_grid_smem_attr() {
  static cudaError_t e = cudaFuncSetAttribute((const void *)lobpcg_grid_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lobpcg_dyn_smem_bytes());
  return e;
}

int lobpcg_grid_blocks(krans_ctx *ctx, int threads) {
  int per_sm = 0;
  if (lobpcg_grid_smem_attr() != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)lobpcg_grid_kernel, threads,
                                                    lobpcg_dyn_smem_bytes()) != cudaSuccess ||
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
    cudaError_t e = lobpcg_grid_smem_attr();
    if (e != cudaSuccess)
      return e;
    void *args[] = {(void *)&d};
    return cudaLaunchCooperativeKernel((const void *)lobpcg_grid_kernel, dim3(blocks), dim3(threads), args,
                                       lobpcg_dyn_smem_bytes(), s);
  }
  return launch_lobpcg_cta(d_dev, threads, s);
}

void preload_lobpcg_kernels() { preload((const void *)lobpcg_grid_kernel); }

} // namespace kr
