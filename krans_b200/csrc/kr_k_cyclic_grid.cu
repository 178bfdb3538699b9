// Kernel TU: cyclic Lanczos on a grid team (one solve on the whole GPU).
#include <algorithm>

#include "kr_cyclic.cuh"
#include "kr_internal.h"

namespace kr {

static const void *grid_kernel(bool mixed) {
  return mixed ? (const void *)cyclic_grid_kernel<float> : (const void *)cyclic_grid_kernel<double>;
}

int cyclic_grid_blocks(krans_ctx *ctx, bool mixed, int threads) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_kernel(mixed), threads, 0) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return ctx->sms * std::min(per_sm, 2);
}

cudaError_t launch_cyclic_grid(bool mixed, const CyclicDesc &d, int blocks, int threads, cudaStream_t s) {
  void *args[] = {(void *)&d};
  return cudaLaunchCooperativeKernel(grid_kernel(mixed), dim3(blocks), dim3(threads), args, 0, s);
}

void preload_cyclic_grid_kernels() {
  preload((const void *)cyclic_grid_kernel<float>);
  preload((const void *)cyclic_grid_kernel<double>);
}

} // namespace kr
