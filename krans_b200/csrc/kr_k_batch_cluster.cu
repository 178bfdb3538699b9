// Kernel TU: cyclic Lanczos with one thread-block cluster per request.
#include <algorithm>

#include "kr_batch.cuh"
#include "kr_internal.h"

namespace kr {

static const void *cl_kernel(bool mixed) {
  return mixed ? (const void *)cyclic_batch_cluster_kernel<float> : (const void *)cyclic_batch_cluster_kernel<double>;
}

static cudaLaunchConfig_t cl_config(int nclusters, int csize, size_t dyn_smem, cudaStream_t s,
                                    cudaLaunchAttribute *at) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * csize);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = dyn_smem;
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = csize;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

int cyclic_batch_cluster_max(bool mixed, int csize, int sms, size_t dyn_smem) {
  if (csize > 8)
    cudaFuncSetAttribute(cl_kernel(mixed), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(cl_kernel(mixed), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem);
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = cl_config(64, csize, dyn_smem, nullptr, at);
  int maxc = 0;
  if (cudaOccupancyMaxActiveClusters(&maxc, cl_kernel(mixed), &cfg) != cudaSuccess || maxc < 1) {
    cudaGetLastError();
    maxc = std::max(1, sms / (2 * csize));
  }
  return maxc;
}

cudaError_t launch_cyclic_batch_cluster(bool mixed, int nclusters, int csize, size_t dyn_smem, cudaStream_t s,
                                        const CyclicRequestDev *reqs_large, int n_large, int *queue_large,
                                        char *ws_large, size_t stride_large, const CyclicRequestDev *reqs_small,
                                        int n_small, int *queue_small, char *ws_small, size_t stride_small,
                                        const LaunchFeed *feed, int feed_large) {
  cudaLaunchAttribute at[1];
  cudaError_t e = cudaFuncSetAttribute(cl_kernel(mixed), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem);
  if (e != cudaSuccess)
    return e;
  cudaLaunchConfig_t cfg = cl_config(nclusters, csize, dyn_smem, s, at);
  if (mixed)
    return cudaLaunchKernelEx(&cfg, cyclic_batch_cluster_kernel<float>, reqs_large, n_large, queue_large, ws_large,
                              stride_large, reqs_small, n_small, queue_small, ws_small, stride_small, feed,
                              feed_large);
  return cudaLaunchKernelEx(&cfg, cyclic_batch_cluster_kernel<double>, reqs_large, n_large, queue_large, ws_large,
                            stride_large, reqs_small, n_small, queue_small, ws_small, stride_small, feed, feed_large);
}

void preload_batch_cluster_kernels() {
  preload(cl_kernel(true));
  preload(cl_kernel(false));
}

} // namespace kr
