// Kernel TU: cyclic Lanczos with one thread block per request (persistent,
// device work queue). Also serves single small requests.
#include "kr_batch.cuh"
#include "kr_internal.h"

namespace kr {

int cyclic_batch_cta_per_sm(bool mixed) {
  const void *k = mixed ? (const void *)cyclic_batch_kernel<float> : (const void *)cyclic_batch_kernel<double>;
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 512, 0) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return per_sm;
}

cudaError_t launch_cyclic_batch_cta(bool mixed, int grid, int block, size_t dyn_smem, cudaStream_t s, const CyclicRequestDev *reqs,
                                    int count, int *queue, char *ws, size_t stride, const LaunchFeed *feed) {
  const void *k = mixed ? (const void *)cyclic_batch_kernel<float> : (const void *)cyclic_batch_kernel<double>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem);
  if (e != cudaSuccess)
    return e;
  if (mixed)
    cyclic_batch_kernel<float><<<grid, block, dyn_smem, s>>>(reqs, count, queue, ws, stride, feed);
  else
    cyclic_batch_kernel<double><<<grid, block, dyn_smem, s>>>(reqs, count, queue, ws, stride, feed);
  return cudaGetLastError();
}

void preload_batch_cta_kernels() {
  preload((const void *)cyclic_batch_kernel<float>);
  preload((const void *)cyclic_batch_kernel<double>);
}

} // namespace kr
