// Kernel TU: block LOBPCG on a thread-block cluster (served requests), and
// the max ||A u|| of a returned basis on one block.
#define KR_LOBPCG_CLUSTER_KERNEL
#include "kr_batch.cuh"
#include "kr_internal.h"
#include "kr_lobpcg.cuh"

namespace kr {

cudaError_t launch_lobpcg_cluster(const LobpcgDesc *d_dev, int csize, cudaStream_t s) {
  const void *k = (const void *)lobpcg_cluster_kernel;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lobpcg_dyn_smem_bytes());
  if (e == cudaSuccess && csize > 8)
    e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess)
    return e;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  cfg.gridDim = dim3(csize);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = lobpcg_dyn_smem_bytes();
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = csize;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, lobpcg_cluster_kernel, d_dev);
}

__global__ void __launch_bounds__(512) basis_max_residual_kernel(CsrView F, const double *basis, int64_t ldb,
                                                                 const int64_t *nf, double *out) {
  __shared__ TeamShared sh;
  __shared__ int err;
  if (threadIdx.x == 0)
    err = 0;
  __syncthreads();
  TeamCta tm{&sh, &err, 0};
  const double mr = team_max_residual(tm, F, basis, ldb, *nf);
  if (threadIdx.x == 0)
    *out = mr;
}

// *out = max_i ||F u_i|| over the *nf vectors of `basis` (stride ldb)
cudaError_t launch_basis_max_residual(const CsrView &F, const double *basis, int64_t ldb, const int64_t *nf,
                                      double *out, cudaStream_t s) {
  basis_max_residual_kernel<<<1, 512, 0, s>>>(F, basis, ldb, nf, out);
  return cudaGetLastError();
}

void preload_lobpcg_cluster_kernels() {
  preload((const void *)lobpcg_cluster_kernel);
  preload((const void *)basis_max_residual_kernel);
}

} // namespace kr
