// Kernel TU: block LOBPCG on one thread block (small problems).
#define KR_LOBPCG_CTA_KERNEL
#include "kr_internal.h"
#include "kr_lobpcg.cuh"

namespace kr {

cudaError_t launch_lobpcg_cta(const LobpcgDesc *d_dev, int threads, cudaStream_t s) {
  static const cudaError_t attr = cudaFuncSetAttribute(
      (const void *)lobpcg_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lobpcg_dyn_smem_bytes());
  if (attr != cudaSuccess)
    return attr;
  lobpcg_cta_kernel<<<1, threads, lobpcg_dyn_smem_bytes(), s>>>(d_dev);
  return cudaGetLastError();
}

void preload_lobpcg_cta_kernels() { preload((const void *)lobpcg_cta_kernel); }

} // namespace kr
