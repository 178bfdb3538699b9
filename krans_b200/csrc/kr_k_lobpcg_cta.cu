// Kernel TU: block LOBPCG on one thread block (small problems).
#define KR_LOBPCG_CTA_KERNEL
#include "kr_internal.h"
#include "kr_lobpcg.cuh"

namespace kr {

cudaError_t launch_lobpcg_cta(const LobpcgDesc *d_dev, int threads, cudaStream_t s) {
  lobpcg_cta_kernel<<<1, threads, 0, s>>>(d_dev);
  return cudaGetLastError();
}

} // namespace kr
