// Allocation-free dot product: krans_vec_dot_noalloc (see include/krans_cuda.h).
//
// Some callers cannot call cudaMalloc: runtimes that hand out device memory
// only from their own pre-planned pool and treat any other allocation as a
// bug, and code paths that must not synchronize the device (cudaFree and, in
// many configurations, cudaMalloc implicitly synchronize). For them this entry
// point computes x.y with the same two reduction kernels as krans_vec_dot,
// but takes its scratch (one partial sum per thread block) from a
// file-scope device array instead of a context allocation.
//
// The array is KRANS_NOALLOC_DOT_MAX_BLOCKS doubles (128 KiB) and every GPU
// that loads this library keeps it until the process exits. Its device
// address is looked up once per CUDA context (normally the device's primary
// context), on the first call made with that context current; make that
// first call before any stream capture. The address is kept by the context's
// unique ID (cuCtxGetId, never reused within a process), so a call made after
// cudaDeviceReset, or under a context the caller created with the driver API,
// looks the address up again instead of writing through an address of a
// context that no longer exists. All calls on a device share
// the array: calls whose kernels overlap on the GPU race on it, so callers
// must order them (one stream, or events). Each call overwrites every slot it
// reads, so nothing has to be zeroed between calls.
#include <cuda.h> // CUcontext (type only; the driver entry point comes through the runtime)
#include <cuda_runtime.h>

#include <mutex>

#include "kr_internal.h"

namespace kr {
__global__ void dot_partial_kernel(int64_t n, const double *x, const double *y, double *part);
__global__ void sum_partials_kernel(int nb, const double *part, double *out, int take_sqrt);
} // namespace kr

static __device__ __align__(256) double g_noalloc_dot_partials[KRANS_NOALLOC_DOT_MAX_BLOCKS];

namespace {
// scratch addresses by context: a small table, oldest entry replaced when full
constexpr int kMaxContexts = 64;
std::mutex g_mu;
struct Slot {
  unsigned long long ctx_id; // cuCtxGetId: unique for the life of the process, never reused
  double *scratch;
};
Slot g_slots[kMaxContexts] = {};
int g_next = 0;

void *driver_entry(const char *name) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return nullptr;
  return p;
}
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// ID of the context current on this thread (0 if none)
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_cur = (CtxGetCurrentFn)driver_entry("cuCtxGetCurrent");
  static CtxGetIdFn get_id = (CtxGetIdFn)driver_entry("cuCtxGetId");
  CUcontext cu = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&cu) != CUDA_SUCCESS || !cu || get_id(cu, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}
} // namespace

extern "C" int krans_vec_dot_noalloc(const double *x, const double *y, int64_t n, double *result, void *stream) {
  if (n < 0 || !result || (n > 0 && (!x || !y))) {
    kr::set_error("krans_vec_dot_noalloc: NULL pointer or negative size");
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  const int64_t blocks = (n + KRANS_NOALLOC_DOT_PER_BLOCK - 1) / KRANS_NOALLOC_DOT_PER_BLOCK;
  if (blocks > KRANS_NOALLOC_DOT_MAX_BLOCKS) {
    kr::set_error("krans_vec_dot_noalloc: n = %lld exceeds the maximum of %lld elements",
                  (long long)n, (long long)KRANS_NOALLOC_DOT_MAX_N);
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return kr::cuda_fail(e, "cudaGetDevice", __FILE__, __LINE__);
  unsigned long long cid = current_context_id();
  if (!cid) {
    // no context current yet on this thread: make the device's primary one current
    e = cudaSetDevice(dev);
    if (e != cudaSuccess)
      return kr::cuda_fail(e, "cudaSetDevice", __FILE__, __LINE__);
    cid = current_context_id();
    if (!cid) {
      kr::set_error("krans_vec_dot_noalloc: no CUDA context is current");
      return KRANS_ERR_CUDA;
    }
  }
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (const Slot &sl : g_slots)
      if (sl.ctx_id == cid && sl.scratch) {
        scratch = sl.scratch;
        break;
      }
    if (!scratch) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_dot_partials);
      if (e != cudaSuccess)
        return kr::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_dot_partials)", __FILE__, __LINE__);
      scratch = (double *)p;
      g_slots[g_next] = Slot{cid, scratch};
      g_next = (g_next + 1) % kMaxContexts;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (blocks > 0)
    kr::dot_partial_kernel<<<(unsigned)blocks, 256, 0, s>>>(n, x, y, scratch);
  kr::sum_partials_kernel<<<1, 256, 0, s>>>((int)blocks, scratch, result, 0);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return kr::cuda_fail(e, "krans_vec_dot_noalloc launch", __FILE__, __LINE__);
  return KRANS_OK;
}
