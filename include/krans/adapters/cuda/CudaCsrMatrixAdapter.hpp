#pragma once
// MatrixInterface over a device CSR matrix with a stored transpose
// (header-only). Replaces EigenSparseMatrixAdapter, which owns A and caches
// A^T the same way (reference:
// include/krans/adapters/eigen/EigenSparseMatrixAdapter.hpp:20-57); like it,
// vectors of another backend are rejected with std::invalid_argument.
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "krans/MatrixInterface.hpp"
#include "krans/adapters/cuda/CudaVectorAdapter.hpp"

namespace krans {
namespace cuda {

class CudaCsrMatrixAdapter final : public MatrixInterface {
public:
  /** copy a host CSR matrix (0-based, row_ptr has m+1 entries); fp32 also keeps
   * FP32 values for the mixed-precision engine */
  CudaCsrMatrixAdapter(krans_ctx *ctx, std::size_t m, std::size_t n, const std::vector<int32_t> &row_ptr,
                       const std::vector<int32_t> &col_idx, const std::vector<double> &values, bool fp32 = false)
      : ctx_(ctx), m_(m), n_(n) {
    if (row_ptr.size() != m + 1)
      throw std::invalid_argument("CudaCsrMatrixAdapter: row_ptr must have m+1 entries");
    const int64_t nnz = row_ptr.empty() ? 0 : row_ptr.back();
    if ((int64_t)col_idx.size() < nnz || (int64_t)values.size() < nnz)
      throw std::invalid_argument("CudaCsrMatrixAdapter: col_idx/values shorter than nnz");
    check(krans_csr_create(ctx, (int64_t)m, (int64_t)n, nnz, row_ptr.data(), col_idx.data(), values.data(),
                           KRANS_CSR_FP64 | (fp32 ? KRANS_CSR_FP32 : 0), &A_),
          "krans_csr_create");
  }
  /** adopt a matrix created through the C ABI (e.g. krans_csr_load) */
  CudaCsrMatrixAdapter(krans_ctx *ctx, krans_mat *adopt) : ctx_(ctx), A_(adopt) {
    int64_t m = 0, n = 0, nnz = 0;
    check(krans_csr_dims(adopt, &m, &n, &nnz), "krans_csr_dims");
    m_ = (std::size_t)m;
    n_ = (std::size_t)n;
  }
  /** load a .mtx / .ija file straight into device memory */
  static std::unique_ptr<CudaCsrMatrixAdapter> load(krans_ctx *ctx, const std::string &path, bool fp32 = false) {
    krans_mat *A = nullptr;
    check(krans_csr_load(ctx, path.c_str(), KRANS_FMT_AUTO, KRANS_CSR_FP64 | (fp32 ? KRANS_CSR_FP32 : 0), &A),
          "krans_csr_load");
    return std::unique_ptr<CudaCsrMatrixAdapter>(new CudaCsrMatrixAdapter(ctx, A));
  }
  ~CudaCsrMatrixAdapter() override { krans_csr_destroy(A_); }
  CudaCsrMatrixAdapter(const CudaCsrMatrixAdapter &) = delete;
  CudaCsrMatrixAdapter &operator=(const CudaCsrMatrixAdapter &) = delete;

  std::size_t rows() const override { return m_; }
  std::size_t cols() const override { return n_; }
  void multiply(const VectorInterface &x, VectorInterface &y) const override { apply(0, x, y, "multiply"); }
  void multiply_transpose(const VectorInterface &x, VectorInterface &y) const override {
    apply(1, x, y, "multiply_transpose");
  }
  krans_mat *handle() const { return A_; }
  krans_ctx *context() const { return ctx_; }

private:
  void apply(int trans, const VectorInterface &x, VectorInterface &y, const char *what) const {
    const auto *cx = dynamic_cast<const CudaVectorAdapter *>(&x);
    auto *cy = dynamic_cast<CudaVectorAdapter *>(&y);
    if (!cx || !cy)
      throw std::invalid_argument(std::string("CudaCsrMatrixAdapter::") + what + " backend mismatch");
    const std::size_t xs = trans ? m_ : n_, ys = trans ? n_ : m_;
    if (x.size() != xs || y.size() != ys)
      throw std::invalid_argument(std::string("CudaCsrMatrixAdapter::") + what + " size mismatch");
    check(krans_spmv(A_, trans, cx->handle(), cy->handle()), what);
    cy->invalidate_host();
  }
  krans_ctx *ctx_;
  krans_mat *A_ = nullptr;
  std::size_t m_, n_;
};

} // namespace cuda
} // namespace krans
