#pragma once
// Matrix file loaders with the reference's names and rules
// (include/krans/IO/MatrixLoader.hpp, src/IO/MatrixLoader.cpp:12-56). The
// reference returns Eigen::SparseMatrix<double>; without Eigen these return a
// host CSR matrix (columns sorted per row, duplicates summed), which
// CudaCsrMatrixAdapter takes directly. Errors throw std::runtime_error (file
// cannot be opened or parsed) or std::invalid_argument (entry out of range).
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "krans_cuda.h"

namespace krans {
namespace io {

struct CsrMatrix {
  std::size_t rows = 0, cols = 0;
  std::vector<int32_t> row_ptr, col_idx;
  std::vector<double> values;
};

inline CsrMatrix read_csr(const std::string &path, int format) {
  int64_t m = 0, n = 0, nnz = 0;
  int32_t *rp = nullptr, *ci = nullptr;
  double *v = nullptr;
  const int rc = krans_csr_read_host(path.c_str(), format, &m, &n, &nnz, &rp, &ci, &v);
  if (rc == KRANS_ERR_INVALID_ARGUMENT)
    throw std::invalid_argument(krans_last_error());
  if (rc != KRANS_OK)
    throw std::runtime_error(krans_last_error());
  CsrMatrix A;
  A.rows = (std::size_t)m;
  A.cols = (std::size_t)n;
  A.row_ptr.assign(rp, rp + m + 1);
  A.col_idx.assign(ci, ci + nnz);
  A.values.assign(v, v + nnz);
  krans_host_free(rp);
  krans_host_free(ci);
  krans_host_free(v);
  return A;
}

/** Matrix Market coordinate file (load_matrix_market) */
inline CsrMatrix load_matrix_market(const std::string &path) { return read_csr(path, KRANS_FMT_MTX); }

/** IJA triplet file (load_ija_triplet_matrix); rows/cols < 0 take the
 * header's, others set the matrix size (every entry must fit) */
inline CsrMatrix load_ija_triplet_matrix(const std::string &path, int rows = -1, int cols = -1) {
  CsrMatrix A = read_csr(path, KRANS_FMT_IJA);
  const int32_t nnz = A.row_ptr.back();
  if (rows >= 0) {
    if ((std::size_t)rows < A.rows && A.row_ptr[(std::size_t)rows] != nnz)
      throw std::invalid_argument("load_ija_triplet_matrix: entries beyond the requested rows");
    A.row_ptr.resize((std::size_t)rows + 1, nnz);
    A.rows = (std::size_t)rows;
  }
  if (cols >= 0) {
    for (int32_t c : A.col_idx)
      if (c >= cols)
        throw std::invalid_argument("load_ija_triplet_matrix: entries beyond the requested cols");
    A.cols = (std::size_t)cols;
  }
  return A;
}

} // namespace io
} // namespace krans
