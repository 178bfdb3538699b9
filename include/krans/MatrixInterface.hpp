#pragma once
// The matrix-free operator of the KraNS plug-in API. Declared exactly as the
// reference's include/krans/MatrixInterface.hpp:10-24 so that existing code
// compiles against this library unchanged.
#include <cstddef>

namespace krans {

class VectorInterface;

class MatrixInterface {
public:
  virtual ~MatrixInterface() = default;
  /** result <- A * x */
  virtual void multiply(const VectorInterface &x, VectorInterface &result) const = 0;
  /** result <- A^T * x */
  virtual void multiply_transpose(const VectorInterface &x, VectorInterface &result) const = 0;
  virtual std::size_t rows() const = 0;
  virtual std::size_t cols() const = 0;
};

} // namespace krans
