#pragma once
// The vector of the KraNS plug-in API, declared as the reference's
// include/krans/VectorInterface.hpp:8-34.
#include <cstddef>
#include <memory>

namespace krans {

class VectorInterface {
public:
  virtual ~VectorInterface() = default;
  virtual double dot(const VectorInterface &other) const = 0;
  /** this <- this + alpha * other */
  virtual void add_scaled(const VectorInterface &other, double alpha) = 0;
  virtual void scale(double alpha) = 0;
  /** unit 2-norm if the norm is > 0 */
  virtual void normalize() = 0;
  virtual double norm() const = 0;
  virtual std::size_t size() const = 0;
  virtual void set_zero() = 0;
  virtual void copy_from(const VectorInterface &other) = 0;
  [[nodiscard]] virtual std::unique_ptr<VectorInterface> clone() const = 0;
  /** raw host data, or nullptr if not available */
  virtual double *data() = 0;
  virtual const double *data() const = 0;
};

} // namespace krans
