#pragma once
// The vector factory of the KraNS plug-in API, declared as the reference's
// include/krans/VectorFactory.hpp:9-23.
#include <cstddef>
#include <memory>

#include "VectorInterface.hpp"

namespace krans {

class VectorFactory {
public:
  virtual ~VectorFactory() = default;
  virtual std::unique_ptr<VectorInterface> create_zero() const = 0;
  virtual std::unique_ptr<VectorInterface> create_random() const = 0;
  virtual std::unique_ptr<VectorInterface> create_zero_of_size(std::size_t n) const = 0;
  virtual std::unique_ptr<VectorInterface> create_random_of_size(std::size_t n) const = 0;
};

} // namespace krans
