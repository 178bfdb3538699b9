#pragma once
// VectorFactory whose vectors live on the GPU (header-only). Replaces
// StdVectorFactory / EigenVectorFactory (reference:
// include/krans/adapters/universal/StdVectorFactory.hpp:16-57). With the
// default MT19937 mode its random vectors are the reference's sequence:
// std::mt19937(seed) + std::normal_distribution<double>(0,1), state carried
// across calls; seed 0 draws a random seed.
#include <memory>

#include "krans/VectorFactory.hpp"
#include "krans/adapters/cuda/CudaVectorAdapter.hpp"

namespace krans {
namespace cuda {

class CudaVectorFactory final : public VectorFactory {
public:
  CudaVectorFactory(krans_ctx *ctx, std::size_t default_size, unsigned seed = 0, int mode = KRANS_RNG_MT19937)
      : ctx_(ctx), default_size_(default_size) {
    check(krans_rng_create(ctx, seed, mode, &rng_), "krans_rng_create");
  }
  ~CudaVectorFactory() override { krans_rng_destroy(rng_); }
  CudaVectorFactory(const CudaVectorFactory &) = delete;
  CudaVectorFactory &operator=(const CudaVectorFactory &) = delete;

  std::unique_ptr<VectorInterface> create_zero() const override { return create_zero_of_size(default_size_); }
  std::unique_ptr<VectorInterface> create_random() const override { return create_random_of_size(default_size_); }
  std::unique_ptr<VectorInterface> create_zero_of_size(std::size_t n) const override {
    return std::make_unique<CudaVectorAdapter>(ctx_, n);
  }
  std::unique_ptr<VectorInterface> create_random_of_size(std::size_t n) const override {
    auto v = std::make_unique<CudaVectorAdapter>(ctx_, n);
    check(krans_rng_normal(rng_, v->handle()), "create_random_of_size");
    v->invalidate_host();
    return v;
  }
  unsigned seed() const {
    uint32_t s = 0;
    check(krans_rng_seed(rng_, &s), "krans_rng_seed");
    return s;
  }
  krans_ctx *context() const { return ctx_; }
  krans_rng *rng() const { return rng_; }

private:
  krans_ctx *ctx_;
  krans_rng *rng_ = nullptr;
  std::size_t default_size_;
};

} // namespace cuda
} // namespace krans
