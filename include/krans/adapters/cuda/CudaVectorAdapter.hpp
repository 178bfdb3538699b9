#pragma once
// VectorInterface over a device FP64 vector of libkrans_cuda.so (header-only).
// Replaces StdVectorAdapter / EigenVectorAdapter
// (reference: include/krans/adapters/universal/StdVectorAdapter.hpp:23-104).
//
// Every operation runs on the GPU; dot() and norm() return their scalar to the
// host (the interface requires it). data() gives a host mirror: the non-const
// overload marks it dirty and the next device operation uploads it first, so
// code that edits entries through data() (e.g. the reference's RREF subspace
// compare) keeps working.
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "krans/VectorInterface.hpp"
#include "krans_cuda.h"

namespace krans {
namespace cuda {

inline void check(int rc, const char *what) {
  if (rc == KRANS_OK)
    return;
  const std::string msg = std::string(what) + ": " + krans_last_error();
  if (rc == KRANS_ERR_INVALID_ARGUMENT)
    throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

class CudaVectorAdapter final : public VectorInterface {
public:
  /** zero vector of size n on the context's device */
  CudaVectorAdapter(krans_ctx *ctx, std::size_t n) : ctx_(ctx) {
    check(krans_vec_create(ctx, (int64_t)n, &v_), "krans_vec_create");
    n_ = n;
  }
  /** adopt a vector handle (takes ownership) */
  CudaVectorAdapter(krans_ctx *ctx, krans_vec *owned) : ctx_(ctx), v_(owned) {
    int64_t n = 0;
    check(krans_vec_size(v_, &n), "krans_vec_size");
    n_ = (std::size_t)n;
  }
  ~CudaVectorAdapter() override { krans_vec_destroy(v_); }
  CudaVectorAdapter(const CudaVectorAdapter &) = delete;
  CudaVectorAdapter &operator=(const CudaVectorAdapter &) = delete;

  double dot(const VectorInterface &other) const override {
    const auto &o = peer(other, "dot");
    flush();
    o.flush();
    double r = 0.0;
    check(krans_vec_dot(v_, o.v_, &r), "CudaVectorAdapter::dot");
    return r;
  }
  void add_scaled(const VectorInterface &other, double alpha) override {
    const auto &o = peer(other, "add_scaled");
    flush();
    o.flush();
    check(krans_vec_axpy(v_, alpha, o.v_), "CudaVectorAdapter::add_scaled");
    stale_ = true;
  }
  void scale(double alpha) override {
    flush();
    check(krans_vec_scale(v_, alpha), "CudaVectorAdapter::scale");
    stale_ = true;
  }
  void normalize() override {
    flush();
    check(krans_vec_normalize(v_), "CudaVectorAdapter::normalize");
    stale_ = true;
  }
  double norm() const override {
    flush();
    double r = 0.0;
    check(krans_vec_nrm2(v_, &r), "CudaVectorAdapter::norm");
    return r;
  }
  std::size_t size() const override { return n_; }
  void set_zero() override {
    dirty_ = false;
    check(krans_vec_fill(v_, 0.0), "CudaVectorAdapter::set_zero");
    stale_ = true;
  }
  void copy_from(const VectorInterface &other) override {
    const auto &o = peer(other, "copy_from");
    o.flush();
    dirty_ = false;
    check(krans_vec_copy(v_, o.v_), "CudaVectorAdapter::copy_from");
    stale_ = true;
  }
  std::unique_ptr<VectorInterface> clone() const override {
    flush();
    krans_vec *c = nullptr;
    check(krans_vec_clone(v_, &c), "CudaVectorAdapter::clone");
    return std::make_unique<CudaVectorAdapter>(ctx_, c);
  }
  double *data() override {
    download();
    dirty_ = true; // the caller may write; upload before the next device op
    return host_.data();
  }
  const double *data() const override {
    download();
    return host_.data();
  }

  krans_vec *handle() const {
    flush();
    return v_;
  }
  krans_ctx *context() const { return ctx_; }
  /** mark device contents changed by a direct C-ABI call */
  void invalidate_host() { stale_ = true; }

private:
  const CudaVectorAdapter &peer(const VectorInterface &other, const char *op) const {
    const auto *o = dynamic_cast<const CudaVectorAdapter *>(&other);
    if (!o)
      throw std::invalid_argument(std::string("CudaVectorAdapter::") + op + " backend mismatch");
    if (o->n_ != n_)
      throw std::invalid_argument(std::string("CudaVectorAdapter::") + op + " size mismatch");
    return *o;
  }
  void download() const {
    if (!stale_ && host_.size() == n_)
      return;
    if (dirty_)
      return; // host mirror holds the newest values
    host_.resize(n_);
    check(krans_vec_download(v_, host_.data(), (int64_t)n_), "CudaVectorAdapter::data");
    stale_ = false;
  }
  void flush() const {
    if (!dirty_)
      return;
    check(krans_vec_upload(v_, host_.data(), (int64_t)n_), "CudaVectorAdapter::flush");
    dirty_ = false;
  }

  krans_ctx *ctx_ = nullptr;
  krans_vec *v_ = nullptr;
  std::size_t n_ = 0;
  mutable std::vector<double> host_;
  mutable bool stale_ = true;
  mutable bool dirty_ = false;
};

} // namespace cuda
} // namespace krans
