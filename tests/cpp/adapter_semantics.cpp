// VectorInterface / MatrixInterface / VectorFactory semantics of the CUDA
// adapters, including the host mirror behind data() that the reference's
// RREF subspace compare (include/krans/Utils/SubspaceCompare.hpp) edits in
// place, and the error behaviour (std::invalid_argument on mismatches).
#include <cmath>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <vector>

#include "krans/adapters/cuda/CudaCsrMatrixAdapter.hpp"
#include "krans/adapters/cuda/CudaVectorFactory.hpp"

#define CHECK(c)                                                                                   \
  do {                                                                                             \
    if (!(c)) {                                                                                    \
      std::printf("CHECK failed: %s (line %d)\n", #c, __LINE__);                                  \
      return 1;                                                                                    \
    }                                                                                              \
  } while (0)

int main() {
  using krans::cuda::CudaVectorAdapter;
  krans_ctx *ctx = nullptr;
  krans::cuda::check(krans_ctx_create(0, 0, &ctx), "ctx");
  {
    krans::cuda::CudaVectorFactory vf(ctx, 5, 42);
    CHECK(vf.seed() == 42);
    auto a = vf.create_zero();
    CHECK(a->size() == 5 && a->norm() == 0.0);
    double *d = a->data();
    for (int i = 0; i < 5; i++)
      d[i] = i + 1.0; // host edit, uploaded before the next device op
    CHECK(std::fabs(a->norm() - std::sqrt(55.0)) < 1e-14);
    auto b = a->clone();
    b->scale(2.0);
    CHECK(std::fabs(a->dot(*b) - 110.0) < 1e-12);
    b->add_scaled(*a, -2.0);
    CHECK(b->norm() == 0.0);
    a->normalize();
    CHECK(std::fabs(a->norm() - 1.0) < 1e-15);
    b->copy_from(*a);
    CHECK(std::fabs(b->data()[4] - 5.0 / std::sqrt(55.0)) < 1e-15);
    b->set_zero();
    CHECK(b->data()[2] == 0.0);
    auto z = vf.create_zero_of_size(3);
    z->normalize(); // norm 0: unchanged
    CHECK(z->norm() == 0.0);
    bool threw = false;
    try {
      a->dot(*z);
    } catch (const std::invalid_argument &) {
      threw = true;
    }
    CHECK(threw);
    // 2x3 matrix [[1,0,1],[0,1,1]]
    krans::cuda::CudaCsrMatrixAdapter A(ctx, 2, 3, {0, 2, 4}, {0, 2, 1, 2}, {1, 1, 1, 1});
    CudaVectorAdapter x(ctx, 3), y(ctx, 2), t(ctx, 3);
    double *xd = x.data();
    xd[0] = -1;
    xd[1] = -1;
    xd[2] = 1;
    A.multiply(x, y);
    CHECK(y.norm() == 0.0);
    y.data()[0] = 1.0;
    y.data()[1] = 2.0;
    A.multiply_transpose(y, t);
    CHECK(t.data()[0] == 1.0 && t.data()[1] == 2.0 && t.data()[2] == 3.0);
    threw = false;
    try {
      A.multiply(y, t);
    } catch (const std::invalid_argument &) {
      threw = true;
    }
    CHECK(threw);
  }
  krans_ctx_destroy(ctx);
  std::printf("adapter semantics OK\n");
  return 0;
}
