// The reference's quickstart (examples/quickstart.cpp) with the CUDA
// adapters dropped in: the same operator (A x)_i = x_{i+N} - c x_i, n = 1000,
// N = 3, c = 0.5, the same factory seed 42, cyclic then LOBPCG on one factory,
// the same check against the analytic kernel. Exits non-zero on failure.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <vector>

#include "krans/Solvers/CyclicLanczosSolver.hpp"
#include "krans/Solvers/LOBPCGSolver.hpp"
#include "krans/adapters/cuda/CudaCsrMatrixAdapter.hpp"
#include "krans/adapters/cuda/CudaVectorFactory.hpp"

int main() {
  const std::size_t n = 1000, N = 3;
  const double c = 0.5;
  std::vector<int32_t> rp{0}, ci;
  std::vector<double> val;
  for (std::size_t i = 0; i + N < n; ++i) {
    ci.push_back((int32_t)i);
    val.push_back(-c);
    ci.push_back((int32_t)(i + N));
    val.push_back(1.0);
    rp.push_back((int32_t)ci.size());
  }
  krans_ctx *ctx = nullptr;
  krans::cuda::check(krans_ctx_create(0, 0, &ctx), "ctx");
  int failures = 0;
  {
    krans::cuda::CudaCsrMatrixAdapter A(ctx, n - N, n, rp, ci, val);
    krans::cuda::CudaVectorFactory vf(ctx, n, /*seed=*/42);
    auto report = [&](const char *name, const auto &U, double s) {
      double max_res = 0.0, max_dist = 0.0;
      krans::cuda::CudaVectorAdapter r(ctx, n - N);
      for (const auto &u : U) {
        A.multiply(*u, r);
        max_res = std::max(max_res, r.norm());
        std::vector<double> d(u->data(), u->data() + n);
        for (std::size_t j = 0; j < N; ++j) {
          double dot = 0.0, vv = 0.0;
          for (std::size_t i = j, k = 0; i < n; i += N, ++k) {
            dot += d[i] * std::pow(c, k);
            vv += std::pow(c, 2 * k);
          }
          for (std::size_t i = j, k = 0; i < n; i += N, ++k)
            d[i] -= dot / vv * std::pow(c, k);
        }
        double dist = 0.0;
        for (double e : d)
          dist += e * e;
        max_dist = std::max(max_dist, std::sqrt(dist));
      }
      std::printf("%-8s %-9zu %-13.1e %-20.1e %.4f s\n", name, U.size(), max_res, max_dist, s);
      if (U.size() != N || max_dist > 1e-8)
        ++failures;
    };
    auto since = [](auto t0) {
      return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    };
    std::printf("solver   vectors   max ||A u||   max dist(u, ker A)   time\n");
    {
      krans::solvers::CyclicLanczosOptions opt;
      opt.k = N;
      auto t0 = std::chrono::steady_clock::now();
      auto U = krans::solvers::find_nullspace_cyclic_lanczos(A, vf, opt);
      report("cyclic", U, since(t0));
    }
    {
      krans::solvers::LOBPCGOptions opt;
      opt.nev = N;
      auto t0 = std::chrono::steady_clock::now();
      auto U = krans::solvers::find_nullspace_lobpcg(A, vf, opt);
      report("lobpcg", U, since(t0));
    }
  }
  krans_ctx_destroy(ctx);
  return failures == 0 ? 0 : 1;
}
