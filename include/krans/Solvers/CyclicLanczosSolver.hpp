#pragma once
// Cyclic Lanczos (Golub-Kahan) right-null-space solver: options, result and
// entry points with the names, fields and defaults of the reference's
// include/krans/Solvers/CyclicLanczosSolver.hpp:77-178. The entry points run
// the B200 device engine (libkrans_cuda.so) and need a
// cuda::CudaCsrMatrixAdapter and a cuda::CudaVectorFactory; any other
// backend is rejected with std::invalid_argument (there is no CPU path).
#include <algorithm>
#include <cstddef>
#include <functional>
#include <memory>
#include <stdexcept>
#include <vector>

#include "krans/MatrixInterface.hpp"
#include "krans/VectorFactory.hpp"
#include "krans/VectorInterface.hpp"
#include "krans/adapters/cuda/CudaCsrMatrixAdapter.hpp"
#include "krans/adapters/cuda/CudaVectorFactory.hpp"

namespace krans::solvers {

using AAtPreconditioner = std::function<void(const VectorInterface &r_m, VectorInterface &y_m)>;

enum class ReorthMode { None = 0, Single = 1, Double = 2 };

struct CyclicLanczosOptions {
  std::size_t k = 1;
  std::size_t ncv = 48;
  std::size_t max_restarts = 80;
  double tol_abs = 1e-12;
  double tol_rel = 1e-10;
  ReorthMode reorth = ReorthMode::Double;
  bool use_harmonic = true;
  double target_tau = 0.0;
  int nullity_known = -1;
  int rank_known = -1;
  std::vector<std::unique_ptr<VectorInterface>> initial_right_space;
  AAtPreconditioner precond_AAt = nullptr;
  std::size_t cg_maxit = 80;
  double cg_rel_tol = 1e-10;
  double cg_breakdown_tol = 1e-30;
  int projector_passes = 1;
  int grad_max_iters = 3000;
  int frob_samples = 4;
  double prescreen_factor = 0.8;
  std::size_t stagnation_restarts = 30;
  bool return_left_space = false;
  bool verbose = false;
  // B200 engine knobs (no reference counterpart)
  int precision = KRANS_PREC_FP64; // KRANS_PREC_MIXED: FP32 SpMV/Lanczos, FP64 reorth/SVD/polish
  int team = KRANS_TEAM_AUTO;
  int polish_block = 0; // 1: project up to 8 candidates per restart with one block CG
  int precond_device = KRANS_PRECOND_NONE; // device form of precond_AAt (KRANS_PRECOND_JACOBI / _SD)
  int precond_steps = 8;
  bool mixed_fallback = true; // MIXED: continue in FP64 when the FP64 polish cannot finish FP32 Ritz vectors
};

struct CyclicLanczosResult {
  std::vector<std::unique_ptr<VectorInterface>> right_null;
  std::vector<std::unique_ptr<VectorInterface>> left_null;
  std::size_t restarts = 0;
  std::size_t krylov_steps_total = 0;
  double frob_norm_est = 0.0;
  bool converged_to_target = false;
  std::size_t cg_solves = 0;
  std::size_t cg_maxit_hits = 0;
};

inline CyclicLanczosResult find_nullspace_cyclic_lanczos_ex(const MatrixInterface &A, const VectorFactory &vf,
                                                            const CyclicLanczosOptions &opt) {
  const auto *cA = dynamic_cast<const cuda::CudaCsrMatrixAdapter *>(&A);
  const auto *cf = dynamic_cast<const cuda::CudaVectorFactory *>(&vf);
  if (!cA || !cf)
    throw std::invalid_argument(
        "find_nullspace_cyclic_lanczos: the B200 engine needs a CudaCsrMatrixAdapter and a CudaVectorFactory");
  if (opt.precond_AAt)
    throw std::invalid_argument("find_nullspace_cyclic_lanczos: host precond_AAt callbacks cannot run inside "
                                "the device engine; use precond_device (KRANS_PRECOND_JACOBI or KRANS_PRECOND_SD)");
  krans_cyclic_opts o;
  krans_cyclic_opts_init(&o);
  o.k = (int64_t)opt.k;
  o.ncv = (int64_t)opt.ncv;
  o.max_restarts = (int64_t)opt.max_restarts;
  o.tol_abs = opt.tol_abs;
  o.tol_rel = opt.tol_rel;
  o.reorth = (int32_t)opt.reorth;
  o.use_harmonic = opt.use_harmonic;
  o.target_tau = opt.target_tau;
  o.nullity_known = opt.nullity_known;
  o.rank_known = opt.rank_known;
  o.cg_maxit = (int64_t)opt.cg_maxit;
  o.cg_rel_tol = opt.cg_rel_tol;
  o.cg_breakdown_tol = opt.cg_breakdown_tol;
  o.projector_passes = opt.projector_passes;
  o.grad_max_iters = opt.grad_max_iters;
  o.frob_samples = opt.frob_samples;
  o.prescreen_factor = opt.prescreen_factor;
  o.stagnation_restarts = (int64_t)opt.stagnation_restarts;
  o.return_left_space = opt.return_left_space;
  o.verbose = opt.verbose;
  o.precision = opt.precision;
  o.team = opt.team;
  o.polish_block = opt.polish_block;
  o.precond_aat = opt.precond_device;
  o.precond_steps = opt.precond_steps;
  o.mixed_fallback = opt.mixed_fallback ? 1 : 0;
  const krans_vec *y0 = nullptr;
  if (!opt.initial_right_space.empty() && opt.initial_right_space.front()) {
    const auto *c = dynamic_cast<const cuda::CudaVectorAdapter *>(opt.initial_right_space.front().get());
    if (!c)
      throw std::invalid_argument("find_nullspace_cyclic_lanczos: initial_right_space backend mismatch");
    y0 = c->handle();
  }
  const std::size_t k_target = opt.nullity_known >= 0 ? (std::size_t)opt.nullity_known : opt.k;
  std::vector<krans_vec *> right(std::max<std::size_t>({k_target, opt.k, 1}), nullptr);
  std::vector<krans_vec *> left(std::max<std::size_t>(opt.k, 1), nullptr);
  krans_cyclic_result r;
  krans_ctx *ctx = cA->context();
  cuda::check(krans_solve_cyclic(ctx, cA->handle(), cf->rng(), &o, y0, right.data(), left.data(), &r),
              "find_nullspace_cyclic_lanczos");
  CyclicLanczosResult R;
  for (int64_t i = 0; i < r.n_right; i++)
    R.right_null.push_back(std::make_unique<cuda::CudaVectorAdapter>(ctx, right[(std::size_t)i]));
  for (int64_t i = 0; i < r.n_left; i++)
    R.left_null.push_back(std::make_unique<cuda::CudaVectorAdapter>(ctx, left[(std::size_t)i]));
  R.restarts = (std::size_t)r.restarts;
  R.krylov_steps_total = (std::size_t)r.krylov_steps_total;
  R.frob_norm_est = r.frob_norm_est;
  R.converged_to_target = r.converged_to_target != 0;
  R.cg_solves = (std::size_t)r.cg_solves;
  R.cg_maxit_hits = (std::size_t)r.cg_maxit_hits;
  return R;
}

inline std::vector<std::unique_ptr<VectorInterface>>
find_nullspace_cyclic_lanczos(const MatrixInterface &A, const VectorFactory &vf, const CyclicLanczosOptions &opt) {
  return std::move(find_nullspace_cyclic_lanczos_ex(A, vf, opt).right_null);
}

} // namespace krans::solvers
