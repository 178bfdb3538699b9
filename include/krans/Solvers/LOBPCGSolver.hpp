#pragma once
// Block LOBPCG on A^T A for the right null space: options, result and entry
// points with the names, fields and defaults of the reference's
// include/krans/Solvers/LOBPCGSolver.hpp:68-149, running the B200 device
// engine. Needs a cuda::CudaCsrMatrixAdapter and a cuda::CudaVectorFactory.
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

using NormalPreconditioner = std::function<void(const VectorInterface &r_n, VectorInterface &y_n)>;

struct LOBPCGOptions {
  std::size_t nev = 1;
  std::size_t block_size = 0;
  std::size_t max_iters = 1000;
  double tol_abs = 1e-12;
  double tol_rel = 1e-10;
  bool soft_locking = true;
  double restart = 0.9;
  double gs_tol = 1e-14;
  bool gs_reorth = true;
  NormalPreconditioner M_inv = nullptr;
  std::vector<std::unique_ptr<VectorInterface>> initial_block;
  int frob_samples = 4;
  std::size_t max_tiny_dim = 0;
  int nullity_known = -1;
  int rank_known = -1;
  bool verbose = false;
  std::size_t progress_every = 100;
  int team = KRANS_TEAM_AUTO; // B200 engine knob
  int precond_device = KRANS_PRECOND_NONE; // device form of M_inv (KRANS_PRECOND_JACOBI / _SD)
  int precond_steps = 6;
};

struct LOBPCGResult {
  std::vector<std::unique_ptr<VectorInterface>> right_null;
  std::vector<double> theta;
  std::vector<double> residuals_Av;
  std::size_t iters = 0;
  std::size_t locked = 0;
  double frob_norm_est = 0.0;
  double accept_threshold = 0.0;
  double best_unaccepted_residual = 0.0;
  std::size_t block_size = 0;
  bool converged_to_target = false;
};

inline LOBPCGResult find_nullspace_lobpcg_ex(const MatrixInterface &A, const VectorFactory &vf,
                                             const LOBPCGOptions &opt) {
  const auto *cA = dynamic_cast<const cuda::CudaCsrMatrixAdapter *>(&A);
  const auto *cf = dynamic_cast<const cuda::CudaVectorFactory *>(&vf);
  if (!cA || !cf)
    throw std::invalid_argument(
        "find_nullspace_lobpcg: the B200 engine needs a CudaCsrMatrixAdapter and a CudaVectorFactory");
  if (opt.M_inv)
    throw std::invalid_argument("find_nullspace_lobpcg: host M_inv callbacks cannot run inside the device "
                                "engine; use precond_device (KRANS_PRECOND_JACOBI or KRANS_PRECOND_SD)");
  krans_lobpcg_opts o;
  krans_lobpcg_opts_init(&o);
  o.nev = (int64_t)opt.nev;
  o.block_size = (int64_t)opt.block_size;
  o.max_iters = (int64_t)opt.max_iters;
  o.tol_abs = opt.tol_abs;
  o.tol_rel = opt.tol_rel;
  o.soft_locking = opt.soft_locking;
  o.restart = opt.restart;
  o.gs_tol = opt.gs_tol;
  o.gs_reorth = opt.gs_reorth;
  o.frob_samples = opt.frob_samples;
  o.max_tiny_dim = (int64_t)opt.max_tiny_dim;
  o.nullity_known = opt.nullity_known;
  o.rank_known = opt.rank_known;
  o.verbose = opt.verbose;
  o.progress_every = (int64_t)opt.progress_every;
  o.team = opt.team;
  o.precond_normal = opt.precond_device;
  o.precond_steps = opt.precond_steps;
  std::vector<const krans_vec *> init;
  for (const auto &v : opt.initial_block) {
    const auto *c = dynamic_cast<const cuda::CudaVectorAdapter *>(v.get());
    if (!c)
      throw std::invalid_argument("find_nullspace_lobpcg: initial_block backend mismatch");
    init.push_back(c->handle());
  }
  std::size_t k_target = std::max<std::size_t>(1, opt.nev);
  if (opt.nullity_known >= 0)
    k_target = (std::size_t)opt.nullity_known;
  else if (opt.rank_known >= 0 && (std::size_t)opt.rank_known <= A.cols())
    k_target = A.cols() - (std::size_t)opt.rank_known;
  const std::size_t cap = std::max<std::size_t>(k_target, 1);
  std::vector<krans_vec *> right(cap, nullptr);
  std::vector<double> theta(cap), resid(cap);
  krans_lobpcg_result r;
  krans_ctx *ctx = cA->context();
  cuda::check(krans_solve_lobpcg(ctx, cA->handle(), cf->rng(), &o, init.empty() ? nullptr : init.data(),
                                 (int64_t)init.size(), right.data(), theta.data(), resid.data(), &r),
              "find_nullspace_lobpcg");
  LOBPCGResult R;
  for (int64_t i = 0; i < r.n_right; i++) {
    R.right_null.push_back(std::make_unique<cuda::CudaVectorAdapter>(ctx, right[(std::size_t)i]));
    R.theta.push_back(theta[(std::size_t)i]);
    R.residuals_Av.push_back(resid[(std::size_t)i]);
  }
  R.iters = (std::size_t)r.iters;
  R.locked = (std::size_t)r.locked;
  R.frob_norm_est = r.frob_norm_est;
  R.accept_threshold = r.accept_threshold;
  R.best_unaccepted_residual = r.best_unaccepted_residual;
  R.block_size = (std::size_t)r.block_size;
  R.converged_to_target = r.converged_to_target != 0;
  return R;
}

inline std::vector<std::unique_ptr<VectorInterface>>
find_nullspace_lobpcg(const MatrixInterface &A, const VectorFactory &vf, const LOBPCGOptions &opt) {
  return std::move(find_nullspace_lobpcg_ex(A, vf, opt).right_null);
}

} // namespace krans::solvers
