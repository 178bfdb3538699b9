// C entry points over the reference's own solvers (TEST INFRASTRUCTURE ONLY).
//
// oracle/Makefile's `ref` target compiles the reference's solver sources
// where they lie (src/Solvers/CyclicLanczosSolver.cpp,
// src/Solvers/LOBPCGSolver.cpp, src/Utils/GramSchmidt.cpp,
// src/Utils/Projection.cpp of Deep-SANE/krans) unchanged, against the
// project's Eigen-subset shim (oracle/eigen_subset/Eigen/Dense), together
// with this file, into oracle/_ref/libkrans_ref.so. The matrix is the
// reference's StdMatrixAdapter over CSR callbacks (row sums in storage order)
// and the vectors come from the reference's StdVectorFactory
// (include/krans/adapters/universal/), so everything except the Eigen dense
// kernels is the reference's code. Options and results use the C structs of
// oracle/krans_oracle.h, so the C restatement and this build are called the
// same way and can be compared directly. Only tests/, __graft_entry__ and
// bench.py's CPU legs load it.
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "krans/Solvers/CyclicLanczosSolver.hpp"
#include "krans/Solvers/LOBPCGSolver.hpp"
#include "krans/adapters/universal/StdMatrixAdapter.hpp"
#include "krans/adapters/universal/StdVectorAdapter.hpp"
#include "krans/adapters/universal/StdVectorFactory.hpp"
#include "krans_oracle.h"

using krans::VectorInterface;
using krans::universal::StdMatrixAdapter;
using krans::universal::StdVectorAdapter;
using krans::universal::StdVectorFactory;

namespace {
thread_local std::string g_err;

struct Counters {
  int64_t spmv = 0, spmvT = 0;
};

// y = A x over CSR rows, s += v[k] * x[c[k]] in storage order
void csr_apply(int64_t rows, const int32_t *rp, const int32_t *ci, const double *v, const std::vector<double> &x,
               std::vector<double> &y) {
  for (int64_t i = 0; i < rows; i++) {
    double s = 0.0;
    for (int32_t k = rp[i]; k < rp[i + 1]; k++)
      s += v[k] * x[(size_t)ci[k]];
    y[(size_t)i] = s;
  }
}

StdMatrixAdapter make_matrix(const ko_csr *A, Counters *cnt) {
  return StdMatrixAdapter(
      (size_t)A->m, (size_t)A->n,
      [A, cnt](const std::vector<double> &x, std::vector<double> &y) {
        cnt->spmv++;
        csr_apply(A->m, A->rp, A->ci, A->v, x, y);
      },
      [A, cnt](const std::vector<double> &x, std::vector<double> &y) {
        cnt->spmvT++;
        csr_apply(A->n, A->rpT, A->ciT, A->vT, x, y);
      });
}

void copy_out(const std::vector<std::unique_ptr<VectorInterface>> &vs, size_t n, double *out) {
  for (size_t i = 0; i < vs.size(); i++)
    std::memcpy(out + i * n, vs[i]->data(), n * sizeof(double));
}

std::unique_ptr<VectorInterface> vec_from(const double *p, size_t n) {
  return std::make_unique<StdVectorAdapter>(std::vector<double>(p, p + n));
}
} // namespace

struct kref_factory {
  StdVectorFactory f;
  kref_factory(size_t n, unsigned seed) : f(n, seed) {}
};

extern "C" {

const char *kref_last_error(void) { return g_err.c_str(); }

// StdVectorFactory(default_size, seed): the reference's factory, whose RNG
// state carries over from one solve to the next
kref_factory *kref_factory_create(int64_t default_size, uint32_t seed) {
  return new kref_factory((size_t)default_size, seed);
}
void kref_factory_destroy(kref_factory *f) { delete f; }

// find_nullspace_cyclic_lanczos_ex; right_out: capacity k_target x n,
// left_out: k x m (or NULL). Returns 0, 1 on std::invalid_argument, 2 on
// another exception (message in kref_last_error).
int kref_cyclic(const ko_csr *A, kref_factory *vf, const ko_cyclic_opts *o, double *right_out, double *left_out,
                ko_cyclic_result *res) {
  try {
    Counters cnt;
    StdMatrixAdapter M = make_matrix(A, &cnt);
    krans::solvers::CyclicLanczosOptions opt;
    opt.k = (size_t)o->k;
    opt.ncv = (size_t)o->ncv;
    opt.max_restarts = (size_t)o->max_restarts;
    opt.tol_abs = o->tol_abs;
    opt.tol_rel = o->tol_rel;
    opt.reorth = (krans::solvers::ReorthMode)o->reorth;
    opt.use_harmonic = o->use_harmonic != 0;
    opt.target_tau = o->target_tau;
    opt.nullity_known = o->nullity_known;
    opt.rank_known = o->rank_known;
    if (o->initial_right)
      opt.initial_right_space.push_back(vec_from(o->initial_right, (size_t)A->n));
    if (o->precond_AAt) {
      ko_precond_fn fn = o->precond_AAt;
      void *user = o->precond_user;
      opt.precond_AAt = [fn, user](const VectorInterface &r, VectorInterface &y) {
        fn(user, r.data(), y.data());
      };
    }
    opt.cg_maxit = (size_t)o->cg_maxit;
    opt.cg_rel_tol = o->cg_rel_tol;
    opt.cg_breakdown_tol = o->cg_breakdown_tol;
    opt.projector_passes = o->projector_passes;
    opt.grad_max_iters = o->grad_max_iters;
    opt.frob_samples = o->frob_samples;
    opt.prescreen_factor = o->prescreen_factor;
    opt.stagnation_restarts = (size_t)o->stagnation_restarts;
    opt.return_left_space = o->return_left_space != 0;
    opt.verbose = o->verbose != 0;
    auto R = krans::solvers::find_nullspace_cyclic_lanczos_ex(M, vf->f, opt);
    copy_out(R.right_null, (size_t)A->n, right_out);
    if (left_out)
      copy_out(R.left_null, (size_t)A->m, left_out);
    std::memset(res, 0, sizeof *res);
    res->n_right = (int64_t)R.right_null.size();
    res->n_left = (int64_t)R.left_null.size();
    res->restarts = (int64_t)R.restarts;
    res->krylov_steps_total = (int64_t)R.krylov_steps_total;
    res->frob_norm_est = R.frob_norm_est;
    res->converged_to_target = R.converged_to_target ? 1 : 0;
    res->cg_solves = (int64_t)R.cg_solves;
    res->cg_maxit_hits = (int64_t)R.cg_maxit_hits;
    res->spmv = cnt.spmv;
    res->spmvT = cnt.spmvT;
    return 0;
  } catch (const std::invalid_argument &e) {
    g_err = e.what();
    return 1;
  } catch (const std::exception &e) {
    g_err = e.what();
    return 2;
  }
}

// find_nullspace_lobpcg_ex; right_out: capacity x n; theta_out / resid_out:
// capacity doubles (LOBPCGResult::theta / residuals_Av).
int kref_lobpcg(const ko_csr *A, kref_factory *vf, const ko_lobpcg_opts *o, int64_t capacity, double *right_out,
                double *theta_out, double *resid_out, ko_lobpcg_result *res) {
  try {
    Counters cnt;
    StdMatrixAdapter M = make_matrix(A, &cnt);
    krans::solvers::LOBPCGOptions opt;
    opt.nev = (size_t)o->nev;
    opt.block_size = (size_t)o->block_size;
    opt.max_iters = (size_t)o->max_iters;
    opt.tol_abs = o->tol_abs;
    opt.tol_rel = o->tol_rel;
    opt.soft_locking = o->soft_locking != 0;
    opt.restart = o->restart;
    opt.gs_tol = o->gs_tol;
    opt.gs_reorth = o->gs_reorth != 0;
    if (o->M_inv) {
      ko_precond_fn fn = o->M_inv;
      void *user = o->M_user;
      opt.M_inv = [fn, user](const VectorInterface &r, VectorInterface &y) { fn(user, r.data(), y.data()); };
    }
    for (int64_t i = 0; o->initial_block && i < o->n_initial; i++)
      opt.initial_block.push_back(vec_from(o->initial_block + i * A->n, (size_t)A->n));
    opt.frob_samples = o->frob_samples;
    opt.max_tiny_dim = (size_t)o->max_tiny_dim;
    opt.nullity_known = o->nullity_known;
    opt.rank_known = o->rank_known;
    opt.verbose = o->verbose != 0;
    auto R = krans::solvers::find_nullspace_lobpcg_ex(M, vf->f, opt);
    if ((int64_t)R.right_null.size() > capacity) {
      g_err = "kref_lobpcg: more vectors than the output capacity";
      return 2;
    }
    copy_out(R.right_null, (size_t)A->n, right_out);
    for (size_t i = 0; i < R.theta.size() && (int64_t)i < capacity; i++)
      theta_out[i] = R.theta[i];
    for (size_t i = 0; i < R.residuals_Av.size() && (int64_t)i < capacity; i++)
      resid_out[i] = R.residuals_Av[i];
    std::memset(res, 0, sizeof *res);
    res->n_right = (int64_t)R.right_null.size();
    res->iters = (int64_t)R.iters;
    res->locked = (int64_t)R.locked;
    res->frob_norm_est = R.frob_norm_est;
    res->accept_threshold = R.accept_threshold;
    res->best_unaccepted_residual = R.best_unaccepted_residual;
    res->block_size = (int64_t)R.block_size;
    res->converged_to_target = R.converged_to_target ? 1 : 0;
    res->spmv = cnt.spmv;
    res->spmvT = cnt.spmvT;
    return 0;
  } catch (const std::invalid_argument &e) {
    g_err = e.what();
    return 1;
  } catch (const std::exception &e) {
    g_err = e.what();
    return 2;
  }
}

} // extern "C"
