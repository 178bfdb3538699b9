/*
 * KraNS oracle: a plain-C, single-threaded CPU restatement of the reference
 * null-space solvers (Deep-SANE/krans). TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and there only as the reference result / CPU baseline. The
 * product path (krans_b200/, libkrans_cuda.so) never links or calls it.
 *
 * What it restates (reference file:line):
 *   - std::mt19937 + std::normal_distribution<double> as used by
 *     StdVectorFactory / EigenVectorFactory
 *     (include/krans/adapters/universal/StdVectorFactory.hpp:16-20,38-44)
 *   - CSR SpMV / SpM^T V (StdMatrixAdapter over CSR callbacks,
 *     include/krans/adapters/universal/StdMatrixAdapter.hpp:47-87)
 *   - find_nullspace_cyclic_lanczos_ex (src/Solvers/CyclicLanczosSolver.cpp:291-660)
 *   - find_nullspace_lobpcg_ex (src/Solvers/LOBPCGSolver.cpp:443-834)
 *   - modified_gram_schmidt / max_pairwise_abs_dot (src/Utils/GramSchmidt.cpp:55-91)
 *   - subspace_diff (RREF) (include/krans/Utils/SubspaceCompare.hpp:17-110)
 *
 * The reference's small dense problems use Eigen 3.4 (JacobiSVD,
 * SelfAdjointEigenSolver, LLT). Eigen is not available here, so this file
 * uses its own textbook routines (one-sided Jacobi SVD, cyclic Jacobi
 * symmetric eigensolver, Cholesky). They agree with Eigen to rounding, not
 * bitwise; singular/eigen vectors may differ in sign or within degenerate
 * clusters, so results are compared at the subspace level.
 *
 * Pinning: tests/test_oracle_pins.py checks this oracle against the known
 * answers of the reference's own tests and examples (quickstart analytic
 * kernel, tests/test_cyclic_lanczos.cpp, tests/test_lobpcg.cpp,
 * tests/test_difference_operator.cpp, tests/test_universal_adapter.cpp,
 * tests/test_subspace_compare.cpp, the nullities of data/mat1-6) and the RNG
 * bit-for-bit against libstdc++'s std::mt19937/std::normal_distribution.
 */
#ifndef KRANS_ORACLE_H
#define KRANS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- RNG: std::mt19937(seed) feeding std::normal_distribution<double>(0,1) */
typedef struct ko_rng {
  uint32_t mt[624];
  int32_t idx;
  int32_t has_saved;
  double saved;
} ko_rng;

void ko_rng_seed(ko_rng *r, uint32_t seed);
uint32_t ko_rng_u32(ko_rng *r);
double ko_rng_normal(ko_rng *r);
void ko_rng_fill_normal(ko_rng *r, double *x, int64_t n);
size_t ko_rng_sizeof(void);

/* ---- CSR matrix A (m x n) plus its explicit transpose (n x m) ------------ */
typedef struct ko_csr {
  int64_t m, n;
  const int32_t *rp, *ci;   /* A: m+1 row pointers, nnz columns */
  const double *v;
  const int32_t *rpT, *ciT; /* A^T: n+1 row pointers */
  const double *vT;
} ko_csr;

void ko_spmv(const ko_csr *A, int trans, const double *x, double *y);

/* preconditioner callback y <- M^{-1} r (sizes implied by the solver) */
typedef void (*ko_precond_fn)(void *user, const double *r, double *y);

/* ---- cyclic Lanczos (CyclicLanczosOptions, CyclicLanczosSolver.hpp:84-146) */
typedef struct ko_cyclic_opts {
  int64_t k, ncv, max_restarts;
  double tol_abs, tol_rel;
  int32_t reorth;          /* 0 none, 1 single, 2 double */
  int32_t use_harmonic;
  double target_tau;
  int32_t nullity_known, rank_known;
  const double *initial_right; /* optional n-vector (first initial_right_space) */
  ko_precond_fn precond_AAt;
  void *precond_user;
  int64_t cg_maxit;
  double cg_rel_tol, cg_breakdown_tol;
  int32_t projector_passes;
  int32_t grad_max_iters;
  int32_t frob_samples;
  double prescreen_factor;
  int64_t stagnation_restarts;
  int32_t return_left_space;
  int32_t verbose;
} ko_cyclic_opts;

typedef struct ko_cyclic_result {
  int64_t n_right, n_left;
  int64_t restarts, krylov_steps_total;
  double frob_norm_est;
  int32_t converged_to_target;
  int64_t cg_solves, cg_maxit_hits;
  int64_t spmv, spmvT; /* operator applications (CountingMatrixAdapter) */
} ko_cyclic_result;

void ko_cyclic_opts_default(ko_cyclic_opts *o);
/* right_out: capacity k_target x n (row i = vector i); left_out: k x m or NULL */
int ko_cyclic(const ko_csr *A, ko_rng *rng, const ko_cyclic_opts *o,
              double *right_out, double *left_out, ko_cyclic_result *res);

/* ---- LOBPCG (LOBPCGOptions, LOBPCGSolver.hpp:71-115) --------------------- */
typedef struct ko_lobpcg_opts {
  int64_t nev, block_size, max_iters;
  double tol_abs, tol_rel;
  int32_t soft_locking;
  double restart;
  double gs_tol;
  int32_t gs_reorth;
  ko_precond_fn M_inv;
  void *M_user;
  const double *initial_block; /* n_initial x n row-major, or NULL */
  int64_t n_initial;
  int32_t frob_samples;
  int64_t max_tiny_dim;
  int32_t nullity_known, rank_known;
  int32_t verbose;
} ko_lobpcg_opts;

typedef struct ko_lobpcg_result {
  int64_t n_right;
  int64_t iters, locked;
  double frob_norm_est, accept_threshold, best_unaccepted_residual;
  int64_t block_size;
  int32_t converged_to_target;
  int64_t spmv, spmvT;
} ko_lobpcg_result;

void ko_lobpcg_opts_default(ko_lobpcg_opts *o);
/* right_out: capacity k_target x n; theta_out/resid_out: capacity k_target */
int ko_lobpcg(const ko_csr *A, ko_rng *rng, const ko_lobpcg_opts *o,
              double *right_out, double *theta_out, double *resid_out,
              ko_lobpcg_result *res);

/* error codes (the reference throws; the oracle returns) */
#define KO_OK 0
#define KO_ERR_INVALID_ARGUMENT 1 /* std::invalid_argument */
#define KO_ERR_RUNTIME 2          /* std::runtime_error */
#define KO_ERR_NOMEM 3
const char *ko_last_error(void);

/* ---- utilities ------------------------------------------------------------ */
/* MGS with optional second pass over k row-vectors of length n (in place). */
int ko_mgs(int64_t k, int64_t n, double *V, double tol, int reorth);
double ko_max_pairwise_abs_dot(int64_t k, int64_t n, const double *V);
/* RREF Frobenius difference (SubspaceCompare.hpp:86-110); 1e9 on mismatch. */
double ko_subspace_diff_rref(int64_t k1, int64_t k2, int64_t n,
                             const double *B1, const double *B2, double tol);
/* Largest principal-angle sine ||V - U (U^T V)||_2 for orthonormal U, V
 * (k x n row-major each); returns 1.0 when ku != kv. */
double ko_subspace_dist(int64_t ku, int64_t kv, int64_t n, const double *U,
                        const double *V);
/* dense helpers exposed for tests */
int ko_svd_right(int r, int c, const double *M_colmajor, double *sv,
                 double *V_colmajor);
int ko_sym_eig(int n, const double *A_colmajor, double *w, double *Q_colmajor);

#ifdef __cplusplus
}
#endif
#endif
