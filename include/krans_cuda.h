/*
 * krans_cuda.h - C ABI of the B200-native KraNS null-space engine
 * (libkrans_cuda.so). Plain pointers and sizes only; no C++ or torch types.
 *
 * Every function returns KRANS_OK (0) or a negative KRANS_ERR_* code; no C++
 * exception crosses this boundary. The message of the last failure on the
 * calling thread is available from krans_last_error().
 *
 * Each entry point below replaces one piece of the reference's C++ plug-in
 * API (Deep-SANE/krans, paths relative to its root):
 *   MatrixInterface        include/krans/MatrixInterface.hpp:10-24
 *   VectorInterface        include/krans/VectorInterface.hpp:8-34
 *   VectorFactory          include/krans/VectorFactory.hpp:9-23
 *   CyclicLanczosOptions / find_nullspace_cyclic_lanczos[_ex]
 *                          include/krans/Solvers/CyclicLanczosSolver.hpp:84-178
 *   LOBPCGOptions / find_nullspace_lobpcg[_ex]
 *                          include/krans/Solvers/LOBPCGSolver.hpp:71-149
 * The header-only C++ adapters in include/krans/adapters/cuda/ bind these
 * functions back to the reference's class interfaces.
 *
 * Threading: a context owns one CUDA stream; calls on one context must not
 * overlap from several host threads. Use one context per host thread.
 */
#ifndef KRANS_CUDA_H
#define KRANS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
#define KRANS_OK 0
#define KRANS_ERR_INVALID_ARGUMENT (-1) /* std::invalid_argument in the reference */
#define KRANS_ERR_RUNTIME (-2)          /* std::runtime_error in the reference */
#define KRANS_ERR_CUDA (-3)             /* a CUDA runtime call failed */
#define KRANS_ERR_OUT_OF_MEMORY (-4)    /* device allocation or HBM budget exceeded */
#define KRANS_ERR_TIMEOUT (-5)          /* a bounded device-side wait gave up */
#define KRANS_ERR_NOT_FOUND (-6)        /* unknown ticket */
#define KRANS_ERR_CANCELLED (-7)        /* request cancelled before it ran */

typedef struct krans_ctx krans_ctx;
typedef struct krans_mat krans_mat;
typedef struct krans_vec krans_vec;
typedef struct krans_rng krans_rng;

/* Message of the last failed call on this thread ("" if none). */
const char *krans_last_error(void);
/* Library version string. */
const char *krans_version(void);
/* sizeof of the ABI structs as this library was compiled, for bindings to
 * check their layouts against: out[0..8] = krans_cyclic_opts,
 * krans_cyclic_result, krans_lobpcg_opts, krans_lobpcg_result, krans_request,
 * krans_request_result, krans_server_opts, krans_spmv_tuning,
 * krans_batch_tuning. Returns the number of entries (9). */
int krans_abi_sizes(int64_t *out, int capacity);

/* ---- context --------------------------------------------------------------- */
/* Opens `device`, creates the context's stream. hbm_budget_bytes = 0 means
 * no budget beyond the device's free memory. */
int krans_ctx_create(int device, size_t hbm_budget_bytes, krans_ctx **out);
int krans_ctx_destroy(krans_ctx *ctx);
int krans_ctx_synchronize(krans_ctx *ctx);
/* Bytes currently held by the context's allocations. */
int krans_ctx_memory_in_use(const krans_ctx *ctx, size_t *bytes);
/* Number of SMs of the context's device. */
int krans_ctx_sm_count(const krans_ctx *ctx, int *sms);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events against the library's. */
int krans_ctx_stream(const krans_ctx *ctx, void **stream);

/* Self-test of failure detection (no reference counterpart): runs a two-block
 * cooperative kernel whose first block waits at a grid barrier that the second
 * never reaches. The wait is bounded by timeout_ms (the solvers' barriers use
 * 8 s); when it runs out the kernel returns with KRANS_ERR_TIMEOUT in
 * *status_out (0 would mean the wait did not give up), *elapsed_ms gets the
 * kernel's device time, and the context stays usable. */
int krans_selftest_barrier_timeout(krans_ctx *ctx, double timeout_ms, int *status_out, double *elapsed_ms);

/* ---- CSR matrix: MatrixInterface (rows, cols, multiply, multiply_transpose) --
 * Replaces EigenSparseMatrixAdapter(A), which owns A and a cached transpose
 * (include/krans/adapters/eigen/EigenSparseMatrixAdapter.hpp:20-24,56).
 * Host arrays are copied before the call returns (they may be reused at
 * once); the transpose is then built on the device, asynchronously on the
 * context's stream, which every entry point of this library orders against
 * (work a caller queues on other streams with the raw device arrays must
 * wait for that stream). Column indices within a row need not be sorted;
 * duplicates are kept as given. */
#define KRANS_CSR_FP64 1 /* keep FP64 values (needed by every FP64 path) */
#define KRANS_CSR_FP32 2 /* also keep an FP32 copy of the values (mixed precision) */
int krans_csr_create(krans_ctx *ctx, int64_t m, int64_t n, int64_t nnz,
                     const int32_t *row_ptr, const int32_t *col_idx,
                     const double *values, int flags, krans_mat **out);
int krans_csr_destroy(krans_mat *A);

/* ---- Matrix files (src/IO/MatrixLoader.cpp:12-56 in the reference:
 * load_matrix_market, load_ija_triplet_matrix). KRANS_FMT_AUTO picks the format
 * from the extension (.mtx / .ija), as the reference CLI does
 * (apps/krans_nullspace.cpp, "Unsupported input format"). IJA: header
 * "rows cols nnz", then 0-based "i j v" triplets up to the first incomplete
 * one (a count mismatch only warns on stderr). Matrix Market: coordinate
 * real/integer/pattern, general/symmetric/skew-symmetric (mirrored), 1-based.
 * Duplicates are summed; columns are sorted within each row. A file that
 * cannot be opened or parsed is KRANS_ERR_RUNTIME (std::runtime_error);
 * an entry outside the stated size is KRANS_ERR_INVALID_ARGUMENT. */
#define KRANS_FMT_AUTO 0
#define KRANS_FMT_MTX 1
#define KRANS_FMT_IJA 2
/* Parse on the host only: CSR arrays allocated by the library, released
 * with krans_host_free. */
int krans_csr_read_host(const char *path, int format, int64_t *m, int64_t *n, int64_t *nnz,
                        int32_t **row_ptr, int32_t **col_idx, double **values);
void krans_host_free(void *p);
/* Parse and create the device matrix (flags as krans_csr_create). */
int krans_csr_load(krans_ctx *ctx, const char *path, int format, int flags, krans_mat **out);
int krans_csr_dims(const krans_mat *A, int64_t *m, int64_t *n, int64_t *nnz);
/* Device pointers of the stored arrays (trans=1: the explicit transpose). */
int krans_csr_device_arrays(const krans_mat *A, int trans, const int32_t **row_ptr,
                            const int32_t **col_idx, const double **values,
                            const float **values32);

/* ---- vectors: VectorInterface (FP64, device resident) ----------------------- */
int krans_vec_create(krans_ctx *ctx, int64_t n, krans_vec **out); /* zero-filled */
int krans_vec_destroy(krans_vec *v);
int krans_vec_size(const krans_vec *v, int64_t *n);
int krans_vec_device_ptr(krans_vec *v, double **dptr);
int krans_vec_upload(krans_vec *v, const double *host, int64_t n);
int krans_vec_download(const krans_vec *v, double *host, int64_t n);
int krans_vec_dot(const krans_vec *x, const krans_vec *y, double *out);   /* dot */
int krans_vec_axpy(krans_vec *y, double alpha, const krans_vec *x);      /* add_scaled */
int krans_vec_scale(krans_vec *v, double alpha);                         /* scale */
int krans_vec_nrm2(const krans_vec *v, double *out);                     /* norm */
int krans_vec_normalize(krans_vec *v);                                   /* normalize */
int krans_vec_fill(krans_vec *v, double value);                          /* set_zero */
int krans_vec_copy(krans_vec *dst, const krans_vec *src);                /* copy_from */
int krans_vec_clone(const krans_vec *src, krans_vec **out);              /* clone */

/* Allocation-free dot product (no counterpart in the reference). For callers
 * that cannot call cudaMalloc: runtimes that give out device memory only from
 * their own pre-planned pool, and code that must not synchronize the device
 * (cudaFree, and often cudaMalloc, synchronize implicitly). Computes
 * *result = x . y for device arrays x, y of n doubles into a device double,
 * enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream) of
 * the current device, without allocating anything and without a context.
 * Scratch comes from a file-scope device array of KRANS_NOALLOC_DOT_MAX_BLOCKS
 * doubles (128 KiB, held by every GPU that loads the library until exit); n
 * above KRANS_NOALLOC_DOT_MAX_N is rejected with KRANS_ERR_INVALID_ARGUMENT.
 * The first call under each CUDA context (normally the device's primary
 * context) looks up the array's address, which is then kept by the context's
 * unique ID: make that first call before any stream capture, and again after
 * a cudaDeviceReset. Calls that overlap on the GPU share the array and race. */
#define KRANS_NOALLOC_DOT_PER_BLOCK 2048LL
#define KRANS_NOALLOC_DOT_MAX_BLOCKS 16384LL
#define KRANS_NOALLOC_DOT_MAX_N (KRANS_NOALLOC_DOT_PER_BLOCK * KRANS_NOALLOC_DOT_MAX_BLOCKS)
int krans_vec_dot_noalloc(const double *x, const double *y, int64_t n, double *result, void *stream);

/* y <- A x (trans = 0) or y <- A^T x (trans = 1): multiply / multiply_transpose
 * (EigenSparseMatrixAdapter.hpp:34-57: A_ * x and AT_ * x on the cached
 * transpose). precision: 0 = FP64 values, 1 = FP32 values with FP32
 * accumulation. Each row is summed in storage order, one rounded product and
 * one rounded addition per entry, so the FP64 result equals the reference's
 * sequential CSR loop bit for bit (kernels KRANS_SPMV_UNIFORM / ROWTILE). */
int krans_spmv(const krans_mat *A, int trans, const krans_vec *x, krans_vec *y);
int krans_spmv_ex(const krans_mat *A, int trans, int precision, const krans_vec *x,
                  krans_vec *y);

/* Kernel choice of krans_spmv_ex for one stored operand (no reference
 * counterpart; the autotuner and the benchmark set it). Zeroed = automatic:
 * UNIFORM when every row holds exactly 1, 2 or 4 entries, else ROWTILE.
 *   KRANS_SPMV_ROWTILE  blocks of rows_per_block consecutive rows (0 = from
 *                       the mean row length); entries streamed in tiles of
 *                       2048, products staged in shared memory, per-row sums
 *                       in storage order
 *   KRANS_SPMV_UNIFORM  one thread per row, vector loads (uniform rows only)
 *   KRANS_SPMV_LANES    the solver teams' form: a power-of-two group of lanes
 *                       per row and a warp butterfly (not bit-identical to the
 *                       sequential loop) */
#define KRANS_SPMV_AUTO 0
#define KRANS_SPMV_ROWTILE 1
#define KRANS_SPMV_UNIFORM 2
#define KRANS_SPMV_LANES 3
typedef struct krans_spmv_tuning {
  int32_t kernel;         /* KRANS_SPMV_* */
  int32_t rows_per_block; /* ROWTILE: rows per block, 1..2048 (0 = automatic) */
  int32_t x_evict_last;   /* UNIFORM / ROWTILE: gather x with the L2 evict-last policy (0 = normal) */
  int32_t reserved;
} krans_spmv_tuning;
int krans_csr_set_spmv_tuning(krans_mat *A, int trans, const krans_spmv_tuning *t);
int krans_csr_get_spmv_tuning(const krans_mat *A, int trans, krans_spmv_tuning *t);

/* ---- the block solver's dense products on raw device arrays -----------------
 * (no reference counterpart: the device code that LOBPCG runs inside its
 * kernel, exposed for tests and benchmarks; FP64 tensor cores). Z, W are
 * column-major n x p blocks with leading dimension ld >= n; results are
 * column-major with leading dimension p (Gram) or ld (combine). Synchronous
 * on the context's stream.
 * krans_block_gram: S = Z^T Z and, when W is given, G = Z^T W, formed on the
 *   upper triangle and mirrored as form_gram does (LOBPCGSolver.cpp:67-80);
 *   W and G are both NULL or both given.
 * krans_block_gemm_tn: C = A^T B (a x b, leading dimension a) for n x a and
 *   n x b blocks A, B (the projections onto the locked basis of
 *   orthonormalize_block, LOBPCGSolver.cpp:137-160).
 * krans_block_combine: out = Z C for C zc x q (leading dimension ldc), as
 *   combine_columns (LOBPCGSolver.cpp:122-134).
 * device_ms (may be NULL) receives the kernel's device time. */
int krans_block_gram(krans_ctx *ctx, int64_t n, int64_t p, const double *Z, const double *W, int64_t ld,
                     double *S, double *G, double *device_ms);
int krans_block_gemm_tn(krans_ctx *ctx, int64_t n, int64_t a, const double *A, int64_t b, const double *B,
                        int64_t ld, double *C, double *device_ms);
int krans_block_combine(krans_ctx *ctx, int64_t n, int64_t zc, int64_t q, const double *Z, int64_t ld,
                        const double *C, int64_t ldc, double *out, double *device_ms);

/* ---- random vectors: VectorFactory::create_random_of_size ------------------
 * KRANS_RNG_MT19937 reproduces std::mt19937(seed) + std::normal_distribution
 * <double>(0,1) as used by StdVectorFactory/EigenVectorFactory
 * (include/krans/adapters/universal/StdVectorFactory.hpp:16-20,38-44),
 * including the state carried from one vector to the next. Seed 0 draws a
 * seed from the host's random device, as the reference does.
 * KRANS_RNG_PHILOX is a counter-based stream (Philox4x32-10 + Box-Muller):
 * not the reference's sequence, but fully parallel. */
#define KRANS_RNG_MT19937 0
#define KRANS_RNG_PHILOX 1
int krans_rng_create(krans_ctx *ctx, uint32_t seed, int mode, krans_rng **out);
int krans_rng_destroy(krans_rng *r);
int krans_rng_normal(krans_rng *r, krans_vec *out); /* next size(out) normals */
int krans_rng_seed(const krans_rng *r, uint32_t *seed);

/* ---- solver options (field names, meanings and defaults of the reference) -- */
#define KRANS_PREC_FP64 0  /* plain FP64 throughout */
#define KRANS_PREC_MIXED 1 /* FP32 SpMV + Krylov recurrence, FP64 reorth/tiny/polish */

#define KRANS_TEAM_AUTO 0 /* pick by problem size */
#define KRANS_TEAM_CTA 1  /* one thread block runs the solve */
#define KRANS_TEAM_GRID 2 /* the whole GPU runs the solve (cooperative launch) */

/* Device preconditioners for the CG projector on A A^T (precond_AAt,
 * CyclicLanczosSolver.hpp:115) and for LOBPCG's N = A^T A (M_inv,
 * LOBPCGSolver.hpp:98). The reference takes host callbacks, which a solver
 * running whole on the GPU cannot call; these are the callbacks its own tests
 * use, computed on the device:
 *   KRANS_PRECOND_NONE     z = r (also the tests' identity callback)
 *   KRANS_PRECOND_JACOBI   z_i = r_i / diag_i (diag of A A^T: squared row norms;
 *                          of A^T A: squared column norms; 1 where the diagonal is 0)
 *   KRANS_PRECOND_SD       precond_steps steps of steepest descent on the operator
 *                          from z = 0 (tests/test_cyclic_lanczos.cpp:339-377,
 *                          tests/test_lobpcg.cpp:179-205): q = r; per step
 *                          alpha = q.q / q.Oq, z += alpha q, q -= alpha Oq, stopping
 *                          when |q.Oq| < 1e-30 or q.q <= 1e-30 */
#define KRANS_PRECOND_NONE 0
#define KRANS_PRECOND_JACOBI 1
#define KRANS_PRECOND_SD 2

typedef struct krans_cyclic_opts {
  int64_t k;                 /* 1    number of right null vectors wanted */
  int64_t ncv;               /* 48   Krylov dimension (Lanczos vectors of H(A)) */
  int64_t max_restarts;      /* 80 */
  double tol_abs;            /* 1e-12 accept if ||Av|| <= max(tol_abs, tol_rel*max(1,||A||_F~)) */
  double tol_rel;            /* 1e-10 */
  int32_t reorth;            /* 2    ReorthMode: 0 None, 1 Single, 2 Double */
  int32_t use_harmonic;      /* 1    refined interior extraction (else plain Ritz) */
  double target_tau;         /* 0 */
  int32_t nullity_known;     /* -1 */
  int32_t rank_known;        /* -1 */
  int64_t cg_maxit;          /* 80 */
  double cg_rel_tol;         /* 1e-10 */
  double cg_breakdown_tol;   /* 1e-30 */
  int32_t projector_passes;  /* 1 */
  int32_t grad_max_iters;    /* 3000 */
  int32_t frob_samples;      /* 4 */
  double prescreen_factor;   /* 0.8 */
  int64_t stagnation_restarts; /* 30 */
  int32_t return_left_space; /* 0 */
  int32_t verbose;           /* 0 (device engine: ignored) */
  /* B200 engine knobs (no reference counterpart) */
  int32_t precision;         /* KRANS_PREC_FP64 */
  int32_t team;              /* KRANS_TEAM_AUTO */
  int32_t precond_aat;       /* KRANS_PRECOND_NONE: the device form of precond_AAt */
  int32_t precond_steps;     /* steps of KRANS_PRECOND_SD (8) */
  int32_t polish_block;      /* (ignored when precond_aat is set)
                                0: polish candidates one by one (the reference's order);
                                1: project up to 8 candidates of a restart with one block CG
                                (matrix read once per iteration for all of them) */
  int32_t mixed_fallback;    /* 1    KRANS_PREC_MIXED only: when the mixed run stops short of k
                                with its FP64 CG polish at cg_maxit (FP32 Ritz vectors too far
                                from the null space for the projector to finish), the solve
                                continues in FP64 from the vectors already accepted (same RNG
                                stream; krans_cyclic_result.fp64_fallback reports it). Single
                                solves only: the batched and served paths keep the mixed result. */
} krans_cyclic_opts;

typedef struct krans_cyclic_result {
  int64_t n_right, n_left;   /* sizes of right_null / left_null */
  int64_t restarts;          /* CyclicLanczosResult::restarts */
  int64_t krylov_steps_total;
  double frob_norm_est;
  int32_t converged_to_target;
  int32_t status;            /* KRANS_OK or a device-side error code */
  int64_t cg_solves, cg_maxit_hits;
  /* B200 engine diagnostics */
  int64_t spmv, spmvT;       /* operator applications (CountingMatrixAdapter) */
  double algo_bytes;         /* algorithmic HBM bytes of the solve */
  double device_ms;          /* device time of the solve kernel(s) */
  double phase_ms[4];        /* device time in Golub-Kahan+reorth, tiny SVD, CG polish, rest */
  int32_t fp64_fallback;     /* 1 when a mixed solve continued in FP64 (mixed_fallback) */
  int32_t fallback_from;     /* vectors the mixed run had accepted before it */
} krans_cyclic_result;

typedef struct krans_lobpcg_opts {
  int64_t nev;               /* 1 */
  int64_t block_size;        /* 0 = auto min(16, nev) */
  int64_t max_iters;         /* 1000 */
  double tol_abs;            /* 1e-12 */
  double tol_rel;            /* 1e-10 */
  int32_t soft_locking;      /* 1 */
  double restart;            /* 0.9 */
  double gs_tol;             /* 1e-14 */
  int32_t gs_reorth;         /* 1 */
  int32_t frob_samples;      /* 4 */
  int64_t max_tiny_dim;      /* 0 */
  int32_t nullity_known;     /* -1 */
  int32_t rank_known;        /* -1 */
  int32_t verbose;           /* 0 (device engine: ignored) */
  int64_t progress_every;    /* 100 (device engine: ignored) */
  int32_t precision;         /* KRANS_PREC_FP64 */
  int32_t team;              /* KRANS_TEAM_AUTO */
  int32_t precond_normal;    /* KRANS_PRECOND_NONE: the device form of M_inv */
  int32_t precond_steps;     /* steps of KRANS_PRECOND_SD (6) */
} krans_lobpcg_opts;

typedef struct krans_lobpcg_result {
  int64_t n_right;
  int64_t iters, locked;
  double frob_norm_est, accept_threshold, best_unaccepted_residual;
  int64_t block_size;
  int32_t converged_to_target;
  int32_t status;
  int64_t spmv, spmvT;
  double algo_bytes, gram_flops;
  double device_ms;
  double phase_ms[5]; /* device time (ms): apply_normal (SpMV pairs), Gram, tiny GEP,
                         orthonormalisation, the rest */
  double final_polish_ms; /* part of the rest: the closing block_rr_polish, two_vec_rr_sharpen
                             and MGS of the accepted basis (their operator products included) */
} krans_lobpcg_result;

int krans_cyclic_opts_init(krans_cyclic_opts *o);
int krans_lobpcg_opts_init(krans_lobpcg_opts *o);

/* find_nullspace_cyclic_lanczos_ex on the device engine
 * (src/Solvers/CyclicLanczosSolver.cpp:618-660 in the reference).
 * rng: the factory's stream (consumed and advanced exactly as the reference
 *      consumes VectorFactory::create_random_of_size).
 * initial_right: optional start vector y0 (CyclicLanczosOptions::
 *      initial_right_space.front()), or NULL.
 * right_out: caller array of capacity max(k, nullity_known) handles; filled
 *      with newly created vectors owned by the caller (result->n_right).
 * left_out: capacity k handles, used when return_left_space (may be NULL). */
int krans_solve_cyclic(krans_ctx *ctx, const krans_mat *A, krans_rng *rng,
                       const krans_cyclic_opts *opts, const krans_vec *initial_right,
                       krans_vec **right_out, krans_vec **left_out,
                       krans_cyclic_result *result);

/* find_nullspace_lobpcg_ex on the device engine
 * (src/Solvers/LOBPCGSolver.cpp:443-834 in the reference).
 * initial_block: optional array of n_initial seed vectors, or NULL.
 * right_out: capacity = the reference's k_target; theta_out/resid_out
 *      (host, may be NULL) receive LOBPCGResult::theta / residuals_Av. */
int krans_solve_lobpcg(krans_ctx *ctx, const krans_mat *A, krans_rng *rng,
                       const krans_lobpcg_opts *opts, const krans_vec *const *initial_block,
                       int64_t n_initial, krans_vec **right_out, double *theta_out,
                       double *resid_out, krans_lobpcg_result *result);

/* ---- batched solves: many independent requests in one persistent launch --- */
#define KRANS_SOLVER_CYCLIC 0 /* find_nullspace_cyclic_lanczos_ex */
#define KRANS_SOLVER_LOBPCG 1 /* find_nullspace_lobpcg_ex (served requests) */
typedef struct krans_request {
  const krans_mat *A;        /* matrix of this request */
  krans_cyclic_opts opts;    /* options of a cyclic request (k, tolerances, precision) */
  uint32_t seed;             /* RNG seed of the request's own stream */
  int32_t rng_mode;          /* KRANS_RNG_PHILOX or KRANS_RNG_MT19937 */
  double *basis_out;         /* DEVICE pointer: basis_capacity x cols(A) doubles, row i = vector i;
                                NULL: the basis stays in the request's workspace and is dropped
                                (the result, max_residual included, is still reported) */
  int64_t basis_capacity;    /* vectors that fit in basis_out */
  int32_t solver;            /* KRANS_SOLVER_CYCLIC; KRANS_SOLVER_LOBPCG for krans_submit only */
  int32_t reserved;
  krans_lobpcg_opts lobpcg;  /* options of a LOBPCG request (FP64; its nev / nullity_known set the target) */
} krans_request;

typedef struct krans_request_result {
  int32_t status;            /* KRANS_OK or error */
  int32_t converged_to_target;
  int64_t n_right;
  int64_t restarts, krylov_steps_total, cg_solves, cg_maxit_hits;
  int64_t spmv, spmvT;
  double frob_norm_est;
  double max_residual;       /* max ||A u||_2 over the returned basis (FP64) */
  double algo_bytes;
  double queue_ms, device_ms, latency_ms; /* see krans_solve_batch / krans_poll */
  double phase_ms[4];        /* device time in Golub-Kahan+reorth, tiny SVD, CG polish, rest */
  int64_t launch_id;         /* server: sequence number of the launch that ran the request */
} krans_request_result;

/* Solve `count` cyclic requests in one persistent launch (one thread block
 * per request at a time, largest first). basis_out of each request is a
 * DEVICE pointer to basis_capacity x cols(A) doubles (row i = vector i). */
int krans_solve_batch(krans_ctx *ctx, int64_t count, const krans_request *reqs,
                      krans_request_result *results, double *device_ms);

/* ---- batched-launch tuning (no reference counterpart) ------------------------
 * Knobs of krans_solve_batch and of the server's launches, held per context.
 * The project's autotuner (krans_b200/autotune.py) measures them on probe
 * batches and caches the winners per device; zero fields keep the built-in
 * value (in parentheses).
 *   cluster_min   requests with m + n >= cluster_min run on thread-block
 *                 clusters, smaller ones on single blocks (16384)
 *   pair_max      cluster requests with m + n < pair_max run on 2-block
 *                 clusters of a second launch beside the big clusters (120000)
 *   cluster_size  blocks per big cluster, 2..16 (8)
 *   lanes[6]      threads per row of the solvers' SpMV for operands whose mean
 *                 row length is <= 3, <= 8, <= 16, <= 32, <= 64, > 64
 *                 (1, 2, 4, 8, 16, 32); powers of two up to 32. Operands whose
 *                 rows all hold exactly 1, 2 or 4 entries use one thread per
 *                 row whatever the table says.
 * The lanes apply to every solve of the context (single and batched); a
 * request's rounding depends on them, so results are reproducible for a
 * given table. */
typedef struct krans_batch_tuning {
  int64_t cluster_min;
  int64_t pair_max;
  int32_t cluster_size;
  int32_t lanes[6];
} krans_batch_tuning;
int krans_ctx_set_batch_tuning(krans_ctx *ctx, const krans_batch_tuning *t);
int krans_ctx_get_batch_tuning(const krans_ctx *ctx, krans_batch_tuning *t); /* values in effect */

/* ---- serving: continuous batching against an HBM budget ---------------------- */
typedef struct krans_server krans_server;
typedef struct krans_server_opts {
  size_t hbm_budget_bytes;   /* admission budget for request state (0 = 150 GB) */
  int32_t max_inflight_launches; /* concurrent persistent launches (streams) */
  int32_t max_batch;         /* requests per launch */
  double batch_window_ms;    /* how long the scheduler waits to fill a launch */
} krans_server_opts;

int krans_server_opts_init(krans_server_opts *o);
int krans_server_create(krans_ctx *ctx, const krans_server_opts *opts, krans_server **out);
int krans_server_destroy(krans_server *s);
/* Queue a request; the server copies the descriptor (A must stay alive until
 * the ticket completes). basis_out is a device pointer as in krans_request.
 * Cyclic requests join a running persistent launch when one has a free team
 * of their size class: the launch stays resident while requests keep
 * arriving (its teams leave after 20 ms without work) and leaves 20 SMs free
 * for other work; its thread-block clusters take large requests whenever
 * one waits and single-block requests otherwise. A request that does not fit
 * it (another precision, a larger workspace than its slots) starts the next
 * launch. LOBPCG requests
 * run one per launch, on one thread block (m + n below the context's
 * cluster_min) or on a cluster of up to 4 blocks, FP64; their result reports
 * LOBPCG iterations in `restarts` and locked vectors in `krylov_steps_total`. */
int krans_submit(krans_server *s, const krans_request *req, uint64_t *ticket);
/* status: 0 queued, 1 running, 2 done, 3 failed, 4 cancelled */
int krans_poll(krans_server *s, uint64_t ticket, int *status, krans_request_result *result);
/* A queued request is dropped at once. A running one is stopped: the server
 * writes KRANS_ERR_CANCELLED into its device status word, its team unwinds at
 * its next check (every solver loop checks it), and the ticket ends as
 * cancelled (status 4), or as done if it finished first. */
int krans_cancel(krans_server *s, uint64_t ticket);
/* Tickets finished (done, failed or cancelled) since the last call, oldest
 * first, at most `capacity` of them; *count = how many were written. */
int krans_server_completed(krans_server *s, uint64_t *tickets, int64_t capacity, int64_t *count);
/* Block until every submitted request has finished or timeout_ms passes. */
int krans_server_drain(krans_server *s, double timeout_ms);
/* Scheduler state: out[0] queued tickets (cancelled ones not yet dropped
 * included), out[1] launches in flight, out[2] of them LOBPCG, out[3] cyclic
 * requests published into running launches and not finished. Returns
 * KRANS_ERR_TIMEOUT at once, without waiting, while the scheduler holds its
 * lock. */
int krans_server_stats(krans_server *s, int64_t out[4]);

#ifdef __cplusplus
}
#endif
#endif /* KRANS_CUDA_H */
