/*
 * KraNS oracle: plain-C CPU restatement of the reference null-space solvers.
 * TEST INFRASTRUCTURE ONLY (checker and CPU baseline); see krans_oracle.h.
 *
 * Build: oracle/Makefile (gcc -O3 -ffp-contract=off, no -ffast-math), so
 * that dot/norm/axpy evaluate in the same sequential order and without FMA
 * contraction, like the reference's StdVectorAdapter loops
 * (include/krans/adapters/universal/StdVectorAdapter.hpp:23-74).
 */
#include "krans_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_err[256];
static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char *ko_last_error(void) { return g_err; }

/* ======================================================================== */
/* RNG: std::mt19937 + std::normal_distribution<double> (libstdc++).        */
/* Restates StdVectorFactory's generator (StdVectorFactory.hpp:16-20,38-44): */
/* the Mersenne Twister MT19937 (Matsumoto & Nishimura 1998), the            */
/* generate_canonical<double,53> combination of two 32-bit draws, and the    */
/* Marsaglia polar method that libstdc++ uses for normal_distribution,       */
/* including the cached second variate that persists across vectors.       */
/* ======================================================================== */
size_t ko_rng_sizeof(void) { return sizeof(ko_rng); }

void ko_rng_seed(ko_rng *r, uint32_t seed) {
  r->mt[0] = seed;
  for (int i = 1; i < 624; i++)
    r->mt[i] = 1812433253u * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (uint32_t)i;
  r->idx = 624;
  r->has_saved = 0;
  r->saved = 0.0;
}

static void mt_regenerate(uint32_t *mt) {
  for (int i = 0; i < 624; i++) {
    const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
    uint32_t v = mt[(i + 397) % 624] ^ (y >> 1);
    if (y & 1u)
      v ^= 0x9908b0dfu;
    mt[i] = v;
  }
}

uint32_t ko_rng_u32(ko_rng *r) {
  if (r->idx >= 624) {
    mt_regenerate(r->mt);
    r->idx = 0;
  }
  uint32_t y = r->mt[r->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

static double rng_canonical(ko_rng *r) {
  const double lo = (double)ko_rng_u32(r);
  const double hi = (double)ko_rng_u32(r);
  const double sum = lo + hi * 4294967296.0;
  double u = sum / 18446744073709551616.0;
  if (u >= 1.0)
    u = nextafter(1.0, 0.0);
  return u;
}

double ko_rng_normal(ko_rng *r) {
  if (r->has_saved) {
    r->has_saved = 0;
    return r->saved;
  }
  double x, y, r2;
  do {
    x = 2.0 * rng_canonical(r) - 1.0;
    y = 2.0 * rng_canonical(r) - 1.0;
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0.0);
  const double mult = sqrt(-2.0 * log(r2) / r2);
  r->saved = x * mult;
  r->has_saved = 1;
  return y * mult;
}

void ko_rng_fill_normal(ko_rng *r, double *x, int64_t n) {
  for (int64_t i = 0; i < n; i++)
    x[i] = ko_rng_normal(r);
}

/* ======================================================================== */
/* CSR SpMV: y = A x (trans=0) or y = A^T x through the stored transpose.   */
/* Sum order per row follows the stored column order.                       */
/* ======================================================================== */
void ko_spmv(const ko_csr *A, int trans, const double *x, double *y) {
  const int64_t rows = trans ? A->n : A->m;
  const int32_t *rp = trans ? A->rpT : A->rp;
  const int32_t *ci = trans ? A->ciT : A->ci;
  const double *v = trans ? A->vT : A->v;
  for (int64_t i = 0; i < rows; i++) {
    double s = 0.0;
    for (int32_t k = rp[i]; k < rp[i + 1]; k++)
      s += v[k] * x[ci[k]];
    y[i] = s;
  }
}

/* ---- BLAS-1 in the StdVectorAdapter order -------------------------------- */
static double vdot(int64_t n, const double *a, const double *b) {
  double s = 0.0;
  for (int64_t i = 0; i < n; i++)
    s += a[i] * b[i];
  return s;
}
static double vnorm(int64_t n, const double *a) {
  double s = 0.0;
  for (int64_t i = 0; i < n; i++)
    s += a[i] * a[i];
  return sqrt(s);
}
/* this <- this + alpha * other (VectorInterface::add_scaled) */
static void vaxpy(int64_t n, double alpha, const double *x, double *y) {
  for (int64_t i = 0; i < n; i++)
    y[i] += alpha * x[i];
}
static void vscale(int64_t n, double alpha, double *x) {
  for (int64_t i = 0; i < n; i++)
    x[i] *= alpha;
}
static void vcopy(int64_t n, const double *src, double *dst) {
  memcpy(dst, src, (size_t)n * sizeof(double));
}
static void vzero(int64_t n, double *x) { memset(x, 0, (size_t)n * sizeof(double)); }
static double *dvec(int64_t n) {
  double *p = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  return p;
}

/* ---- operator wrapper (plain or TransposedMatrix, CyclicLanczosSolver.cpp:266-281) */
typedef struct op_t {
  const ko_csr *A;
  int trans;
  int64_t *spmv, *spmvT; /* counters on the underlying A */
} op_t;
static int64_t op_rows(const op_t *o) { return o->trans ? o->A->n : o->A->m; }
static int64_t op_cols(const op_t *o) { return o->trans ? o->A->m : o->A->n; }
static void op_mul(const op_t *o, const double *x, double *y) {
  if (o->trans)
    (*o->spmvT)++;
  else
    (*o->spmv)++;
  ko_spmv(o->A, o->trans, x, y);
}
static void op_mulT(const op_t *o, const double *x, double *y) {
  if (o->trans)
    (*o->spmv)++;
  else
    (*o->spmvT)++;
  ko_spmv(o->A, !o->trans, x, y);
}

/* ======================================================================== */
/* Small dense routines (column-major). Written from textbook methods:      */
/*  - one-sided (Hestenes) Jacobi SVD, right vectors accumulated            */
/*  - cyclic two-sided Jacobi for symmetric eigenproblems                   */
/*  - Cholesky (lower) failing on a non-positive pivot, like Eigen::LLT     */
/* ======================================================================== */
int ko_svd_right(int r, int c, const double *M, double *sv, double *V) {
  double *W = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1) * (size_t)(c > 0 ? c : 1));
  if (!W)
    return KO_ERR_NOMEM;
  memcpy(W, M, sizeof(double) * (size_t)r * (size_t)c);
  for (int j = 0; j < c; j++)
    for (int i = 0; i < c; i++)
      V[i + (size_t)j * c] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    int rotated = 0;
    for (int p = 0; p < c - 1; p++) {
      for (int q = p + 1; q < c; q++) {
        double a = 0.0, b = 0.0, g = 0.0;
        const double *wp = W + (size_t)p * r, *wq = W + (size_t)q * r;
        for (int i = 0; i < r; i++) {
          a += wp[i] * wp[i];
          b += wq[i] * wq[i];
          g += wp[i] * wq[i];
        }
        if (g == 0.0 || fabs(g) <= 1e-15 * sqrt(a * b))
          continue;
        rotated = 1;
        const double zeta = (b - a) / (2.0 * g);
        const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        double *Wp = W + (size_t)p * r, *Wq = W + (size_t)q * r;
        for (int i = 0; i < r; i++) {
          const double x = Wp[i], y = Wq[i];
          Wp[i] = cs * x - sn * y;
          Wq[i] = sn * x + cs * y;
        }
        double *Vp = V + (size_t)p * c, *Vq = V + (size_t)q * c;
        for (int i = 0; i < c; i++) {
          const double x = Vp[i], y = Vq[i];
          Vp[i] = cs * x - sn * y;
          Vq[i] = sn * x + cs * y;
        }
      }
    }
    if (!rotated)
      break;
  }
  for (int j = 0; j < c; j++) {
    double s = 0.0;
    for (int i = 0; i < r; i++)
      s += W[i + (size_t)j * r] * W[i + (size_t)j * r];
    sv[j] = sqrt(s);
  }
  free(W);
  return KO_OK;
}

/* eigenvalues ascending, eigenvectors in the columns of Q */
int ko_sym_eig(int n, const double *A0, double *w, double *Q) {
  double *A = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * (size_t)(n > 0 ? n : 1));
  if (!A)
    return KO_ERR_NOMEM;
  memcpy(A, A0, sizeof(double) * (size_t)n * (size_t)n);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++)
      Q[i + (size_t)j * n] = (i == j) ? 1.0 : 0.0;
  double fro = 0.0;
  for (size_t i = 0; i < (size_t)n * n; i++)
    fro += A[i] * A[i];
  fro = sqrt(fro);
  if (!isfinite(fro)) {
    free(A);
    for (int i = 0; i < n; i++)
      w[i] = NAN;
    return KO_ERR_RUNTIME;
  }
  for (int sweep = 0; sweep < 100; sweep++) {
    int rotated = 0;
    for (int p = 0; p < n - 1; p++) {
      for (int q = p + 1; q < n; q++) {
        const double apq = A[p + (size_t)q * n];
        const double app = A[p + (size_t)p * n], aqq = A[q + (size_t)q * n];
        if (fabs(apq) <= fmax(1e-18 * fro, 1e-16 * sqrt(fabs(app * aqq))) || apq == 0.0)
          continue;
        rotated = 1;
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = copysign(1.0, theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; k++) { /* columns p,q */
          const double akp = A[k + (size_t)p * n], akq = A[k + (size_t)q * n];
          A[k + (size_t)p * n] = c * akp - s * akq;
          A[k + (size_t)q * n] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) { /* rows p,q */
          const double apk = A[p + (size_t)k * n], aqk = A[q + (size_t)k * n];
          A[p + (size_t)k * n] = c * apk - s * aqk;
          A[q + (size_t)k * n] = s * apk + c * aqk;
        }
        A[p + (size_t)q * n] = 0.0;
        A[q + (size_t)p * n] = 0.0;
        for (int k = 0; k < n; k++) {
          const double qkp = Q[k + (size_t)p * n], qkq = Q[k + (size_t)q * n];
          Q[k + (size_t)p * n] = c * qkp - s * qkq;
          Q[k + (size_t)q * n] = s * qkp + c * qkq;
        }
      }
    }
    if (!rotated)
      break;
  }
  /* sort ascending (stable selection on a copy) */
  int *ord = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  double *Qs = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++)
    ord[i] = i;
  for (int i = 1; i < n; i++) { /* insertion sort: stable */
    int key = ord[i], j = i - 1;
    while (j >= 0 && A[ord[j] + (size_t)ord[j] * n] > A[key + (size_t)key * n]) {
      ord[j + 1] = ord[j];
      j--;
    }
    ord[j + 1] = key;
  }
  for (int j = 0; j < n; j++) {
    w[j] = A[ord[j] + (size_t)ord[j] * n];
    memcpy(Qs + (size_t)j * n, Q + (size_t)ord[j] * n, sizeof(double) * (size_t)n);
  }
  memcpy(Q, Qs, sizeof(double) * (size_t)n * (size_t)n);
  free(Qs);
  free(ord);
  free(A);
  return KO_OK;
}

/* Cholesky of the lower triangle; returns 0 on success. Fails when a pivot
 * is <= 0 (a NaN pivot passes through, as in Eigen's LLT). */
static int cholesky_lower(int n, double *A) {
  for (int k = 0; k < n; k++) {
    double x = A[k + (size_t)k * n];
    for (int j = 0; j < k; j++)
      x -= A[k + (size_t)j * n] * A[k + (size_t)j * n];
    if (x <= 0.0)
      return k + 1;
    x = sqrt(x);
    A[k + (size_t)k * n] = x;
    for (int i = k + 1; i < n; i++) {
      double s = A[i + (size_t)k * n];
      for (int j = 0; j < k; j++)
        s -= A[i + (size_t)j * n] * A[k + (size_t)j * n];
      A[i + (size_t)k * n] = s / x;
    }
  }
  for (int j = 0; j < n; j++)
    for (int i = 0; i < j; i++)
      A[i + (size_t)j * n] = 0.0;
  return 0;
}

/* inverse of a lower-triangular L (forward substitution per column) */
static void lower_inverse(int n, const double *L, double *Li) {
  for (int j = 0; j < n; j++) {
    for (int i = 0; i < n; i++) {
      if (i < j) {
        Li[i + (size_t)j * n] = 0.0;
        continue;
      }
      double s = (i == j) ? 1.0 : 0.0;
      for (int k = j; k < i; k++)
        s -= L[i + (size_t)k * n] * Li[k + (size_t)j * n];
      Li[i + (size_t)j * n] = s / L[i + (size_t)i * n];
    }
  }
}

/* ======================================================================== */
/* Gram-Schmidt utilities (src/Utils/GramSchmidt.cpp:55-91)                 */
/* ======================================================================== */
static int mgs_ptrs(int64_t k, int64_t n, double **V, double tol, int reorth) {
  for (int64_t i = 0; i < k; i++) {
    for (int64_t j = 0; j < i; j++) {
      const double c = vdot(n, V[i], V[j]);
      vaxpy(n, -c, V[j], V[i]);
    }
    double n1 = vnorm(n, V[i]);
    if (n1 < tol)
      return 0;
    if (reorth) {
      for (int64_t j = 0; j < i; j++) {
        const double c = vdot(n, V[i], V[j]);
        vaxpy(n, -c, V[j], V[i]);
      }
      const double n2 = vnorm(n, V[i]);
      if (n2 < tol)
        return 0;
      n1 = n2;
    }
    vscale(n, 1.0 / n1, V[i]);
  }
  return 1;
}

int ko_mgs(int64_t k, int64_t n, double *V, double tol, int reorth) {
  double **P = (double **)malloc(sizeof(double *) * (size_t)(k > 0 ? k : 1));
  for (int64_t i = 0; i < k; i++)
    P[i] = V + i * n;
  const int ok = mgs_ptrs(k, n, P, tol, reorth);
  free(P);
  return ok;
}

double ko_max_pairwise_abs_dot(int64_t k, int64_t n, const double *V) {
  double m = 0.0;
  for (int64_t i = 0; i < k; i++)
    for (int64_t j = i + 1; j < k; j++)
      m = fmax(m, fabs(vdot(n, V + i * n, V + j * n)));
  return m;
}

/* ======================================================================== */
/* Subspace comparison                                                      */
/* ======================================================================== */
/* RREF of k row vectors (include/krans/Utils/SubspaceCompare.hpp:17-79) */
static void rref_rows(int64_t k, int64_t N, double **rows, double tol) {
  if (k == 0)
    return;
  int64_t pivot_row = 0;
  for (int64_t pc = 0; pc < N && pivot_row < k; pc++) {
    int64_t best = pivot_row;
    double maxv = 0.0;
    for (int64_t r = pivot_row; r < k; r++) {
      const double v = fabs(rows[r][pc]);
      if (v > maxv) {
        maxv = v;
        best = r;
      }
    }
    if (maxv < tol) {
      for (int64_t r = pivot_row; r < k; r++)
        rows[r][pc] = 0.0;
      continue;
    }
    if (best != pivot_row) {
      double *t = rows[pivot_row];
      rows[pivot_row] = rows[best];
      rows[best] = t;
    }
    const double pv = rows[pivot_row][pc];
    vscale(N, 1.0 / pv, rows[pivot_row]);
    rows[pivot_row][pc] = 1.0;
    for (int64_t r = 0; r < k; r++) {
      if (r == pivot_row)
        continue;
      const double f = rows[r][pc];
      if (fabs(f) > tol)
        vaxpy(N, -f, rows[pivot_row], rows[r]);
      rows[r][pc] = 0.0;
    }
    pivot_row++;
  }
  for (int64_t r = 0; r < k; r++)
    for (int64_t c = 0; c < N; c++)
      if (fabs(rows[r][c]) < tol)
        rows[r][c] = 0.0;
}

double ko_subspace_diff_rref(int64_t k1, int64_t k2, int64_t n, const double *B1,
                             const double *B2, double tol) {
  if (k1 == 0 && k2 == 0)
    return 0.0;
  if (k1 != k2)
    return 1e9;
  double *c1 = dvec(k1 * n), *c2 = dvec(k2 * n);
  double **r1 = (double **)malloc(sizeof(double *) * (size_t)k1);
  double **r2 = (double **)malloc(sizeof(double *) * (size_t)k2);
  memcpy(c1, B1, sizeof(double) * (size_t)(k1 * n));
  memcpy(c2, B2, sizeof(double) * (size_t)(k2 * n));
  for (int64_t i = 0; i < k1; i++) {
    r1[i] = c1 + i * n;
    r2[i] = c2 + i * n;
  }
  rref_rows(k1, n, r1, tol);
  rref_rows(k2, n, r2, tol);
  double sum_sq = 0.0;
  for (int64_t i = 0; i < k1; i++) {
    vaxpy(n, -1.0, r2[i], r1[i]);
    const double nn = vnorm(n, r1[i]);
    sum_sq += nn * nn;
  }
  free(r1);
  free(r2);
  free(c1);
  free(c2);
  return sqrt(sum_sq);
}

double ko_subspace_dist(int64_t ku, int64_t kv, int64_t n, const double *U, const double *V) {
  if (ku != kv)
    return 1.0;
  if (kv == 0)
    return 0.0;
  double *E = dvec(kv * n);
  memcpy(E, V, sizeof(double) * (size_t)(kv * n));
  for (int64_t i = 0; i < kv; i++)
    for (int64_t j = 0; j < ku; j++) {
      const double c = vdot(n, V + i * n, U + j * n);
      vaxpy(n, -c, U + j * n, E + i * n);
    }
  const int k = (int)kv;
  double *G = dvec((int64_t)k * k), *w = dvec(k), *Q = dvec((int64_t)k * k);
  for (int i = 0; i < k; i++)
    for (int j = 0; j < k; j++)
      G[i + (size_t)j * k] = vdot(n, E + (int64_t)i * n, E + (int64_t)j * n);
  ko_sym_eig(k, G, w, Q);
  const double lmax = w[k - 1] > 0.0 ? w[k - 1] : 0.0;
  free(G);
  free(w);
  free(Q);
  free(E);
  return sqrt(lmax);
}

/* ======================================================================== */
/* Cyclic Lanczos (src/Solvers/CyclicLanczosSolver.cpp)                     */
/* ======================================================================== */
void ko_cyclic_opts_default(ko_cyclic_opts *o) {
  memset(o, 0, sizeof *o);
  o->k = 1;
  o->ncv = 48;
  o->max_restarts = 80;
  o->tol_abs = 1e-12;
  o->tol_rel = 1e-10;
  o->reorth = 2;
  o->use_harmonic = 1;
  o->target_tau = 0.0;
  o->nullity_known = -1;
  o->rank_known = -1;
  o->cg_maxit = 80;
  o->cg_rel_tol = 1e-10;
  o->cg_breakdown_tol = 1e-30;
  o->projector_passes = 1;
  o->grad_max_iters = 3000;
  o->frob_samples = 4;
  o->prescreen_factor = 0.8;
  o->stagnation_restarts = 30;
}

/* Hutchinson estimate of ||A||_F (CyclicLanczosSolver.cpp:115-127) */
static double fro_est(const op_t *A, ko_rng *rng, int64_t samples) {
  const int64_t m = op_rows(A), n = op_cols(A);
  if (samples < 1)
    samples = 1;
  double *r = dvec(n), *Ar = dvec(m);
  double sum2 = 0.0;
  for (int64_t s = 0; s < samples; s++) {
    ko_rng_fill_normal(rng, r, n);
    op_mul(A, r, Ar);
    const double nr = vnorm(m, Ar);
    sum2 += nr * nr;
  }
  free(r);
  free(Ar);
  return sqrt(sum2 / (double)samples);
}

/* CG on (A A^T) w = rhs (CyclicLanczosSolver.cpp:48-113) */
typedef struct cg_ret {
  int64_t its;
  double rnorm;
} cg_ret;
static cg_ret cg_normal_eq(const op_t *A, const double *rhs, double *w, ko_precond_fn M,
                           void *Mu, int64_t maxit, double rel_tol, double bd_tol) {
  const int64_t m = op_rows(A), n = op_cols(A);
  cg_ret ret = {0, 0.0};
  double *r = dvec(m), *z = dvec(m), *p = dvec(m), *Ap = dvec(m), *tn = dvec(n);
  vzero(m, w);
  vcopy(m, rhs, r);
  const double rr = vdot(m, r, r);
  const double rhsn = sqrt(rr > 0.0 ? rr : 0.0);
  if (!(rhsn > 0.0) || !isfinite(rhsn)) {
    ret.rnorm = rhsn;
    goto done;
  }
  if (M)
    M(Mu, r, z);
  else
    vcopy(m, r, z);
  vcopy(m, z, p);
  double rz = vdot(m, r, z);
  if (!(rz > 0.0) || !isfinite(rz)) {
    ret.rnorm = rhsn;
    goto done;
  }
  double rnorm = sqrt(rz);
  const double tol = fmax(rel_tol * rnorm, 1e-30);
  if (rnorm <= tol) {
    ret.rnorm = rnorm;
    goto done;
  }
  int64_t k = 0;
  for (; k < maxit; ++k) {
    op_mulT(A, p, tn);
    op_mul(A, tn, Ap);
    const double pAp = vdot(m, p, Ap);
    if (!isfinite(pAp) || fabs(pAp) <= bd_tol)
      break;
    const double alpha = rz / pAp;
    vaxpy(m, alpha, p, w);
    vaxpy(m, -alpha, Ap, r);
    if (M)
      M(Mu, r, z);
    else
      vcopy(m, r, z);
    const double rz_new = vdot(m, r, z);
    if (!isfinite(rz_new))
      break;
    rnorm = sqrt(rz_new > 0.0 ? rz_new : 0.0);
    if (rnorm <= tol) {
      ++k;
      break;
    }
    const double beta = rz_new / fmax(1e-300, rz);
    rz = rz_new;
    vscale(m, beta, p);
    vaxpy(m, 1.0, z, p);
  }
  ret.its = k;
  ret.rnorm = rnorm;
done:
  free(r);
  free(z);
  free(p);
  free(Ap);
  free(tn);
  return ret;
}

/* two Gram-Schmidt passes against the accepted basis (CyclicLanczosSolver.cpp:324-330) */
static void gs2_basis(int64_t n, double *v, double **basis, int64_t nb) {
  for (int pass = 0; pass < 2; pass++)
    for (int64_t q = 0; q < nb; q++) {
      const double c = vdot(n, v, basis[q]);
      vaxpy(n, -c, basis[q], v);
    }
}

static void orth_pass(int64_t len, double *w, double **S, int64_t ns) {
  for (int64_t s = 0; s < ns; s++) {
    const double c = vdot(len, S[s], w);
    vaxpy(len, -c, S[s], w);
  }
}

/* randomized projector + gradient fallback (CyclicLanczosSolver.cpp:140-214) */
static int try_project_random(const op_t *A, ko_rng *rng, double tol_accept, double **basis,
                              int64_t *nb, int grad_max_iters, int frob_samples) {
  const int64_t m = op_rows(A), n = op_cols(A);
  double *v = dvec(n);
  ko_rng_fill_normal(rng, v, n);
  for (int64_t q = 0; q < *nb; q++) {
    const double c = vdot(n, v, basis[q]);
    vaxpy(n, -c, basis[q], v);
  }
  double nv = vnorm(n, v);
  int ok = 0;
  double *tm = dvec(m), *wm = dvec(m), *tn = dvec(n);
  if (nv < 1e-14)
    goto out;
  vscale(n, 1.0 / nv, v);
  op_mul(A, v, tm);
  {
    cg_ret cr = cg_normal_eq(A, tm, wm, NULL, NULL, 500, 1e-12, 1e-30);
    if (cr.its > 0 || cr.rnorm < vnorm(m, tm)) {
      op_mulT(A, wm, tn);
      vaxpy(n, -1.0, tn, v);
    }
  }
  for (int64_t q = 0; q < *nb; q++) {
    const double c = vdot(n, v, basis[q]);
    vaxpy(n, -c, basis[q], v);
  }
  nv = vnorm(n, v);
  if (nv >= 1e-14)
    vscale(n, 1.0 / nv, v);
  op_mul(A, v, tm);
  double res = vnorm(m, tm);
  if (res <= tol_accept) {
    ok = 1;
    goto accept;
  }
  {
    const double fn = fro_est(A, rng, frob_samples > 1 ? frob_samples : 1);
    const double L2 = fmax(1e-30, fn * fn);
    const double tau = 0.9 / L2;
    for (int it = 0; it < grad_max_iters && res > tol_accept; ++it) {
      op_mul(A, v, tm);
      op_mulT(A, tm, tn);
      vaxpy(n, -tau, tn, v);
      for (int64_t q = 0; q < *nb; q++) {
        const double c = vdot(n, v, basis[q]);
        vaxpy(n, -c, basis[q], v);
      }
      nv = vnorm(n, v);
      if (nv < 1e-14)
        goto out;
      vscale(n, 1.0 / nv, v);
      op_mul(A, v, tm);
      res = vnorm(m, tm);
    }
  }
  if (res <= tol_accept)
    ok = 1;
accept:
  if (ok) {
    vcopy(n, v, basis[*nb]);
    (*nb)++;
  }
out:
  free(v);
  free(tm);
  free(wm);
  free(tn);
  return ok;
}

typedef struct sortpair {
  double key;
  int idx;
} sortpair;
static void stable_sort_pairs(sortpair *a, int n) { /* insertion sort, stable */
  for (int i = 1; i < n; i++) {
    sortpair k = a[i];
    int j = i - 1;
    while (j >= 0 && a[j].key > k.key) {
      a[j + 1] = a[j];
      j--;
    }
    a[j + 1] = k;
  }
}

/* find_right_nullspace (CyclicLanczosSolver.cpp:291-616). basis_out has
 * capacity k_target vectors of length cols(A). */
static int find_right(const op_t *A, ko_rng *rng, const ko_cyclic_opts *o, double *basis_out,
                      int64_t *n_found, ko_cyclic_result *R) {
  const int64_t m = op_rows(A), n = op_cols(A);
  *n_found = 0;
  if (n == 0 || m == 0)
    return KO_OK;
  const int64_t k_target = (o->nullity_known >= 0) ? (int64_t)o->nullity_known : o->k;
  if (k_target == 0) {
    R->converged_to_target = 1;
    return KO_OK;
  }
  if (o->rank_known >= 0 && n <= (int64_t)o->rank_known)
    return KO_OK;
  int64_t ncv = o->ncv > 2 ? o->ncv : 2;
  if (ncv < k_target + 2)
    ncv = k_target + 2;

  R->frob_norm_est = fro_est(A, rng, o->frob_samples > 1 ? o->frob_samples : 1);
  const double fmx = fmax(1.0, R->frob_norm_est);
  const double accept = fmax(o->tol_abs, o->tol_rel * fmx);
  const double prescreen = fmax(0.0, o->prescreen_factor) * fmx;

  double **basis = (double **)malloc(sizeof(double *) * (size_t)k_target);
  for (int64_t i = 0; i < k_target; i++)
    basis[i] = basis_out + i * n;
  int64_t nb = 0;

  const int64_t cap = ncv / 2 + 2;
  double **Y = (double **)malloc(sizeof(double *) * (size_t)cap);
  double **X = (double **)malloc(sizeof(double *) * (size_t)cap);
  for (int64_t i = 0; i < cap; i++) {
    Y[i] = dvec(n);
    X[i] = dvec(m);
  }
  double *alpha = dvec(ncv + 1), *beta = dvec(ncv + 1);
  double *y0 = dvec(n), *best_v = dvec(n), *v = dvec(n), *vp = dvec(n);
  double *tm = dvec(m), *wm = dvec(m), *tn = dvec(n);
  double *wx = dvec(m), *wy = dvec(n);
  int have_best = 0;
  const int L = (int)ncv;
  double *Tb = dvec((int64_t)(L + 1) * L), *sv = dvec(L), *Vv = dvec((int64_t)L * L);
  sortpair *ord = (sortpair *)malloc(sizeof(sortpair) * (size_t)(L > 0 ? L : 1));

  if (o->initial_right)
    vcopy(n, o->initial_right, y0);
  else
    ko_rng_fill_normal(rng, y0, n);

  int64_t restarts_since_accept = 0;
  for (int64_t restart = 0; restart < o->max_restarts; ++restart) {
    R->restarts = restart;
    int64_t na = 0, nbeta = 0;

    gs2_basis(n, y0, basis, nb);
    double ny = vnorm(n, y0);
    if (!isfinite(ny) || ny < 1e-14) {
      ko_rng_fill_normal(rng, y0, n); /* random_right() */
      gs2_basis(n, y0, basis, nb);
      ny = vnorm(n, y0);
      if (!(ny >= 1e-14))
        break;
    }
    vscale(n, 1.0 / ny, y0);
    int64_t nY = 0, nX = 0;
    vcopy(n, y0, Y[nY++]);

    int64_t local_steps = 0;
    double beta_last = 0.0;
    for (int64_t j = 0; j < ncv; ++j) {
      const int from_y = nY > nX;
      double *w = from_y ? wx : wy;
      if (from_y) {
        op_mul(A, Y[nY - 1], w);
        if (nbeta > 0)
          vaxpy(m, -beta[nbeta - 1], X[nX - 1], w);
      } else {
        op_mulT(A, X[nX - 1], w);
        vaxpy(n, -beta[nbeta - 1], Y[nY - 1], w);
      }
      for (int pass = 0; pass < o->reorth; ++pass) {
        if (from_y) {
          orth_pass(m, w, X, nX);
        } else {
          orth_pass(n, w, basis, nb);
          orth_pass(n, w, Y, nY);
        }
      }
      const int64_t len = from_y ? m : n;
      const double bj = sqrt(vdot(len, w, w));
      alpha[na++] = 0.0;
      beta_last = bj;
      if (!isfinite(bj) || bj < 1e-14 || nY + nX >= ncv)
        break;
      beta[nbeta++] = bj;
      double *dst = from_y ? X[nX++] : Y[nY++];
      vcopy(len, w, dst);
      vscale(len, 1.0 / bj, dst);
      ++local_steps;
    }
    R->krylov_steps_total += local_steps;

    const int l = (int)na;
    if (l == 0 || !isfinite(beta_last))
      break;

    /* tiny problem and interior selection (CyclicLanczosSolver.cpp:428-453) */
    int finite_ok = 1;
    if (o->use_harmonic) {
      memset(Tb, 0, sizeof(double) * (size_t)(l + 1) * (size_t)l);
      for (int i = 0; i < l; i++) {
        Tb[i + (size_t)i * (l + 1)] = alpha[i] - o->target_tau;
        if (i + 1 < l) {
          Tb[i + (size_t)(i + 1) * (l + 1)] = beta[i];
          Tb[(i + 1) + (size_t)i * (l + 1)] = beta[i];
        }
      }
      Tb[l + (size_t)(l - 1) * (l + 1)] = beta_last;
      ko_svd_right(l + 1, l, Tb, sv, Vv);
      for (int i = 0; i < l; i++) {
        ord[i].key = sv[i];
        ord[i].idx = i;
      }
      stable_sort_pairs(ord, l);
    } else {
      memset(Tb, 0, sizeof(double) * (size_t)l * (size_t)l);
      for (int i = 0; i < l; i++) {
        Tb[i + (size_t)i * l] = alpha[i];
        if (i + 1 < l) {
          Tb[i + (size_t)(i + 1) * l] = beta[i];
          Tb[(i + 1) + (size_t)i * l] = beta[i];
        }
      }
      ko_sym_eig(l, Tb, sv, Vv);
      for (int i = 0; i < l; i++) {
        ord[i].key = fabs(sv[i] - o->target_tau);
        ord[i].idx = i;
      }
      stable_sort_pairs(ord, l);
    }
    for (int i = 0; i < l && finite_ok; i++) {
      if (!isfinite(sv[i]))
        finite_ok = 0;
      for (int j = 0; j < l; j++)
        if (!isfinite(Vv[i + (size_t)j * l]))
          finite_ok = 0;
    }
    if (!finite_ok) {
      ko_rng_fill_normal(rng, y0, n);
      gs2_basis(n, y0, basis, nb);
      continue;
    }

    int64_t test_cap = k_target > 8 ? k_target : 8;
    if (test_cap > l)
      test_cap = l;
    double best_res = INFINITY;
    have_best = 0;
    int accepted_this_cycle = 0;
    int64_t tested = 0;
    int polish_stalled = 0;
    for (int t = 0; t < l && tested < test_cap; ++t) {
      const int jb = ord[t].idx;
      double c_even2 = 0.0;
      for (int i = 0; i < l; i += 2)
        c_even2 += Vv[i + (size_t)jb * l] * Vv[i + (size_t)jb * l];
      if (!(c_even2 >= 1e-20))
        continue;
      vzero(n, v);
      for (int i = 0; i < l; i += 2)
        vaxpy(n, Vv[i + (size_t)jb * l], Y[i / 2], v);
      gs2_basis(n, v, basis, nb);
      double nv = vnorm(n, v);
      if (!isfinite(nv) || nv < 1e-8)
        continue;
      vscale(n, 1.0 / nv, v);
      ++tested;

      op_mul(A, v, tm);
      double res = vnorm(m, tm);
      if (!isfinite(res))
        continue;
      if (res > prescreen || polish_stalled) {
        if (res < best_res) {
          best_res = res;
          vcopy(n, v, best_v);
          have_best = 1;
        }
        continue;
      }
      int64_t cg_its = 0;
      int hit_maxit = 0;
      const int passes = o->projector_passes > 1 ? o->projector_passes : 1;
      for (int pass = 0; pass < passes && res > accept; ++pass) {
        cg_its = cg_normal_eq(A, tm, wm, o->precond_AAt, o->precond_user, o->cg_maxit,
                              o->cg_rel_tol, o->cg_breakdown_tol)
                     .its;
        ++R->cg_solves;
        if (cg_its >= o->cg_maxit) {
          ++R->cg_maxit_hits;
          hit_maxit = 1;
        }
        op_mulT(A, wm, tn);
        vcopy(n, v, vp);
        vaxpy(n, -1.0, tn, vp);
        gs2_basis(n, vp, basis, nb);
        const double np = vnorm(n, vp);
        if (!isfinite(np) || np < 1e-14)
          break;
        vscale(n, 1.0 / np, vp);
        op_mul(A, vp, wm);
        const double res_p = vnorm(m, wm);
        if (!(res_p < res))
          break;
        vcopy(n, vp, v);
        res = res_p;
        vcopy(m, wm, tm);
      }
      if (o->verbose)
        fprintf(stderr, "[oracle cyclic] restart=%lld res=%.3e accept=%.3e cg_its=%lld\n",
                (long long)restart, res, accept, (long long)cg_its);
      if (res <= accept) {
        vcopy(n, v, basis[nb++]);
        accepted_this_cycle = 1;
        if (nb >= k_target) {
          R->converged_to_target = 1;
          goto finish;
        }
      } else {
        polish_stalled = polish_stalled || hit_maxit;
        if (res < best_res) {
          best_res = res;
          vcopy(n, v, best_v);
          have_best = 1;
        }
      }
    }

    if (!accepted_this_cycle) {
      ++restarts_since_accept;
      if (o->stagnation_restarts > 0 && restarts_since_accept >= o->stagnation_restarts)
        break;
    } else {
      restarts_since_accept = 0;
    }
    if (have_best) {
      vcopy(n, best_v, y0);
    } else {
      ko_rng_fill_normal(rng, y0, n);
      gs2_basis(n, y0, basis, nb);
    }
  }

  if (nb < k_target) {
    int64_t failures = 0;
    while (nb < k_target && failures < 8) {
      if (try_project_random(A, rng, accept, basis, &nb, o->grad_max_iters, o->frob_samples))
        failures = 0;
      else
        ++failures;
    }
    R->converged_to_target = nb >= k_target;
  }

finish:
  *n_found = nb;
  for (int64_t i = 0; i < cap; i++) {
    free(Y[i]);
    free(X[i]);
  }
  free(Y);
  free(X);
  free(alpha);
  free(beta);
  free(y0);
  free(best_v);
  free(v);
  free(vp);
  free(tm);
  free(wm);
  free(tn);
  free(wx);
  free(wy);
  free(Tb);
  free(sv);
  free(Vv);
  free(ord);
  free(basis);
  return KO_OK;
}

/* find_nullspace_cyclic_lanczos_ex (CyclicLanczosSolver.cpp:618-660) */
int ko_cyclic(const ko_csr *Am, ko_rng *rng, const ko_cyclic_opts *o, double *right_out,
              double *left_out, ko_cyclic_result *res) {
  memset(res, 0, sizeof *res);
  op_t A = {Am, 0, &res->spmv, &res->spmvT};
  int64_t nr = 0;
  int rc = find_right(&A, rng, o, right_out, &nr, res);
  res->n_right = nr;
  if (rc != KO_OK)
    return rc;
  if (!o->return_left_space || Am->m == 0 || Am->n == 0)
    return KO_OK;
  ko_cyclic_opts lo;
  ko_cyclic_opts_default(&lo);
  lo.k = o->k;
  lo.ncv = o->ncv;
  lo.max_restarts = o->max_restarts;
  lo.tol_abs = o->tol_abs;
  lo.tol_rel = o->tol_rel;
  lo.reorth = o->reorth;
  lo.use_harmonic = o->use_harmonic;
  lo.target_tau = o->target_tau;
  lo.cg_maxit = o->cg_maxit;
  lo.cg_rel_tol = o->cg_rel_tol;
  lo.cg_breakdown_tol = o->cg_breakdown_tol;
  lo.projector_passes = o->projector_passes;
  lo.grad_max_iters = o->grad_max_iters;
  lo.frob_samples = o->frob_samples;
  lo.prescreen_factor = o->prescreen_factor;
  lo.stagnation_restarts = o->stagnation_restarts;
  lo.verbose = o->verbose;
  lo.rank_known = o->rank_known;
  if (o->rank_known >= 0) {
    int left_nullity = (int)Am->m - o->rank_known;
    int kk = (int)o->k;
    int v = left_nullity < kk ? left_nullity : kk;
    lo.nullity_known = v > 0 ? v : 0;
  }
  op_t At = {Am, 1, &res->spmv, &res->spmvT};
  ko_cyclic_result L;
  memset(&L, 0, sizeof L);
  L.spmv = 0;
  int64_t nl = 0;
  /* the left run shares the counters of the underlying A */
  rc = find_right(&At, rng, &lo, left_out, &nl, &L);
  res->n_left = nl;
  res->cg_solves += L.cg_solves;
  res->cg_maxit_hits += L.cg_maxit_hits;
  return rc;
}

/* ======================================================================== */
/* LOBPCG (src/Solvers/LOBPCGSolver.cpp)                                    */
/* ======================================================================== */
void ko_lobpcg_opts_default(ko_lobpcg_opts *o) {
  memset(o, 0, sizeof *o);
  o->nev = 1;
  o->block_size = 0;
  o->max_iters = 1000;
  o->tol_abs = 1e-12;
  o->tol_rel = 1e-10;
  o->soft_locking = 1;
  o->restart = 0.9;
  o->gs_tol = 1e-14;
  o->gs_reorth = 1;
  o->frob_samples = 4;
  o->max_tiny_dim = 0;
  o->nullity_known = -1;
  o->rank_known = -1;
}

/* a dense small matrix */
typedef struct dmat {
  int r, c;
  double *a; /* col-major */
} dmat;
static dmat dm_new(int r, int c) {
  dmat d = {r, c, dvec((int64_t)(r > 0 ? r : 1) * (c > 0 ? c : 1))};
  return d;
}
static void dm_free(dmat *d) {
  free(d->a);
  d->a = NULL;
}
#define DM(d, i, j) ((d).a[(size_t)(i) + (size_t)(j) * (size_t)(d).r])

/* AZ := A^T (A Z) column by column (LOBPCGSolver.cpp:54-64) */
static void apply_normal(const op_t *A, double **Z, int64_t k, double **AZ, double *tmp_m) {
  for (int64_t j = 0; j < k; j++) {
    op_mul(A, Z[j], tmp_m);
    op_mulT(A, tmp_m, AZ[j]);
  }
}

/* S = Z^T Z, G = Z^T AZ (LOBPCGSolver.cpp:67-80) */
static void form_gram(int64_t n, double **Z, double **AZ, int k, dmat *S, dmat *G) {
  for (int j = 0; j < k; j++)
    for (int i = 0; i <= j; i++) {
      const double sij = vdot(n, Z[i], Z[j]);
      const double gij = vdot(n, Z[i], AZ[j]);
      DM(*S, i, j) = DM(*S, j, i) = sij;
      DM(*G, i, j) = DM(*G, j, i) = gij;
    }
}

/* solve_tiny_gep (LOBPCGSolver.cpp:88-119): theta ascending (k), Y (k x k) */
static int solve_tiny_gep(int k, dmat *G, dmat *S, double *theta, dmat *Y) {
  for (int j = 0; j < k; j++)
    for (int i = 0; i < k; i++) {
      if (i < j)
        continue;
      const double g = 0.5 * (DM(*G, i, j) + DM(*G, j, i));
      const double s = 0.5 * (DM(*S, i, j) + DM(*S, j, i));
      DM(*G, i, j) = DM(*G, j, i) = g;
      DM(*S, i, j) = DM(*S, j, i) = s;
    }
  double sn = 0.0;
  for (size_t i = 0; i < (size_t)k * k; i++)
    sn += S->a[i] * S->a[i];
  const double s_norm = fmax(1.0, sqrt(sn));
  const double jit[4] = {0.0, 1e-14, 1e-12, 1e-10};
  dmat Sj = dm_new(k, k), Li = dm_new(k, k), T = dm_new(k, k), C = dm_new(k, k), Q = dm_new(k, k);
  int ok = 0;
  for (int t = 0; t < 4 && !ok; t++) {
    memcpy(Sj.a, S->a, sizeof(double) * (size_t)k * k);
    if (jit[t] > 0.0)
      for (int i = 0; i < k; i++)
        DM(Sj, i, i) += jit[t] * s_norm;
    if (cholesky_lower(k, Sj.a) != 0)
      continue;
    lower_inverse(k, Sj.a, Li.a);
    /* C = Li * G * Li^T */
    for (int j = 0; j < k; j++)
      for (int i = 0; i < k; i++) {
        double s = 0.0;
        for (int p = 0; p < k; p++)
          s += DM(Li, i, p) * DM(*G, p, j);
        DM(T, i, j) = s;
      }
    for (int j = 0; j < k; j++)
      for (int i = 0; i < k; i++) {
        double s = 0.0;
        for (int p = 0; p < k; p++)
          s += DM(T, i, p) * DM(Li, j, p);
        DM(C, i, j) = s;
      }
    if (ko_sym_eig(k, C.a, theta, Q.a) != KO_OK)
      continue;
    int fin = 1;
    for (int i = 0; i < k; i++)
      if (!isfinite(theta[i]))
        fin = 0;
    if (!fin)
      continue;
    /* Y = Li^T Q */
    for (int j = 0; j < k; j++)
      for (int i = 0; i < k; i++) {
        double s = 0.0;
        for (int p = 0; p < k; p++)
          s += DM(Li, p, i) * DM(Q, p, j);
        DM(*Y, i, j) = s;
      }
    ok = 1;
  }
  dm_free(&Sj);
  dm_free(&Li);
  dm_free(&T);
  dm_free(&C);
  dm_free(&Q);
  if (!ok) {
    set_err("LOBPCG tiny GEP: S not SPD (after jitter)");
    return KO_ERR_RUNTIME;
  }
  return KO_OK;
}

/* out[i] = sum_j Y(j,i) Z[j], skipping zero coefficients (LOBPCGSolver.cpp:122-134).
 * Y is read with row offset roff within a dmat. */
static void combine_columns(int64_t n, double **Z, int zc, const dmat *Y, int roff, int p,
                            double **out) {
  for (int i = 0; i < p; i++) {
    vzero(n, out[i]);
    for (int j = 0; j < zc; j++) {
      const double c = DM(*Y, roff + j, i);
      if (c != 0.0)
        vaxpy(n, c, Z[j], out[i]);
    }
  }
}

/* orthonormalize_block (LOBPCGSolver.cpp:137-160). Modifies X in place;
 * on failure X may be partially modified, as in the reference. */
static int orthonormalize_block(int64_t n, double **X, int64_t k, double **basis, int64_t nb,
                                double tol, int reorth) {
  for (int64_t i = 0; i < k; i++) {
    for (int64_t q = 0; q < nb; q++) {
      const double c = vdot(n, X[i], basis[q]);
      vaxpy(n, -c, basis[q], X[i]);
    }
    const double nrm = vnorm(n, X[i]);
    if (nrm < tol)
      return 0;
    vscale(n, 1.0 / nrm, X[i]);
  }
  /* MGS on clones; copied back only on success */
  double **tmp = (double **)malloc(sizeof(double *) * (size_t)(k > 0 ? k : 1));
  for (int64_t i = 0; i < k; i++) {
    tmp[i] = dvec(n);
    vcopy(n, X[i], tmp[i]);
  }
  const int indep = mgs_ptrs(k, n, tmp, tol, reorth);
  if (indep)
    for (int64_t i = 0; i < k; i++)
      vcopy(n, tmp[i], X[i]);
  for (int64_t i = 0; i < k; i++)
    free(tmp[i]);
  free(tmp);
  return indep;
}

static void project_out(int64_t n, double **basis, int64_t nb, double *x) {
  for (int64_t q = 0; q < nb; q++) {
    const double c = vdot(n, x, basis[q]);
    if (c != 0.0)
      vaxpy(n, -c, basis[q], x);
  }
}

/* two_vec_rr_sharpen (LOBPCGSolver.cpp:199-278) */
static int two_vec_rr_sharpen(const op_t *A, double **V, int64_t k, int64_t idx, double target,
                              ko_precond_fn M, void *Mu, int max_iters) {
  if (idx >= k)
    return 1;
  const int64_t m = op_rows(A), n = op_cols(A);
  double *Av = dvec(m), *t = dvec(n), *d = dvec(n), *Ad = dvec(m), *Nd = dvec(n),
         *vn = dvec(n);
  double **basis = (double **)malloc(sizeof(double *) * (size_t)(k > 0 ? k : 1));
  int64_t nb = 0;
  for (int64_t j = 0; j < k; j++)
    if (j != idx) {
      basis[nb] = dvec(n);
      vcopy(n, V[j], basis[nb]);
      nb++;
    }
  int ret = 0;
  for (int it = 0; it < max_iters; ++it) {
    op_mul(A, V[idx], Av);
    const double res = vnorm(m, Av);
    if (res <= target) {
      ret = 1;
      break;
    }
    op_mulT(A, Av, t);
    if (M)
      M(Mu, t, d);
    else
      vcopy(n, t, d);
    project_out(n, basis, nb, d);
    const double nd = vnorm(n, d);
    if (nd <= 1e-14)
      break;
    vscale(n, 1.0 / fmax(nd, 1e-300), d);
    op_mul(A, d, Ad);
    vcopy(n, t, Nd);
    op_mulT(A, Ad, Nd);
    const double vNv = vdot(n, V[idx], t);
    const double vNd = vdot(n, V[idx], Nd);
    const double dNv = vdot(n, d, t);
    const double dNd = vdot(n, d, Nd);
    /* symmetric 2x2 [[vNv, g],[g, dNd]] with g the averaged off-diagonal */
    const double a = vNv, g = 0.5 * (dNv + vNd), e = dNd;
    double y0, y1;
    if (g == 0.0) {
      if (a <= e) {
        y0 = 1.0;
        y1 = 0.0;
      } else {
        y0 = 0.0;
        y1 = 1.0;
      }
    } else {
      const double theta = (e - a) / (2.0 * g);
      const double tt = copysign(1.0, theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(tt * tt + 1.0), s = tt * c;
      const double lp = a - tt * g, lq = e + tt * g; /* eigenvalues for (c,-s), (s,c) */
      if (lp <= lq) {
        y0 = c;
        y1 = -s;
      } else {
        y0 = s;
        y1 = c;
      }
    }
    if (!isfinite(y0) || !isfinite(y1))
      break;
    vcopy(n, V[idx], vn);
    vscale(n, y0, vn);
    vaxpy(n, y1, d, vn);
    project_out(n, basis, nb, vn);
    const double nv = vnorm(n, vn);
    if (nv <= 1e-14)
      break;
    vscale(n, 1.0 / nv, vn);
    vcopy(n, vn, V[idx]);
  }
  for (int64_t j = 0; j < nb; j++)
    free(basis[j]);
  free(basis);
  free(Av);
  free(t);
  free(d);
  free(Ad);
  free(Nd);
  free(vn);
  return ret;
}

/* block_rr_polish (LOBPCGSolver.cpp:286-440) */
static int block_rr_polish(const op_t *A, ko_rng *rng, double **V, int64_t k, double target,
                           int max_sweeps, ko_precond_fn M, void *Mu) {
  if (k == 0)
    return KO_OK;
  const int64_t m = op_rows(A), n = op_cols(A);
  double *r = dvec(m), *g = dvec(n), *gp = dvec(n), *tmp = dvec(m);
  double **Vb = (double **)malloc(sizeof(double *) * (size_t)k);
  double **D = (double **)malloc(sizeof(double *) * (size_t)(k + 2));
  double **Z = (double **)malloc(sizeof(double *) * (size_t)(2 * k + 2));
  double **AZ = (double **)malloc(sizeof(double *) * (size_t)(2 * k + 2));
  double **Vn = (double **)malloc(sizeof(double *) * (size_t)k);
  for (int64_t i = 0; i < k; i++) {
    Vb[i] = dvec(n);
    Vn[i] = dvec(n);
  }
  for (int64_t i = 0; i < k + 2; i++)
    D[i] = dvec(n);
  for (int64_t i = 0; i < 2 * k + 2; i++)
    AZ[i] = dvec(n);
  int rc = KO_OK;
  mgs_ptrs(k, n, V, 1e-14, 1);
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    double max_res = 0.0;
    for (int64_t i = 0; i < k; i++) {
      op_mul(A, V[i], r);
      max_res = fmax(max_res, vnorm(m, r));
    }
    if (max_res <= target)
      break;
    int64_t nd = 0;
    for (int64_t i = 0; i < k; i++)
      vcopy(n, V[i], Vb[i]);
    for (int64_t j = 0; j < k; j++) {
      op_mul(A, V[j], r);
      const double res = vnorm(m, r);
      if (res <= target)
        continue;
      op_mulT(A, r, g);
      if (M) {
        vcopy(n, g, gp);
        M(Mu, g, gp);
        vcopy(n, gp, g);
      }
      project_out(n, Vb, k, g);
      const double gn = vnorm(n, g);
      if (gn <= 1e-14)
        continue;
      vscale(n, 1.0 / gn, g);
      int dup = 0;
      for (int64_t q = 0; q < nd; q++)
        if (fabs(vdot(n, g, D[q])) >= 1.0 - 1e-8) {
          dup = 1;
          break;
        }
      if (!dup)
        vcopy(n, g, D[nd++]);
    }
    if (nd == 0) {
      for (int64_t i = 0; i < k; i++) {
        for (int it = 0; it < 50; ++it) {
          op_mul(A, V[i], r);
          const double res = vnorm(m, r);
          if (res <= target)
            break;
          op_mulT(A, r, g);
          for (int64_t t = 0; t < k; t++) {
            if (t == i)
              continue;
            const double c = vdot(n, g, V[t]);
            if (c != 0.0)
              vaxpy(n, -c, V[t], g);
          }
          const double gg = vdot(n, g, g);
          if (gg <= 0.0)
            break;
          op_mul(A, g, tmp);
          const double Ag2 = vdot(m, tmp, tmp);
          if (Ag2 <= 0.0)
            break;
          const double alpha = gg / Ag2;
          vaxpy(n, -alpha, g, V[i]);
          for (int64_t t = 0; t < k; t++)
            if (t != i) {
              const double c = vdot(n, V[i], V[t]);
              if (c != 0.0)
                vaxpy(n, -c, V[t], V[i]);
            }
          const double nv = vnorm(n, V[i]);
          if (nv > 0.0)
            vscale(n, 1.0 / nv, V[i]);
        }
      }
      mgs_ptrs(k, n, V, 1e-14, 1);
      const int enrich = k < 2 ? (int)k : 2;
      for (int e = 0; e < enrich; e++) {
        ko_rng_fill_normal(rng, D[nd], n);
        project_out(n, Vb, k, D[nd]);
        const double nq = vnorm(n, D[nd]);
        if (nq > 1e-14) {
          vscale(n, 1.0 / nq, D[nd]);
          nd++;
        }
      }
      if (nd > 0)
        (void)orthonormalize_block(n, D, nd, Vb, k, 1e-14, 1);
      else
        continue;
    }
    if (!orthonormalize_block(n, D, nd, Vb, k, 1e-14, 1))
      continue;
    const int64_t zc = k + nd;
    for (int64_t i = 0; i < k; i++)
      Z[i] = V[i];
    for (int64_t i = 0; i < nd; i++)
      Z[k + i] = D[i];
    apply_normal(A, Z, zc, AZ, tmp);
    dmat S = dm_new((int)zc, (int)zc), G = dm_new((int)zc, (int)zc), Y = dm_new((int)zc, (int)zc);
    double *th = dvec(zc);
    form_gram(n, Z, AZ, (int)zc, &S, &G);
    rc = solve_tiny_gep((int)zc, &G, &S, th, &Y);
    if (rc == KO_OK) {
      combine_columns(n, Z, (int)zc, &Y, 0, (int)k, Vn);
      mgs_ptrs(k, n, Vn, 1e-14, 1);
      for (int64_t i = 0; i < k; i++)
        vcopy(n, Vn[i], V[i]);
    }
    dm_free(&S);
    dm_free(&G);
    dm_free(&Y);
    free(th);
    if (rc != KO_OK)
      goto out;
    max_res = 0.0;
    for (int64_t i = 0; i < k; i++) {
      op_mul(A, V[i], r);
      max_res = fmax(max_res, vnorm(m, r));
    }
    if (max_res <= target)
      break;
  }
  mgs_ptrs(k, n, V, 1e-14, 1);
out:
  for (int64_t i = 0; i < k; i++) {
    free(Vb[i]);
    free(Vn[i]);
  }
  for (int64_t i = 0; i < k + 2; i++)
    free(D[i]);
  for (int64_t i = 0; i < 2 * k + 2; i++)
    free(AZ[i]);
  free(Vb);
  free(Vn);
  free(D);
  free(Z);
  free(AZ);
  free(r);
  free(g);
  free(gp);
  free(tmp);
  return rc;
}

static void theta_from(double *theta, int64_t bs, const double *t, int64_t tn) {
  for (int64_t j = 0; j < bs; j++)
    theta[j] = 0.0;
  const int64_t lim = tn < bs ? tn : bs;
  for (int64_t j = 0; j < lim; j++)
    theta[j] = fmax(0.0, t[j]);
}

/* find_nullspace_lobpcg_ex (LOBPCGSolver.cpp:443-834) */
int ko_lobpcg(const ko_csr *Am, ko_rng *rng, const ko_lobpcg_opts *o, double *right_out,
              double *theta_out, double *resid_out, ko_lobpcg_result *R) {
  memset(R, 0, sizeof *R);
  op_t Aop = {Am, 0, &R->spmv, &R->spmvT};
  const op_t *A = &Aop;
  const int64_t m = Am->m, n = Am->n;
  if (n == 0 || m == 0)
    return KO_OK;
  int64_t k_target = o->nev > 1 ? o->nev : 1;
  if (o->nullity_known >= 0) {
    if ((int64_t)o->nullity_known > n) {
      set_err("LOBPCG: nullity_known > n");
      return KO_ERR_INVALID_ARGUMENT;
    }
    k_target = o->nullity_known;
  }
  if (o->rank_known >= 0) {
    const int64_t rk = o->rank_known;
    if (rk > n) {
      set_err("LOBPCG: rank_known > n");
      return KO_ERR_INVALID_ARGUMENT;
    }
    const int64_t implied = n - rk;
    if (o->nullity_known >= 0 && implied != k_target) {
      set_err("LOBPCG: inconsistent rank_known vs nullity_known");
      return KO_ERR_INVALID_ARGUMENT;
    }
    if (o->nullity_known < 0)
      k_target = implied;
    if (n <= rk) {
      R->frob_norm_est = 0.0;
      R->converged_to_target = (k_target == 0);
      return KO_OK;
    }
  }
  int64_t bs = o->block_size > 0 ? o->block_size : (k_target < 16 ? (k_target > 1 ? k_target : 1) : 16);
  if (bs > n)
    bs = n;
  R->block_size = bs;
  const int64_t guards =
      (bs == 1) ? 0
                : ((int64_t)((1.0 - o->restart) * (double)bs + 0.45) < bs - 1
                       ? (int64_t)((1.0 - o->restart) * (double)bs + 0.45)
                       : bs - 1);

  R->frob_norm_est = fro_est(A, rng, o->frob_samples > 1 ? o->frob_samples : 1);
  const double accept_thr = fmax(o->tol_abs, o->tol_rel * fmax(1.0, R->frob_norm_est));
  R->accept_threshold = accept_thr;

  int rc = KO_OK;
  const int64_t kcap = k_target > 0 ? k_target : 1;
  double **Yl = (double **)malloc(sizeof(double *) * (size_t)kcap);
  double **RN = (double **)malloc(sizeof(double *) * (size_t)kcap);
  for (int64_t i = 0; i < kcap; i++) {
    Yl[i] = dvec(n);
    RN[i] = right_out ? right_out + i * n : dvec(n);
  }
  int64_t nlocked = 0, nright = 0;

  double **X = (double **)malloc(sizeof(double *) * (size_t)bs);
  double **AX = (double **)malloc(sizeof(double *) * (size_t)bs);
  double **Rb = (double **)malloc(sizeof(double *) * (size_t)bs);
  double **W = (double **)malloc(sizeof(double *) * (size_t)bs);
  double **P = (double **)malloc(sizeof(double *) * (size_t)bs);
  double **T1 = (double **)malloc(sizeof(double *) * (size_t)bs);
  double **T2 = (double **)malloc(sizeof(double *) * (size_t)bs);
  double **Zs = (double **)malloc(sizeof(double *) * (size_t)(3 * bs));
  double **AZ = (double **)malloc(sizeof(double *) * (size_t)(3 * bs));
  for (int64_t j = 0; j < bs; j++) {
    X[j] = dvec(n);
    AX[j] = dvec(n);
    Rb[j] = dvec(n);
    W[j] = dvec(n);
    P[j] = dvec(n);
    T1[j] = dvec(n);
    T2[j] = dvec(n);
  }
  for (int64_t j = 0; j < 3 * bs; j++)
    AZ[j] = dvec(n);
  double *tmp_m = dvec(m), *vacc = dvec(n);
  double *theta = dvec(bs), *th = dvec(3 * bs);

  /* initial block: seeds, then random */
  int64_t filled = 0;
  const int64_t seeds = o->initial_block ? (o->n_initial < bs ? o->n_initial : bs) : 0;
  for (; filled < seeds; ++filled)
    vcopy(n, o->initial_block + filled * n, X[filled]);
  for (; filled < bs; ++filled)
    ko_rng_fill_normal(rng, X[filled], n);
  if (!orthonormalize_block(n, X, bs, Yl, nlocked, o->gs_tol, o->gs_reorth)) {
    set_err("LOBPCG: initial block is dependent");
    rc = KO_ERR_RUNTIME;
    goto cleanup;
  }
  {
    apply_normal(A, X, bs, AX, tmp_m);
    dmat S = dm_new((int)bs, (int)bs), G = dm_new((int)bs, (int)bs), Y = dm_new((int)bs, (int)bs);
    form_gram(n, X, AX, (int)bs, &S, &G);
    rc = solve_tiny_gep((int)bs, &G, &S, th, &Y);
    if (rc == KO_OK) {
      combine_columns(n, X, (int)bs, &Y, 0, (int)bs, T1);
      for (int64_t j = 0; j < bs; j++)
        vcopy(n, T1[j], X[j]);
      apply_normal(A, X, bs, AX, tmp_m);
      theta_from(theta, bs, th, bs);
    }
    dm_free(&S);
    dm_free(&G);
    dm_free(&Y);
    if (rc != KO_OK)
      goto cleanup;
  }

  int64_t its = 0;
  while (nlocked < k_target && its < o->max_iters) {
    ++its;
    int64_t nconv = 0;
    double best_unaccepted = INFINITY;
    for (int64_t j = 0; j < bs; ++j) {
      vcopy(n, AX[j], Rb[j]);
      vaxpy(n, -theta[j], X[j], Rb[j]);
      op_mul(A, X[j], tmp_m);
      const double Av_orig = vnorm(m, tmp_m);
      if (Av_orig <= accept_thr) {
        vcopy(n, X[j], vacc);
        for (int64_t q = 0; q < nlocked; q++) {
          const double c = vdot(n, vacc, Yl[q]);
          vaxpy(n, -c, Yl[q], vacc);
        }
        const double nv = vnorm(n, vacc);
        int reject = 0;
        if (nv <= fmax(1e-14, 10.0 * o->gs_tol)) {
          reject = 1;
        } else {
          vscale(n, 1.0 / nv, vacc);
          for (int64_t q = 0; q < nlocked; q++)
            if (fabs(vdot(n, vacc, Yl[q])) >= 1.0 - 1e-8) {
              reject = 1;
              break;
            }
        }
        double Av_acc = INFINITY;
        if (!reject) {
          op_mul(A, vacc, tmp_m);
          Av_acc = vnorm(m, tmp_m);
          if (Av_acc > accept_thr)
            reject = 1;
        }
        if (!reject) {
          vcopy(n, vacc, Yl[nlocked]);
          vcopy(n, vacc, RN[nright]);
          if (theta_out)
            theta_out[nright] = theta[j];
          if (resid_out)
            resid_out[nright] = Av_acc;
          nright++;
          nlocked++;
          nconv++;
          if (o->verbose)
            fprintf(stderr, "[oracle lobpcg] accept ||Av||=%.3e locked=%lld/%lld\n", Av_acc,
                    (long long)nlocked, (long long)k_target);
          if (nlocked >= k_target)
            break;
        } else {
          best_unaccepted = fmin(best_unaccepted, Av_orig);
        }
      } else {
        best_unaccepted = fmin(best_unaccepted, Av_orig);
      }
    }
    R->locked = nlocked;
    R->iters = its;
    R->best_unaccepted_residual = isfinite(best_unaccepted) ? best_unaccepted : 0.0;
    if (nlocked >= k_target)
      break;

    const int64_t ini = o->soft_locking ? nconv : 0;
    if (nconv >= bs - guards) {
      const int64_t remain = bs - nconv;
      for (int64_t j = 0; j < remain; j++) {
        vcopy(n, X[nconv + j], X[j]);
        vcopy(n, AX[nconv + j], AX[j]);
        theta[j] = theta[nconv + j];
        vcopy(n, P[nconv + j], P[j]);
      }
      for (int64_t j = remain; j < bs; j++)
        ko_rng_fill_normal(rng, X[j], n);
      if (!orthonormalize_block(n, X, bs, Yl, nlocked, o->gs_tol, o->gs_reorth)) {
        set_err("LOBPCG: restart orthogonalization failed");
        rc = KO_ERR_RUNTIME;
        goto cleanup;
      }
      apply_normal(A, X, bs, AX, tmp_m);
      dmat S = dm_new((int)bs, (int)bs), G = dm_new((int)bs, (int)bs), Y = dm_new((int)bs, (int)bs);
      form_gram(n, X, AX, (int)bs, &S, &G);
      rc = solve_tiny_gep((int)bs, &G, &S, th, &Y);
      if (rc == KO_OK)
        theta_from(theta, bs, th, bs);
      dm_free(&S);
      dm_free(&G);
      dm_free(&Y);
      if (rc != KO_OK)
        goto cleanup;
      continue;
    }

    for (int64_t j = ini; j < bs; j++) {
      if (o->M_inv)
        o->M_inv(o->M_user, Rb[j], W[j]);
      else
        vcopy(n, Rb[j], W[j]);
    }
    {
      const int64_t na = bs - ini;
      for (int64_t t = 0; t < na; t++)
        vcopy(n, W[ini + t], T1[t]);
      if (!orthonormalize_block(n, T1, na, Yl, nlocked, o->gs_tol, o->gs_reorth)) {
        for (int64_t j = ini; j < bs; j++)
          ko_rng_fill_normal(rng, W[j], n);
        for (int64_t j = ini; j < bs; j++)
          for (int64_t q = 0; q < nlocked; q++) {
            const double c = vdot(n, W[j], Yl[q]);
            vaxpy(n, -c, Yl[q], W[j]);
          }
      } else {
        for (int64_t t = 0; t < na; t++)
          vcopy(n, T1[t], W[ini + t]);
      }
    }
    if (its > 1) {
      const int64_t na = bs - ini;
      for (int64_t t = 0; t < na; t++)
        vcopy(n, P[ini + t], T1[t]);
      (void)orthonormalize_block(n, T1, na, Yl, nlocked, o->gs_tol, o->gs_reorth);
      for (int64_t t = 0; t < na; t++)
        vcopy(n, T1[t], P[ini + t]);
    }
    const int64_t na = bs - ini;
    const int64_t np = (its > 1) ? na : 0;
    const int64_t nv = na + na + np;
    if (nv == 0)
      continue;
    if (o->max_tiny_dim > 0 && nv > o->max_tiny_dim) {
      set_err("LOBPCG: tiny problem too large (nv cap)");
      rc = KO_ERR_RUNTIME;
      goto cleanup;
    }
    for (int64_t t = 0; t < na; t++) {
      Zs[t] = X[ini + t];
      Zs[na + t] = W[ini + t];
      if (np)
        Zs[2 * na + t] = P[ini + t];
    }
    apply_normal(A, Zs, nv, AZ, tmp_m);
    {
      dmat S = dm_new((int)nv, (int)nv), G = dm_new((int)nv, (int)nv), Y = dm_new((int)nv, (int)nv);
      form_gram(n, Zs, AZ, (int)nv, &S, &G);
      rc = solve_tiny_gep((int)nv, &G, &S, th, &Y);
      if (rc == KO_OK) {
        const int64_t take = na < nv ? na : nv;
        /* P_new = [W P] * [Yw; Yp] */
        combine_columns(n, Zs + na, (int)(na + np), &Y, (int)na, (int)take, T1);
        /* X_new = X * Yx (uses the pre-update X columns) */
        combine_columns(n, Zs, (int)na, &Y, 0, (int)take, T2);
        for (int64_t j = 0; j < take; j++)
          vcopy(n, T1[j], P[ini + j]);
        for (int64_t j = 0; j < take; j++) {
          vcopy(n, T2[j], X[ini + j]);
          vaxpy(n, 1.0, P[ini + j], X[ini + j]);
        }
        if (!orthonormalize_block(n, X + ini, take, Yl, nlocked, o->gs_tol, o->gs_reorth)) {
          /* the reference orthonormalizes clones and throws; X is left
           * untouched there, which only matters for the error path */
          set_err("LOBPCG: X slice orthonormalization failed");
          rc = KO_ERR_RUNTIME;
        }
      }
      dm_free(&S);
      dm_free(&G);
      dm_free(&Y);
      if (rc != KO_OK)
        goto cleanup;
    }
    /* full RR for ordering */
    apply_normal(A, X, bs, AX, tmp_m);
    {
      dmat S = dm_new((int)bs, (int)bs), G = dm_new((int)bs, (int)bs), Y = dm_new((int)bs, (int)bs);
      form_gram(n, X, AX, (int)bs, &S, &G);
      rc = solve_tiny_gep((int)bs, &G, &S, th, &Y);
      if (rc == KO_OK) {
        combine_columns(n, X, (int)bs, &Y, 0, (int)bs, T1);
        for (int64_t j = 0; j < bs; j++)
          vcopy(n, T1[j], X[j]);
        apply_normal(A, X, bs, AX, tmp_m);
        theta_from(theta, bs, th, bs);
      }
      dm_free(&S);
      dm_free(&G);
      dm_free(&Y);
      if (rc != KO_OK)
        goto cleanup;
    }
  }
  R->converged_to_target = (R->locked >= k_target);

  if (nright > 0) {
    const double desired = fmax(o->tol_abs, o->tol_rel * fmax(1.0, R->frob_norm_est));
    const double target = fmax(1e-14, fmin(1e-10, 0.01 * desired));
    rc = block_rr_polish(A, rng, RN, nright, target, 80, o->M_inv, o->M_user);
    if (rc != KO_OK)
      goto cleanup;
    for (int64_t i = 0; i < nright; i++) {
      op_mul(A, RN[i], tmp_m);
      if (vnorm(m, tmp_m) <= target)
        continue;
      (void)two_vec_rr_sharpen(A, RN, nright, i, target, o->M_inv, o->M_user, 120);
    }
    mgs_ptrs(nright, n, RN, 1e-14, 1);
  }

cleanup:
  R->n_right = nright;
  for (int64_t i = 0; i < kcap; i++) {
    free(Yl[i]);
    if (!right_out)
      free(RN[i]);
  }
  free(Yl);
  free(RN);
  for (int64_t j = 0; j < bs; j++) {
    free(X[j]);
    free(AX[j]);
    free(Rb[j]);
    free(W[j]);
    free(P[j]);
    free(T1[j]);
    free(T2[j]);
  }
  for (int64_t j = 0; j < 3 * bs; j++)
    free(AZ[j]);
  free(X);
  free(AX);
  free(Rb);
  free(W);
  free(P);
  free(T1);
  free(T2);
  free(Zs);
  free(AZ);
  free(tmp_m);
  free(vacc);
  free(theta);
  free(th);
  return rc;
}
