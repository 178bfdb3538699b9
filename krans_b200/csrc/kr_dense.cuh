// Small dense FP64 problems solved by one thread block (the projected
// problems of the Krylov solvers: the (l+1) x l refined-extraction SVD of
// the cyclic solver and the Rayleigh-Ritz pencil of LOBPCG).
//
// Methods (textbook, parallel orderings):
//  - one-sided Hestenes-Jacobi SVD with round-robin (circle) pair ordering,
//    one warp per column pair;
//  - two-sided cyclic Jacobi for symmetric matrices, Brent-Luk parallel
//    ordering (all disjoint rotations of a round applied at once);
//  - Householder tridiagonalisation + implicit QL for symmetric matrices;
//  - Cholesky and a triangular inverse.
// Orders up to 32 run on warp 0 with warp barriers (block barriers dominate
// such tiny problems); larger ones use the whole block.
// Matrices are column-major in global memory owned by the solve.
#pragma once

#include "kr_device.cuh"

namespace kr {

// Pair k of round r in the circle method for cp (even) players.
KR_DEV void rr_pair(int r, int k, int cp, int &p, int &q) {
  const int m = cp - 1;
  if (k == 0) {
    p = r;
    q = m;
  } else {
    p = (r + k) % m;
    q = (r - k + m) % m;
  }
  if (p > q) {
    const int t = p;
    p = q;
    q = t;
  }
}

// One-sided Jacobi SVD of M (r x c, column-major, leading dim ldm). On return
// V (c x c, leading dim c) holds the right singular vectors and sv the
// singular values (unsorted). M is overwritten with U*diag(sv).
KR_DEV void block_jacobi_svd(int r, int c, double *M, int ldm, double *V, double *sv) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __shared__ int s_rot;
  for (int i = threadIdx.x; i < c * c; i += blockDim.x)
    V[i] = (i % c == i / c) ? 1.0 : 0.0;
  __syncthreads();
  const int cp = c + (c & 1);
  for (int sweep = 0; sweep < 60 && c > 1; sweep++) {
    if (threadIdx.x == 0)
      s_rot = 0;
    __syncthreads();
    for (int round = 0; round < cp - 1; round++) {
      for (int k = wid; k < cp / 2; k += nw) {
        int p, q;
        rr_pair(round, k, cp, p, q);
        if (q >= c)
          continue;
        double *Mp = M + (size_t)p * ldm, *Mq = M + (size_t)q * ldm;
        double a = 0.0, b = 0.0, g = 0.0;
        for (int i = lane; i < r; i += 32) {
          const double x = Mp[i], y = Mq[i];
          a += x * x;
          b += y * y;
          g += x * y;
        }
        a = warp_sum(a);
        b = warp_sum(b);
        g = warp_sum(g);
        if (g == 0.0 || fabs(g) <= 1e-15 * sqrt(a * b))
          continue;
        const double zeta = (b - a) / (2.0 * g);
        const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        for (int i = lane; i < r; i += 32) {
          const double x = Mp[i], y = Mq[i];
          Mp[i] = cs * x - sn * y;
          Mq[i] = sn * x + cs * y;
        }
        double *Vp = V + (size_t)p * c, *Vq = V + (size_t)q * c;
        for (int i = lane; i < c; i += 32) {
          const double x = Vp[i], y = Vq[i];
          Vp[i] = cs * x - sn * y;
          Vq[i] = sn * x + cs * y;
        }
        if (lane == 0)
          s_rot = 1;
      }
      __syncthreads();
    }
    const int rot = s_rot;
    __syncthreads();
    if (!rot)
      break;
  }
  for (int j = wid; j < c; j += nw) {
    double s = 0.0;
    for (int i = lane; i < r; i += 32)
      s += M[(size_t)j * ldm + i] * M[(size_t)j * ldm + i];
    s = warp_sum(s);
    if (lane == 0)
      sv[j] = sqrt(s);
  }
  __syncthreads();
}

// Symmetric eigendecomposition of A (n x n, column-major, ld n, overwritten)
// by parallel two-sided Jacobi. w ascending, Q columns = eigenvectors.
// rot is scratch of 3*(n/2+1) doubles + (n/2+1)*2 ints (global).
KR_DEV void block_jacobi_eig(int n, double *A, double *w, double *Q, double *rot_cs,
                             int *rot_pq, int *ord_scratch) {
  __shared__ int s_rot;
  __shared__ double s_fro;
  const int tid = threadIdx.x, bd = blockDim.x;
  for (int i = tid; i < n * n; i += bd)
    Q[i] = (i % n == i / n) ? 1.0 : 0.0;
  // Frobenius norm
  {
    double s = 0.0;
    for (int i = tid; i < n * n; i += bd)
      s += A[i] * A[i];
    s = warp_sum(s);
    __shared__ double s_part[KR_MAX_WARPS];
    if ((tid & 31) == 0)
      s_part[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int i = 0; i < (bd + 31) / 32; i++)
        t += s_part[i];
      s_fro = sqrt(t);
    }
    __syncthreads();
  }
  const double fro = s_fro;
  const int cp = n + (n & 1), half = cp / 2;
  for (int sweep = 0; sweep < 60 && n > 1 && isfinite(fro); sweep++) {
    if (tid == 0)
      s_rot = 0;
    __syncthreads();
    for (int round = 0; round < cp - 1; round++) {
      for (int k = tid; k < half; k += bd) {
        int p, q;
        rr_pair(round, k, cp, p, q);
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = A[p + (size_t)q * n];
          const double app = A[p + (size_t)p * n], aqq = A[q + (size_t)q * n];
          if (apq != 0.0 && fabs(apq) > fmax(1e-18 * fro, 1e-16 * sqrt(fabs(app * aqq)))) {
            const double theta = (aqq - app) / (2.0 * apq);
            const double t = copysign(1.0, theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            s = t * c;
            s_rot = 1;
          }
        }
        rot_cs[2 * k] = c;
        rot_cs[2 * k + 1] = s;
        rot_pq[2 * k] = p;
        rot_pq[2 * k + 1] = q;
      }
      __syncthreads();
      // columns: A <- A J ; Q <- Q J
      for (int e = tid; e < half * n; e += bd) {
        const int k = e / n, row = e % n;
        const int p = rot_pq[2 * k], q = rot_pq[2 * k + 1];
        const double c = rot_cs[2 * k], s = rot_cs[2 * k + 1];
        if (q >= n || s == 0.0)
          continue;
        const double x = A[row + (size_t)p * n], y = A[row + (size_t)q * n];
        A[row + (size_t)p * n] = c * x - s * y;
        A[row + (size_t)q * n] = s * x + c * y;
        const double u = Q[row + (size_t)p * n], v = Q[row + (size_t)q * n];
        Q[row + (size_t)p * n] = c * u - s * v;
        Q[row + (size_t)q * n] = s * u + c * v;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int e = tid; e < half * n; e += bd) {
        const int k = e / n, col = e % n;
        const int p = rot_pq[2 * k], q = rot_pq[2 * k + 1];
        const double c = rot_cs[2 * k], s = rot_cs[2 * k + 1];
        if (q >= n || s == 0.0)
          continue;
        const double x = A[p + (size_t)col * n], y = A[q + (size_t)col * n];
        A[p + (size_t)col * n] = c * x - s * y;
        A[q + (size_t)col * n] = s * x + c * y;
      }
      __syncthreads();
      for (int k = tid; k < half; k += bd) {
        const int p = rot_pq[2 * k], q = rot_pq[2 * k + 1];
        if (q < n && rot_cs[2 * k + 1] != 0.0) {
          A[p + (size_t)q * n] = 0.0;
          A[q + (size_t)p * n] = 0.0;
        }
      }
      __syncthreads();
    }
    const int rot = s_rot;
    __syncthreads();
    if (!rot)
      break;
  }
  // sort ascending (stable by index): rank of each eigenvalue
  for (int i = tid; i < n; i += bd) {
    const double di = A[i + (size_t)i * n];
    int rank = 0;
    for (int j = 0; j < n; j++) {
      const double dj = A[j + (size_t)j * n];
      if (dj < di || (dj == di && j < i))
        rank++;
    }
    ord_scratch[rank] = i;
  }
  __syncthreads();
  for (int i = tid; i < n; i += bd)
    w[i] = A[ord_scratch[i] + (size_t)ord_scratch[i] * n];
  // permute Q columns into A (as scratch), then back
  for (int e = tid; e < n * n; e += bd) {
    const int j = e / n, row = e % n;
    A[row + (size_t)j * n] = Q[row + (size_t)ord_scratch[j] * n];
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += bd)
    Q[e] = A[e];
  __syncthreads();
}

// Block-wide sum of one value per thread; every thread receives the total
// (fixed order: warp butterfly, then warps in index order). `red` is shared
// scratch of KR_MAX_WARPS doubles.
KR_DEV double blk_allsum(double v, double *red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0)
    red[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < nw; i++)
    t += red[i];
  return t;
}

#define KR_EIG_MAX 512

// Thread groups of the eigensolver: the whole block, or warp 0 alone (small
// pencils, where block barriers dominate: the same steps with warp barriers).
struct EigBlock {
  KR_DEV static int tid() { return threadIdx.x; }
  KR_DEV static int size() { return blockDim.x; }
  KR_DEV static void sync() { __syncthreads(); }
  KR_DEV static double allsum(double v, double *red) { return blk_allsum(v, red); }
};
struct EigWarp { // called by warp 0 only
  KR_DEV static int tid() { return threadIdx.x & 31; }
  KR_DEV static int size() { return 32; }
  KR_DEV static void sync() { __syncwarp(); }
  KR_DEV static double allsum(double v, double *) { return warp_sum(v); }
};

// Symmetric eigendecomposition of A (n x n, column-major, ld n; both
// triangles referenced, destroyed) on a thread group: Householder reduction
// to tridiagonal form with the orthogonal factor accumulated explicitly, then
// the implicit QL algorithm with shifts for the tridiagonal matrix (Golub &
// Van Loan, Matrix Computations, 4th ed., 8.3.1 and 8.3.3; QL as in Bowdler,
// Martin, Reinsch and Wilkinson, Numer. Math. 11 (1968) 293-306). One thread
// runs the scalar recurrence of each QL sweep into shared arrays of rotations;
// all threads then apply the sweep to the rows of Z in parallel (the rows are
// independent). w ascending (ties keep index order), Z columns = eigenvectors.
// Returns 0, or nonzero if n > KR_EIG_MAX or an eigenvalue needed more than 60
// sweeps (the caller then falls back to Jacobi).
template <class G, int NMAX> KR_DEV int sym_eig_ql(int n, double *A, double *w, double *Z, int *ord) {
  __shared__ double s_d[NMAX], s_e[NMAX], s_c[NMAX], s_s[NMAX];
  __shared__ double s_red[KR_MAX_WARPS];
  __shared__ int s_m, s_lo, s_fail;
  __shared__ double s_tn;
  const int tid = G::tid(), bd = G::size(), lane = tid & 31, wid = tid >> 5, nw = bd >> 5;
  if (n > NMAX || n < 1)
    return -1;
  // ---- 1) Householder reduction: column k below the subdiagonal -> alpha e1
  for (int k = 0; k + 2 < n; k++) {
    const int r0 = k + 1, r = n - r0;
    double *x = A + r0 + (size_t)k * n; // A[r0:n, k]; becomes the Householder vector
    double t2 = 0.0;
    for (int i = 1 + tid; i < r; i += bd)
      t2 += x[i] * x[i];
    t2 = G::allsum(t2, s_red);
    const double x0 = x[0];
    if (!(t2 > 0.0)) { // nothing to annihilate: H_k = I
      if (tid == 0) {
        s_d[k] = A[k + (size_t)k * n];
        s_e[k] = x0;
        s_s[k] = 0.0;
      }
      G::sync();
      continue;
    }
    const double sig = sqrt(x0 * x0 + t2);
    const double alpha = x0 >= 0.0 ? -sig : sig;
    const double beta = 1.0 / (sig * (sig + fabs(x0))); // H = I - beta v v^T, v = x - alpha e1
    G::sync();
    if (tid == 0) {
      x[0] = x0 - alpha;
      s_d[k] = A[k + (size_t)k * n];
      s_e[k] = alpha;
      s_s[k] = beta;
    }
    G::sync();
    // p = beta * A_sub v (A_sub symmetric: row i read as column i, coalesced)
    double *pv = s_c;
    for (int i = wid; i < r; i += nw) {
      const double *col = A + r0 + (size_t)(r0 + i) * n;
      double acc = 0.0;
      for (int j = lane; j < r; j += 32)
        acc += col[j] * x[j];
      acc = warp_sum(acc);
      if (lane == 0)
        pv[i] = beta * acc;
    }
    G::sync();
    double vp = 0.0;
    for (int i = tid; i < r; i += bd)
      vp += x[i] * pv[i];
    vp = G::allsum(vp, s_red);
    const double K = 0.5 * beta * vp;
    for (int i = tid; i < r; i += bd)
      pv[i] -= K * x[i]; // w = p - K v
    G::sync();
    // A_sub -= v w^T + w v^T
    for (int e = tid; e < r * r; e += bd) {
      const int j = e / r, i = e % r;
      A[r0 + i + (size_t)(r0 + j) * n] -= x[i] * pv[j] + pv[i] * x[j];
    }
    G::sync();
  }
  if (tid == 0) {
    if (n >= 2) {
      s_d[n - 2] = A[(n - 2) + (size_t)(n - 2) * n];
      s_e[n - 2] = A[(n - 1) + (size_t)(n - 2) * n];
    }
    s_d[n - 1] = A[(n - 1) + (size_t)(n - 1) * n];
    s_e[n - 1] = 0.0;
    s_fail = 0;
    double tn = 0.0; // ||T||_inf: the deflation floor eps ||T|| (absolute accuracy)
    for (int i = 0; i < n; i++)
      tn = fmax(tn, fabs(s_d[i]) + fabs(s_e[i]) + (i ? fabs(s_e[i - 1]) : 0.0));
    s_tn = tn;
  }
  // ---- 2) Z = H_0 H_1 ... H_{n-3}, accumulated backwards
  for (int e = tid; e < n * n; e += bd)
    Z[e] = (e % n == e / n) ? 1.0 : 0.0;
  G::sync();
  for (int k = n - 3; k >= 0; k--) {
    const double beta = s_s[k];
    if (beta == 0.0)
      continue;
    const int r0 = k + 1, r = n - r0;
    const double *v = A + r0 + (size_t)k * n;
    for (int j = wid; j < r; j += nw) {
      double *zc = Z + r0 + (size_t)(r0 + j) * n;
      double acc = 0.0;
      for (int i = lane; i < r; i += 32)
        acc += v[i] * zc[i];
      acc = beta * warp_sum(acc);
      for (int i = lane; i < r; i += 32)
        zc[i] -= acc * v[i];
    }
    G::sync();
  }
  // ---- 3) implicit QL on (d, e), rotations applied to the rows of Z
  for (int l = 0; l < n; l++) {
    for (int iter = 0;; iter++) {
      if (tid == 0) {
        int m = l;
        for (; m < n - 1; m++) {
          const double dd = fabs(s_d[m]) + fabs(s_d[m + 1]);
          if (fabs(s_e[m]) <= 2.2204460492503131e-16 * dd || fabs(s_e[m]) <= 2.2204460492503131e-16 * s_tn)
            break;
        }
        s_m = m;
        s_lo = m;
        if (m != l) {
          if (iter >= 60) {
            s_fail = 1;
          } else {
            double g = (s_d[l + 1] - s_d[l]) / (2.0 * s_e[l]);
            double r = hypot(g, 1.0);
            g = s_d[m] - s_d[l] + s_e[l] / (g + copysign(r, g));
            double sn = 1.0, cs = 1.0, pp = 0.0;
            int i = m - 1;
            bool early = false;
            for (; i >= l; i--) {
              const double f = sn * s_e[i], b = cs * s_e[i];
              r = hypot(f, g);
              s_e[i + 1] = r;
              if (r == 0.0) {
                s_d[i + 1] -= pp;
                s_e[m] = 0.0;
                early = true;
                break;
              }
              sn = f / r;
              cs = g / r;
              g = s_d[i + 1] - pp;
              r = (s_d[i] - g) * sn + 2.0 * cs * b;
              pp = sn * r;
              s_d[i + 1] = g + pp;
              g = cs * r - b;
              s_c[i] = cs;
              s_s[i] = sn;
            }
            s_lo = early ? i + 1 : l;
            if (!early) {
              s_d[l] -= pp;
              s_e[l] = g;
              s_e[m] = 0.0;
            }
          }
        }
      }
      G::sync();
      const int m = s_m, lo = s_lo, fl = s_fail;
      G::sync(); // all have read before thread 0 writes the next sweep
      if (m == l || fl)
        break;
      // rotation i mixes columns i and i+1 of every row, for i = m-1 down to
      // lo; eight columns are loaded ahead at a time (each is read before the
      // rotation that overwrites it, as in the plain loop, so the values are
      // the same) to keep eight loads in flight per row
      for (int row = tid; row < n; row += bd) {
        double xr = Z[row + (size_t)m * n];
        int i0 = m - 1;
        for (; i0 - 7 >= lo; i0 -= 8) {
          double zi[8];
#pragma unroll
          for (int u = 0; u < 8; u++)
            zi[u] = Z[row + (size_t)(i0 - u) * n];
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const int i = i0 - u;
            const double cs = s_c[i], sn = s_s[i];
            Z[row + (size_t)(i + 1) * n] = sn * zi[u] + cs * xr;
            xr = cs * zi[u] - sn * xr;
          }
        }
        for (int i = i0; i >= lo; i--) {
          const double zi = Z[row + (size_t)i * n];
          const double cs = s_c[i], sn = s_s[i];
          Z[row + (size_t)(i + 1) * n] = sn * zi + cs * xr;
          xr = cs * zi - sn * xr;
        }
        Z[row + (size_t)lo * n] = xr;
      }
      G::sync();
    }
    if (s_fail)
      break;
    G::sync();
  }
  const int fail = s_fail;
  G::sync();
  if (fail)
    return 1;
  // ---- 4) ascending order (ties by index), columns permuted through A
  for (int i = tid; i < n; i += bd) {
    const double di = s_d[i];
    int rank = 0;
    for (int j = 0; j < n; j++) {
      const double dj = s_d[j];
      if (dj < di || (dj == di && j < i))
        rank++;
    }
    ord[rank] = i;
  }
  G::sync();
  for (int i = tid; i < n; i += bd)
    w[i] = s_d[ord[i]];
  for (int e = tid; e < n * n; e += bd) {
    const int j = e / n, row = e % n;
    A[row + (size_t)j * n] = Z[row + (size_t)ord[j] * n];
  }
  G::sync();
  for (int e = tid; e < n * n; e += bd)
    Z[e] = A[e];
  G::sync();
  return 0;
}

// The block's entry: warp 0 alone for n <= 32, else the whole block. Every
// thread of the block calls it and gets the same return value.
KR_DEV int block_sym_eig_ql(int n, double *A, double *w, double *Z, int *ord) {
  if (n <= 32) {
    __shared__ int s_rc;
    if (threadIdx.x < 32) {
      const int rc = sym_eig_ql<EigWarp, 32>(n, A, w, Z, ord);
      if (threadIdx.x == 0)
        s_rc = rc;
    }
    __syncthreads();
    const int rc = s_rc;
    __syncthreads();
    return rc;
  }
  return sym_eig_ql<EigBlock, KR_EIG_MAX>(n, A, w, Z, ord);
}

// In-place Cholesky of the lower triangle of A (n x n, ld n). Returns 0 on
// success or k+1 when pivot k is <= 0 (NaN pivots pass, like Eigen::LLT).
// Every entry sees the same subtractions in the same order (j = 0, 1, ...)
// in both forms below, so the factor is the same to the last bit.
KR_DEV int block_cholesky(int n, double *A) {
  __shared__ int s_fail;
  __shared__ double s_piv;
  if (n <= 32) {
    // one warp, lane i on row i: the same updates in the same order, with
    // warp barriers instead of block barriers (the tiny pencils of small
    // solves are latency-bound on the barriers)
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      int fail = 0;
      for (int k = 0; k < n; k++) {
        double x = A[k + (size_t)k * n];
        if (x <= 0.0) {
          fail = k + 1;
          break;
        }
        x = sqrt(x);
        __syncwarp();
        if (lane == k)
          A[k + (size_t)k * n] = x;
        if (lane > k && lane < n)
          A[lane + (size_t)k * n] = A[lane + (size_t)k * n] / x;
        __syncwarp();
        if (lane > k && lane < n) {
          const double lik = A[lane + (size_t)k * n];
          for (int j = k + 1; j <= lane; j++)
            A[lane + (size_t)j * n] -= lik * A[j + (size_t)k * n];
        }
        __syncwarp();
      }
      if (lane == 0)
        s_fail = fail;
    }
    __syncthreads();
    const int f = s_fail;
    __syncthreads();
    if (f)
      return f;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int j = e / n, i = e % n;
      if (i < j)
        A[e] = 0.0;
    }
    __syncthreads();
    return 0;
  }
  // left-looking: pivot k from a dot over row k (thread 0), then every entry
  // below it from a dot over its row (one thread per row); measured faster
  // than the right-looking update above 32 (p = 288: 2.0 ms against 3.5 ms
  // on one block), whose trailing update rewrites the matrix at every step
  if (threadIdx.x == 0)
    s_fail = 0;
  __syncthreads();
  for (int k = 0; k < n; k++) {
    if (threadIdx.x == 0) {
      double x = A[k + (size_t)k * n];
      for (int j = 0; j < k; j++)
        x -= A[k + (size_t)j * n] * A[k + (size_t)j * n];
      if (x <= 0.0) {
        s_fail = k + 1;
      } else {
        x = sqrt(x);
        A[k + (size_t)k * n] = x;
      }
      s_piv = x;
    }
    __syncthreads();
    if (s_fail)
      break;
    const double piv = s_piv;
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
      double s = A[i + (size_t)k * n];
      for (int j = 0; j < k; j++)
        s -= A[i + (size_t)j * n] * A[k + (size_t)j * n];
      A[i + (size_t)k * n] = s / piv;
    }
    __syncthreads();
  }
  const int f = s_fail;
  __syncthreads();
  if (f)
    return f;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int j = e / n, i = e % n;
    if (i < j)
      A[e] = 0.0;
  }
  __syncthreads();
  return 0;
}

// Li = L^{-1} for lower-triangular L (n x n): forward substitution on all
// columns at once, row by row. Row k of Li is final once divided by L[k, k];
// it is then subtracted, times L[i, k], from every later row i. Each entry
// sees the same operations in the same order as column-by-column forward
// substitution (subtractions for k = j, ..., i-1, then the division).
KR_DEV void block_lower_inverse(int n, const double *L, double *Li) {
  if (n <= 32) {
    // one thread per column (same operations, no barrier inside)
    if (threadIdx.x < (unsigned)n) {
      const int j = threadIdx.x;
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
    __syncthreads();
    return;
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x)
    Li[e] = (e % n == e / n) ? 1.0 : 0.0;
  __syncthreads();
  for (int k = 0; k < n; k++) {
    const double lkk = L[k + (size_t)k * n];
    for (int j = threadIdx.x; j <= k; j += blockDim.x)
      Li[k + (size_t)j * n] = Li[k + (size_t)j * n] / lkk;
    __syncthreads();
    const int r = n - k - 1;
    for (int e = threadIdx.x; e < r * (k + 1); e += blockDim.x) {
      const int j = e / r, i = k + 1 + e % r;
      Li[i + (size_t)j * n] -= L[i + (size_t)k * n] * Li[k + (size_t)j * n];
    }
    __syncthreads();
  }
}

// C = op(A) * op(B) for small n x n matrices (ld n); ta/tb transpose flags.
KR_DEV void block_gemm_nn(int n, const double *A, bool ta, const double *B, bool tb, double *C) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int j = e / n, i = e % n;
    double s = 0.0;
    for (int p = 0; p < n; p++) {
      const double a = ta ? A[p + (size_t)i * n] : A[i + (size_t)p * n];
      const double b = tb ? B[j + (size_t)p * n] : B[p + (size_t)j * n];
      s += a * b;
    }
    C[e] = s;
  }
  __syncthreads();
}

} // namespace kr
