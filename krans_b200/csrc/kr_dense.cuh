// Small dense FP64 problems solved by one thread block (the projected
// problems of the Krylov solvers: the (l+1) x l refined-extraction SVD of
// the cyclic solver and the Rayleigh-Ritz pencil of LOBPCG).
//
// Methods (textbook, parallel orderings):
//  - one-sided Hestenes-Jacobi SVD with round-robin (circle) pair ordering,
//    one warp per column pair;
//  - two-sided cyclic Jacobi for symmetric matrices, Brent-Luk parallel
//    ordering (all disjoint rotations of a round applied at once);
//  - right-looking Cholesky and a triangular inverse.
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
    TeamShared *dummy = nullptr;
    (void)dummy;
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

// In-place Cholesky of the lower triangle of A (n x n, ld n). Returns 0 on
// success or k+1 when pivot k is <= 0 (NaN pivots pass, like Eigen::LLT).
KR_DEV int block_cholesky(int n, double *A) {
  __shared__ int s_fail;
  __shared__ double s_piv;
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

// Li = L^{-1} for lower-triangular L (n x n): column j by forward
// substitution, one thread per column.
KR_DEV void block_lower_inverse(int n, const double *L, double *Li) {
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
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
