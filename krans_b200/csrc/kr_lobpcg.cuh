// Block LOBPCG on N = A^T A for the right null space, on the device.
//
// Restates find_nullspace_lobpcg_ex of the reference
// (src/Solvers/LOBPCGSolver.cpp:443-834) as team code, including
// orthonormalize_block (137-160), the tiny generalized eigenproblem with
// Cholesky jitter (88-119), block_rr_polish (286-440) and
// two_vec_rr_sharpen (199-278). Blocks are column-major (one contiguous
// n-vector per column, leading dimension ldn). Dot products of a column
// against a group of columns are fused into team reductions; Gram
// matrices are formed in FP64 (tensor cores: kr_gram.cuh). Only
// rounding differs from the reference: classical GS passes replace MGS
// loops, and reductions use fixed trees.
#pragma once

#include "kr_cyclic.cuh"
#include "kr_dense.cuh"
#include "kr_device.cuh"
#include "kr_gram.cuh"

namespace kr {

template <class Team> struct LobpcgSolver {
  Team &tm;
  const LobpcgDesc &d;
  int64_t m, n, ldn;
  Counters c;
  double gram_flops = 0.0;
  uint64_t t_ph[4] = {0, 0, 0, 0}; // apply_normal, Gram, tiny GEP, orthonormalisation (ns)
  int orth_depth = 0;
  int err = 0;

  KR_DEV LobpcgSolver(Team &t, const LobpcgDesc &dd) : tm(t), d(dd) {
    m = d.F.rows;
    n = d.F.cols;
    ldn = d.ldn;
  }
  KR_DEV double *col(double *b, int64_t j) const { return b + j * ldn; }

  // ---- primitives ---------------------------------------------------------
  KR_DEV void mulA(const double *x, double *y) {
    csr_mv(tm, d.F, d.F.v64, x, [&](int64_t i, double s) { y[i] = s; });
    c.spmv++;
    c.bytes += spmv_bytes(m, n, d.F.nnz, 8, 8, 8);
    tm.sync();
  }
  KR_DEV void mulAT(const double *x, double *y) {
    csr_mv(tm, d.B, d.B.v64, x, [&](int64_t i, double s) { y[i] = s; });
    c.spmvT++;
    c.bytes += spmv_bytes(n, m, d.B.nnz, 8, 8, 8);
    tm.sync();
  }
  KR_DEV double normA(const double *x, double *y) { // ||A x||, y = A x
    double s2 = 0.0;
    csr_mv(tm, d.F, d.F.v64, x, [&](int64_t i, double s) {
      y[i] = s;
      s2 += s * s;
    });
    c.spmv++;
    c.bytes += spmv_bytes(m, n, d.F.nnz, 8, 8, 8);
    return sqrt(tm.sum1(s2));
  }
  KR_DEV double dot(const double *a, const double *b) {
    c.bytes += 16.0 * n;
    return team_dot(tm, n, a, b);
  }
  KR_DEV double nrm(const double *a) {
    c.bytes += 8.0 * n;
    return team_nrm2(tm, n, a);
  }
  KR_DEV void copy(const double *s, double *dd) {
    team_for(tm, n, [&](int64_t i) { dd[i] = s[i]; });
    c.bytes += 16.0 * n;
    tm.sync();
  }
  // k consecutive columns (ld ldn) in one pass; src and dst must not overlap
  KR_DEV void copy_cols(const double *s, double *dd, int64_t k) {
    team_for(tm, k * ldn, [&](int64_t i) { dd[i] = s[i]; });
    c.bytes += 16.0 * n * k;
    tm.sync();
  }
  KR_DEV void scale(double a, double *x) {
    team_for(tm, n, [&](int64_t i) { x[i] *= a; });
    c.bytes += 16.0 * n;
    tm.sync();
  }
  KR_DEV void axpy(double a, const double *x, double *y) {
    team_for(tm, n, [&](int64_t i) { y[i] += a * x[i]; });
    c.bytes += 24.0 * n;
    tm.sync();
  }
  KR_DEV void random(double *out) {
    team_random_normal(tm, d.rng, out, n);
    c.bytes += 8.0 * n;
  }
  // x -= sum_q <x, B_q> B_q over nb columns (one classical pass); when
  // skip_zero, coefficients that are exactly 0 are dropped (project_out).
  __device__ __noinline__ void gs_pass(const double *Bk, int64_t nb, double *x) {
    if (nb <= 0)
      return;
    for (int64_t q0 = 0; q0 < nb; q0 += 128) {
      const int cnt = (int)imin64(128, nb - q0);
      team_multidot(tm, n, Bk + q0 * ldn, ldn, cnt, x);
      team_multi_axpy(tm, n, Bk + q0 * ldn, ldn, cnt, tm.sh->h, x);
      c.bytes += (double)(2 * cnt + 3) * 8.0 * n;
      tm.sync();
    }
  }
  // same against an arbitrary list of columns given by index set of a block
  __device__ __noinline__ void gs_pass_excl(const double *Bk, int64_t nb, int64_t excl, double *x) {
    // project x against columns q != excl, one at a time in the group form
    for (int64_t q0 = 0; q0 < nb; q0 += 128) {
      const int cnt = (int)imin64(128, nb - q0);
      team_multidot(tm, n, Bk + q0 * ldn, ldn, cnt, x);
      if (excl >= q0 && excl < q0 + cnt && threadIdx.x == 0)
        tm.sh->h[excl - q0] = 0.0;
      __syncthreads();
      team_multi_axpy(tm, n, Bk + q0 * ldn, ldn, cnt, tm.sh->h, x);
      c.bytes += (double)(2 * cnt + 3) * 8.0 * n;
      tm.sync();
    }
  }

  // Jacobi weights of N = A^T A: 1 / squared column norms of A (rows of the
  // stored transpose; 1 for empty columns)
  __device__ __noinline__ void jacobi_weights_n() {
    team_for(tm, n, [&](int64_t i) {
      double s2 = 0.0;
      for (int32_t k = d.B.rp[i]; k < d.B.rp[i + 1]; k++) {
        const double v = d.B.v64[k];
        s2 += v * v;
      }
      d.pc_dinv[i] = s2 > 0.0 ? 1.0 / s2 : 1.0;
    });
    c.bytes += 4.0 * n + 12.0 * d.B.nnz + 8.0 * n;
    tm.sync();
  }
  // y = M^-1 x for N = A^T A (n-vectors, y != x): the device form of M_inv.
  // Jacobi, or precond_steps steps of steepest descent on N from y = 0 (the
  // M_inv callback of tests/test_lobpcg.cpp:179-205: the residual q is also
  // the next direction). With no preconditioner y = x.
  __device__ __noinline__ void apply_minv(const double *x, double *y) {
    const int kind = d.o.precond_normal;
    if (kind == KRANS_PRECOND_JACOBI) {
      team_for(tm, n, [&](int64_t i) { y[i] = d.pc_dinv[i] * x[i]; });
      c.bytes += 24.0 * n;
      tm.sync();
      return;
    }
    if (kind != KRANS_PRECOND_SD) {
      copy(x, y);
      return;
    }
    double *q = d.pc_q, *Nq = d.pc_nq;
    team_for(tm, n, [&](int64_t i) {
      y[i] = 0.0;
      q[i] = x[i];
    });
    c.bytes += 24.0 * n;
    tm.sync();
    for (int it = 0; it < d.o.precond_steps && tm.ok(); it++) {
      mulA(q, d.pc_tm);
      double acc[2] = {0.0, 0.0}; // q.Nq, q.q
      csr_mv(tm, d.B, d.B.v64, d.pc_tm, [&](int64_t i, double s) {
        Nq[i] = s;
        const double qi = q[i];
        acc[0] += qi * s;
        acc[1] += qi * qi;
      });
      c.spmvT++;
      c.bytes += spmv_bytes(d.B.rows, d.B.cols, d.B.nnz, 8, 8, 8) + 8.0 * n;
      tm.template sum<2>(acc);
      if (!(fabs(acc[0]) >= 1e-30))
        break;
      const double alpha = acc[1] / acc[0];
      double q2 = 0.0;
      team_for(tm, n, [&](int64_t i) {
        const double qi = q[i];
        y[i] += alpha * qi;
        const double qn = qi - alpha * Nq[i];
        q[i] = qn;
        q2 += qn * qn;
      });
      c.bytes += 48.0 * n;
      q2 = tm.sum1(q2);
      if (q2 <= 1e-30)
        break;
    }
  }

  // MGS with optional reorth (GramSchmidt.cpp:55-82) on k columns of block V.
  __device__ __noinline__ bool mgs(double *V, int64_t k, double tol, bool reorth) {
    const uint64_t t0 = globaltimer_ns();
    orth_depth++;
    const bool ok = mgs_cols(V, k, tol, reorth);
    if (--orth_depth == 0)
      t_ph[3] += globaltimer_ns() - t0;
    return ok;
  }
  __device__ __noinline__ bool mgs_cols(double *V, int64_t k, double tol, bool reorth) {
    for (int64_t i = 0; i < k; i++) {
      double *vi = col(V, i);
      gs_pass(V, i, vi);
      double n1 = nrm(vi);
      if (n1 < tol)
        return false;
      if (reorth) {
        gs_pass(V, i, vi);
        const double n2 = nrm(vi);
        if (n2 < tol)
          return false;
        n1 = n2;
      }
      scale(1.0 / n1, vi);
    }
    return true;
  }

  // orthonormalize_block (LOBPCGSolver.cpp:137-160): project each column vs
  // basis and normalise (in place), then MGS on a copy in `scratch`, copied
  // back only on success.
  __device__ __noinline__ bool orthonormalize_block(double *Xb, int64_t k, const double *basis, int64_t nb, double tol,
                                   bool reorth, double *scratch) {
    const uint64_t t0 = globaltimer_ns();
    orth_depth++;
    const bool ok = orthonormalize_cols(Xb, k, basis, nb, tol, reorth, scratch);
    if (--orth_depth == 0)
      t_ph[3] += globaltimer_ns() - t0;
    return ok;
  }
  // Block form of orthonormalize_cols_mgs below, same result up to rounding:
  // (1) every column gets one classical projection against the basis
  //     (C = B^T X, X -= B C on the tensor cores) and is normalised;
  // (2) the MGS (with reorthogonalisation) of the block is done as Cholesky
  //     QR, twice: G = V^T V = L L^T, V <- V L^-T. For full-rank input both
  //     give the same Q (the QR factor with positive diagonal R), and MGS's
  //     failure test (a column norm below tol after removing the earlier
  //     columns) is the test on the Cholesky pivots. When a Cholesky fails
  //     (dependent columns, or a block too ill-conditioned for Cholesky QR),
  //     the column-wise path decides on the same input.
  __device__ __noinline__ bool orthonormalize_cols(double *Xb, int64_t k, const double *basis, int64_t nb, double tol,
                                                   bool reorth, double *scratch) {
    if (k <= 0)
      return true;
    if (nb > 0) {
      team_gemm_tn(tm, n, basis, (int)nb, Xb, (int)k, ldn, d.Cm, d.gram_part);
      team_combine_sub(tm, n, basis, ldn, (int)nb, d.Cm, (int)nb, (int)k, Xb);
      tm.sync();
      gram_flops += 4.0 * (double)n * nb * k;
      c.bytes += 8.0 * n * (2.0 * nb + 3.0 * k);
    }
    if (!normalize_cols(Xb, k, tol))
      return false;
    if (cholqr_round(Xb, k, tol, scratch) && (!reorth || cholqr_round(scratch, k, tol, Xb))) {
      if (!reorth)
        for (int64_t i = 0; i < k; i++)
          copy(col(scratch, i), col(Xb, i));
      return true;
    }
    for (int64_t i = 0; i < k; i++)
      copy(col(Xb, i), col(scratch, i));
    if (!mgs_cols(scratch, k, tol, reorth))
      return false;
    for (int64_t i = 0; i < k; i++)
      copy(col(scratch, i), col(Xb, i));
    return true;
  }

  // scale each of k columns to unit norm; false if a norm is below tol
  __device__ __noinline__ bool normalize_cols(double *Xb, int64_t k, double tol) {
    for (int64_t q0 = 0; q0 < k; q0 += KR_RED_K) {
      const int cnt = (int)imin64(KR_RED_K, k - q0);
      double acc[KR_RED_K];
#pragma unroll
      for (int t = 0; t < KR_RED_K; t++)
        acc[t] = 0.0;
      for (int64_t i = tm.tid(); i < n; i += tm.nthreads()) {
#pragma unroll
        for (int t = 0; t < KR_RED_K; t++)
          if (t < cnt) {
            const double x = Xb[(q0 + t) * ldn + i];
            acc[t] += x * x;
          }
      }
      tm.template sum<KR_RED_K>(acc);
      double inv[KR_RED_K];
      bool bad = false;
#pragma unroll
      for (int t = 0; t < KR_RED_K; t++) {
        const double nr = sqrt(acc[t]);
        inv[t] = 1.0;
        if (t < cnt) {
          if (!(nr >= tol))
            bad = true;
          inv[t] = 1.0 / nr;
        }
      }
      if (bad)
        return false;
      for (int64_t i = tm.tid(); i < n; i += tm.nthreads()) {
#pragma unroll
        for (int t = 0; t < KR_RED_K; t++)
          if (t < cnt)
            Xb[(q0 + t) * ldn + i] *= inv[t];
      }
      c.bytes += 24.0 * n * cnt;
    }
    tm.sync();
    return true;
  }

  // d.Tm <- L^-T for the Cholesky factor L of the k x k matrix in d.Sj (lead
  // block). False if a pivot is not positive or below tol.
  __device__ __noinline__ bool chol_inv_t(int k, double tol) {
    if (tm.lead_cta()) {
      __shared__ int s_bad;
      const int f = block_cholesky(k, d.Sj);
      if (threadIdx.x == 0)
        s_bad = f != 0;
      __syncthreads();
      if (!s_bad) {
        for (int i = threadIdx.x; i < k; i += blockDim.x)
          if (!(d.Sj[i + (size_t)i * k] >= tol))
            s_bad = 1;
        __syncthreads();
      }
      if (!s_bad) {
        block_lower_inverse(k, d.Sj, d.Li);
        for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
          const int j = e / k, i = e % k;
          d.Tm[e] = d.Li[j + (size_t)i * k];
        }
        __syncthreads();
      }
      if (threadIdx.x == 0)
        *d.flag = s_bad;
      __syncthreads();
    }
    tm.publish();
    return *(volatile int32_t *)d.flag == 0;
  }

  // one Cholesky-QR round: out = V chol(V^T V)^-T (V unchanged)
  __device__ __noinline__ bool cholqr_round(const double *V, int64_t k, double tol, double *out) {
    if (n >= 131072 && k >= 32)
      team_gram_sym_tiled(tm, n, V, nullptr, ldn, (int)k, d.Sj, nullptr, d.gram_part);
    else
      team_gemm_tn(tm, n, V, (int)k, V, (int)k, ldn, d.Sj, d.gram_part);
    gram_flops += 2.0 * (double)n * k * k;
    c.bytes += 8.0 * n * k;
    if (!chol_inv_t((int)k, tol))
      return false;
    team_combine(tm, n, V, ldn, (int)k, d.Tm, (int)k, 0, (int)k, out);
    c.bytes += 16.0 * n * k;
    tm.sync();
    return true;
  }

  __device__ __noinline__ bool orthonormalize_cols_mgs(double *Xb, int64_t k, const double *basis, int64_t nb,
                                                       double tol, bool reorth, double *scratch) {
    for (int64_t i = 0; i < k; i++) {
      double *xi = col(Xb, i);
      gs_pass(basis, nb, xi);
      const double nr = nrm(xi);
      if (nr < tol)
        return false;
      scale(1.0 / nr, xi);
    }
    for (int64_t i = 0; i < k; i++)
      copy(col(Xb, i), col(scratch, i));
    if (!mgs(scratch, k, tol, reorth))
      return false;
    for (int64_t i = 0; i < k; i++)
      copy(col(scratch, i), col(Xb, i));
    return true;
  }

  // The k columns of a block, KR_NBP at a time: Zi holds the group
  // interleaved (row i's KR_NBP entries in 64 contiguous bytes), so the
  // multi-right-hand-side SpMV (team_spmv_block) reads the operator once per
  // group and every gather reads 64 contiguous bytes; each row is summed in
  // storage order.
  KR_DEV void interleave(const double *Zg, int gc) {
    team_for(tm, n * KR_NBP, [&](int64_t e) {
      const int64_t i = e / KR_NBP;
      const int j = (int)(e % KR_NBP);
      d.Zi[e] = j < gc ? Zg[(int64_t)j * ldn + i] : 0.0;
    });
    c.bytes += 16.0 * n * gc;
    tm.sync();
  }
  // AZ = A^T (A Z) (LOBPCGSolver.cpp:54-64, column by column there): per
  // group, Ti = A Zi, then the columns of A^T Ti straight into AZb
  __device__ __noinline__ void apply_normal(const double *Zb, int64_t k, double *AZb) {
    const uint64_t t0 = globaltimer_ns();
    const int jc = (int)(tm.tid() % KR_NBP); // this thread's column within a group
    for (int64_t g0 = 0; g0 < k; g0 += KR_NBP) {
      const int gc = (int)imin64(KR_NBP, k - g0);
      interleave(Zb + g0 * ldn, gc);
      team_spmv_block(
          tm, m, d.F.rp, d.F.ci, d.F.v64, d.F.ulen, jc < gc,
          [&](int32_t cc) { return d.Zi[(int64_t)cc * KR_NBP + jc]; },
          [&](int64_t i, double s) { d.Ti[i * KR_NBP + jc] = s; });
      tm.sync();
      double *out = AZb + (g0 + (jc < gc ? jc : 0)) * ldn;
      team_spmv_block(
          tm, n, d.B.rp, d.B.ci, d.B.v64, d.B.ulen, jc < gc,
          [&](int32_t cc) { return d.Ti[(int64_t)cc * KR_NBP + jc]; }, [&](int64_t i, double s) { out[i] = s; });
      tm.sync();
      c.spmv += gc;
      c.spmvT += gc;
      c.bytes += gc * (spmv_bytes(m, n, d.F.nnz, 8, 8, 8) + spmv_bytes(n, m, d.B.nnz, 8, 8, 8));
    }
    t_ph[0] += globaltimer_ns() - t0;
  }
  // d.avn[j] = ||A x_j|| for the k columns of a block (the acceptance test's
  // norms, LOBPCGSolver.cpp:545-560), through the same grouped SpMV; every
  // block writes the team-wide totals and reads back only its own writes
  __device__ __noinline__ void block_norms(const double *Xb, int64_t k) {
    const uint64_t t0 = globaltimer_ns();
    const int jc = (int)(tm.tid() % KR_NBP);
    for (int64_t g0 = 0; g0 < k; g0 += KR_NBP) {
      const int gc = (int)imin64(KR_NBP, k - g0);
      interleave(Xb + g0 * ldn, gc);
      double s2 = 0.0;
      team_spmv_block(
          tm, m, d.F.rp, d.F.ci, d.F.v64, d.F.ulen, jc < gc,
          [&](int32_t cc) { return d.Zi[(int64_t)cc * KR_NBP + jc]; }, [&](int64_t, double s) { s2 += s * s; });
      double v[KR_NBP];
#pragma unroll
      for (int j = 0; j < KR_NBP; j++)
        v[j] = j == jc ? s2 : 0.0;
      tm.template sum<KR_NBP>(v);
      if (threadIdx.x == 0)
        for (int j = 0; j < gc; j++)
          d.avn[g0 + j] = sqrt(v[j]);
      __syncthreads();
      c.spmv += gc;
      c.bytes += gc * spmv_bytes(m, n, d.F.nnz, 8, 8, 8);
    }
    t_ph[0] += globaltimer_ns() - t0;
  }

  __device__ __noinline__ void form_gram(const double *Zb, const double *AZb, int p) {
    const uint64_t t0 = globaltimer_ns();
    if (n >= 131072 && p >= 32) {
      team_gram_sym_tiled(tm, n, Zb, AZb, ldn, p, d.S, d.G, d.gram_part); // both in one pass
    } else {
      team_gram2_direct(tm, n, Zb, AZb, ldn, p, d.S, d.G, d.gram_part); // both in one pass
    }
    t_ph[1] += globaltimer_ns() - t0;
    gram_flops += 2.0 * 2.0 * (double)n * p * p;
    c.bytes += 2.0 * 8.0 * n * p;
  }

  // solve_tiny_gep (LOBPCGSolver.cpp:88-119): symmetrise, Cholesky of S with
  // the reference's jitter ladder, C = L^-1 G L^-T, eigenpairs of C (theta
  // ascending in d.th), Y = L^-T Q in d.Ym (ld p). The three p x p products
  // run on the whole team; the factorisations and the eigensolver run on the
  // leader block. Returns false if no jitter makes S positive definite (or
  // the eigenvalues are not finite).
  __device__ __noinline__ bool tiny_gep(int p) {
    const uint64_t t0 = globaltimer_ns();
    if (tm.lead_cta())
      gep_prep(p);
    tm.publish();
    bool ok = false;
    for (int t = 0; t < 4 && !ok; t++) {
      if (tm.lead_cta())
        gep_chol(p, t);
      tm.publish();
      const bool chol_ok = *(volatile int32_t *)d.flag == 0;
      tm.sync(); // every block has read the flag before the leader writes it again
      if (!chol_ok)
        continue;
      team_small_gemm(p, d.Li, false, d.G, false, d.Tm);  // T = L^-1 G
      team_small_gemm(p, d.Tm, false, d.Li, true, d.Cm); // C = T L^-T
      if (tm.lead_cta())
        gep_eig(p);
      tm.publish();
      const bool eig_ok = *(volatile int32_t *)d.flag == 0;
      tm.sync();
      if (!eig_ok)
        continue;
      team_small_gemm(p, d.Li, true, d.Q, false, d.Ym); // Y = L^-T Q
      ok = true;
    }
    t_ph[2] += globaltimer_ns() - t0;
    return ok;
  }
  // C = op(A) op(B) for p x p matrices (ld p) on the whole team
  KR_DEV void team_small_gemm(int p, const double *A, bool ta, const double *B, bool tb, double *C) {
    const int64_t nt = tm.nthreads();
    for (int64_t e = tm.tid(); e < (int64_t)p * p; e += nt) {
      const int j = (int)(e / p), i = (int)(e % p);
      double s = 0.0;
      for (int q = 0; q < p; q++) {
        const double x = ta ? A[q + (size_t)i * p] : A[i + (size_t)q * p];
        const double y = tb ? B[j + (size_t)q * p] : B[q + (size_t)j * p];
        s += x * y;
      }
      C[e] = s;
    }
    tm.sync();
  }
  // leader block: symmetrise S and G; ||S||_F (floored at 1) into d.dflag[0]
  __device__ __noinline__ void gep_prep(int p) {
    double *S = d.S, *G = d.G;
    for (int e = threadIdx.x; e < p * p; e += blockDim.x) {
      const int j = e / p, i = e % p;
      if (i >= j) {
        const double g = 0.5 * (G[i + (size_t)j * p] + G[j + (size_t)i * p]);
        const double s = 0.5 * (S[i + (size_t)j * p] + S[j + (size_t)i * p]);
        G[i + (size_t)j * p] = g;
        G[j + (size_t)i * p] = g;
        S[i + (size_t)j * p] = s;
        S[j + (size_t)i * p] = s;
      }
    }
    __syncthreads();
    double s = 0.0;
    for (int e = threadIdx.x; e < p * p; e += blockDim.x)
      s += S[e] * S[e];
    int b = 0;
    double v[1] = {s};
    block_sum<1>(tm.sh, b, v);
    if (threadIdx.x == 0)
      d.dflag[0] = fmax(1.0, sqrt(v[0]));
    __syncthreads();
  }
  // leader block: Cholesky of S + jitter_t ||S|| I and L^-1 into d.Li;
  // d.flag = 0 on success
  __device__ __noinline__ void gep_chol(int p, int t) {
    const double jit[4] = {0.0, 1e-14, 1e-12, 1e-10};
    const double sn = *(volatile double *)d.dflag;
    for (int e = threadIdx.x; e < p * p; e += blockDim.x) {
      double v = d.S[e];
      if (jit[t] > 0.0 && (e % p) == (e / p))
        v += jit[t] * sn;
      d.Sj[e] = v;
    }
    __syncthreads();
    const int f = block_cholesky(p, d.Sj);
    if (f == 0)
      block_lower_inverse(p, d.Sj, d.Li);
    if (threadIdx.x == 0)
      *d.flag = f != 0;
    __syncthreads();
  }
  // leader block: eigenpairs of C (made exactly symmetric): tridiagonal QL on
  // a copy, Jacobi on C itself if QL does not converge; d.flag = 0 when all
  // eigenvalues are finite
  __device__ __noinline__ void gep_eig(int p) {
    for (int e = threadIdx.x; e < p * p; e += blockDim.x) {
      const int j = e / p, i = e % p;
      if (i > j) {
        const double c = 0.5 * (d.Cm[e] + d.Cm[j + (size_t)i * p]);
        d.Cm[e] = c;
        d.Cm[j + (size_t)i * p] = c;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < p * p; e += blockDim.x)
      d.Tm[e] = d.Cm[e];
    __syncthreads();
    if (block_sym_eig_ql(p, d.Tm, d.th, d.Q, d.eig_ord) != 0)
      block_jacobi_eig(p, d.Cm, d.th, d.Q, d.eig_cs, d.eig_pq, d.eig_ord);
    __shared__ int s_bad;
    if (threadIdx.x == 0)
      s_bad = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < p; i += blockDim.x)
      if (!isfinite(d.th[i]))
        s_bad = 1;
    __syncthreads();
    if (threadIdx.x == 0)
      *d.flag = s_bad;
    __syncthreads();
  }

  // out[i] = sum_{j<zc} Y(roff+j, i) Z_j for i < q (Y has leading dim ldy)
  __device__ __noinline__ void combine(const double *Zb, int zc, const double *Y, int ldy, int roff, int q, double *out) {
    team_combine(tm, n, Zb, ldn, zc, Y, ldy, roff, q, out);
    c.bytes += (double)(zc + q) * 8.0 * n;
    tm.sync();
  }

  // X <- X Y and AX <- AX Y with Y the tiny GEP's eigenvectors (d.Ym, ld
  // bs): the reference recomputes AX = N (X Y) with bs operator pairs
  // (LOBPCGSolver.cpp:520-521, 779-781); N (X Y) = (N X) Y, so one more
  // product gives it. The three blocks trade places instead of being copied.
  __device__ __noinline__ void rotate_block(double *&X, double *&AX, double *&T, int bs) {
    combine(X, bs, d.Ym, bs, 0, bs, T);
    double *t = X;
    X = T;
    T = t;
    combine(AX, bs, d.Ym, bs, 0, bs, T);
    t = AX;
    AX = T;
    T = t;
  }

  KR_DEV void theta_from(int64_t bs, int tn) {
    if (tm.leader()) {
      for (int64_t j = 0; j < bs; j++)
        d.theta[j] = 0.0;
      const int64_t lim = tn < bs ? tn : bs;
      for (int64_t j = 0; j < lim; j++)
        d.theta[j] = fmax(0.0, d.th[j]);
    }
    tm.publish();
  }
  KR_DEV double theta_of(int64_t j) const { return *(volatile double *)&d.theta[j]; }

  // ---- two_vec_rr_sharpen (LOBPCGSolver.cpp:199-278) ------------------------
  __device__ __noinline__ bool sharpen(double *V, int64_t k, int64_t idx, double target, int max_iters) {
    if (idx >= k)
      return true;
    double *Av = d.sv_av, *t = d.sv_t, *dd = d.sv_d, *Ad = d.sv_ad, *Nd = d.sv_nd, *vn = d.sv_vn;
    double *vi = col(V, idx);
    for (int it = 0; it < max_iters && tm.ok(); ++it) {
      const double res = normA(vi, Av);
      if (res <= target)
        return true;
      mulAT(Av, t);
      apply_minv(t, dd); // d = M^-1 t (or t)
      gs_pass_excl(V, k, idx, dd);
      const double nd = nrm(dd);
      if (nd <= 1e-14)
        return false;
      scale(1.0 / fmax(nd, 1e-300), dd);
      mulA(dd, Ad);
      mulAT(Ad, Nd);
      double acc[4] = {0, 0, 0, 0};
      team_for(tm, n, [&](int64_t i) {
        acc[0] += vi[i] * t[i];
        acc[1] += vi[i] * Nd[i];
        acc[2] += dd[i] * t[i];
        acc[3] += dd[i] * Nd[i];
      });
      tm.template sum<4>(acc);
      c.bytes += 32.0 * n;
      const double a = acc[0], g = 0.5 * (acc[2] + acc[1]), e = acc[3];
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
        const double cc = 1.0 / sqrt(tt * tt + 1.0), s = tt * cc;
        if (a - tt * g <= e + tt * g) {
          y0 = cc;
          y1 = -s;
        } else {
          y0 = s;
          y1 = cc;
        }
      }
      if (!isfinite(y0) || !isfinite(y1))
        return false;
      team_for(tm, n, [&](int64_t i) { vn[i] = vi[i] * y0 + y1 * dd[i]; });
      tm.sync();
      gs_pass_excl(V, k, idx, vn);
      const double nv = nrm(vn);
      if (nv <= 1e-14)
        return false;
      scale(1.0 / nv, vn);
      copy(vn, vi);
    }
    return false;
  }

  // ---- block_rr_polish (LOBPCGSolver.cpp:286-440) ---------------------------
  __device__ __noinline__ bool polish(double *V, int64_t k, double target, int max_sweeps) {
    if (k == 0)
      return true;
    double *r = d.pr, *g = d.pg, *tmp = d.ptmp;
    mgs(V, k, 1e-14, true);
    for (int sweep = 0; sweep < max_sweeps && tm.ok(); ++sweep) {
      double max_res = 0.0;
      for (int64_t i = 0; i < k; i++)
        max_res = fmax(max_res, normA(col(V, i), r));
      if (max_res <= target)
        break;
      int64_t nd = 0;
      for (int64_t i = 0; i < k; i++)
        copy(col(V, i), col(d.Vb, i));
      for (int64_t j = 0; j < k; j++) {
        const double res = normA(col(V, j), r);
        if (res <= target)
          continue;
        mulAT(r, g);
        if (d.o.precond_normal != KRANS_PRECOND_NONE) {
          apply_minv(g, d.vacc); // g <- M^-1 g
          copy(d.vacc, g);
        }
        gs_pass(d.Vb, k, g);
        const double gn = nrm(g);
        if (gn <= 1e-14)
          continue;
        scale(1.0 / gn, g);
        bool dup = false;
        if (nd > 0) {
          team_multidot(tm, n, d.D, ldn, (int)nd, g);
          for (int64_t q = 0; q < nd; q++)
            if (fabs(tm.sh->h[q]) >= 1.0 - 1e-8)
              dup = true;
          __syncthreads();
        }
        if (!dup) {
          copy(g, col(d.D, nd));
          nd++;
        }
      }
      if (nd == 0) {
        for (int64_t i = 0; i < k; i++) {
          double *vi = col(V, i);
          for (int it = 0; it < 50 && tm.ok(); ++it) {
            const double res = normA(vi, r);
            if (res <= target)
              break;
            mulAT(r, g);
            gs_pass_excl(V, k, i, g);
            const double gg = dot(g, g);
            if (gg <= 0.0)
              break;
            const double ag = normA(g, tmp);
            const double Ag2 = ag * ag;
            if (Ag2 <= 0.0)
              break;
            axpy(-(gg / Ag2), g, vi);
            gs_pass_excl(V, k, i, vi);
            const double nv = nrm(vi);
            if (nv > 0.0)
              scale(1.0 / nv, vi);
          }
        }
        mgs(V, k, 1e-14, true);
        const int enrich = k < 2 ? (int)k : 2;
        for (int e = 0; e < enrich; e++) {
          double *q = col(d.D, nd);
          random(q);
          gs_pass(d.Vb, k, q);
          const double nq = nrm(q);
          if (nq > 1e-14) {
            scale(1.0 / nq, q);
            nd++;
          }
        }
        if (nd > 0)
          (void)orthonormalize_block(d.D, nd, d.Vb, k, 1e-14, true, d.Vn);
        else
          continue;
      }
      if (!orthonormalize_block(d.D, nd, d.Vb, k, 1e-14, true, d.Vn))
        continue;
      const int64_t zc = k + nd;
      for (int64_t i = 0; i < k; i++)
        copy(col(V, i), col(d.Zp, i));
      for (int64_t i = 0; i < nd; i++)
        copy(col(d.D, i), col(d.Zp, k + i));
      apply_normal(d.Zp, zc, d.AZp);
      form_gram(d.Zp, d.AZp, (int)zc);
      if (!tiny_gep((int)zc)) {
        err = kLobErrGep;
        return false;
      }
      combine(d.Zp, (int)zc, d.Ym, (int)zc, 0, (int)k, d.Vn);
      mgs(d.Vn, k, 1e-14, true);
      for (int64_t i = 0; i < k; i++)
        copy(col(d.Vn, i), col(V, i));
      max_res = 0.0;
      for (int64_t i = 0; i < k; i++)
        max_res = fmax(max_res, normA(col(V, i), r));
      if (max_res <= target)
        break;
    }
    mgs(V, k, 1e-14, true);
    return true;
  }

  __device__ __noinline__ void run() {
    const krans_lobpcg_opts &o = d.o;
    const int64_t bs = d.bs, k_target = d.k_target, guards = d.guards;
    LobpcgDevResult R;
    memset(&R, 0, sizeof R);
    R.block_size = bs;
    double *X = d.X, *AX = d.AX, *Rb = d.Rb, *W = d.W, *P = d.P, *T1 = d.T1, *T2 = d.T2;
    int64_t nlocked = 0, nright = 0, its = 0;
    uint64_t t_pol0 = 0; // start of the closing polish (0: not reached)
    const uint64_t t_run0 = globaltimer_ns();

    // ||A||_F estimate (LOBPCGSolver.cpp:163-178)
    {
      const int samples = o.frob_samples > 1 ? o.frob_samples : 1;
      double sum2 = 0.0;
      for (int s = 0; s < samples; s++) {
        random(d.vacc);
        const double nr = normA(d.vacc, d.tmv);
        sum2 += nr * nr;
      }
      R.frob = sqrt(sum2 / (double)samples);
    }
    if (o.precond_normal == KRANS_PRECOND_JACOBI)
      jacobi_weights_n();
    const double accept_thr = fmax(o.tol_abs, o.tol_rel * fmax(1.0, R.frob));
    R.accept = accept_thr;

    // initial block: seeds, then random
    int64_t filled = 0;
    const int64_t seeds = d.initial ? min(d.n_initial, bs) : 0;
    for (; filled < seeds; ++filled)
      copy(d.initial[filled], col(X, filled));
    for (; filled < bs; ++filled)
      random(col(X, filled));
    if (!orthonormalize_block(X, bs, d.Yl, 0, o.gs_tol, o.gs_reorth != 0, T1)) {
      err = kLobErrInitialDependent;
      goto finish;
    }
    apply_normal(X, bs, AX);
    form_gram(X, AX, (int)bs);
    if (!tiny_gep((int)bs)) {
      err = kLobErrGep;
      goto finish;
    }
    rotate_block(X, AX, T1, (int)bs);
    theta_from(bs, (int)bs);

    while (nlocked < k_target && its < o.max_iters && tm.ok()) {
      ++its;
      int64_t nconv = 0;
      double best_unacc = INFINITY;
      // residuals of all columns in one pass, R = AX - theta X, and the norms
      // ||A x_j|| of the acceptance test for the whole block
      {
        for (int j = threadIdx.x; j < (int)bs; j += blockDim.x)
          tm.sh->h[j] = theta_of(j);
        __syncthreads();
        const double *sth = tm.sh->h;
        team_for(tm, bs * ldn, [&](int64_t e) { Rb[e] = AX[e] - sth[e / ldn] * X[e]; });
        c.bytes += 24.0 * n * bs;
        tm.sync();
      }
      block_norms(X, bs);
      for (int64_t j = 0; j < bs; ++j) {
        const double th = theta_of(j);
        double *xj = col(X, j);
        const double av_orig = *(volatile double *)&d.avn[j];
        if (av_orig <= accept_thr) {
          copy(xj, d.vacc);
          gs_pass(d.Yl, nlocked, d.vacc);
          const double nv = nrm(d.vacc);
          bool reject = false;
          if (nv <= fmax(1e-14, 10.0 * o.gs_tol)) {
            reject = true;
          } else {
            scale(1.0 / nv, d.vacc);
            if (nlocked > 0) {
              for (int64_t q0 = 0; q0 < nlocked; q0 += 128) {
                const int cnt = (int)imin64(128, nlocked - q0);
                team_multidot(tm, n, d.Yl + q0 * ldn, ldn, cnt, d.vacc);
                for (int q = 0; q < cnt; q++)
                  if (fabs(tm.sh->h[q]) >= 1.0 - 1e-8)
                    reject = true;
                __syncthreads();
              }
            }
          }
          double av_acc = INFINITY;
          if (!reject) {
            av_acc = normA(d.vacc, d.tmv);
            if (av_acc > accept_thr)
              reject = true;
          }
          if (!reject) {
            copy(d.vacc, col(d.Yl, nlocked));
            copy(d.vacc, col(d.RN, nright));
            if (tm.leader()) {
              d.theta_out[nright] = th;
              d.resid_out[nright] = av_acc;
            }
            nright++;
            nlocked++;
            nconv++;
            if (nlocked >= k_target)
              break;
          } else {
            best_unacc = fmin(best_unacc, av_orig);
          }
        } else {
          best_unacc = fmin(best_unacc, av_orig);
        }
      }
      R.locked = nlocked;
      R.iters = its;
      R.best_unaccepted = isfinite(best_unacc) ? best_unacc : 0.0;
      if (nlocked >= k_target)
        break;

      const int64_t ini = o.soft_locking ? nconv : 0;
      if (nconv >= bs - guards) {
        const int64_t remain = bs - nconv;
        for (int64_t j = 0; j < remain; j++) {
          copy(col(X, nconv + j), col(X, j));
          copy(col(AX, nconv + j), col(AX, j));
          copy(col(P, nconv + j), col(P, j));
        }
        if (tm.leader())
          for (int64_t j = 0; j < remain; j++)
            d.theta[j] = d.theta[nconv + j];
        tm.publish();
        for (int64_t j = remain; j < bs; j++)
          random(col(X, j));
        if (!orthonormalize_block(X, bs, d.Yl, nlocked, o.gs_tol, o.gs_reorth != 0, T1)) {
          err = kLobErrRestartOrth;
          goto finish;
        }
        apply_normal(X, bs, AX);
        form_gram(X, AX, (int)bs);
        if (!tiny_gep((int)bs)) {
          err = kLobErrGep;
          goto finish;
        }
        theta_from(bs, (int)bs);
        continue;
      }

      // W = M^-1 R (LOBPCGSolver.cpp:655-656), W = R without M_inv
      for (int64_t j = ini; j < bs; j++)
        apply_minv(col(Rb, j), col(W, j));
      const int64_t na = bs - ini;
      copy_cols(col(W, ini), T1, na);
      if (!orthonormalize_block(T1, na, d.Yl, nlocked, o.gs_tol, o.gs_reorth != 0, T2)) {
        for (int64_t j = ini; j < bs; j++)
          random(col(W, j));
        for (int64_t j = ini; j < bs; j++)
          gs_pass(d.Yl, nlocked, col(W, j));
      } else {
        copy_cols(T1, col(W, ini), na);
      }
      if (its > 1) {
        copy_cols(col(P, ini), T1, na);
        (void)orthonormalize_block(T1, na, d.Yl, nlocked, o.gs_tol, o.gs_reorth != 0, T2);
        copy_cols(T1, col(P, ini), na);
      }
      const int64_t np = (its > 1) ? na : 0;
      const int64_t nv = na + na + np;
      if (nv == 0)
        continue;
      if (o.max_tiny_dim > 0 && nv > o.max_tiny_dim) {
        err = kLobErrTinyDim;
        goto finish;
      }
      // Z = [X_act | W_act | P_act] (contiguous copy)
      copy_cols(col(X, ini), d.Z, na);
      copy_cols(col(W, ini), col(d.Z, na), na);
      if (np)
        copy_cols(col(P, ini), col(d.Z, 2 * na), na);
      apply_normal(d.Z, nv, d.AZ);
      form_gram(d.Z, d.AZ, (int)nv);
      if (!tiny_gep((int)nv)) {
        err = kLobErrGep;
        goto finish;
      }
      {
        const int64_t take = na < nv ? na : nv;
        // P_new = [W P] [Yw; Yp]; X_new = X_act Yx + P_new
        combine(d.Z + na * ldn, (int)(na + np), d.Ym, (int)nv, (int)na, (int)take, T1);
        combine(d.Z, (int)na, d.Ym, (int)nv, 0, (int)take, T2);
        copy_cols(T1, col(P, ini), take);
        {
          double *xo = col(X, ini);
          const double *a = T2, *b = col(P, ini);
          team_for(tm, take * ldn, [&](int64_t i) { xo[i] = a[i] + b[i]; });
          c.bytes += 24.0 * n * take;
          tm.sync();
        }
        if (!orthonormalize_block(X + ini * ldn, take, d.Yl, nlocked, o.gs_tol, o.gs_reorth != 0, T1)) {
          err = kLobErrXSlice;
          goto finish;
        }
      }
      // full Rayleigh-Ritz for ordering
      apply_normal(X, bs, AX);
      form_gram(X, AX, (int)bs);
      if (!tiny_gep((int)bs)) {
        err = kLobErrGep;
        goto finish;
      }
      rotate_block(X, AX, T1, (int)bs);
      theta_from(bs, (int)bs);
    }
    R.converged = (R.locked >= k_target) ? 1 : 0;

    t_pol0 = globaltimer_ns();
    if (nright > 0 && tm.ok()) {
      const double desired = fmax(o.tol_abs, o.tol_rel * fmax(1.0, R.frob));
      const double target = fmax(1e-14, fmin(1e-10, 0.01 * desired));
      if (!polish(d.RN, nright, target, 80))
        goto finish;
      for (int64_t i = 0; i < nright; i++) {
        if (normA(col(d.RN, i), d.ptmp) <= target)
          continue;
        (void)sharpen(d.RN, nright, i, target, 120);
      }
      mgs(d.RN, nright, 1e-14, true);
    }
  finish:
    tm.sync();
    if (t_pol0)
      R.final_polish_ms = (double)(globaltimer_ns() - t_pol0) * 1e-6;
    if (tm.leader()) {
      R.n_right = nright;
      R.status = *(volatile int *)d.status;
      R.err_code = err;
      R.spmv = c.spmv;
      R.spmvT = c.spmvT;
      R.bytes = c.bytes;
      R.gram_flops = gram_flops;
      const double tot = (double)(globaltimer_ns() - t_run0) * 1e-6;
      double acc = 0.0;
      for (int i = 0; i < 4; i++) {
        R.phase_ms[i] = (double)t_ph[i] * 1e-6;
        acc += R.phase_ms[i];
      }
      R.phase_ms[4] = tot - acc;
      *d.res = R;
    }
  }
};

#ifdef KR_LOBPCG_GRID_KERNEL
__global__ void __launch_bounds__(512) lobpcg_grid_kernel(LobpcgDesc d) {
  __shared__ TeamShared sh;
  TeamGrid tm{&sh, d.status, d.gb, d.gpart, 0, 0};
  LobpcgSolver<TeamGrid> s(tm, d);
  s.run();
}
#endif

#ifdef KR_LOBPCG_CLUSTER_KERNEL
// one solve on a thread-block cluster (served LOBPCG requests)
__global__ void __launch_bounds__(512) lobpcg_cluster_kernel(const LobpcgDesc *dp) {
  __shared__ TeamShared sh;
  const LobpcgDesc &d = *dp;
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  TeamCluster tm{&sh, d.status, 0, 0, cl.block_rank(), cl.num_blocks()};
  LobpcgSolver<TeamCluster> s(tm, d);
  s.run();
}
#endif

#ifdef KR_LOBPCG_CTA_KERNEL
__global__ void __launch_bounds__(512) lobpcg_cta_kernel(const LobpcgDesc *dp) {
  __shared__ TeamShared sh;
  const LobpcgDesc &d = *dp;
  TeamCta tm{&sh, d.status, 0};
  LobpcgSolver<TeamCta> s(tm, d);
  s.run();
}
#endif

} // namespace kr
