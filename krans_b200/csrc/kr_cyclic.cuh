// Cyclic Lanczos (Golub-Kahan) null-space solver on the device.
//
// Restates find_right_nullspace of the reference
// (src/Solvers/CyclicLanczosSolver.cpp:291-616) as team code: the whole
// restart / candidate / polish control flow runs on the GPU, with every
// decision taken from team-wide reductions so all threads follow one path.
// Differences that only change rounding:
//  - reorthogonalisation is block classical Gram-Schmidt, two passes (CGS2)
//    instead of vector-by-vector MGS (CyclicLanczosSolver.cpp:26-33,399-407);
//  - dot products are fixed-tree reductions instead of sequential sums;
//  - the refined-extraction SVD uses the even/odd decoupling of Tbar when
//    tau = 0 (all alpha are zero, so right singular vectors live on either
//    the [0;y] or the [x;0] Lanczos vectors; only the [0;y] ones can be
//    candidates, CyclicLanczosSolver.cpp:474-480).
// Precision: KT is the storage type of the Krylov vectors and of the
// SpMV in the Golub-Kahan recurrence (double: plain FP64 path; float: mixed
// path with FP32 SpMV and FP32 accumulation). Reorthogonalisation inner
// products, the projected SVD, the candidate vectors, the CG projector polish
// and the acceptance residuals are FP64 with FP64 matrix values in both.
#pragma once

#include "kr_dense.cuh"
#include "kr_device.cuh"

namespace kr {

// counters kept identically by every thread (uniform control flow)
struct Counters {
  int64_t spmv = 0, spmvT = 0, cg_solves = 0, cg_maxit_hits = 0, steps = 0, restarts = 0;
  double bytes = 0.0;
  uint64_t t_gk = 0, t_tiny = 0, t_cg = 0; // device time per phase (ns), leader's clock
};

template <class Team, class KT> struct CyclicSolver {
  Team &tm;
  const CyclicDesc &d;
  Counters c;
  int64_t m, n, nb = 0;
  double frob = 0.0;

  KR_DEV CyclicSolver(Team &t, const CyclicDesc &dd) : tm(t), d(dd) {
    m = d.F.rows;
    n = d.F.cols;
  }

  KR_DEV void count_F() {
    if (d.trans_run)
      c.spmvT++;
    else
      c.spmv++;
  }
  KR_DEV void count_B() {
    if (d.trans_run)
      c.spmv++;
    else
      c.spmvT++;
  }

  // y = F x (FP64)
  KR_DEV void mulF(const double *x, double *y) {
    csr_mv(tm, d.F, d.F.v64, x,
              [&](int64_t i, double s) { y[i] = s; });
    count_F();
    c.bytes += spmv_bytes(d.F.rows, d.F.cols, d.F.nnz, 8, 8, 8);
    tm.sync();
  }
  KR_DEV void mulB(const double *x, double *y) {
    csr_mv(tm, d.B, d.B.v64, x,
              [&](int64_t i, double s) { y[i] = s; });
    count_B();
    c.bytes += spmv_bytes(d.B.rows, d.B.cols, d.B.nnz, 8, 8, 8);
    tm.sync();
  }
  // ||F x|| with y = F x stored (fused norm)
  KR_DEV double mulF_norm(const double *x, double *y) {
    double s2 = 0.0;
    csr_mv(tm, d.F, d.F.v64, x, [&](int64_t i, double s) {
      y[i] = s;
      s2 += s * s;
    });
    count_F();
    c.bytes += spmv_bytes(d.F.rows, d.F.cols, d.F.nnz, 8, 8, 8);
    return sqrt(tm.sum1(s2)); // the reduction's barrier also publishes y
  }

  KR_DEV double nrm2(int64_t len, const double *x) {
    c.bytes += 8.0 * len;
    return team_nrm2(tm, len, x);
  }
  KR_DEV void scale(int64_t len, double a, double *x) {
    team_for(tm, len, [&](int64_t i) { x[i] *= a; });
    c.bytes += 16.0 * len;
    tm.sync();
  }
  KR_DEV void copy(int64_t len, const double *s, double *dd) {
    team_for(tm, len, [&](int64_t i) { dd[i] = s[i]; });
    c.bytes += 16.0 * len;
    tm.sync();
  }
  KR_DEV void random(double *out) {
    team_random_normal(tm, d.rng, out, n);
    c.bytes += 8.0 * n;
  }

  // two classical Gram-Schmidt passes against the accepted basis (double)
  __device__ __noinline__ void gs2_basis(double *v) {
    if (nb == 0)
      return;
    for (int pass = 0; pass < 2; pass++) {
      team_multidot(tm, n, d.basis, d.ldb, (int)nb, v);
      team_multi_axpy(tm, n, d.basis, d.ldb, (int)nb, tm.sh->h, v);
      c.bytes += 2.0 * (nb + 1) * 8.0 * n + 8.0 * n;
      tm.sync();
    }
  }
  // one CGS pass of w (len) against ns stored vectors S (type TS)
  template <class TS, class TW> KR_DEV void cgs_pass(int64_t len, const TS *S, int64_t ld, int ns, TW *w) {
    if (ns == 0)
      return;
    team_multidot(tm, len, S, ld, ns, w);
    team_multi_axpy(tm, len, S, ld, ns, tm.sh->h, w);
    c.bytes += (double)(2 * ns + 3) * sizeof(TS) * len;
    tm.sync();
  }

  __device__ __noinline__ double fro_est() {
    const int samples = d.o.frob_samples > 1 ? d.o.frob_samples : 1;
    double sum2 = 0.0;
    for (int s = 0; s < samples; s++) {
      random(d.tn);
      const double nr = mulF_norm(d.tn, d.tmv);
      sum2 += nr * nr;
    }
    return sqrt(sum2 / (double)samples);
  }

  // CG on (F F^T) w = rhs (CyclicLanczosSolver.cpp:48-113), no preconditioner.
  // The callers only use F^T w, so this returns u = F^T w instead of w: u
  // accumulates alpha_k F^T p_k, and F^T p_k is the vector the first SpMV of
  // iteration k forms anyway. The m-vector w and the closing F^T w product
  // are never needed (same value in exact arithmetic; rounding differs).
  // r and p are stored interleaved, so the gather of r + beta p at each entry
  // of F^T is one 16-byte load.
  // `precond`: use the request's precond_aat (the candidate polish does; the
  // random-projector fallback of try_project_random does not,
  // CyclicLanczosSolver.cpp:140-214).
  __device__ __noinline__ int64_t cg(const double *rhs, double *u, int64_t maxit, double rel_tol, double bd_tol,
                                     double *rnorm_out, bool precond = true) {
    if (precond && d.o.precond_aat != KRANS_PRECOND_NONE)
      return cg_pre(rhs, u, maxit, rel_tol, bd_tol, rnorm_out);
    double2 *rp = d.rp;
    double *Ap = d.Ap, *tn = d.tn;
    double rr = 0.0;
    team_for(tm, n, [&](int64_t i) { u[i] = 0.0; });
    team_for4(tm, m, [&](const int64_t *ix, int cnt) {
      double xv[4];
#pragma unroll
      for (int u4 = 0; u4 < 4; u4++)
        if (u4 < cnt)
          xv[u4] = rhs[ix[u4]];
#pragma unroll
      for (int u4 = 0; u4 < 4; u4++)
        if (u4 < cnt) {
          rp[ix[u4]] = make_double2(xv[u4], xv[u4]);
          rr += xv[u4] * xv[u4];
        }
    });
    rr = tm.sum1(rr);
    c.bytes += 24.0 * m + 8.0 * n;
    const double rhsn = sqrt(rr > 0.0 ? rr : 0.0);
    *rnorm_out = rhsn;
    if (!(rhsn > 0.0) || !isfinite(rhsn))
      return 0;
    double rz = rr; // z = r without a preconditioner
    if (!(rz > 0.0) || !isfinite(rz))
      return 0;
    double rnorm = sqrt(rz);
    const double tol = fmax(rel_tol * rnorm, 1e-30);
    *rnorm_out = rnorm;
    if (rnorm <= tol)
      return 0;
    // p = r at entry. Each iteration first forms p <- r + beta p; that
    // update is folded into the gather of the first SpMV (t = F^T p) and into
    // the epilogue of the second (which stores p), so CG needs no separate
    // pass over p (fma(beta, p, r) in both places: the same values).
    int64_t k = 0;
    double beta = 0.0;
    for (; k < maxit && tm.ok(); ++k) {
      const double bq = beta;
      team_spmv_x(
          tm, d.B.rows, d.B.rp, d.B.ci, d.B.v64,
          [&](int32_t cc) {
            const double2 q = rp[cc];
            return q.x + bq * q.y;
          },
          d.B.lanes, d.B.ulen, [&](int64_t i, double s) { tn[i] = s; });
      count_B();
      c.bytes += spmv_bytes(d.B.rows, d.B.cols, d.B.nnz, 8, 16, 8);
      tm.sync();
      double pap = 0.0;
      csr_mv(tm, d.F, d.F.v64, tn, [&](int64_t i, double s) {
        const double2 q = rp[i];
        const double pn = q.x + bq * q.y;
        rp[i].y = pn;
        Ap[i] = s;
        pap += pn * s;
      });
      count_F();
      c.bytes += spmv_bytes(d.F.rows, d.F.cols, d.F.nnz, 8, 8, 8) + 24.0 * m;
      pap = tm.sum1(pap);
      if (!isfinite(pap) || fabs(pap) <= bd_tol)
        break;
      const double alpha = rz / pap;
      double rzn = 0.0;
      team_for4(tm, m, [&](const int64_t *ix, int cnt) {
        double rv[4], av[4];
#pragma unroll
        for (int u4 = 0; u4 < 4; u4++)
          if (u4 < cnt) {
            rv[u4] = rp[ix[u4]].x;
            av[u4] = Ap[ix[u4]];
          }
#pragma unroll
        for (int u4 = 0; u4 < 4; u4++)
          if (u4 < cnt) {
            const double ri = rv[u4] - alpha * av[u4];
            rp[ix[u4]].x = ri;
            rzn += ri * ri;
          }
      });
      team_for4(tm, n, [&](const int64_t *ix, int cnt) {
        double uv[4], tv[4];
#pragma unroll
        for (int u4 = 0; u4 < 4; u4++)
          if (u4 < cnt) {
            uv[u4] = u[ix[u4]];
            tv[u4] = tn[ix[u4]];
          }
#pragma unroll
        for (int u4 = 0; u4 < 4; u4++)
          if (u4 < cnt)
            u[ix[u4]] = uv[u4] + alpha * tv[u4];
      });
      rzn = tm.sum1(rzn); // its barrier also publishes r for the next gather
      c.bytes += 24.0 * m + 24.0 * n;
      if (!isfinite(rzn))
        break;
      rnorm = sqrt(rzn > 0.0 ? rzn : 0.0);
      if (rnorm <= tol) {
        ++k;
        break;
      }
      beta = rzn / fmax(1e-300, rz);
      rz = rzn;
    }
    *rnorm_out = rnorm;
    return k;
  }

  // Jacobi weights 1 / diag(F F^T) (squared row norms of F; 1 for empty rows)
  __device__ __noinline__ void jacobi_weights() {
    team_for(tm, m, [&](int64_t i) {
      double s2 = 0.0;
      for (int32_t k = d.F.rp[i]; k < d.F.rp[i + 1]; k++) {
        const double v = d.F.v64[k];
        s2 += v * v;
      }
      d.dinv[i] = s2 > 0.0 ? 1.0 / s2 : 1.0;
    });
    c.bytes += 4.0 * m + 12.0 * d.F.nnz + 8.0 * m;
    tm.sync();
  }

  // z = M^-1 r into zp[i].x: Jacobi (z = r / diag(F F^T)) or precond_steps
  // steps of steepest descent on F F^T from z = 0 (the precond_AAt callback of
  // tests/test_cyclic_lanczos.cpp:339-377: residual and direction coincide at
  // the start of each step, so one vector q carries both)
  __device__ __noinline__ void apply_precond(const double *r, double2 *zp) {
    if (d.o.precond_aat == KRANS_PRECOND_JACOBI) {
      team_for(tm, m, [&](int64_t i) { zp[i].x = d.dinv[i] * r[i]; });
      c.bytes += 32.0 * m;
      tm.sync();
      return;
    }
    double *q = d.sd_q, *Oq = d.sd_Oq, *tn = d.tn;
    team_for(tm, m, [&](int64_t i) {
      zp[i].x = 0.0;
      q[i] = r[i];
    });
    c.bytes += 24.0 * m;
    tm.sync();
    for (int it = 0; it < d.o.precond_steps && tm.ok(); it++) {
      mulB(q, tn);
      double acc[2] = {0.0, 0.0}; // q.Oq, q.q
      csr_mv(tm, d.F, d.F.v64, tn, [&](int64_t i, double s) {
        Oq[i] = s;
        const double qi = q[i];
        acc[0] += qi * s;
        acc[1] += qi * qi;
      });
      count_F();
      c.bytes += spmv_bytes(d.F.rows, d.F.cols, d.F.nnz, 8, 8, 8) + 8.0 * m;
      tm.template sum<2>(acc);
      if (!(fabs(acc[0]) >= 1e-30))
        break;
      const double alpha = acc[1] / acc[0];
      double q2 = 0.0;
      team_for(tm, m, [&](int64_t i) {
        const double qi = q[i];
        zp[i].x += alpha * qi;
        const double qn = qi - alpha * Oq[i];
        q[i] = qn;
        q2 += qn * qn;
      });
      c.bytes += 48.0 * m;
      q2 = tm.sum1(q2);
      if (q2 <= 1e-30)
        break;
    }
  }

  // Preconditioned CG (cg_normal_eq_prec, CyclicLanczosSolver.cpp:48-113):
  // z = M^-1 r, rz = r.z, p = z, tolerance on sqrt(r.z); otherwise as cg()
  // (u = F^T w returned, direction update folded into the SpMVs, z and p
  // interleaved for the gather of z + beta p).
  __device__ __noinline__ int64_t cg_pre(const double *rhs, double *u, int64_t maxit, double rel_tol,
                                         double bd_tol, double *rnorm_out) {
    double2 *zp = d.rp;
    double *r = d.r_pre, *Ap = d.Ap, *tn = d.tn;
    double rr = 0.0;
    team_for(tm, n, [&](int64_t i) { u[i] = 0.0; });
    team_for(tm, m, [&](int64_t i) {
      const double x = rhs[i];
      r[i] = x;
      rr += x * x;
    });
    rr = tm.sum1(rr);
    c.bytes += 16.0 * m + 8.0 * n;
    const double rhsn = sqrt(rr > 0.0 ? rr : 0.0);
    *rnorm_out = rhsn;
    if (!(rhsn > 0.0) || !isfinite(rhsn))
      return 0;
    apply_precond(r, zp);
    double rz = 0.0;
    team_for(tm, m, [&](int64_t i) {
      const double z = zp[i].x;
      zp[i].y = z;
      rz += r[i] * z;
    });
    rz = tm.sum1(rz);
    c.bytes += 32.0 * m;
    if (!(rz > 0.0) || !isfinite(rz))
      return 0;
    double rnorm = sqrt(rz);
    const double tol = fmax(rel_tol * rnorm, 1e-30);
    *rnorm_out = rnorm;
    if (rnorm <= tol)
      return 0;
    int64_t k = 0;
    double beta = 0.0;
    for (; k < maxit && tm.ok(); ++k) {
      const double bq = beta;
      team_spmv_x(
          tm, d.B.rows, d.B.rp, d.B.ci, d.B.v64,
          [&](int32_t cc) {
            const double2 q = zp[cc];
            return q.x + bq * q.y;
          },
          d.B.lanes, d.B.ulen, [&](int64_t i, double s) { tn[i] = s; });
      count_B();
      c.bytes += spmv_bytes(d.B.rows, d.B.cols, d.B.nnz, 8, 16, 8);
      tm.sync();
      double pap = 0.0;
      csr_mv(tm, d.F, d.F.v64, tn, [&](int64_t i, double s) {
        const double2 q = zp[i];
        const double pn = q.x + bq * q.y;
        zp[i].y = pn;
        Ap[i] = s;
        pap += pn * s;
      });
      count_F();
      c.bytes += spmv_bytes(d.F.rows, d.F.cols, d.F.nnz, 8, 8, 8) + 24.0 * m;
      pap = tm.sum1(pap);
      if (!isfinite(pap) || fabs(pap) <= bd_tol)
        break;
      const double alpha = rz / pap;
      team_for(tm, m, [&](int64_t i) { r[i] -= alpha * Ap[i]; });
      team_for(tm, n, [&](int64_t i) { u[i] += alpha * tn[i]; });
      c.bytes += 24.0 * m + 24.0 * n;
      tm.sync();
      apply_precond(r, zp);
      double rzn = 0.0;
      team_for(tm, m, [&](int64_t i) { rzn += r[i] * zp[i].x; });
      rzn = tm.sum1(rzn); // its barrier also publishes z for the next gather
      c.bytes += 16.0 * m;
      if (!isfinite(rzn))
        break;
      rnorm = sqrt(rzn > 0.0 ? rzn : 0.0);
      if (rnorm <= tol) {
        ++k;
        break;
      }
      beta = rzn / fmax(1e-300, rz);
      rz = rzn;
    }
    *rnorm_out = rnorm;
    return k;
  }

  // Per-column totals of a value each thread holds for its own column
  // (column = thread index mod KR_NBP); every thread receives all KR_NBP totals.
  KR_DEV void col_sums(double x, double (&t)[KR_NBP]) {
    const int col = (int)(threadIdx.x & (KR_NBP - 1));
#pragma unroll
    for (int q = 0; q < KR_NBP; q++)
      t[q] = q == col ? x : 0.0;
    tm.template sum<KR_NBP>(t);
  }
  KR_DEV static double pick(const double (&t)[KR_NBP], int col) {
    double r = 0.0;
#pragma unroll
    for (int q = 0; q < KR_NBP; q++)
      if (q == col)
        r = t[q];
    return r;
  }

  // Block CG on (F F^T) W = H for the first nc <= KR_NBP interleaved columns
  // of d.Hb (solutions in d.Wb). Every column follows the rules of cg()
  // above on its own: same start, breakdown, finiteness and tolerance tests,
  // and a column that stops is never touched again; one iteration reads the
  // matrix once for all columns still running. The iteration count of column
  // q is left in tm.sh->ibuf[q].
  __device__ __noinline__ void cg_block(int nc, int64_t maxit, double rel_tol, double bd_tol) {
    const int col = (int)(threadIdx.x & (KR_NBP - 1));
    double *R = d.Rk, *P = d.Pk, *AP = d.Ak, *W = d.Wb, *T = d.Tk;
    const double *H = d.Hb;
    const int64_t mb = m * KR_NBP;
    double t[KR_NBP];
    double rr = 0.0;
    team_for(tm, mb, [&](int64_t e) {
      const double h = col < nc ? H[e] : 0.0;
      W[e] = 0.0;
      R[e] = h;
      P[e] = h;
      rr += h * h;
    });
    col_sums(rr, t);
    c.bytes += 32.0 * m * nc;
    unsigned act = 0;
    double tol[KR_NBP];
    int64_t its[KR_NBP];
#pragma unroll
    for (int q = 0; q < KR_NBP; q++) {
      its[q] = 0;
      const double rn = sqrt(t[q] > 0.0 ? t[q] : 0.0);
      tol[q] = fmax(rel_tol * rn, 1e-30);
      if (q < nc && rn > 0.0 && isfinite(rn) && rn > tol[q])
        act |= 1u << q;
    }
    double rz = pick(t, col), beta = 0.0; // this thread's column
    int64_t k = 0;
    for (; k < maxit && act && tm.ok(); ++k) {
      const int na = __popc(act);
      const bool mine = (act >> col) & 1u;
      const double bq = beta;
      // T = F^T (R + beta P): the direction update folded into the gather
      team_spmv_block(
          tm, d.B.rows, d.B.rp, d.B.ci, d.B.v64, d.B.ulen, mine,
          [&](int32_t cc) {
            const int64_t e = (int64_t)cc * KR_NBP + col;
            return R[e] + bq * P[e];
          },
          [&](int64_t i, double s) { T[i * KR_NBP + col] = s; });
      c.spmvT += d.trans_run ? 0 : na;
      c.spmv += d.trans_run ? na : 0;
      c.bytes += spmv_bytes(d.B.rows, d.B.cols, d.B.nnz, 8, 16 * na, 8 * na);
      tm.sync();
      double pap = 0.0;
      team_spmv_block(
          tm, d.F.rows, d.F.rp, d.F.ci, d.F.v64, d.F.ulen, mine, [&](int32_t cc) { return T[(int64_t)cc * KR_NBP + col]; },
          [&](int64_t i, double s) {
            const int64_t e = i * KR_NBP + col;
            const double pn = R[e] + bq * P[e];
            P[e] = pn;
            AP[e] = s;
            pap += pn * s;
          });
      c.spmv += d.trans_run ? 0 : na;
      c.spmvT += d.trans_run ? na : 0;
      c.bytes += spmv_bytes(d.F.rows, d.F.cols, d.F.nnz, 8, 8 * na, 8 * na) + 24.0 * m * na;
      col_sums(pap, t);
#pragma unroll
      for (int q = 0; q < KR_NBP; q++)
        if (((act >> q) & 1u) && (!isfinite(t[q]) || fabs(t[q]) <= bd_tol)) {
          its[q] = k;
          act &= ~(1u << q);
        }
      const bool upd = (act >> col) & 1u;
      const double alpha = upd ? rz / pick(t, col) : 0.0;
      double rzn = 0.0;
      team_for4(tm, mb, [&](const int64_t *ix, int cnt) {
        if (!upd)
          return;
        double pv[4], wv[4], rv[4], av[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (u < cnt) {
            pv[u] = P[ix[u]];
            wv[u] = W[ix[u]];
            rv[u] = R[ix[u]];
            av[u] = AP[ix[u]];
          }
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (u < cnt) {
            W[ix[u]] = wv[u] + alpha * pv[u];
            const double ri = rv[u] - alpha * av[u];
            R[ix[u]] = ri;
            rzn += ri * ri;
          }
      });
      col_sums(rzn, t); // its barrier also publishes R for the next gather
      c.bytes += 40.0 * m * na;
#pragma unroll
      for (int q = 0; q < KR_NBP; q++) {
        if (!((act >> q) & 1u))
          continue;
        if (!isfinite(t[q])) {
          its[q] = k;
          act &= ~(1u << q);
        } else if (sqrt(t[q] > 0.0 ? t[q] : 0.0) <= tol[q]) {
          its[q] = k + 1;
          act &= ~(1u << q);
        }
      }
      if ((act >> col) & 1u) {
        const double rzq = pick(t, col);
        beta = rzq / fmax(1e-300, rz);
        rz = rzq;
      }
    }
    // columns still running ran out of iterations
#pragma unroll
    for (int q = 0; q < KR_NBP; q++)
      if ((act >> q) & 1u)
        its[q] = k;
    if (threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < KR_NBP; q++)
        tm.sh->ibuf[q] = (int)its[q];
    }
    __syncthreads();
  }

  // try_project_random_to_nullspace (CyclicLanczosSolver.cpp:140-214)
  __device__ __noinline__ bool try_project_random(double accept) {
    double *v = d.v, *tmv = d.tmv, *wm = d.wm, *tn = d.tn;
    random(v);
    // single GS pass vs basis
    if (nb > 0) {
      team_multidot(tm, n, d.basis, d.ldb, (int)nb, v);
      team_multi_axpy(tm, n, d.basis, d.ldb, (int)nb, tm.sh->h, v);
      tm.sync();
    }
    double nv = nrm2(n, v);
    if (nv < 1e-14)
      return false;
    scale(n, 1.0 / nv, v);
    const double tnorm = mulF_norm(v, tmv);
    double rn;
    double *u = d.vp;
    const int64_t its = cg(tmv, u, 500, 1e-12, 1e-30, &rn, false);
    if (its > 0 || rn < tnorm) {
      team_for(tm, n, [&](int64_t i) { v[i] -= u[i]; });
      tm.sync();
    }
    if (nb > 0) {
      team_multidot(tm, n, d.basis, d.ldb, (int)nb, v);
      team_multi_axpy(tm, n, d.basis, d.ldb, (int)nb, tm.sh->h, v);
      tm.sync();
    }
    nv = nrm2(n, v);
    if (nv >= 1e-14)
      scale(n, 1.0 / nv, v);
    double res = mulF_norm(v, tmv);
    if (res > accept) {
      const double fn = fro_est();
      const double L2 = fmax(1e-30, fn * fn);
      const double tau = 0.9 / L2;
      for (int it = 0; it < d.o.grad_max_iters && res > accept && tm.ok(); ++it) {
        mulF(v, tmv);
        mulB(tmv, tn);
        team_for(tm, n, [&](int64_t i) { v[i] -= tau * tn[i]; });
        tm.sync();
        if (nb > 0) {
          team_multidot(tm, n, d.basis, d.ldb, (int)nb, v);
          team_multi_axpy(tm, n, d.basis, d.ldb, (int)nb, tm.sh->h, v);
          tm.sync();
        }
        nv = nrm2(n, v);
        if (nv < 1e-14)
          return false;
        scale(n, 1.0 / nv, v);
        res = mulF_norm(v, tmv);
      }
    }
    if (res <= accept) {
      copy(n, v, d.basis + nb * d.ldb);
      nb++;
      return true;
    }
    return false;
  }

  // Build and solve the projected problem on the leader block. Writes the
  // candidate coefficient matrix (over the Y vectors) into d.Vt, their
  // ordering into d.ord; returns the number of candidates (uniform).
  __device__ __noinline__ int tiny_problem(int l, double beta_last, int ny) {
    const double tau = d.o.target_tau;
    const bool harmonic = d.o.use_harmonic != 0;
    const bool split = harmonic && tau == 0.0;
    int ncand = 0;
    if (split)
      ncand = (l + 1) / 2;
    else
      ncand = l;
    if (tm.lead_cta()) {
      double *Tb = d.Tb, *Vt = d.Vt, *sv = d.sv;
      int32_t *ord = d.ord;
      if (split) {
        // even columns of Tbar: column i=2t has beta[i-1] at row i-1 and
        // beta[i] (or beta_last for i = l-1) at row i+1
        const int ce = ncand, r = l + 1;
        for (int e = threadIdx.x; e < r * ce; e += blockDim.x) {
          const int t = e / r, row = e % r, i = 2 * t;
          double val = 0.0;
          if (row == i - 1)
            val = d.beta[i - 1];
          else if (row == i + 1)
            val = (i + 1 < l) ? d.beta[i] : beta_last;
          Tb[e] = val;
        }
        __syncthreads();
        block_jacobi_svd(r, ce, Tb, r, Vt, sv);
        // ascending, ties by index
        for (int i = threadIdx.x; i < ce; i += blockDim.x) {
          int rank = 0;
          for (int j = 0; j < ce; j++)
            if (sv[j] < sv[i] || (sv[j] == sv[i] && j < i))
              rank++;
          ord[rank] = i;
        }
        __syncthreads();
      } else if (harmonic) {
        const int r = l + 1;
        for (int e = threadIdx.x; e < r * l; e += blockDim.x) {
          const int j = e / r, i = e % r;
          double val = 0.0;
          if (i < l) {
            if (i == j)
              val = d.alpha[i] - tau;
            else if (j == i + 1 && i + 1 < l)
              val = d.beta[i];
            else if (i == j + 1 && j + 1 < l)
              val = d.beta[j];
          } else if (j == l - 1) {
            val = beta_last;
          }
          Tb[e] = val;
        }
        __syncthreads();
        block_jacobi_svd(r, l, Tb, r, d.eig_cs + 0, sv); // V into eig_cs scratch
        // move V (l x l) into Vt keeping only even rows as Y coefficients
        for (int e = threadIdx.x; e < l * l; e += blockDim.x)
          Vt[e] = d.eig_cs[e];
        __syncthreads();
        for (int i = threadIdx.x; i < l; i += blockDim.x) {
          int rank = 0;
          for (int j = 0; j < l; j++)
            if (sv[j] < sv[i] || (sv[j] == sv[i] && j < i))
              rank++;
          ord[rank] = i;
        }
        __syncthreads();
      } else {
        for (int e = threadIdx.x; e < l * l; e += blockDim.x) {
          const int j = e / l, i = e % l;
          double val = 0.0;
          if (i == j)
            val = d.alpha[i];
          else if (j == i + 1)
            val = d.beta[i];
          else if (i == j + 1)
            val = d.beta[j];
          Tb[e] = val;
        }
        __syncthreads();
        block_jacobi_eig(l, Tb, sv, Vt, d.eig_cs, d.eig_pq, d.eig_ord);
        // already ascending by value; reorder by |lambda - tau| (stable)
        for (int i = threadIdx.x; i < l; i += blockDim.x) {
          const double ki = fabs(sv[i] - tau);
          int rank = 0;
          for (int j = 0; j < l; j++) {
            const double kj = fabs(sv[j] - tau);
            if (kj < ki || (kj == ki && j < i))
              rank++;
          }
          ord[rank] = i;
        }
        __syncthreads();
      }
      // finiteness flag
      __shared__ int s_bad;
      if (threadIdx.x == 0)
        s_bad = 0;
      __syncthreads();
      const int nv = split ? ncand * ncand : l * l;
      for (int e = threadIdx.x; e < nv; e += blockDim.x)
        if (!isfinite(Vt[e]))
          s_bad = 1;
      for (int e = threadIdx.x; e < ncand; e += blockDim.x)
        if (!isfinite(sv[e]))
          s_bad = 1;
      __syncthreads();
      if (threadIdx.x == 0)
        d.ord[ncand] = s_bad; // flag slot after the ordering
    }
    tm.publish();
    const int bad = *(volatile int32_t *)&d.ord[ncand];
    (void)ny;
    return bad ? -1 : ncand;
  }

  // coefficient of Y[t] in candidate column jb
  KR_DEV double coef(bool split, int l, int jb, int t) const {
    if (split)
      return *(volatile double *)&d.Vt[(size_t)jb * ((l + 1) / 2) + t];
    return *(volatile double *)&d.Vt[(size_t)jb * l + 2 * t];
  }

  // candidate v = sum_q coef_q Y[q] (CyclicLanczosSolver.cpp:496-503)
  KR_DEV void form_candidate(const KT *Y, bool split, int l, int jb, int ny_used, double *v) {
    for (int q = threadIdx.x; q < ny_used; q += blockDim.x)
      tm.sh->h[q] = coef(split, l, jb, q);
    __syncthreads();
    const int64_t ldn = d.ldn;
    team_for4(tm, n, [&](const int64_t *ix, int cnt) {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int q = 0; q < ny_used; q++) {
        const double hq = tm.sh->h[q];
        const KT *yq = Y + (int64_t)q * ldn;
        double yv[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
          yv[u] = u < cnt ? (double)yq[ix[u]] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; u++)
          acc[u] += hq * yv[u];
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (u < cnt)
          v[ix[u]] = acc[u];
    });
    c.bytes += (double)(ny_used * sizeof(KT) + 8) * n;
    tm.sync();
  }

  struct CandState {
    double best_res;
    bool have_best, accepted_this, polish_stalled, converged;
  };

  // Candidate phase with the block polish: candidates are taken in the same
  // order and screened by the same rules as the one-by-one loop of run(), but
  // up to KR_NBP of those that need the projector are collected first and
  // polished by one block CG. Each is then finished in order against the
  // basis as it stands at that point (Gram-Schmidt, residual, acceptance), so
  // an accepted vector is always orthogonal to the earlier ones. A candidate
  // that already meets the tolerance is accepted when it is formed.
  __device__ __noinline__ void candidates_block(const KT *Y, bool split, int l, int ncand, int64_t test_cap,
                                                int ny_used, double prescreen, double accept, CandState &st) {
    const krans_cyclic_opts &o = d.o;
    const int64_t ldn = d.ldn;
    double *Hb = d.Hb, *Tk = d.Tk;
    double mres[KR_NBP];
    int t = 0;
    int64_t tested = 0;
    while (t < ncand && tested < test_cap && tm.ok() && !st.converged) {
      int g = 0;
      while (g < KR_NBP && t < ncand && tested < test_cap && tm.ok()) {
        const int jb = *(volatile int32_t *)&d.ord[t++];
        double ce2 = 0.0;
        for (int q = 0; q < ny_used; q++) {
          const double cq = coef(split, l, jb, q);
          ce2 += cq * cq;
        }
        if (!(ce2 >= 1e-20))
          continue;
        double *vg = d.Vc + (int64_t)g * ldn;
        form_candidate(Y, split, l, jb, ny_used, vg);
        gs2_basis(vg);
        const double nv = nrm2(n, vg);
        if (!isfinite(nv) || nv < 1e-8)
          continue;
        scale(n, 1.0 / nv, vg);
        ++tested;
        // residual, with F v stored as column g of the block right-hand side
        double s2 = 0.0;
        csr_mv(tm, d.F, d.F.v64, vg, [&](int64_t i, double s) {
          Hb[i * KR_NBP + g] = s;
          s2 += s * s;
        });
        count_F();
        c.bytes += spmv_bytes(d.F.rows, d.F.cols, d.F.nnz, 8, 8, 8);
        const double res = sqrt(tm.sum1(s2));
        if (!isfinite(res))
          continue;
        if (res <= accept) {
          copy(n, vg, d.basis + nb * d.ldb);
          nb++;
          st.accepted_this = true;
          if (nb >= d.k_target) {
            st.converged = true;
            break;
          }
          continue;
        }
        if (res > prescreen || st.polish_stalled) {
          if (res < st.best_res) {
            st.best_res = res;
            copy(n, vg, d.best_v);
            st.have_best = true;
          }
          continue;
        }
        mres[g] = res;
        g++;
      }
      if (st.converged || g == 0)
        break;
      const uint64_t t_cg0 = globaltimer_ns();
      cg_block(g, o.cg_maxit, o.cg_rel_tol, o.cg_breakdown_tol);
      c.t_cg += globaltimer_ns() - t_cg0;
      // Tk = F^T W for all members at once
      {
        const int col = (int)(threadIdx.x & (KR_NBP - 1));
        const double *W = d.Wb;
        team_spmv_block(
            tm, d.B.rows, d.B.rp, d.B.ci, d.B.v64, d.B.ulen, col < g, [&](int32_t cc) { return W[(int64_t)cc * KR_NBP + col]; },
            [&](int64_t i, double s) { Tk[i * KR_NBP + col] = s; });
        c.spmvT += d.trans_run ? 0 : g;
        c.spmv += d.trans_run ? g : 0;
        c.bytes += spmv_bytes(d.B.rows, d.B.cols, d.B.nnz, 8, 8 * g, 8 * g);
        tm.sync();
      }
      int its[KR_NBP];
#pragma unroll
      for (int q = 0; q < KR_NBP; q++)
        its[q] = tm.sh->ibuf[q];
      __syncthreads();
      const int passes = o.projector_passes > 1 ? o.projector_passes : 1;
      for (int q = 0; q < g && tm.ok(); q++) {
        double *v = d.Vc + (int64_t)q * ldn, *vp = d.vp, *tmv = d.tmv, *wm = d.wm;
        double res = mres[q];
        bool hit_maxit = false;
        int its_q = 0;
#pragma unroll
        for (int u = 0; u < KR_NBP; u++)
          if (u == q)
            its_q = its[u];
        c.cg_solves++;
        if (its_q >= o.cg_maxit) {
          c.cg_maxit_hits++;
          hit_maxit = true;
        }
        for (int pass = 0; pass < passes && res > accept && tm.ok(); ++pass) {
          if (pass == 0) {
            team_for(tm, n, [&](int64_t i) { vp[i] = v[i] - Tk[i * KR_NBP + q]; });
          } else {
            double rn;
            const uint64_t t_cg1 = globaltimer_ns();
            const int64_t cg_its = cg(tmv, vp, o.cg_maxit, o.cg_rel_tol, o.cg_breakdown_tol, &rn);
            c.t_cg += globaltimer_ns() - t_cg1;
            c.cg_solves++;
            if (cg_its >= o.cg_maxit) {
              c.cg_maxit_hits++;
              hit_maxit = true;
            }
            team_for(tm, n, [&](int64_t i) { vp[i] = v[i] - vp[i]; });
          }
          c.bytes += 24.0 * n;
          tm.sync();
          gs2_basis(vp);
          const double np = nrm2(n, vp);
          if (!isfinite(np) || np < 1e-14)
            break;
          scale(n, 1.0 / np, vp);
          const double res_p = mulF_norm(vp, wm);
          if (!(res_p < res))
            break;
          double *t1 = v;
          v = vp;
          vp = t1;
          res = res_p;
          t1 = tmv;
          tmv = wm;
          wm = t1;
        }
        if (res <= accept) {
          copy(n, v, d.basis + nb * d.ldb);
          nb++;
          st.accepted_this = true;
          if (nb >= d.k_target) {
            st.converged = true;
            break;
          }
        } else {
          st.polish_stalled = st.polish_stalled || hit_maxit;
          if (res < st.best_res) {
            st.best_res = res;
            copy(n, v, d.best_v);
            st.have_best = true;
          }
        }
      }
    }
  }

  __device__ __noinline__ void run() {
    const krans_cyclic_opts &o = d.o;
    KT *Y = (KT *)d.Y, *X = (KT *)d.X, *wx = (KT *)d.wx, *wy = (KT *)d.wy;
    const int64_t ldn = d.ldn, ldm = d.ldm;
    const int64_t k_target = d.k_target, ncv = d.ncv;
    bool converged = false;

    const uint64_t t_run0 = globaltimer_ns();
    // a continued run (the FP64 continuation of a mixed solve) keeps the
    // estimate and the vectors its predecessor accepted
    frob = d.frob_init > 0.0 ? d.frob_init : fro_est();
    nb = d.nb_init;
    if (d.o.precond_aat == KRANS_PRECOND_JACOBI)
      jacobi_weights();
    const double fmx = fmax(1.0, frob);
    const double accept = fmax(o.tol_abs, o.tol_rel * fmx);
    const double prescreen = fmax(0.0, o.prescreen_factor) * fmx;

    double *y0 = d.y0, *v = d.v, *vp = d.vp, *best_v = d.best_v, *tn = d.tn;
    double *tmv = d.tmv, *wm = d.wm;
    if (d.initial_right)
      copy(n, d.initial_right, y0);
    else
      random(y0);

    int64_t rsa = 0;
    for (int64_t restart = 0; restart < o.max_restarts && tm.ok(); ++restart) {
      c.restarts = restart;
      gs2_basis(y0);
      double ny = nrm2(n, y0);
      if (!isfinite(ny) || ny < 1e-14) {
        random(y0);
        gs2_basis(y0);
        ny = nrm2(n, y0);
        if (!(ny >= 1e-14))
          break;
      }
      {
        const double s = 1.0 / ny;
        team_for(tm, n, [&](int64_t i) {
          const double t = y0[i] * s;
          y0[i] = t;
          Y[i] = (KT)t;
        });
        c.bytes += (8.0 + 8.0 + sizeof(KT)) * n;
        tm.sync();
      }
      const uint64_t t_gk0 = globaltimer_ns();
      int nY = 1, nX = 0, na = 0, nbeta = 0;
      int64_t local_steps = 0;
      double beta_last = 0.0, beta_prev = 0.0; // beta_prev: uniform register copy
      for (int64_t j = 0; j < ncv && tm.ok(); ++j) {
        const bool from_y = nY > nX;
        if (from_y) {
          const KT *yj = Y + (int64_t)(nY - 1) * ldn;
          const KT *xp = X + (int64_t)(nX > 0 ? nX - 1 : 0) * ldm;
          const KT bp = (KT)(nbeta > 0 ? beta_prev : 0.0);
          const bool sub = nbeta > 0;
          if constexpr (sizeof(KT) == 8) {
            csr_mv(tm, d.F, d.F.v64, yj,
                      [&](int64_t i, double s) { wx[i] = sub ? (KT)(s - (double)bp * (double)xp[i]) : (KT)s; });
          } else {
            csr_mv(tm, d.F, d.F.v32, yj,
                      [&](int64_t i, float s) { wx[i] = sub ? (KT)(s - (float)bp * (float)xp[i]) : (KT)s; });
          }
          count_F();
          c.bytes += spmv_bytes(m, n, d.F.nnz, sizeof(KT), sizeof(KT), sizeof(KT)) +
                     (sub ? sizeof(KT) * (double)m : 0.0);
          tm.sync();
          for (int pass = 0; pass < o.reorth; ++pass)
            cgs_pass(m, X, ldm, nX, wx);
        } else {
          const KT *xj = X + (int64_t)(nX - 1) * ldm;
          const KT *yp = Y + (int64_t)(nY - 1) * ldn;
          const KT bp = (KT)beta_prev;
          if constexpr (sizeof(KT) == 8) {
            csr_mv(tm, d.B, d.B.v64, xj,
                      [&](int64_t i, double s) { wy[i] = (KT)(s - (double)bp * (double)yp[i]); });
          } else {
            csr_mv(tm, d.B, d.B.v32, xj,
                      [&](int64_t i, float s) { wy[i] = (KT)(s - (float)bp * (float)yp[i]); });
          }
          count_B();
          c.bytes += spmv_bytes(n, m, d.B.nnz, sizeof(KT), sizeof(KT), sizeof(KT)) + sizeof(KT) * (double)n;
          tm.sync();
          for (int pass = 0; pass < o.reorth; ++pass) {
            cgs_pass(n, d.basis, d.ldb, (int)nb, wy);
            cgs_pass(n, Y, ldn, nY, wy);
          }
        }
        const int64_t len = from_y ? m : n;
        KT *w = from_y ? wx : wy;
        double bj;
        if constexpr (sizeof(KT) == 8)
          bj = nrm2(len, (const double *)w);
        else {
          bj = team_nrm2(tm, len, w);
          c.bytes += 4.0 * len;
        }
        if (tm.leader())
          d.alpha[na] = 0.0;
        na++;
        beta_last = bj;
        if (!isfinite(bj) || bj < 1e-14 || nY + nX >= ncv)
          break;
        if (tm.leader())
          d.beta[nbeta] = bj;
        beta_prev = bj;
        nbeta++;
        KT *dst = from_y ? X + (int64_t)nX * ldm : Y + (int64_t)nY * ldn;
        const double s = 1.0 / bj;
        team_for(tm, len, [&](int64_t i) { dst[i] = (KT)((double)w[i] * s); });
        c.bytes += 2.0 * sizeof(KT) * len;
        tm.sync();
        if (from_y)
          nX++;
        else
          nY++;
        ++local_steps;
      }
      c.steps += local_steps;
      tm.publish(); // alpha/beta written by the leader
      c.t_gk += globaltimer_ns() - t_gk0;
      const int l = na;
      if (l == 0 || !isfinite(beta_last) || !tm.ok())
        break;

      const bool split = (o.use_harmonic != 0) && o.target_tau == 0.0;
      const uint64_t t_ti0 = globaltimer_ns();
      const int ncand = tiny_problem(l, beta_last, nY);
      c.t_tiny += globaltimer_ns() - t_ti0;
      if (ncand < 0) {
        random(y0);
        gs2_basis(y0);
        continue;
      }

      int64_t test_cap = k_target > 8 ? k_target : 8;
      if (test_cap > l)
        test_cap = l;
      double best_res = INFINITY;
      bool have_best = false, accepted_this = false, polish_stalled = false;
      int64_t tested = 0;
      const int ny_used = split ? ncand : (l + 1) / 2;
      if (d.Vc && d.o.precond_aat == KRANS_PRECOND_NONE) {
        CandState st{best_res, have_best, accepted_this, polish_stalled, converged};
        candidates_block(Y, split, l, ncand, test_cap, ny_used, prescreen, accept, st);
        best_res = st.best_res;
        have_best = st.have_best;
        accepted_this = st.accepted_this;
        converged = st.converged;
        tested = test_cap; // the one-by-one loop below is skipped
      }
      for (int t = 0; t < ncand && tested < test_cap && tm.ok() && !(d.Vc && d.o.precond_aat == KRANS_PRECOND_NONE); ++t) {
        const int jb = *(volatile int32_t *)&d.ord[t];
        double ce2 = 0.0;
        for (int q = 0; q < ny_used; q++) {
          const double cq = coef(split, l, jb, q);
          ce2 += cq * cq;
        }
        if (!(ce2 >= 1e-20))
          continue;
        form_candidate(Y, split, l, jb, ny_used, v);
        gs2_basis(v);
        const double nv = nrm2(n, v);
        if (!isfinite(nv) || nv < 1e-8)
          continue;
        scale(n, 1.0 / nv, v);
        ++tested;
        double res = mulF_norm(v, tmv);
        if (!isfinite(res))
          continue;
        if (res > prescreen || polish_stalled) {
          if (res < best_res) {
            best_res = res;
            copy(n, v, best_v);
            have_best = true;
          }
          continue;
        }
        int64_t cg_its = 0;
        bool hit_maxit = false;
        const int passes = o.projector_passes > 1 ? o.projector_passes : 1;
        for (int pass = 0; pass < passes && res > accept && tm.ok(); ++pass) {
          double rn;
          const uint64_t t_cg0 = globaltimer_ns();
          cg_its = cg(tmv, vp, o.cg_maxit, o.cg_rel_tol, o.cg_breakdown_tol, &rn); // vp = F^T w
          c.t_cg += globaltimer_ns() - t_cg0;
          c.cg_solves++;
          if (cg_its >= o.cg_maxit) {
            c.cg_maxit_hits++;
            hit_maxit = true;
          }
          team_for(tm, n, [&](int64_t i) { vp[i] = v[i] - vp[i]; });
          c.bytes += 24.0 * n;
          tm.sync();
          gs2_basis(vp);
          const double np = nrm2(n, vp);
          if (!isfinite(np) || np < 1e-14)
            break;
          scale(n, 1.0 / np, vp);
          const double res_p = mulF_norm(vp, wm);
          if (!(res_p < res))
            break;
          double *t1 = v;
          v = vp;
          vp = t1;
          res = res_p;
          t1 = tmv;
          tmv = wm;
          wm = t1;
        }
        if (res <= accept) {
          copy(n, v, d.basis + nb * d.ldb);
          nb++;
          accepted_this = true;
          if (nb >= k_target) {
            converged = true;
            break;
          }
        } else {
          polish_stalled = polish_stalled || hit_maxit;
          if (res < best_res) {
            best_res = res;
            copy(n, v, best_v);
            have_best = true;
          }
        }
      }
      if (converged)
        break;
      if (!accepted_this) {
        ++rsa;
        if (o.stagnation_restarts > 0 && rsa >= o.stagnation_restarts)
          break;
      } else {
        rsa = 0;
      }
      if (have_best) {
        copy(n, best_v, y0);
      } else {
        random(y0);
        gs2_basis(y0);
      }
    }
    if (!converged && nb < k_target && tm.ok()) {
      int64_t failures = 0;
      while (nb < k_target && failures < 8 && tm.ok()) {
        if (try_project_random(accept))
          failures = 0;
        else
          ++failures;
      }
      converged = nb >= k_target;
    }
    tm.sync();
    if (tm.leader()) {
      CyclicDevResult *R = d.res;
      R->n_found = nb;
      R->restarts = c.restarts;
      R->krylov_steps_total = c.steps;
      R->cg_solves = c.cg_solves;
      R->cg_maxit_hits = c.cg_maxit_hits;
      R->spmv = c.spmv;
      R->spmvT = c.spmvT;
      R->frob = frob;
      R->bytes = c.bytes;
      R->converged = converged ? 1 : 0;
      R->status = *(volatile int *)d.status;
      const double tot = (double)(globaltimer_ns() - t_run0) * 1e-6;
      R->phase_ms[0] = (double)c.t_gk * 1e-6;
      R->phase_ms[1] = (double)c.t_tiny * 1e-6;
      R->phase_ms[2] = (double)c.t_cg * 1e-6;
      R->phase_ms[3] = tot - R->phase_ms[0] - R->phase_ms[1] - R->phase_ms[2];
    }
  }
};

// Entry for the early exits of find_right_nullspace that need no work
// (CyclicLanczosSolver.cpp:297-309) is handled on the host.

template <class KT>
__global__ void __launch_bounds__(512) cyclic_grid_kernel(CyclicDesc d) {
  __shared__ TeamShared sh;
  TeamGrid tm{&sh, d.status, d.gb, d.gpart, 0, 0};
  CyclicSolver<TeamGrid, KT> s(tm, d);
  s.run();
}

} // namespace kr
