// Device building blocks of the KraNS B200 engine.
//
// The solvers are written once against a "team": the set of threads that
// cooperates on one null-space solve.
//   TeamCta  - one thread block (batched serving: many solves side by side,
//              one per block, synchronised with __syncthreads).
//   TeamGrid - every block of a cooperative launch (one large solve on the
//              whole GPU, synchronised with a bounded grid barrier).
// All reductions use a fixed tree whose shape depends only on the team size,
// so a solve gives bit-identical results alone and inside a batch.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/krans_cuda.h"
#include "kr_types.cuh"

#define KR_DEV __device__ __forceinline__
#define KR_MAX_WARPS 32
#ifndef KR_RED_K
#define KR_RED_K 8 // values per fused team reduction
#endif
#ifndef KR_SPMV_ROWS
#define KR_SPMV_ROWS 4 // row groups each warp keeps in flight in team_spmv
#endif

namespace kr {

// ---------------------------------------------------------------------------
// timing / barrier primitives
// ---------------------------------------------------------------------------
KR_DEV uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A grid barrier wait gives up after this long and flags KRANS_ERR_TIMEOUT
// (the longest legitimate wait is a serial section on the leader block).
constexpr uint64_t kBarrierTimeoutNs = 8ull * 1000ull * 1000ull * 1000ull;

// Per-block shared memory used by the team primitives.
struct TeamShared {
  double red[2][KR_MAX_WARPS * KR_RED_K]; // double-buffered warp partials
  double bc[KR_RED_K];                    // broadcast slots (grid reductions)
  double h[160];                          // Gram-Schmidt coefficients
  double cpart[2][KR_RED_K];              // cluster reductions: this block's partials
  int ibuf[64];                           // small integer scratch
};

KR_DEV double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-level sum of K values; every thread receives the totals. Fixed order:
// butterfly inside each warp, then warps summed in index order.
template <int K>
KR_DEV void block_sum(TeamShared *sh, int &buf, double (&v)[K]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; k++)
    v[k] = warp_sum(v[k]);
  double *r = sh->red[buf];
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; k++)
      r[wid * KR_RED_K + k] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) {
    double s = 0.0;
    for (int w = 0; w < nw; w++)
      s += r[w * KR_RED_K + k];
    v[k] = s;
  }
  buf ^= 1;
}

// ---------------------------------------------------------------------------
// Teams
// ---------------------------------------------------------------------------
struct TeamCta {
  TeamShared *sh;
  int *err; // per-solve status word (global)
  int buf;
  KR_DEV int64_t tid() const { return threadIdx.x; }
  KR_DEV int64_t nthreads() const { return blockDim.x; }
  KR_DEV int64_t warp_id() const { return threadIdx.x >> 5; }
  KR_DEV int64_t nwarps() const { return blockDim.x >> 5; }
  KR_DEV bool lead_cta() const { return true; }
  KR_DEV bool leader() const { return threadIdx.x == 0; }
  KR_DEV int cta_rank() const { return 0; }
  KR_DEV int ncta() const { return 1; }
  KR_DEV bool ok() const { return *(volatile int *)err == 0; }
  KR_DEV void sync() { __syncthreads(); }
  template <int K> KR_DEV void sum(double (&v)[K]) { block_sum<K>(sh, buf, v); }
  KR_DEV double sum1(double x) {
    double v[1] = {x};
    sum<1>(v);
    return v[0];
  }
  // make values written by the leader block visible to the team
  KR_DEV void publish() { __syncthreads(); }
};

struct TeamGrid {
  TeamShared *sh;
  int *err;
  GridBarrierState *gb;
  double *gpart; // [2][gridDim.x][KR_RED_K]
  int buf;
  int gbuf;
  KR_DEV int64_t tid() const { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
  KR_DEV int64_t nthreads() const { return (int64_t)gridDim.x * blockDim.x; }
  KR_DEV int64_t warp_id() const { return tid() >> 5; }
  KR_DEV int64_t nwarps() const { return nthreads() >> 5; }
  KR_DEV bool lead_cta() const { return blockIdx.x == 0; }
  KR_DEV bool leader() const { return blockIdx.x == 0 && threadIdx.x == 0; }
  KR_DEV int cta_rank() const { return blockIdx.x; }
  KR_DEV int ncta() const { return gridDim.x; }
  KR_DEV bool ok() const { return *(volatile int *)err == 0 && *(volatile int *)&gb->error == 0; }

  // Sense-counting grid barrier with a bounded wait. On timeout it records
  // KRANS_ERR_TIMEOUT in the solve's status word; afterwards every barrier
  // returns immediately and the solver's bounded loops unwind.
  KR_DEV void sync() {
    __syncthreads();
    if (threadIdx.x == 0) {
      volatile int *verr = &gb->error;
      if (*verr == 0) {
        volatile unsigned *vgen = &gb->gen;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&gb->count, 1u);
        if (arrived == gridDim.x - 1) {
          atomicExch(&gb->count, 0u);
          __threadfence();
          atomicAdd(&gb->gen, 1u);
        } else {
          const uint64_t t0 = globaltimer_ns();
          const uint64_t limit = gb->timeout_ns ? gb->timeout_ns : kBarrierTimeoutNs;
          while (*vgen == g) {
            if (*verr != 0)
              break;
            if (globaltimer_ns() - t0 > limit) {
              atomicCAS(&gb->error, 0, KRANS_ERR_TIMEOUT);
              atomicCAS(err, 0, KRANS_ERR_TIMEOUT);
              break;
            }
            __nanosleep(40);
          }
        }
        __threadfence();
      }
    }
    __syncthreads();
  }

  template <int K> KR_DEV void sum(double (&v)[K]) {
    block_sum<K>(sh, buf, v);
    double *gp = gpart + (size_t)gbuf * gridDim.x * KR_RED_K;
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; k++)
        gp[(size_t)blockIdx.x * KR_RED_K + k] = v[k];
    }
    sync();
    // warp 0 of every block sums the block partials in the same fixed order
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
#pragma unroll
      for (int k = 0; k < K; k++) {
        double s = 0.0;
        for (unsigned b = lane; b < gridDim.x; b += 32)
          s += __ldcg(gp + (size_t)b * KR_RED_K + k);
        s = warp_sum(s);
        if (lane == 0)
          sh->bc[k] = s;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++)
      v[k] = sh->bc[k];
    __syncthreads();
    gbuf ^= 1;
  }
  KR_DEV double sum1(double x) {
    double v[1] = {x};
    sum<1>(v);
    return v[0];
  }
  KR_DEV void publish() { sync(); }
};

// A thread-block cluster (up to 16 blocks on distinct SMs of one GPC) as a
// team: hardware cluster barrier, reductions through distributed shared
// memory (each block publishes its partial in its own shared memory, every
// block sums the partials of ranks 0..size-1 in order).
struct TeamCluster {
  TeamShared *sh;
  int *err;
  int buf;
  int cbuf;
  unsigned rank, csize;
  KR_DEV int64_t tid() const { return (int64_t)rank * blockDim.x + threadIdx.x; }
  KR_DEV int64_t nthreads() const { return (int64_t)csize * blockDim.x; }
  KR_DEV int64_t warp_id() const { return tid() >> 5; }
  KR_DEV int64_t nwarps() const { return nthreads() >> 5; }
  KR_DEV bool lead_cta() const { return rank == 0; }
  KR_DEV bool leader() const { return rank == 0 && threadIdx.x == 0; }
  KR_DEV int cta_rank() const { return (int)rank; }
  KR_DEV int ncta() const { return (int)csize; }
  KR_DEV bool ok() const { return *(volatile int *)err == 0; }
  KR_DEV void sync() { cooperative_groups::this_cluster().sync(); }
  template <int K> KR_DEV void sum(double (&v)[K]) {
    block_sum<K>(sh, buf, v);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; k++)
        sh->cpart[cbuf][k] = v[k];
    }
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    cl.sync();
    // every thread sums the ranks' partials in rank order straight from their
    // shared memory (the same order as a sequential sum from rank 0). The
    // next reduction writes the other buffer, and the one after it is behind
    // that reduction's cluster barrier, which no block passes before all
    // blocks have read this one.
    double t[K];
#pragma unroll
    for (int k = 0; k < K; k++)
      t[k] = 0.0;
    for (unsigned r = 0; r < csize; r++) {
      const double *peer = cl.map_shared_rank(&sh->cpart[cbuf][0], r);
#pragma unroll
      for (int k = 0; k < K; k++)
        t[k] += peer[k];
    }
#pragma unroll
    for (int k = 0; k < K; k++)
      v[k] = t[k];
    cbuf ^= 1;
  }
  KR_DEV double sum1(double x) {
    double v[1] = {x};
    sum<1>(v);
    return v[0];
  }
  KR_DEV void publish() { sync(); }
};

// ---------------------------------------------------------------------------
// Element-wise team loops (grid-stride over the team's threads)
// ---------------------------------------------------------------------------
template <class Team, class F> KR_DEV void team_for(Team &tm, int64_t len, F f) {
  const int64_t nt = tm.nthreads();
  for (int64_t i = tm.tid(); i < len; i += nt)
    f(i);
}

template <class T> KR_DEV double to_d(T x) { return (double)x; }
KR_DEV int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

template <class Team, class TX, class TY>
KR_DEV double team_dot(Team &tm, int64_t len, const TX *x, const TY *y) {
  double s = 0.0;
  const int64_t nt = tm.nthreads();
#pragma unroll 4
  for (int64_t i = tm.tid(); i < len; i += nt)
    s += to_d(x[i]) * to_d(y[i]);
  return tm.sum1(s);
}

template <class Team, class TX> KR_DEV double team_nrm2(Team &tm, int64_t len, const TX *x) {
  double s = 0.0;
  const int64_t nt = tm.nthreads();
  for (int64_t i = tm.tid(); i < len; i += nt) {
    const double v = to_d(x[i]);
    s += v * v;
  }
  return sqrt(tm.sum1(s));
}

// h[q] = <S_q, w> for q < ns (S columns at stride ld); results in tm.sh->h
// (all threads of every block see them after the call).
template <class Team, class TS, class TW>
KR_DEV void team_multidot(Team &tm, int64_t len, const TS *S, int64_t ld, int ns, const TW *w) {
  const int64_t nt = tm.nthreads();
  for (int q0 = 0; q0 < ns; q0 += KR_RED_K) {
    double acc[KR_RED_K];
#pragma unroll
    for (int k = 0; k < KR_RED_K; k++)
      acc[k] = 0.0;
    const int qn = min(KR_RED_K, ns - q0);
#pragma unroll 4
    for (int64_t i = tm.tid(); i < len; i += nt) {
      const double wi = to_d(w[i]);
#pragma unroll
      for (int k = 0; k < KR_RED_K; k++)
        if (k < qn)
          acc[k] += to_d(S[(int64_t)(q0 + k) * ld + i]) * wi;
    }
    tm.template sum<KR_RED_K>(acc);
    if (threadIdx.x < (unsigned)qn)
      tm.sh->h[q0 + threadIdx.x] = acc[threadIdx.x];
  }
  __syncthreads();
}

// w -= sum_q S_q * coef[q]  (coef in shared memory). The subtractions run in
// q order for every element; the loads of several q are issued before their
// subtractions, so a thread keeps 8-16 loads in flight instead of waiting out
// one load per q (the short vectors of small solves are latency-bound on this).
template <class Team, class TS, class TW>
KR_DEV void team_multi_axpy(Team &tm, int64_t len, const TS *S, int64_t ld, int ns,
                            const double *coef, TW *w) {
  const int64_t nt = tm.nthreads();
  int64_t i = tm.tid();
  for (; i + 3 * nt < len; i += 4 * nt) {
    double acc[4];
#pragma unroll
    for (int u = 0; u < 4; u++)
      acc[u] = to_d(w[i + u * nt]);
    int q = 0;
    for (; q + 3 < ns; q += 4) {
      double sv[4][4];
#pragma unroll
      for (int t = 0; t < 4; t++)
#pragma unroll
        for (int u = 0; u < 4; u++)
          sv[t][u] = to_d(S[(int64_t)(q + t) * ld + i + u * nt]);
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const double cq = coef[q + t];
#pragma unroll
        for (int u = 0; u < 4; u++)
          acc[u] -= sv[t][u] * cq;
      }
    }
    for (; q < ns; q++) {
      const double cq = coef[q];
      const TS *sq = S + (int64_t)q * ld + i;
      double sv[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
        sv[u] = to_d(sq[u * nt]);
#pragma unroll
      for (int u = 0; u < 4; u++)
        acc[u] -= sv[u] * cq;
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
      w[i + u * nt] = (TW)acc[u];
  }
  for (; i < len; i += nt) {
    double acc = to_d(w[i]);
    int q = 0;
    for (; q + 7 < ns; q += 8) {
      double sv[8];
#pragma unroll
      for (int t = 0; t < 8; t++)
        sv[t] = to_d(S[(int64_t)(q + t) * ld + i]);
#pragma unroll
      for (int t = 0; t < 8; t++)
        acc -= sv[t] * coef[q + t];
    }
    for (; q < ns; q++)
      acc -= to_d(S[(int64_t)q * ld + i]) * coef[q];
    w[i] = (TW)acc;
  }
}

// Streams `len` elements with each thread handling 4 indices per step; the
// functor gets (index array, count) and must load all inputs before storing.
template <class Team, class F> KR_DEV void team_for4(Team &tm, int64_t len, F f) {
  const int64_t nt = tm.nthreads();
  int64_t i = tm.tid();
  for (; i + 3 * nt < len; i += 4 * nt) {
    const int64_t idx[4] = {i, i + nt, i + 2 * nt, i + 3 * nt};
    f(idx, 4);
  }
  for (; i < len; i += nt) {
    const int64_t idx[4] = {i, i, i, i};
    f(idx, 1);
  }
}

// ---------------------------------------------------------------------------
// CSR SpMV inside a team: `lanes` threads per row (power of two <= 32), rows
// handed out in warp-uniform blocks so the shuffles see full warps. The
// epilogue gets (row, sum) on the first lane of the row group.
// ---------------------------------------------------------------------------
template <class Acc> struct AccOf;
template <> struct AccOf<double> { using T = double; };
template <> struct AccOf<float> { using T = float; };

// Thread-per-row SpMV for matrices whose rows all hold exactly L entries
// (L = 1, 2 or 4): no row pointers, vector loads of the (column, value)
// pairs. The products are combined with the tree of an L-lane butterfly.
template <int L, class Team, class VT, class GX, class Epi>
KR_DEV void team_spmv_uniform(Team &tm, int64_t rows, const int32_t *__restrict__ ci,
                              const VT *__restrict__ val, GX gx, Epi epi) {
  using Acc = typename AccOf<VT>::T;
  using XT = decltype(gx(0));
  constexpr int R = KR_SPMV_ROWS;
  const int64_t nt = tm.nthreads();
  for (int64_t i0 = tm.tid(); i0 < rows; i0 += (int64_t)R * nt) {
    int32_t c[R][L];
    VT v[R][L];
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int64_t i = i0 + (int64_t)u * nt;
      if (i < rows) {
        if constexpr (L == 2) {
          const int2 cc = __ldg(reinterpret_cast<const int2 *>(ci) + i);
          c[u][0] = cc.x;
          c[u][1] = cc.y;
          if constexpr (sizeof(VT) == 8) {
            const double2 vv = __ldg(reinterpret_cast<const double2 *>(val) + i);
            v[u][0] = vv.x;
            v[u][1] = vv.y;
          } else {
            const float2 vv = __ldg(reinterpret_cast<const float2 *>(val) + i);
            v[u][0] = vv.x;
            v[u][1] = vv.y;
          }
        } else if constexpr (L == 4) {
          const int4 cc = __ldg(reinterpret_cast<const int4 *>(ci) + i);
          c[u][0] = cc.x;
          c[u][1] = cc.y;
          c[u][2] = cc.z;
          c[u][3] = cc.w;
#pragma unroll
          for (int j = 0; j < 4; j++)
            v[u][j] = __ldg(val + i * 4 + j);
        } else {
#pragma unroll
          for (int j = 0; j < L; j++) {
            c[u][j] = __ldg(ci + i * L + j);
            v[u][j] = __ldg(val + i * L + j);
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < L; j++) {
          c[u][j] = 0;
          v[u][j] = VT(0);
        }
      }
    }
    XT xv[R][L];
#pragma unroll
    for (int u = 0; u < R; u++)
#pragma unroll
      for (int j = 0; j < L; j++)
        xv[u][j] = (i0 + (int64_t)u * nt < rows) ? gx(c[u][j]) : XT(0);
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int64_t i = i0 + (int64_t)u * nt;
      Acc p[L];
#pragma unroll
      for (int j = 0; j < L; j++)
        p[j] = Acc(0) + (Acc)v[u][j] * (Acc)xv[u][j];
#pragma unroll
      for (int o = L / 2; o > 0; o /= 2)
#pragma unroll
        for (int j = 0; j < o; j++)
          p[j] = p[j] + p[j + o];
      if (i < rows)
        epi(i, p[0]);
    }
  }
}

// CSR SpMV inside a team with a gather functor gx(col) for the input vector.
// `lanes` threads per row (power of two <= 32), rows handed out in
// warp-uniform blocks so the shuffles see full warps; each warp walks R row
// groups at once (all row pointers, then all (column, value) pairs, then all
// gathers are issued before the FMAs). Lane `sub` of a row sums the entries
// b+sub, b+sub+lanes, ... in order, then a fixed butterfly combines the
// lanes: the result does not depend on R or on the team. The epilogue gets
// (row, sum) on the first lane of the row group.
template <class Team, class VT, class GX, class Epi>
KR_DEV void team_spmv_x(Team &tm, int64_t rows, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                        const VT *__restrict__ val, GX gx, int lanes, int32_t ulen, Epi epi) {
  if (ulen == 1 || ulen == 2 || ulen == 4) {
    if (ulen == 2) {
      team_spmv_uniform<2>(tm, rows, ci, val, gx, epi);
      return;
    }
    if (ulen == 4) {
      team_spmv_uniform<4>(tm, rows, ci, val, gx, epi);
      return;
    }
    if (ulen == 1) {
      team_spmv_uniform<1>(tm, rows, ci, val, gx, epi);
      return;
    }
  }
  using Acc = typename AccOf<VT>::T;
  using XT = decltype(gx(0));
  constexpr int R = KR_SPMV_ROWS;
  const int lane = threadIdx.x & 31;
  const int sub = lane & (lanes - 1), grp = lane / lanes;
  const int rpw = 32 / lanes;
  const int64_t chunk = (int64_t)rpw * R;
  const int64_t nw = tm.nwarps();
  for (int64_t base = tm.warp_id() * chunk; base < rows; base += nw * chunk) {
    int32_t b[R], e[R];
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int64_t i = base + (int64_t)u * rpw + grp;
      b[u] = 0;
      e[u] = 0;
      if (i < rows) {
        b[u] = __ldg(rp + i) + sub;
        e[u] = __ldg(rp + i + 1);
      }
    }
    Acc s[R];
#pragma unroll
    for (int u = 0; u < R; u++)
      s[u] = Acc(0);
    for (int32_t j = 0;; j += lanes) {
      int32_t c[R];
      VT v[R];
      bool ok[R], more = false;
#pragma unroll
      for (int u = 0; u < R; u++) {
        const int32_t k = b[u] + j;
        ok[u] = k < e[u];
        more |= (k + lanes) < e[u];
        c[u] = ok[u] ? __ldg(ci + k) : 0;
        v[u] = ok[u] ? __ldg(val + k) : VT(0);
      }
      XT xv[R];
#pragma unroll
      for (int u = 0; u < R; u++)
        xv[u] = ok[u] ? gx(c[u]) : XT(0);
#pragma unroll
      for (int u = 0; u < R; u++)
        if (ok[u])
          s[u] += (Acc)v[u] * (Acc)xv[u];
      if (!more)
        break;
    }
#pragma unroll
    for (int u = 0; u < R; u++) {
      for (int o = lanes >> 1; o > 0; o >>= 1)
        s[u] += __shfl_xor_sync(0xffffffffu, s[u], o);
      const int64_t i = base + (int64_t)u * rpw + grp;
      if (i < rows && sub == 0)
        epi(i, s[u]);
    }
  }
}

template <class Team, class VT, class XT, class Epi>
KR_DEV void team_spmv(Team &tm, int64_t rows, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                      const VT *__restrict__ val, const XT *__restrict__ x, int lanes, Epi epi) {
  team_spmv_x(tm, rows, rp, ci, val, [&](int32_t c) { return x[c]; }, lanes, 0, epi);
}

// y = V x over a CsrView (uses the uniform-row-length path when it applies)
template <class Team, class VT, class XT, class Epi>
KR_DEV void csr_mv(Team &tm, const CsrView &V, const VT *val, const XT *__restrict__ x, Epi epi) {
  team_spmv_x(tm, V.rows, V.rp, V.ci, val, [&](int32_t c) { return x[c]; }, V.lanes, V.ulen, epi);
}

// CSR SpMV over KR_NBP right-hand sides stored interleaved (element (i, j) at
// i * KR_NBP + j). Eight consecutive threads share a row and thread j of the
// group owns column j (the team size is a multiple of KR_NBP, so a thread's
// column never changes): the (column, value) loads are broadcast inside the
// group and the gather reads 64 contiguous bytes per entry. Each thread sums
// its column over the row's entries in storage order (the same order in both
// variants below); threads whose column is not `active` skip the row. Every
// thread keeps R rows in flight so the gathers of several rows overlap.
template <int L, int R, class Team, class GX, class Epi>
KR_DEV void team_spmv_block_uniform(Team &tm, int64_t rows, const int32_t *__restrict__ ci,
                                    const double *__restrict__ val, GX gx, Epi epi) {
  const int64_t ng = tm.nthreads() / KR_NBP;
  for (int64_t i0 = tm.tid() / KR_NBP; i0 < rows; i0 += (int64_t)R * ng) {
    int32_t c[R][L];
    double v[R][L];
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int64_t i = i0 + (int64_t)u * ng;
#pragma unroll
      for (int j = 0; j < L; j++) {
        c[u][j] = i < rows ? __ldg(ci + i * L + j) : 0;
        v[u][j] = i < rows ? __ldg(val + i * L + j) : 0.0;
      }
    }
    double xv[R][L];
#pragma unroll
    for (int u = 0; u < R; u++)
#pragma unroll
      for (int j = 0; j < L; j++)
        xv[u][j] = i0 + (int64_t)u * ng < rows ? gx(c[u][j]) : 0.0;
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int64_t i = i0 + (int64_t)u * ng;
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < L; j++)
        s += v[u][j] * xv[u][j];
      if (i < rows)
        epi(i, s);
    }
  }
}

template <class Team, class GX, class Epi>
KR_DEV void team_spmv_block(Team &tm, int64_t rows, const int32_t *__restrict__ rp,
                            const int32_t *__restrict__ ci, const double *__restrict__ val, int32_t ulen,
                            bool active, GX gx, Epi epi) {
  if (!active)
    return; // no barrier inside: threads of inactive columns simply skip
  if (ulen == 2) {
    team_spmv_block_uniform<2, 4>(tm, rows, ci, val, gx, epi);
    return;
  }
  if (ulen == 1) {
    team_spmv_block_uniform<1, 8>(tm, rows, ci, val, gx, epi);
    return;
  }
  if (ulen == 4) {
    team_spmv_block_uniform<4, 2>(tm, rows, ci, val, gx, epi);
    return;
  }
  constexpr int R = 4;
  const int64_t ng = tm.nthreads() / KR_NBP;
  for (int64_t i0 = tm.tid() / KR_NBP; i0 < rows; i0 += (int64_t)R * ng) {
    int32_t b[R], e[R];
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int64_t i = i0 + (int64_t)u * ng;
      b[u] = 0;
      e[u] = 0;
      if (i < rows) {
        b[u] = __ldg(rp + i);
        e[u] = __ldg(rp + i + 1);
      }
    }
    double s[R];
#pragma unroll
    for (int u = 0; u < R; u++)
      s[u] = 0.0;
    for (int32_t j = 0;; ++j) {
      int32_t c[R];
      double v[R];
      bool ok[R], more = false;
#pragma unroll
      for (int u = 0; u < R; u++) {
        const int32_t k = b[u] + j;
        ok[u] = k < e[u];
        more |= (k + 1) < e[u];
        c[u] = ok[u] ? __ldg(ci + k) : 0;
        v[u] = ok[u] ? __ldg(val + k) : 0.0;
      }
      double xv[R];
#pragma unroll
      for (int u = 0; u < R; u++)
        xv[u] = ok[u] ? gx(c[u]) : 0.0;
#pragma unroll
      for (int u = 0; u < R; u++)
        if (ok[u])
          s[u] += v[u] * xv[u];
      if (!more)
        break;
    }
#pragma unroll
    for (int u = 0; u < R; u++) {
      const int64_t i = i0 + (int64_t)u * ng;
      if (i < rows)
        epi(i, s[u]);
    }
  }
}

// Algorithmic HBM bytes of one CSR SpMV (rows r, cols c, nnz z, value width
// w, x width wx, y width wy): row pointers, columns+values, x once, y once.
__host__ __device__ inline double spmv_bytes(int64_t r, int64_t c, int64_t z, int w, int wx, int wy) {
  return 4.0 * (double)(r + 1) + (double)z * (w + 4) + (double)c * wx + (double)r * wy;
}

// ---------------------------------------------------------------------------
// Random normal vectors
// ---------------------------------------------------------------------------
KR_DEV uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

// Block-cooperative MT19937 regeneration of 624 words: src -> dst. The
// recurrence new[i] = f(old[i], old[i+1], new-or-old[(i+397) mod 624]) is
// evaluated in four dependency waves ([0,227), [227,454), [454,623), 623).
KR_DEV void mt_regen_block(const uint32_t *src, uint32_t *dst) {
  const int t = threadIdx.x;
  auto f = [&](int i, uint32_t a, uint32_t b, uint32_t c) {
    const uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
    uint32_t v = c ^ (y >> 1);
    if (y & 1u)
      v ^= 0x9908b0dfu;
    dst[i] = v;
  };
  for (int i = t; i < 227; i += blockDim.x)
    f(i, src[i], src[i + 1], src[i + 397]);
  __syncthreads();
  for (int i = 227 + t; i < 454; i += blockDim.x)
    f(i, src[i], src[i + 1], dst[i - 227]);
  __syncthreads();
  for (int i = 454 + t; i < 623; i += blockDim.x)
    f(i, src[i], src[i + 1], dst[i - 227]);
  __syncthreads();
  if (t == 0)
    f(623, src[623], dst[0], dst[396]);
  __syncthreads();
}

// One block draws the next n normals of an MT19937 + polar stream, exactly
// as std::normal_distribution<double> consumes std::mt19937 in libstdc++:
// each polar attempt takes four 32-bit words (two 53-bit canonicals); an
// accepted attempt yields y*m then x*m, and an unused x*m is carried over.
// Needs blockDim.x >= 160.
KR_DEV void block_mt_normals(RngState *st, double *out, int64_t n) {
  __shared__ uint32_t smt[2][624];
  __shared__ int s_wsum[8];
  __shared__ int s_last;
  __shared__ double s_saved;
  __shared__ int s_has_saved;
  int cur = 0;
  for (int i = threadIdx.x; i < 624; i += blockDim.x)
    smt[0][i] = st->mt[i];
  int idx = st->idx;
  if (threadIdx.x == 0) {
    s_has_saved = st->has_saved;
    s_saved = st->saved;
  }
  __syncthreads();
  int64_t pos = 0;
  if (n > 0 && s_has_saved) {
    if (threadIdx.x == 0)
      out[0] = s_saved;
    pos = 1;
    __syncthreads();
    if (threadIdx.x == 0)
      s_has_saved = 0;
  }
  __syncthreads();
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  while (pos < n) {
    if (idx >= 624) {
      mt_regen_block(smt[cur], smt[cur ^ 1]);
      cur ^= 1;
      idx = 0;
    }
    const int navail = (624 - idx) >> 2;
    bool acc = false;
    double x = 0.0, y = 0.0, r2 = 0.0;
    if (t < navail) {
      const uint32_t *w = smt[cur] + idx + 4 * t;
      const double a = (double)mt_temper(w[0]), b = (double)mt_temper(w[1]);
      const double c = (double)mt_temper(w[2]), d = (double)mt_temper(w[3]);
      double u1 = __dadd_rn(a, __dmul_rn(b, 4294967296.0)) * 0x1p-64;
      double u2 = __dadd_rn(c, __dmul_rn(d, 4294967296.0)) * 0x1p-64;
      if (u1 >= 1.0)
        u1 = 0x1.fffffffffffffp-1;
      if (u2 >= 1.0)
        u2 = 0x1.fffffffffffffp-1;
      x = __dadd_rn(__dmul_rn(2.0, u1), -1.0);
      y = __dadd_rn(__dmul_rn(2.0, u2), -1.0);
      r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
      acc = !(r2 > 1.0 || r2 == 0.0);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, acc);
    if (lane == 0 && wid < 8)
      s_wsum[wid] = __popc(bal);
    if (t == 0)
      s_last = -1;
    __syncthreads();
    int before = __popc(bal & ((1u << lane) - 1u));
    int total = 0;
    for (int w = 0; w < 5; w++) {
      if (w < wid)
        before += s_wsum[w];
      total += s_wsum[w];
    }
    const int64_t need = (n - pos + 1) >> 1; // pairs still needed
    if (acc && before < need) {
      const double mult = sqrt(-2.0 * log(r2) / r2);
      const int64_t p = pos + 2 * (int64_t)before;
      out[p] = __dmul_rn(y, mult);
      if (p + 1 < n) {
        out[p + 1] = __dmul_rn(x, mult);
      } else {
        s_saved = __dmul_rn(x, mult);
        s_has_saved = 1;
      }
      if (before == need - 1)
        s_last = t;
    }
    __syncthreads();
    if (total >= need) {
      idx += 4 * (s_last + 1);
      pos = n;
    } else {
      idx += 4 * navail;
      pos += 2 * (int64_t)total;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < 624; i += blockDim.x)
    st->mt[i] = smt[cur][i];
  if (threadIdx.x == 0) {
    st->idx = idx;
    st->has_saved = s_has_saved;
    st->saved = s_saved;
  }
  __syncthreads();
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11), counter-based.
KR_DEV uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Normal variate number `ctr` of the stream `key` (Box-Muller on two
// 53-bit uniforms from one Philox block).
KR_DEV double philox_normal(uint64_t key, uint64_t ctr) {
  const uint4 r = philox4x32_10(make_uint4((uint32_t)ctr, (uint32_t)(ctr >> 32), 0x4b52414eu, 0u),
                                make_uint2((uint32_t)key, (uint32_t)(key >> 32)));
  const uint64_t a = ((uint64_t)r.x << 21) ^ (uint64_t)(r.y >> 11);
  const uint64_t b = ((uint64_t)r.z << 21) ^ (uint64_t)(r.w >> 11);
  const double u1 = ((double)(a & ((1ull << 53) - 1)) + 1.0) * 0x1p-53; // (0, 1]
  const double u2 = (double)(b & ((1ull << 53) - 1)) * 0x1p-53;         // [0, 1)
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// Fill out[0..n) with the stream's next n normals, as a team. MT19937 is
// generated by the team's leader block; Philox by every thread.
template <class Team> KR_DEV void team_random_normal(Team &tm, RngState *st, double *out, int64_t n) {
  if (*(volatile int32_t *)&st->mode == KRANS_RNG_PHILOX) {
    const uint64_t key = *(volatile uint64_t *)&st->philox_key;
    const uint64_t base = *(volatile uint64_t *)&st->philox_ctr;
    team_for(tm, n, [&](int64_t i) { out[i] = philox_normal(key, base + (uint64_t)i); });
    tm.sync();
    if (tm.leader())
      st->philox_ctr = base + (uint64_t)n;
    tm.publish();
  } else {
    if (tm.lead_cta())
      block_mt_normals(st, out, n);
    tm.publish();
  }
}

} // namespace kr
