// Tall-skinny products of the block solver:
//   team_gemm_tn:       C = A^T B (Gram matrices S = Z^T Z, G = Z^T (AZ),
//                       Cholesky QR, projections), FP64 tensor cores: tiled
//                       with shared-memory panels for long, wide products,
//                       one warp per output tile otherwise
//   team_gram2_direct:  S = Z^T Z and G = Z^T (AZ) in one pass (short or
//                       narrow blocks)
//   team_combine_sub:   X -= S C
//   team_combine:       out = Z * Y[roff:roff+zc, 0:q] (n x q)
// Sums run in a fixed order that depends only on the team size, so results
// are deterministic for a given team size.
#pragma once

#include "kr_device.cuh"

namespace kr {

// FP64 tensor-core MMA (DMMA) m8n8k4: D = A(8x4, row) * B(4x8, col) + C.
KR_DEV void dmma_8x8x4(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// C = A^T B (a x b, leading dim a) for tall-skinny column-major A (n x a) and
// B (n x b), leading dim ld, on the FP64 tensor cores with shared-memory
// panels. Work items are (64 x 64 tile of C, fixed chunk of rows); a block
// stages 16-row panels of the tile's 64 columns of A and of B in shared
// memory, and each of its 16 warps accumulates a 16 x 16 piece (four DMMA
// 8x8 tiles). Each item leaves its partial tile in `part`; the partials are
// then summed in chunk order, so the result depends only on the team size
// (which fixes the chunking), not on which block ran which item. `part` must
// hold ceil(a/64) * ceil(b/64) * 4096 * nchunks doubles, nchunks <= ncta.
// Blocks of 512 threads.
#define KR_GT 64 // tile edge
#define KR_GK 16 // rows per shared-memory panel
template <class Team>
KR_DEV void team_gemm_tn_tiled(Team &tm, int64_t n, const double *A, int a, const double *B, int b, int64_t ld,
                               double *C, double *part) {
  __shared__ double sA[KR_GT][KR_GK + 1], sB[KR_GT][KR_GK + 1];
  const int ta = (a + KR_GT - 1) / KR_GT, tb = (b + KR_GT - 1) / KR_GT, nt = ta * tb;
  const int ncta = tm.ncta();
  const int64_t kblocks = (n + KR_GK - 1) / KR_GK;
  const int nch = (int)imin64(imin64(ncta, kblocks > 0 ? kblocks : 1), (int64_t)(2 * ncta + nt - 1) / nt);
  const int nchunks = nch > 0 ? nch : 1;
  const int64_t kb_per = (kblocks + nchunks - 1) / nchunks; // panels per chunk
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wr = (wid >> 2) * 16, wc = (wid & 3) * 16; // this warp's 16 x 16 piece
  const int items = nt * nchunks;
  for (int it = tm.cta_rank(); it < items; it += ncta) {
    const int tile = it % nt, ch = it / nt;
    const int ti = tile % ta, tj = tile / ta;
    const int64_t kb0 = (int64_t)ch * kb_per, kb1 = imin64(kb0 + kb_per, kblocks);
    double acc[2][2][2];
#pragma unroll
    for (int x = 0; x < 2; x++)
#pragma unroll
      for (int y = 0; y < 2; y++)
        acc[x][y][0] = acc[x][y][1] = 0.0;
    // panels travel global -> registers two ahead of use -> shared memory, so
    // their loads are in flight while the tensor cores work on the current one
    constexpr int PER = (2 * KR_GT * KR_GK + 511) / 512; // elements per thread and panel (512 threads)
    auto fetch = [&](int64_t kb, double (&v)[PER]) {
      const int64_t r0 = kb * KR_GK;
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int e = threadIdx.x + q * 512;
        const int which = e / (KR_GT * KR_GK), rem = e % (KR_GT * KR_GK);
        const int c = rem / KR_GK, k = rem % KR_GK;
        const int64_t r = r0 + k;
        double x = 0.0;
        if (e < 2 * KR_GT * KR_GK && kb < kb1 && r < n) {
          const int col = (which == 0 ? ti : tj) * KR_GT + c;
          if (col < (which == 0 ? a : b))
            x = (which == 0 ? A : B)[(int64_t)col * ld + r];
        }
        v[q] = x;
      }
    };
    double v0[PER], v1[PER];
    fetch(kb0, v0);
    fetch(kb0 + 1, v1);
    for (int64_t kb = kb0; kb < kb1; kb++) {
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int e = threadIdx.x + q * 512;
        if (e < 2 * KR_GT * KR_GK) {
          const int which = e / (KR_GT * KR_GK), rem = e % (KR_GT * KR_GK);
          const int c = rem / KR_GK, k = rem % KR_GK;
          if (which == 0)
            sA[c][k] = v0[q];
          else
            sB[c][k] = v0[q];
        }
        v0[q] = v1[q];
      }
      __syncthreads();
      fetch(kb + 2, v1);
      if (wid < 16) {
#pragma unroll
        for (int kk = 0; kk < KR_GK; kk += 4) {
          double fa[2], fb[2];
#pragma unroll
          for (int x = 0; x < 2; x++)
            fa[x] = sA[wr + 8 * x + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
          for (int y = 0; y < 2; y++)
            fb[y] = sB[wc + 8 * y + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
          for (int x = 0; x < 2; x++)
#pragma unroll
            for (int y = 0; y < 2; y++)
              dmma_8x8x4(acc[x][y][0], acc[x][y][1], fa[x], fb[y]);
        }
      }
      __syncthreads();
    }
    if (wid < 16) {
      double *pt = part + (size_t)it * (KR_GT * KR_GT);
#pragma unroll
      for (int x = 0; x < 2; x++)
#pragma unroll
        for (int y = 0; y < 2; y++) {
          const int i = wr + 8 * x + (lane >> 2), j = wc + 8 * y + 2 * (lane & 3);
          pt[i + j * KR_GT] = acc[x][y][0];
          pt[i + (j + 1) * KR_GT] = acc[x][y][1];
        }
    }
  }
  tm.sync();
  const int64_t nthr = tm.nthreads();
  for (int64_t e = tm.tid(); e < (int64_t)a * b; e += nthr) {
    const int i = (int)(e % a), j = (int)(e / a);
    const int tile = (i / KR_GT) + ta * (j / KR_GT), li = i % KR_GT, lj = j % KR_GT;
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ch++)
      s += __ldcg(part + (size_t)(tile + ch * nt) * (KR_GT * KR_GT) + li + lj * KR_GT);
    C[e] = s;
  }
  tm.sync();
}

// C = A^T B for tall-skinny A (n x a) and B (n x b), column-major with
// leading dim ld; C is a x b with leading dim a. DMMA 8x8 tiles, one warp per
// tile; each block reduces its fixed row range into a private partial, then
// the partials are summed in block order (deterministic for a team size).
template <class Team>
KR_DEV void team_gemm_tn_direct(Team &tm, int64_t n, const double *A, int a, const double *B, int b, int64_t ld,
                         double *C, double *part) {
  const int ta = (a + 7) / 8, tb = (b + 7) / 8, ntiles = ta * tb;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int ncta = tm.ncta(), rank = tm.cta_rank();
  const int64_t per = (n + ncta - 1) / ncta;
  const int64_t r0 = imin64((int64_t)rank * per, n), r1 = imin64(r0 + per, n);
  double *my = part + (size_t)rank * a * b;
  for (int t = wid; t < ntiles; t += nw) {
    const int bi = t % ta, bj = t / ta;
    const int ia = bi * 8 + (lane >> 2), jb = bj * 8 + (lane >> 2);
    const bool va = ia < a, vb = jb < b;
    const double *pa = A + (int64_t)(va ? ia : 0) * ld;
    const double *pb = B + (int64_t)(vb ? jb : 0) * ld;
    double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0;
    int64_t base = r0;
    for (; base + 8 <= r1; base += 8) { // two independent accumulators
      const int64_t r = base + (lane & 3);
      const double x0 = va ? pa[r] : 0.0, y0 = vb ? pb[r] : 0.0;
      const double x1 = va ? pa[r + 4] : 0.0, y1 = vb ? pb[r + 4] : 0.0;
      dmma_8x8x4(c0, c1, x0, y0);
      dmma_8x8x4(e0, e1, x1, y1);
    }
    for (; base < r1; base += 4) {
      const int64_t r = base + (lane & 3);
      const bool in = r < r1;
      const double x0 = (in && va) ? pa[r] : 0.0, y0 = (in && vb) ? pb[r] : 0.0;
      dmma_8x8x4(c0, c1, x0, y0);
    }
    c0 += e0;
    c1 += e1;
    const int ci = bi * 8 + (lane >> 2), cj = bj * 8 + 2 * (lane & 3);
    if (ci < a) {
      if (cj < b)
        my[ci + (size_t)cj * a] = c0;
      if (cj + 1 < b)
        my[ci + (size_t)(cj + 1) * a] = c1;
    }
  }
  tm.sync();
  const int64_t nt = tm.nthreads();
  for (int64_t e = tm.tid(); e < (int64_t)a * b; e += nt) {
    double s = 0.0;
    for (int r = 0; r < ncta; r++)
      s += __ldcg(part + (size_t)r * a * b + e);
    C[e] = s;
  }
  tm.sync();
}


// S = Z^T Z and G = Z^T (AZ) (p x p) in one pass, one warp per 8x8 tile with
// DMMA, operands straight from global memory; each block reduces its fixed
// row range into a private partial (2 p^2 doubles per block in `part`),
// summed in block order. G is formed on every tile, so its two triangles are
// computed independently (as Z_i^T (AZ)_j and Z_j^T (AZ)_i) and the tiny
// GEP's symmetrisation averages them, as the reference's form_gram + 0.5 (G +
// G^T) does; S is formed on the upper tiles and mirrored (its two triangles
// would be the same products in the same order). Used for short or narrow
// blocks.
template <class Team>
KR_DEV void team_gram2_direct(Team &tm, int64_t n, const double *Z, const double *AZ, int64_t ld, int p,
                       double *S, double *G, double *part) {
  const int nt8 = (p + 7) / 8; // 8x8 tiles per dimension
  const int ntiles = nt8 * nt8;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int ncta = tm.ncta(), rank = tm.cta_rank();
  // fixed row range of this block
  const int64_t per = (n + ncta - 1) / ncta;
  const int64_t r0 = imin64((int64_t)rank * per, n), r1 = imin64(r0 + per, n);
  double *myS = part + (size_t)rank * 2 * p * p;
  double *myG = myS + (size_t)p * p;
  // a warp owns one 8x8 tile at a time; the MMA lane layout of m8n8k4:
  // A(row=lane>>2, k=lane&3), B(k=lane&3, col=lane>>2), C rows lane>>2,
  // cols 2*(lane&3) and 2*(lane&3)+1.
  for (int t = wid; t < ntiles; t += nw) {
    const int bi = t % nt8, bj = t / nt8;
    const bool upper = bi <= bj; // warp-uniform
    const int ia = bi * 8 + (lane >> 2), jb = bj * 8 + (lane >> 2);
    const bool va = ia < p, vb = jb < p;
    const double *za = Z + (int64_t)(va ? ia : 0) * ld;
    const double *zb = Z + (int64_t)(vb ? jb : 0) * ld;
    const double *azb = AZ + (int64_t)(vb ? jb : 0) * ld;
    double s0 = 0.0, s1 = 0.0, g0 = 0.0, g1 = 0.0;
    for (int64_t base = r0; base < r1; base += 4) { // warp-uniform trip count
      const int64_t r = base + (lane & 3);
      const bool in = r < r1;
      const double a = (in && va) ? za[r] : 0.0;
      const double ab = (in && vb) ? azb[r] : 0.0;
      if (upper) {
        const double b = (in && vb) ? zb[r] : 0.0;
        dmma_8x8x4(s0, s1, a, b);
      }
      dmma_8x8x4(g0, g1, a, ab);
    }
    const int ci = bi * 8 + (lane >> 2), cj = bj * 8 + 2 * (lane & 3);
    if (ci < p) {
      if (cj < p) {
        if (upper)
          myS[ci + (size_t)cj * p] = s0;
        myG[ci + (size_t)cj * p] = g0;
      }
      if (cj + 1 < p) {
        if (upper)
          myS[ci + (size_t)(cj + 1) * p] = s1;
        myG[ci + (size_t)(cj + 1) * p] = g1;
      }
    }
  }
  tm.sync();
  // sum the block partials in block order: G entry by entry, S on the upper
  // triangle (mirrored)
  const int64_t nt = tm.nthreads();
  for (int64_t e = tm.tid(); e < (int64_t)p * p; e += nt) {
    const int j = (int)(e / p), i = (int)(e % p);
    double s = 0.0, g = 0.0;
    for (int b = 0; b < ncta; b++) {
      const double *ps = part + (size_t)b * 2 * p * p;
      g += __ldcg(ps + (size_t)p * p + e);
      if (i <= j)
        s += __ldcg(ps + e);
    }
    G[e] = g;
    if (i <= j) {
      S[i + (size_t)j * p] = s;
      S[j + (size_t)i * p] = s;
    }
  }
  tm.sync();
}


// C = A^T B: the tiled kernel for long products with wide blocks, where the
// shared-memory panels pay off; the direct one (one warp per 8 x 8 tile,
// operands straight from global memory) for short or narrow ones, where
// streaming full 64-column panels 16 rows at a time through one block costs
// more than it saves (measured: a 1000-row LOBPCG with 3-column blocks ran
// 3.3x slower tiled). `part` must suit both (see each).
template <class Team>
KR_DEV void team_gemm_tn(Team &tm, int64_t n, const double *A, int a, const double *B, int b, int64_t ld,
                         double *C, double *part) {
  if (n >= 131072 && (a >= 32 || b >= 32))
    team_gemm_tn_tiled(tm, n, A, a, B, b, ld, C, part);
  else
    team_gemm_tn_direct(tm, n, A, a, B, b, ld, C, part);
}

// X[:, i] -= sum_j S[:, j] * Cc(j, i) for i < k, j < ns (X, S column-major
// with leading dim ld; Cc leading dim ldc).
template <class Team>
KR_DEV void team_combine_sub(Team &tm, int64_t n, const double *S, int64_t ld, int ns, const double *Cc, int ldc,
                             int k, double *X) {
  const int64_t nt = tm.nthreads();
  for (int64_t r = tm.tid(); r < n; r += nt) {
    for (int i0 = 0; i0 < k; i0 += 8) {
      double acc[8];
#pragma unroll
      for (int t = 0; t < 8; t++)
        acc[t] = (i0 + t < k) ? X[(int64_t)(i0 + t) * ld + r] : 0.0;
      for (int j = 0; j < ns; j++) {
        const double z = S[(int64_t)j * ld + r];
        const double *cj = Cc + j;
#pragma unroll
        for (int t = 0; t < 8; t++)
          if (i0 + t < k)
            acc[t] -= __ldg(cj + (size_t)(i0 + t) * ldc) * z;
      }
#pragma unroll
      for (int t = 0; t < 8; t++)
        if (i0 + t < k)
          X[(int64_t)(i0 + t) * ld + r] = acc[t];
    }
  }
}

// out[:, i] = sum_j Y(roff + j, i) * Z[:, j], i < q, j < zc (column-major,
// both with leading dim ld; Y leading dim ldy).
template <class Team>
KR_DEV void team_combine(Team &tm, int64_t n, const double *Z, int64_t ld, int zc, const double *Y,
                         int ldy, int roff, int q, double *out) {
  const int64_t nt = tm.nthreads();
  for (int64_t r = tm.tid(); r < n; r += nt) {
    for (int i0 = 0; i0 < q; i0 += 8) {
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int j = 0; j < zc; j++) {
        const double z = Z[(int64_t)j * ld + r];
        const double *yr = Y + (roff + j);
#pragma unroll
        for (int t = 0; t < 8; t++)
          if (i0 + t < q)
            acc[t] += __ldg(yr + (size_t)(i0 + t) * ldy) * z;
      }
#pragma unroll
      for (int t = 0; t < 8; t++)
        if (i0 + t < q)
          out[(int64_t)(i0 + t) * ld + r] = acc[t];
    }
  }
}

} // namespace kr
