// Tall-skinny products of the block solver:
//   team_gemm_tn:       C = A^T B (Cholesky QR of short blocks, projections),
//                       FP64 tensor cores: shared-memory panels for long, wide
//                       products (team_gemm_tn_panel), one warp per output
//                       tile otherwise
//   team_gram_sym_tiled: S = Z^T Z and G = Z^T (AZ), upper tiles, panels
//   team_gram2_direct:  S = Z^T Z and G = Z^T (AZ) in one pass (short or
//                       narrow blocks)
//   team_gemm_nn:       out (-)= Z * Y[roff:roff+zc, 0:q] (n x q), FP64 tensor
//                       cores, shared-memory tiles (team_combine, team_combine_sub)
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


// S = Z^T Z and G = Z^T (AZ) (p x p) in one pass, one warp per 8x8 upper
// tile with DMMA, operands straight from global memory; each block reduces
// its fixed row range into a private partial (2 p^2 doubles per block in
// `part`), summed in block order. Like the reference's form_gram
// (LOBPCGSolver.cpp:67-80), which sets S(i,j) = S(j,i) = Z_i.Z_j and
// G(i,j) = G(j,i) = Z_i.(AZ)_j for i <= j, only the upper triangles are
// formed and then mirrored. Used for short or narrow blocks.
template <class Team>
KR_DEV void team_gram2_direct(Team &tm, int64_t n, const double *Z, const double *AZ, int64_t ld, int p,
                       double *S, double *G, double *part) {
  const int nt8 = (p + 7) / 8;                       // 8x8 tiles per dimension
  const int ntiles = nt8 * (nt8 + 1) / 2;            // upper triangle incl. diagonal
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
    // decode upper-triangular tile index t -> (bi <= bj)
    int bi = 0, rem = t;
    while (rem >= nt8 - bi) {
      rem -= nt8 - bi;
      bi++;
    }
    const int bj = bi + rem;
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
      const double b = (in && vb) ? zb[r] : 0.0;
      const double ab = (in && vb) ? azb[r] : 0.0;
      dmma_8x8x4(s0, s1, a, b);
      dmma_8x8x4(g0, g1, a, ab);
    }
    const int ci = bi * 8 + (lane >> 2), cj = bj * 8 + 2 * (lane & 3);
    if (ci < p) {
      if (cj < p) {
        myS[ci + (size_t)cj * p] = s0;
        myG[ci + (size_t)cj * p] = g0;
      }
      if (cj + 1 < p) {
        myS[ci + (size_t)(cj + 1) * p] = s1;
        myG[ci + (size_t)(cj + 1) * p] = g1;
      }
    }
  }
  tm.sync();
  // sum the block partials in block order; fill both triangles
  const int64_t nt = tm.nthreads();
  for (int64_t e = tm.tid(); e < (int64_t)p * p; e += nt) {
    const int j = (int)(e / p), i = (int)(e % p);
    if (i > j)
      continue;
    double s = 0.0, g = 0.0;
    for (int b = 0; b < ncta; b++) {
      const double *ps = part + (size_t)b * 2 * p * p;
      s += __ldcg(ps + e);
      g += __ldcg(ps + (size_t)p * p + e);
    }
    S[i + (size_t)j * p] = s;
    S[j + (size_t)i * p] = s;
    G[i + (size_t)j * p] = g;
    G[j + (size_t)i * p] = g;
  }
  tm.sync();
}


// S = Z^T Z and, when AZ is given, G = Z^T (AZ) (p x p) in one pass over Z
// and AZ, on the FP64 tensor cores with shared-memory panels: the tiled form
// of team_gram2_direct for long, wide blocks. Only the upper 64 x 64 tiles
// are formed and mirrored, as the reference's form_gram does
// (LOBPCGSolver.cpp:67-80: S(i,j) = S(j,i) = Z_i.Z_j, G(i,j) = G(j,i) =
// Z_i.(AZ)_j for i <= j). Work items are (upper tile, fixed chunk of rows);
// a block stages 32-row panels of the tile's columns of Z (and of AZ) in
// shared memory, fetching the next panel into registers while the current
// one is multiplied, and each of its 16 warps accumulates a 16 x 16 piece of
// S (and of G). Partial tiles are summed in chunk order, so the result
// depends only on the team size. `part` must hold (2 ncta + tiles) * 8192
// doubles; needs 512 threads and gram_tiled_smem_bytes() of dynamic shared
// memory.
#define KR_GT 64 // tile edge of the panel products
#define KR_GP 32 // rows per panel of the panel products
__host__ __device__ constexpr size_t gram_tiled_smem_bytes() { return (size_t)3 * KR_GT * (KR_GP + 1) * 8; }

template <class Team>
KR_DEV void team_gram_sym_tiled(Team &tm, int64_t n, const double *Z, const double *AZ, int64_t ld, int p,
                                double *S, double *G, double *part) {
  extern __shared__ __align__(16) double kr_gemm_smem[];
  typedef double Panel[KR_GP + 1];
  Panel *sA = reinterpret_cast<Panel *>(kr_gemm_smem);
  Panel *sB = sA + KR_GT, *sC = sB + KR_GT;
  const bool withG = AZ != nullptr;
  const int tp = (p + KR_GT - 1) / KR_GT, tu = tp * (tp + 1) / 2;
  const int ncta = tm.ncta();
  const int64_t kblocks = (n + KR_GP - 1) / KR_GP;
  const int nch = (int)imin64(imin64(ncta, kblocks > 0 ? kblocks : 1), (int64_t)(2 * ncta + tu - 1) / tu);
  const int nchunks = nch > 0 ? nch : 1;
  const int64_t kb_per = (kblocks + nchunks - 1) / nchunks; // panels per chunk
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wr = (wid >> 2) * 16, wc = (wid & 3) * 16; // this warp's 16 x 16 piece
  const int items = tu * nchunks;
  constexpr int PER = 3 * KR_GT * KR_GP / 512; // elements per thread and panel (up to three operands)
  for (int it = tm.cta_rank(); it < items; it += ncta) {
    const int tile = it % tu, ch = it / tu;
    int tj = 0;
    while ((tj + 1) * (tj + 2) / 2 <= tile)
      tj++;
    const int ti = tile - tj * (tj + 1) / 2; // ti <= tj
    const bool diag = ti == tj;              // the B panel is the A panel
    const int64_t kb0 = (int64_t)ch * kb_per, kb1 = imin64(kb0 + kb_per, kblocks);
    double aS[2][2][2], aG[2][2][2];
#pragma unroll
    for (int x = 0; x < 2; x++)
#pragma unroll
      for (int y = 0; y < 2; y++)
        aS[x][y][0] = aS[x][y][1] = aG[x][y][0] = aG[x][y][1] = 0.0;
    double v[PER];
    auto fetch = [&](int64_t kb) {
      const int64_t r0 = kb * KR_GP;
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int e = threadIdx.x + q * 512;
        const int which = e / (KR_GT * KR_GP), rem = e % (KR_GT * KR_GP);
        const int c = rem / KR_GP, k = rem % KR_GP;
        const int64_t r = r0 + k;
        double x = 0.0;
        const bool used = which == 0 || (which == 1 && !diag) || (which == 2 && withG);
        if (used && kb < kb1 && r < n) {
          const int colx = (which == 0 ? ti : tj) * KR_GT + c;
          if (colx < p)
            x = (which == 2 ? AZ : Z)[(int64_t)colx * ld + r];
        }
        v[q] = x;
      }
    };
    fetch(kb0);
    for (int64_t kb = kb0; kb < kb1; kb++) {
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int e = threadIdx.x + q * 512;
        const int which = e / (KR_GT * KR_GP), rem = e % (KR_GT * KR_GP);
        (which == 0 ? sA : which == 1 ? sB : sC)[rem / KR_GP][rem % KR_GP] = v[q];
      }
      __syncthreads();
      if (kb + 1 < kb1)
        fetch(kb + 1);
      const Panel *pB = diag ? sA : sB;
#pragma unroll
      for (int kk = 0; kk < KR_GP; kk += 4) {
        double fa[2], fb[2];
#pragma unroll
        for (int x = 0; x < 2; x++)
          fa[x] = sA[wr + 8 * x + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
        for (int y = 0; y < 2; y++)
          fb[y] = pB[wc + 8 * y + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
        for (int x = 0; x < 2; x++)
#pragma unroll
          for (int y = 0; y < 2; y++)
            dmma_8x8x4(aS[x][y][0], aS[x][y][1], fa[x], fb[y]);
        if (withG) {
          double fc[2];
#pragma unroll
          for (int y = 0; y < 2; y++)
            fc[y] = sC[wc + 8 * y + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
          for (int x = 0; x < 2; x++)
#pragma unroll
            for (int y = 0; y < 2; y++)
              dmma_8x8x4(aG[x][y][0], aG[x][y][1], fa[x], fc[y]);
        }
      }
      __syncthreads();
    }
    double *pt = part + (size_t)it * (2 * KR_GT * KR_GT);
#pragma unroll
    for (int x = 0; x < 2; x++)
#pragma unroll
      for (int y = 0; y < 2; y++) {
        const int i = wr + 8 * x + (lane >> 2), j = wc + 8 * y + 2 * (lane & 3);
        pt[i + j * KR_GT] = aS[x][y][0];
        pt[i + (j + 1) * KR_GT] = aS[x][y][1];
        pt[KR_GT * KR_GT + i + j * KR_GT] = aG[x][y][0];
        pt[KR_GT * KR_GT + i + (j + 1) * KR_GT] = aG[x][y][1];
      }
  }
  tm.sync();
  const int64_t nthr = tm.nthreads();
  for (int64_t e = tm.tid(); e < (int64_t)p * p; e += nthr) {
    const int i = (int)(e % p), j = (int)(e / p);
    if (i > j)
      continue;
    const int ti = i / KR_GT, tj = j / KR_GT, li = i % KR_GT, lj = j % KR_GT;
    const int tile = tj * (tj + 1) / 2 + ti;
    double sv = 0.0, gv = 0.0;
    for (int ch = 0; ch < nchunks; ch++) {
      const double *pt = part + (size_t)(tile + ch * tu) * (2 * KR_GT * KR_GT);
      sv += __ldcg(pt + li + lj * KR_GT);
      if (withG)
        gv += __ldcg(pt + KR_GT * KR_GT + li + lj * KR_GT);
    }
    S[i + (size_t)j * p] = sv;
    S[j + (size_t)i * p] = sv;
    if (withG) {
      G[i + (size_t)j * p] = gv;
      G[j + (size_t)i * p] = gv;
    }
  }
  tm.sync();
}

// C = A^T B (a x b, leading dim a) for long, wide products: the general form
// of team_gram_sym_tiled. Work items are (64 x 64 tile of C, fixed chunk of
// rows); a block stages 32-row panels of the tile's columns of A and of B in
// shared memory, fetching the next panel into registers while the current
// one is multiplied, and each of its 16 warps accumulates a 16 x 16 piece of
// the tile (2 x 2 DMMA 8x8 tiles). Partial tiles are summed in chunk order,
// so the result depends only on the team size. `part` must hold
// (2 ncta + tiles) * 4096 doubles, tiles = ceil(a/64) * ceil(b/64); needs 512
// threads and gram_tiled_smem_bytes() of dynamic shared memory.
template <class Team>
KR_DEV void team_gemm_tn_panel(Team &tm, int64_t n, const double *A, int a, const double *B, int b, int64_t ld,
                               double *C, double *part) {
  extern __shared__ __align__(16) double kr_gemm_smem[];
  typedef double Panel[KR_GP + 1];
  Panel *sA = reinterpret_cast<Panel *>(kr_gemm_smem);
  Panel *sB = sA + KR_GT;
  const int ta = (a + KR_GT - 1) / KR_GT, tb = (b + KR_GT - 1) / KR_GT, tiles = ta * tb;
  const int ncta = tm.ncta();
  const int64_t kblocks = (n + KR_GP - 1) / KR_GP;
  const int nch = (int)imin64(imin64(ncta, kblocks > 0 ? kblocks : 1), (int64_t)(2 * ncta + tiles - 1) / tiles);
  const int nchunks = nch > 0 ? nch : 1;
  const int64_t kb_per = (kblocks + nchunks - 1) / nchunks;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wr = (wid >> 2) * 16, wc = (wid & 3) * 16;
  const int items = tiles * nchunks;
  constexpr int PER = 2 * KR_GT * KR_GP / 512; // elements per thread and panel (two operands)
  for (int it = tm.cta_rank(); it < items; it += ncta) {
    const int tile = it % tiles, ch = it / tiles;
    const int ti = tile % ta, tj = tile / ta;
    const int64_t kb0 = (int64_t)ch * kb_per, kb1 = imin64(kb0 + kb_per, kblocks);
    double acc[2][2][2];
#pragma unroll
    for (int x = 0; x < 2; x++)
#pragma unroll
      for (int y = 0; y < 2; y++)
        acc[x][y][0] = acc[x][y][1] = 0.0;
    double v[PER];
    auto fetch = [&](int64_t kb) {
      const int64_t r0 = kb * KR_GP;
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int e = threadIdx.x + q * 512;
        const int which = e / (KR_GT * KR_GP), rem = e % (KR_GT * KR_GP);
        const int c = rem / KR_GP, k = rem % KR_GP;
        const int64_t r = r0 + k;
        double x = 0.0;
        if (kb < kb1 && r < n) {
          const int colx = (which == 0 ? ti : tj) * KR_GT + c;
          if (colx < (which == 0 ? a : b))
            x = (which == 0 ? A : B)[(int64_t)colx * ld + r];
        }
        v[q] = x;
      }
    };
    fetch(kb0);
    for (int64_t kb = kb0; kb < kb1; kb++) {
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int e = threadIdx.x + q * 512;
        const int which = e / (KR_GT * KR_GP), rem = e % (KR_GT * KR_GP);
        (which == 0 ? sA : sB)[rem / KR_GP][rem % KR_GP] = v[q];
      }
      __syncthreads();
      if (kb + 1 < kb1)
        fetch(kb + 1);
#pragma unroll
      for (int kk = 0; kk < KR_GP; kk += 4) {
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
      __syncthreads();
    }
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
  tm.sync();
  const int64_t nthr = tm.nthreads();
  for (int64_t e = tm.tid(); e < (int64_t)a * b; e += nthr) {
    const int i = (int)(e % a), j = (int)(e / a);
    const int ti = i / KR_GT, tj = j / KR_GT, li = i % KR_GT, lj = j % KR_GT;
    const int tile = tj * ta + ti;
    double sv = 0.0;
    for (int ch = 0; ch < nchunks; ch++)
      sv += __ldcg(part + (size_t)(tile + ch * tiles) * (KR_GT * KR_GT) + li + lj * KR_GT);
    C[i + (size_t)j * a] = sv;
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
    team_gemm_tn_panel(tm, n, A, a, B, b, ld, C, part);
  else
    team_gemm_tn_direct(tm, n, A, a, B, b, ld, C, part);
}

// ---- Z * Y products (combine_columns, LOBPCGSolver.cpp:122-134) -----------
// out (n x q) = Z (n x zc) * Y[roff : roff + zc, 0 : q], or out -= that
// product; Z and out column-major with leading dim ld, Y column-major with
// leading dim ldy. On the FP64 tensor cores: a block takes 64-row tiles of
// the tall operand (every 128-column group of the output for one tile before
// the next tile, so the tile is read from HBM once); k runs in chunks of 16
// staged in shared memory (the next chunk is fetched into registers while
// the current one is multiplied); each of the 16 warps owns a 16 x 32 piece
// of the 64 x 128 output group (2 x 4 DMMA 8x8 tiles). Each output is summed
// in a fixed order, independent of the team. Needs 512 threads and
// gemm_nn_smem_bytes() of dynamic shared memory.
#define KR_NT 64  // rows per tile
#define KR_NQ 128 // output columns per group
#define KR_NK 16  // k per chunk
__host__ __device__ constexpr size_t gemm_nn_smem_bytes() { return (size_t)(KR_NT + KR_NQ) * (KR_NK + 1) * 8; }

// Narrow form (q <= KR_NQ_DIRECT outputs): every thread takes whole rows and
// sums over k in order on the CUDA cores, with no shared memory and no
// barrier. For the few-column blocks of small solves the tiled form spends
// two block barriers per 64-row tile on a 64 x 128 output group it barely
// fills; this form costs none (the caller's barrier publishes the result).
#define KR_NQ_DIRECT 16
template <class Team>
KR_DEV void team_gemm_nn_direct(Team &tm, int64_t n, const double *Z, int64_t ld, int zc, const double *Y, int ldy,
                                int roff, int q, double *out, bool subtract) {
  for (int64_t i = tm.tid(); i < n; i += tm.nthreads()) {
    double acc[KR_NQ_DIRECT];
#pragma unroll
    for (int j = 0; j < KR_NQ_DIRECT; j++)
      acc[j] = 0.0;
    for (int k = 0; k < zc; k++) {
      const double z = Z[(int64_t)k * ld + i];
      const double *yk = Y + roff + k;
#pragma unroll
      for (int j = 0; j < KR_NQ_DIRECT; j++)
        if (j < q)
          acc[j] += z * yk[(int64_t)j * ldy];
    }
#pragma unroll
    for (int j = 0; j < KR_NQ_DIRECT; j++)
      if (j < q) {
        double *o = out + (int64_t)j * ld + i;
        *o = subtract ? *o - acc[j] : acc[j];
      }
  }
}

template <class Team>
KR_DEV void team_gemm_nn(Team &tm, int64_t n, const double *Z, int64_t ld, int zc, const double *Y, int ldy,
                         int roff, int q, double *out, bool subtract) {
  if (q <= KR_NQ_DIRECT) {
    team_gemm_nn_direct(tm, n, Z, ld, zc, Y, ldy, roff, q, out, subtract);
    return;
  }
  extern __shared__ __align__(16) double kr_gemm_smem[];
  double(*sZ)[KR_NK + 1] = reinterpret_cast<double(*)[KR_NK + 1]>(kr_gemm_smem);
  double(*sY)[KR_NK + 1] = reinterpret_cast<double(*)[KR_NK + 1]>(kr_gemm_smem + KR_NT * (KR_NK + 1));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wr = (wid >> 2) * 16, wc = (wid & 3) * 32; // this warp's 16 x 32 piece
  const int64_t row_tiles = (n + KR_NT - 1) / KR_NT;
  const int col_groups = (q + KR_NQ - 1) / KR_NQ;
  const int nchunks = (zc + KR_NK - 1) / KR_NK;
  constexpr int PZ = KR_NT * KR_NK / 512, PY = KR_NQ * KR_NK / 512;
  for (int64_t rt = tm.cta_rank(); rt < row_tiles; rt += tm.ncta()) {
    const int64_t r0 = rt * KR_NT;
    for (int cg = 0; cg < col_groups; cg++) {
      const int c0 = cg * KR_NQ;
      double acc[2][4][2];
#pragma unroll
      for (int x = 0; x < 2; x++)
#pragma unroll
        for (int y = 0; y < 4; y++)
          acc[x][y][0] = acc[x][y][1] = 0.0;
      double vz[PZ], vy[PY];
      auto fetch = [&](int ch) {
        const int k0 = ch * KR_NK;
#pragma unroll
        for (int p = 0; p < PZ; p++) {
          const int e = threadIdx.x + p * 512, kk = e / KR_NT, r = e % KR_NT;
          vz[p] = (r0 + r < n && k0 + kk < zc) ? Z[(int64_t)(k0 + kk) * ld + r0 + r] : 0.0;
        }
#pragma unroll
        for (int p = 0; p < PY; p++) {
          const int e = threadIdx.x + p * 512, c = e / KR_NK, kk = e % KR_NK;
          vy[p] = (c0 + c < q && k0 + kk < zc) ? Y[(int64_t)(roff + k0 + kk) + (int64_t)(c0 + c) * ldy] : 0.0;
        }
      };
      fetch(0);
      for (int ch = 0; ch < nchunks; ch++) {
#pragma unroll
        for (int p = 0; p < PZ; p++) {
          const int e = threadIdx.x + p * 512;
          sZ[e % KR_NT][e / KR_NT] = vz[p];
        }
#pragma unroll
        for (int p = 0; p < PY; p++) {
          const int e = threadIdx.x + p * 512;
          sY[e / KR_NK][e % KR_NK] = vy[p];
        }
        __syncthreads();
        if (ch + 1 < nchunks)
          fetch(ch + 1);
        if (c0 + wc < q) { // warp-uniform: warps past the last column have nothing to do
#pragma unroll
          for (int kk = 0; kk < KR_NK; kk += 4) {
            double fa[2], fb[4];
#pragma unroll
            for (int x = 0; x < 2; x++)
              fa[x] = sZ[wr + 8 * x + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
            for (int y = 0; y < 4; y++)
              fb[y] = sY[wc + 8 * y + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
            for (int x = 0; x < 2; x++)
#pragma unroll
              for (int y = 0; y < 4; y++)
                dmma_8x8x4(acc[x][y][0], acc[x][y][1], fa[x], fb[y]);
          }
        }
        __syncthreads();
      }
#pragma unroll
      for (int x = 0; x < 2; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) {
          const int64_t i = r0 + wr + 8 * x + (lane >> 2);
          const int j = c0 + wc + 8 * y + 2 * (lane & 3);
          if (i < n) {
#pragma unroll
            for (int h = 0; h < 2; h++)
              if (j + h < q) {
                double *o = out + (int64_t)(j + h) * ld + i;
                *o = subtract ? *o - acc[x][y][h] : acc[x][y][h];
              }
          }
        }
    }
  }
}

// X[:, i] -= sum_j S[:, j] * Cc(j, i) for i < k, j < ns (X, S column-major
// with leading dim ld; Cc leading dim ldc).
template <class Team>
KR_DEV void team_combine_sub(Team &tm, int64_t n, const double *S, int64_t ld, int ns, const double *Cc, int ldc,
                             int k, double *X) {
  team_gemm_nn(tm, n, S, ld, ns, Cc, ldc, 0, k, X, true);
}

// out[:, i] = sum_j Y(roff + j, i) * Z[:, j], i < q, j < zc (column-major,
// both with leading dim ld; Y leading dim ldy).
template <class Team>
KR_DEV void team_combine(Team &tm, int64_t n, const double *Z, int64_t ld, int zc, const double *Y,
                         int ldy, int roff, int q, double *out) {
  team_gemm_nn(tm, n, Z, ld, zc, Y, ldy, roff, q, out, false);
}

// dynamic shared memory of a kernel that runs the block solver's products
__host__ __device__ constexpr size_t lobpcg_dyn_smem_bytes() {
  return gram_tiled_smem_bytes() > gemm_nn_smem_bytes() ? gram_tiled_smem_bytes() : gemm_nn_smem_bytes();
}

} // namespace kr
