"""Seeded generators of the workloads the engine is measured on.

Each returns a scipy CSR matrix plus an orthonormal basis of its exact null
space (rows = vectors), so results can be checked against the analytic kernel
as well as against the oracle.

  shift_operator      (Ax)_i = x_{i+N} - c x_i, (n-N) x n  (the reference's
                      quickstart operator, examples/quickstart.cpp:29-36)
  difference_operator (Dx)_i = x_{i+1} - x_i (tests/test_difference_operator.cpp:28-37)
  graph_incidence     edges x vertices, +1 tail / -1 head; kernel = component
                      indicators (random multigraph: spanning path + ER edges)
  planted_kernel      A = [B | B W], kernel spanned by the columns of [W; -I_k]
  batch_instances     many small shift / incidence instances of uneven size
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import scipy.sparse as sp


@dataclass
class Instance:
    name: str
    A: sp.csr_matrix
    kernel: Optional[np.ndarray]  # (k, n) orthonormal rows, or None if not materialised
    k: int
    meta: dict


def _csr(rows, cols, vals, m, n):
    A = sp.csr_matrix((np.asarray(vals, np.float64), (np.asarray(rows), np.asarray(cols))),
                      shape=(m, n))
    A.sort_indices()
    return A


def shift_operator(n: int = 1000, N: int = 3, c: float = 0.5, kernel: bool = True) -> Instance:
    m = n - N
    i = np.arange(m)
    rows = np.repeat(i, 2)
    cols = np.stack([i, i + N], 1).ravel()
    vals = np.tile([-c, 1.0], m)
    A = _csr(rows, cols, vals, m, n)
    K = None
    if kernel:
        K = np.zeros((N, n))
        for j in range(N):
            idx = np.arange(j, n, N)
            K[j, idx] = c ** np.arange(len(idx), dtype=np.float64)
        K /= np.linalg.norm(K, axis=1, keepdims=True)
    return Instance("shift", A, K, N, dict(n=n, N=N, c=c))


def difference_operator(n: int) -> Instance:
    m = n - 1
    i = np.arange(m)
    rows = np.repeat(i, 2)
    cols = np.stack([i, i + 1], 1).ravel()
    vals = np.tile([-1.0, 1.0], m)
    A = _csr(rows, cols, vals, m, n)
    K = np.full((1, n), 1.0 / np.sqrt(n))
    return Instance("difference", A, K, 1, dict(n=n))


def graph_incidence(n_vertices: int, n_components: int, mean_degree: float, seed: int = 1,
                    kernel: bool = True, shuffle: bool = True) -> Instance:
    """Random multigraph of `n_components` equal connected components: each a
    spanning path plus Erdos-Renyi edges so that the total edge count is
    n_vertices * mean_degree / 2. Rows are edges (+1 tail, -1 head, random
    orientation); columns are vertices. ker(A) = component indicators."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nc = n_components
    sizes = np.full(nc, n_vertices // nc)
    sizes[: n_vertices - sizes.sum()] += 1
    perm = rng.permutation(n_vertices) if shuffle else np.arange(n_vertices)
    total_edges = int(round(n_vertices * mean_degree / 2))
    tails, heads, comp_of = [], [], np.empty(n_vertices, np.int64)
    start = 0
    path_edges = int((sizes - 1).clip(min=0).sum())
    er_total = max(0, total_edges - path_edges)
    er_per = np.floor(er_total * sizes / n_vertices).astype(np.int64)
    er_per[: er_total - er_per.sum()] += 1
    for c in range(nc):
        s = sizes[c]
        verts = perm[start:start + s]
        comp_of[verts] = c
        start += s
        if s >= 2:
            tails.append(verts[:-1])
            heads.append(verts[1:])
            e = er_per[c]
            if e > 0:
                u = rng.integers(0, s, e)
                v = rng.integers(0, s - 1, e)
                v = v + (v >= u)  # v != u
                tails.append(verts[u])
                heads.append(verts[v])
    t = np.concatenate(tails) if tails else np.zeros(0, np.int64)
    h = np.concatenate(heads) if heads else np.zeros(0, np.int64)
    flip = rng.random(t.shape[0]) < 0.5
    t, h = np.where(flip, h, t), np.where(flip, t, h)
    if shuffle:
        order = rng.permutation(t.shape[0])
        t, h = t[order], h[order]
    m = t.shape[0]
    rows = np.repeat(np.arange(m), 2)
    cols = np.stack([t, h], 1).ravel()
    vals = np.tile([1.0, -1.0], m)
    A = _csr(rows, cols, vals, m, n_vertices)
    K = None
    if kernel:
        K = np.zeros((nc, n_vertices))
        K[comp_of, np.arange(n_vertices)] = 1.0
        K /= np.sqrt(sizes)[:, None]
    return Instance("incidence", A, K, nc, dict(n=n_vertices, components=nc,
                                                 mean_degree=mean_degree, seed=seed))


def planted_kernel(m: int, n_minus_k: int, k: int, nnz_row: int = 8, w_nnz_col: int = 4,
                   seed: int = 1, kernel: bool = True) -> Instance:
    """A = [B | B W] with B (m x (n-k)) holding nnz_row distinct uniform columns
    per row with N(0,1) values (every column forced nonempty) and W
    ((n-k) x k) holding w_nnz_col N(0,1) entries per column. ker(A) is spanned
    by the columns of [W; -I_k]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nk = n_minus_k
    # distinct columns per row: sample with replacement, then resample duplicates
    cols = rng.integers(0, nk, (m, nnz_row))
    for _ in range(16):
        s = np.sort(cols, axis=1)
        dup = np.zeros_like(cols, dtype=bool)
        dup[:, 1:] = s[:, 1:] == s[:, :-1]
        if not dup.any():
            break
        cols = s
        cols[dup] = rng.integers(0, nk, int(dup.sum()))
    cols = np.sort(cols, axis=1)
    vals = rng.standard_normal((m, nnz_row))
    # every column of B nonempty: put missing columns into random rows (replacing
    # an entry whose column still appears elsewhere)
    counts = np.bincount(cols.ravel(), minlength=nk)
    empty = np.flatnonzero(counts == 0)
    for j in empty:
        for _ in range(64):
            r = rng.integers(0, m)
            q = rng.integers(0, nnz_row)
            old = cols[r, q]
            if counts[old] > 1 and j not in cols[r]:
                counts[old] -= 1
                cols[r, q] = j
                counts[j] += 1
                break
    B = _csr(np.repeat(np.arange(m), nnz_row), cols.ravel(), vals.ravel(), m, nk)
    wr = np.concatenate([rng.choice(nk, w_nnz_col, replace=False) for _ in range(k)])
    wc = np.repeat(np.arange(k), w_nnz_col)
    W = sp.csr_matrix((rng.standard_normal(k * w_nnz_col), (wr, wc)), shape=(nk, k))
    BW = (B @ W).tocsr()
    A = sp.hstack([B, BW], format="csr")
    A.sort_indices()
    K = None
    if kernel:
        Z = np.vstack([W.toarray(), -np.eye(k)])  # (n x k)
        Q, _ = np.linalg.qr(Z)
        K = Q.T.copy()
    return Instance("planted", A, K, k, dict(m=m, n=nk + k, k=k, seed=seed))


def batch_instances(count: int = 4096, seed: int = 1, n_lo: float = 1e3, n_hi: float = 2e5,
                    kernel: bool = False) -> List[Instance]:
    """Uneven independent instances: half shift operators (n log-uniform,
    N in 1..16, c in [0.3, 0.9]), half graph incidence matrices (n log-uniform,
    1-16 components, mean degree 6 including the spanning paths). Instance i
    draws from its own stream seeded by (seed, i)."""
    out = []
    for i in range(count):
        r = np.random.Generator(np.random.PCG64([seed, i]))
        n = int(round(np.exp(r.uniform(np.log(n_lo), np.log(n_hi)))))
        if i % 2 == 0:
            N = int(r.integers(1, 17))
            c = float(r.uniform(0.3, 0.9))
            inst = shift_operator(n, N, c, kernel=kernel)
        else:
            comps = int(r.integers(1, 17))
            n = max(n, 2 * comps)
            inst = graph_incidence(n, comps, 6.0, seed=int(r.integers(1 << 31)), kernel=kernel)
        inst.meta["index"] = i
        out.append(inst)
    return out
