"""Independent FP64 oracle — TEST INFRASTRUCTURE ONLY.

Plain scipy.sparse power iteration and a serial level-synchronous BFS, written
from the mathematical definitions (no engine, no push/pull), used to
cross-check both ref_cpu.c and the CUDA path:

  PageRank (plato/algo/pagerank/pagerank.hpp:81-146, un-normalised):
      r_0 = 1;  r_{t+1}(v) = (1-d) + d * sum_{u in in(v)} r_t(u) / deg(u)
      (deg(u) = out-degree; u with deg 0 has no out-edges, so it never
      contributes), and the last epoch returns r, earlier epochs feed r/deg.
  Seed-set PPR (trustrank.hpp:197-245): teleport (1-d)/|S| on seeds, r_0 = 1/|S| on seeds.
  BFS levels: distance in hops from the root over out-edges.
"""
from __future__ import annotations

from collections import deque

import numpy as np
import scipy.sparse as sp


def adjacency(vertices: int, src, dst, is_directed: bool = True) -> sp.csr_matrix:
    """A[v, u] = number of edges u -> v (in-edge matrix, CSR by destination)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if not is_directed:
        src, dst = np.concatenate([src, dst]), np.concatenate([dst, src])
    data = np.ones(src.size, dtype=np.float64)
    return sp.csr_matrix((data, (dst, src)), shape=(vertices, vertices))


def _power(A: sp.csr_matrix, x0: np.ndarray, tele: np.ndarray, d: float, iterations: int,
           eps: float) -> tuple[np.ndarray, int]:
    deg = np.asarray(A.sum(axis=0)).ravel()  # out-degree (column sums)
    safe = np.where(deg > 0, deg, 1.0)
    x = np.where(deg > 0, x0 / safe, x0)
    epochs = 0
    it = 0
    while it < iterations:
        y = A @ x
        r = tele + d * y
        epochs += 1
        if it == iterations - 1:
            return r, epochs
        xn = np.where(deg > 0, r / safe, r)
        delta = float(np.sum(np.where(deg > 0, np.abs(xn - x) * deg, np.abs(xn - x))))
        x = xn
        if eps > 0.0 and delta < eps:
            it = iterations - 1
            continue
        it += 1
    return x, epochs


def pagerank(vertices: int, src, dst, is_directed=True, iterations=100, damping=0.85, eps=0.0):
    """Reference units (initial rank 1, teleport 1-d) -> (ranks, epochs)."""
    A = adjacency(vertices, src, dst, is_directed)
    return _power(A, np.ones(vertices), np.full(vertices, 1.0 - damping), damping, iterations, eps)


def ppr(vertices: int, src, dst, source: int, is_directed=True, iterations=100, damping=0.85,
        eps=0.0):
    A = adjacency(vertices, src, dst, is_directed)
    x0 = np.zeros(vertices)
    x0[source] = 1.0
    tele = np.zeros(vertices)
    tele[source] = 1.0 - damping
    return _power(A, x0, tele, damping, iterations, eps)


def seedset_ppr(vertices: int, src, dst, seeds, is_directed=True, iterations=100, damping=0.85,
                eps=0.0):
    A = adjacency(vertices, src, dst, is_directed)
    s = np.unique(np.asarray(seeds, dtype=np.int64))
    x0 = np.zeros(vertices)
    x0[s] = 1.0 / s.size
    tele = np.zeros(vertices)
    tele[s] = (1.0 - damping) / s.size
    return _power(A, x0, tele, damping, iterations, eps)


def bfs_levels(vertices: int, src, dst, root: int, is_directed=True) -> np.ndarray:
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if not is_directed:
        src, dst = np.concatenate([src, dst]), np.concatenate([dst, src])
    order = np.argsort(src, kind="stable")
    s, d = src[order], dst[order]
    off = np.zeros(vertices + 1, dtype=np.int64)
    np.add.at(off, s + 1, 1)
    off = np.cumsum(off)
    lev = np.full(vertices, 0xFFFFFFFF, dtype=np.uint32)
    lev[root] = 0
    q = deque([root])
    while q:
        u = q.popleft()
        for v in d[off[u]:off[u + 1]]:
            if lev[v] == 0xFFFFFFFF:
                lev[v] = lev[u] + 1
                q.append(v)
    return lev


def cc_labels(vertices: int, src, dst, is_directed=True) -> np.ndarray:
    """Fixed point of plato::algo::connected_component_t's label propagation
    (plato/algo/cgm/connected_component.hpp:173-245): label[v] = the smallest
    id u with a directed path u -> v (u = v included).  On an undirected
    graph that is the smallest id of v's component, which is what the
    reference's own test checks with a BFS from ascending ids
    (plato/algo/cgm/test/test_cgm.cc:81-99, 141-149).  Computed here by
    synchronous min-propagation over the edges until nothing changes."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if not is_directed:
        src, dst = np.concatenate([src, dst]), np.concatenate([dst, src])
    lab = np.arange(vertices, dtype=np.int64)
    while True:
        nxt = lab.copy()
        np.minimum.at(nxt, dst, lab[src])
        if np.array_equal(nxt, lab):
            return lab.astype(np.uint32)
        lab = nxt


def cc_components_bfs(vertices: int, src, dst) -> np.ndarray:
    """The reference test's own labelling of an undirected graph
    (test_cgm.cc:81-99): scan ids in ascending order, BFS from each unlabelled
    one and give its whole component that id."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    s, d = np.concatenate([src, dst]), np.concatenate([dst, src])
    order = np.argsort(s, kind="stable")
    s, d = s[order], d[order]
    off = np.zeros(vertices + 1, dtype=np.int64)
    np.add.at(off, s + 1, 1)
    off = np.cumsum(off)
    label = np.full(vertices, -1, dtype=np.int64)
    for i in range(vertices):
        if label[i] != -1:
            continue
        label[i] = i
        q = deque([i])
        while q:
            u = q.popleft()
            for v in d[off[u]:off[u + 1]]:
                if label[v] == -1:
                    label[v] = i
                    q.append(v)
    return label.astype(np.uint32)


def weighted_pagerank(vertices: int, src, dst, weights, is_directed=True, iterations=100, damping=0.85,
                      eps=0.001):
    """algo::weighted_pagerank (plato/algo/pagerank/weighted_pagerank.hpp:60-149)
    in double: v_weight_sum[u] = sum of u's out-edge weights (:86-99), ranks
    start at 1 (:104-109); each epoch rank'(v) = 1 - d + d * sum over in-edges
    (u, v, w) of rank[u] * w / v_weight_sum[u] (:112-130); delta = sum
    |rank' - rank| except in the last epoch, and eps > 0 with delta < eps
    jumps to the last epoch (:131-137).  Undirected edges count both ways.
    Returns (ranks, epochs run, last delta)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    w = np.asarray(weights, dtype=np.float64)
    if not is_directed:
        src, dst, w = np.concatenate([src, dst]), np.concatenate([dst, src]), np.concatenate([w, w])
    wsum = np.zeros(vertices)
    np.add.at(wsum, src, w)
    with np.errstate(divide="ignore", invalid="ignore"):
        beta = w / wsum[src]
    A = sp.csr_matrix((beta, (dst, src)), shape=(vertices, vertices))
    rank = np.ones(vertices)
    epochs, delta = 0, 0.0
    epoch = 0
    while epoch < iterations:
        nxt = (1.0 - damping) + damping * (A @ rank)
        epochs += 1
        if epoch == iterations - 1:
            rank = nxt
            break
        delta = float(np.abs(nxt - rank).sum())
        rank = nxt
        if eps > 0.0 and delta < eps:
            epoch = iterations - 2
        epoch += 1
    return rank, epochs, delta
