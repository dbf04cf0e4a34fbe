"""HyperLogLog propagation oracle (HyperANF, n-step degrees) — TEST
INFRASTRUCTURE ONLY: imported by tests/, bench.py's CPU leg and smoke() as
the checker, never by the plato_b200 package.

A numpy restatement of
  plato/util/hash.hpp:33-88            murmurhash3 (MurmurHash3_x86_32, the
                                       published algorithm) of a 4-byte id
  plato/util/hyperloglog.hpp:32-142    hyperloglog_t<P>: add, estimate, merge
  plato/algo/hyperanf/hyperanf.hpp:61-195
                                       hyperanf() and GetAvgDistance
  plato/algo/nstepdegrees/nstepdegrees.hpp:160-402
                                       mark_target, spread, propagate, compute
with the dual-mode engine's switch (plato/engine/dualmode.hpp:245-297: push
iff sum of out-degrees of the actives / edges < push_threshold; out-degrees
from the in-edges, edges doubled on undirected graphs).

Parity pins: murmurhash3, add and estimate against the reference's own
headers compiled by oracle/build.py (build_ref) into golden vectors
(tests/golden/hll_golden.npz); n-step degrees against the values the
reference's test asserts (test_nstepdegrees.cc:92-95) and HyperANF against
its exact-average-distance test (test_hyperanf.cc:190-217), both on
raw_graph_7_7.csv.
"""
from __future__ import annotations

import numpy as np

HLL_SEED = 0x5F61767A  # hyperloglog.hpp:64
DBL_EPSILON = np.finfo(np.float64).eps
U32 = np.uint32


def _rotl(x: np.ndarray, r: int) -> np.ndarray:
    return (x << U32(r)) | (x >> U32(32 - r))


def murmur3_u32(ids, seed: int = HLL_SEED) -> np.ndarray:
    """MurmurHash3_x86_32 of each id's 4 little-endian bytes (one block, no
    tail), as hash.hpp:33-88 computes it for len = 4."""
    k = np.asarray(ids, dtype=np.uint32).copy()
    with np.errstate(over="ignore"):
        k *= U32(0xCC9E2D51)
        k = _rotl(k, 15)
        k *= U32(0x1B873593)
        h = np.full_like(k, U32(seed)) ^ k
        h = _rotl(h, 13)
        h = h * U32(5) + U32(0xE6546B64)
        h ^= U32(4)  # length
        h ^= h >> U32(16)
        h *= U32(0x85EBCA6B)
        h ^= h >> U32(13)
        h *= U32(0xC2B2AE35)
        h ^= h >> U32(16)
    return h


def _clz32(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint64)
    n = np.zeros(x.shape, dtype=np.int64)
    for s in (16, 8, 4, 2, 1):
        small = x < (np.uint64(1) << np.uint64(32 - s))
        n += np.where(small, s, 0)
        x = np.where(small, x << np.uint64(s), x)
    return np.where(np.asarray(x) == 0, 32, n)


def index_rank(ids, P: int) -> tuple[np.ndarray, np.ndarray]:
    """Register index and rank of hyperloglog_t<P>::add (hyperloglog.hpp:53-70):
    index = top P bits of the hash; rank = 1 + leading zeros of the hash
    shifted left by P, capped at Q + 1 (Q = 32 - P)."""
    h = murmur3_u32(ids)
    Q = 32 - P
    idx = (h >> U32(Q)).astype(np.int64)
    shifted = (h.astype(np.uint64) << np.uint64(P)) & np.uint64(0xFFFFFFFF)
    rank = np.minimum(_clz32(shifted), Q) + 1
    return idx, rank.astype(np.uint8)


def add(regs: np.ndarray, ids, P: int) -> None:
    """hyperloglog_t<P>::add of every id into one register row (in place)."""
    idx, rank = index_rank(ids, P)
    np.maximum.at(regs, idx, rank)


def single(ids, P: int) -> np.ndarray:
    """One row per id holding that id alone (hyperanf.hpp:111-121)."""
    ids = np.asarray(ids, dtype=np.uint32)
    regs = np.zeros((ids.size, 1 << P), dtype=np.uint8)
    idx, rank = index_rank(ids, P)
    regs[np.arange(ids.size), idx] = rank
    return regs


def alpha_mm(P: int) -> float:
    m = float(1 << P)
    a = {4: 0.673, 5: 0.697, 6: 0.709}.get(P, 0.7213 / (1.0 + 1.079 / m))
    return a * (m * m)


def estimate(regs: np.ndarray, P: int) -> np.ndarray:
    """hyperloglog_t<P>::estimate (hyperloglog.hpp:76-113) of each row.  The
    register sum is exact in double (terms 2^-r, r <= 33 - P), so the row
    order of the sum does not matter."""
    regs = np.atleast_2d(regs)
    m = float(1 << P)
    s = np.ldexp(1.0, -regs.astype(np.int64)).sum(axis=1)
    est = alpha_mm(P) / s
    zeros = (regs == 0).sum(axis=1)
    small = est <= 5.0 / 2.0 * m
    lc = small & (zeros > 0)
    with np.errstate(divide="ignore"):
        est = np.where(lc, m * np.log(m / np.maximum(zeros, 1).astype(np.float64)), est)
    big = (~small) & (est > (1.0 / 30.0) * 4294967296.0)
    with np.errstate(invalid="ignore"):
        est = np.where(big, -4294967296.0 * np.log(1.0 - est / 4294967296.0), est)
    return est


def _stored(V: int, src, dst, is_directed: bool):
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if not is_directed:
        src, dst = np.concatenate([src, dst]), np.concatenate([dst, src])
    return src, dst


def _is_push(active: np.ndarray, outdeg: np.ndarray, edges: int, thr: float) -> bool:
    """dualmode.hpp:262-279 (edges = stored directed edges)."""
    ae = int(outdeg[active].sum())
    return edges > 0 and (ae / edges) < thr


def _gather(books: np.ndarray, frm: np.ndarray, to: np.ndarray, use: np.ndarray) -> np.ndarray:
    """delta[v] = register max over the rows books[u] of the edges u -> v
    with use[u] (a vertex that receives nothing keeps an empty row, so it
    cannot change: the reference's delta_active bookkeeping drops out)."""
    sel = use[frm]
    delta = np.zeros_like(books)
    np.maximum.at(delta, to[sel], books[frm[sel]])
    return delta


def hyperanf(V: int, src, dst, is_directed: bool, bits: int = 6, iterations: int = 20,
             push_threshold: float = 0.05):
    """algo::hyperanf (hyperanf.hpp:83-195).  Returns (avg_distance, anfs,
    registers [V, 2^bits], modes) with modes[i] True for a push epoch.

    Every epoch merges, into each vertex, the rows of its in-neighbours as
    they stood before the epoch.  Push epochs scatter only the rows that
    changed in the previous epoch (hyperanf.hpp:133-147), pull epochs gather
    every in-neighbour (:148-164); with every vertex active in the first
    epoch the two give the same registers, so both are computed here by
    gathering from the active in-neighbours."""
    s, d = _stored(V, src, dst, is_directed)
    outdeg = np.bincount(s, minlength=V)
    ids = np.arange(V, dtype=np.uint32)
    labels = single(ids, bits)
    anfs = [float(estimate(labels, bits).sum())]
    active = np.ones(V, dtype=bool)
    modes = []
    for _ in range(iterations):
        modes.append(_is_push(active, outdeg, s.size, push_threshold))
        merged = np.maximum(labels, _gather(labels, s, d, active))
        changed = (merged != labels).any(axis=1)
        labels = merged
        anf = float(estimate(labels, bits).sum())
        if anf - anfs[-1] < DBL_EPSILON:  # hyperanf.hpp:185-187
            break
        anfs.append(anf)
        active = changed
    return avg_distance(anfs), np.asarray(anfs), labels, modes


def avg_distance(anfs) -> float:
    """GetAvgDistance (hyperanf.hpp:61-70)."""
    a = 0.0
    for i in range(1, len(anfs)):
        a += i * (anfs[i] - anfs[i - 1])
    den = anfs[-1] - anfs[0]
    return a / den if den != 0 else float("nan")


def exact_avg_distance(V: int, src, dst) -> float:
    """The reference test's exact answer on an undirected graph
    (test_hyperanf.cc:80-119, 190-215): per root, the mean hop distance from
    cumulative reach counts; averaged over all roots."""
    from collections import deque
    s, d = _stored(V, src, dst, False)
    adj = [[] for _ in range(V)]
    for a, b in zip(s.tolist(), d.tolist()):
        adj[a].append(b)
    total = 0.0
    for root in range(V):
        dist = [-1] * V
        dist[root] = 0
        q = deque([root])
        while q:
            u = q.popleft()
            for v in adj[u]:
                if dist[v] == -1:
                    dist[v] = dist[u] + 1
                    q.append(v)
        md = max(dist)
        friends = [0] * V
        for x in dist:
            if x >= 0:  # the test's graphs are connected; unreached vertices are not counted
                friends[x] += 1
        for i in range(md):
            friends[i + 1] += friends[i]
        num = sum(i * (friends[i] - friends[i - 1]) for i in range(1, md + 1))
        total += num / (friends[md] - friends[0]) if md > 0 else 0.0
    return total / V


def nstep_degrees(V: int, src, dst, graph_directed: bool, step: int = 20, bits: int = 6,
                  kind: str = "both", is_directed: bool | None = None, targets=None,
                  push_threshold: float = 0.05):
    """nstepdegrees_t::compute (nstepdegrees.hpp:380-402).  Returns
    (in_degrees, out_degrees, modes), uint32 per vertex (0 for non-targets),
    modes = one (phase, push?) entry per epoch.

    Engine rules reproduced as the reference runs them:
    * the switch uses forward out-degrees even while the engine is reversed
      (out_degrees_ is built once from the in-edges, dualmode.hpp:250-259);
    * reversed pull epochs walk the out-edges (dualmode.hpp:302-308), but the
      push slots of spread() and propagate() always scatter over
      engine_->out_edges() (nstepdegrees.hpp:217-229, 316-327), i.e. forward,
      even while reversed;
    * pull epochs of propagate() merge every neighbour's row, push epochs
      only the rows of the actives; spread() pull epochs test the actives.
    """
    if is_directed is None:
        is_directed = graph_directed
    s, d = _stored(V, src, dst, graph_directed)
    E = s.size
    outdeg = np.bincount(s, minlength=V)  # forward out-degrees (from the in-edges)
    target = np.ones(V, dtype=bool) if targets is None else np.asarray(targets, dtype=bool).copy()
    steps = 0xFFFFFFFF if step < 0 else int(step)
    deg_in = np.zeros(V, dtype=np.uint32)
    deg_out = np.zeros(V, dtype=np.uint32)
    modes = []

    def spread(covered, active, reversed_):
        actives = 1
        i = 0
        while i < steps and actives > 0:
            push = _is_push(active, outdeg, E, push_threshold)
            modes.append(("spread", push))
            if push or not reversed_:  # forward: dst with an active in-neighbour
                hit = np.zeros(V, dtype=bool)
                hit[d[active[s]]] = True
            else:  # reversed pull: u with an active out-neighbour
                hit = np.zeros(V, dtype=bool)
                hit[s[active[d]]] = True
            new = hit & ~covered
            actives = int(new.sum())
            covered |= new
            active = new
            i += 1
        return covered

    def propagate(covered, reversed_):
        books = np.zeros((V, 1 << bits), dtype=np.uint8)
        cov_ids = np.flatnonzero(covered).astype(np.uint32)
        books[cov_ids] = single(cov_ids, bits)
        active = covered.copy()
        actives = int(active.sum())
        i = 0
        while i < steps and actives > 0:
            push = _is_push(active, outdeg, E, push_threshold)
            modes.append(("propagate", push))
            every = np.ones(V, dtype=bool)
            if push:  # forward scatter from the actives
                delta = _gather(books, s, d, active)
            elif not reversed_:  # pull over the in-edges: every in-neighbour
                delta = _gather(books, s, d, every)
            else:  # reversed pull over the out-edges: every out-neighbour
                delta = _gather(books, d, s, every)
            merged = np.maximum(books, delta)
            changed = covered & (merged != books).any(axis=1)
            books[changed] = merged[changed]
            actives = int(changed.sum())
            active = changed
            i += 1
        est = estimate(books[target], bits)
        return (est.astype(np.int64).astype(np.uint32) - np.uint32(1)).astype(np.uint32)

    if kind in ("in", "both"):
        covered = target.copy()
        covered = spread(covered, target.copy(), True)
        deg_in[target] = propagate(covered, False)
    if kind in ("out", "both"):
        if kind == "out" or is_directed:
            covered = target.copy()
            covered = spread(covered, target.copy(), False)
            deg_out[target] = propagate(covered, True)
        else:
            deg_out[:] = deg_in
    return deg_in, deg_out, modes
