"""numpy restatement of the RMAT edge-list spec documented in
plato_b200/csrc/rmat.cpp (counter-based stream, compaction, optional
symmetrisation and permutation), used to check the C++ generator."""
from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def mix64(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z + np.uint64(0x9E3779B97F4A7C15)) & M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M64
        return z ^ (z >> np.uint64(31))


def rmat(scale, edgefactor, seed, a=0.57, b=0.19, c=0.19, symmetrize=False, permute=False):
    M = edgefactor << scale
    ta = int(a * 4294967296.0)
    tb = int((a + b) * 4294967296.0)
    tc = int((a + b + c) * 4294967296.0)
    base = mix64(np.array([seed], dtype=np.uint64))[0]
    i = np.arange(M, dtype=np.uint64)
    u = np.zeros(M, dtype=np.uint64)
    v = np.zeros(M, dtype=np.uint64)
    h = None
    for lvl in range(scale):
        if lvl % 2 == 0:
            with np.errstate(over="ignore"):
                h = mix64(base + np.uint64(32) * i + np.uint64(lvl >> 1))
        r = (h >> np.uint64(32)) if lvl % 2 else (h & np.uint64(0xFFFFFFFF))
        r = r.astype(np.int64)
        bu = (r >= tb).astype(np.uint64)
        bv = (((r >= ta) & (r < tb)) | (r >= tc)).astype(np.uint64)
        u = (u << np.uint64(1)) | bu
        v = (v << np.uint64(1)) | bv
    keep = u != v
    u, v = u[keep], v[keep]
    if symmetrize:
        u, v = np.minimum(u, v), np.maximum(u, v)
    keys = np.unique((u << np.uint64(32)) | v)
    u = keys >> np.uint64(32)
    v = keys & np.uint64(0xFFFFFFFF)
    present = np.zeros(1 << scale, dtype=bool)
    present[u.astype(np.int64)] = True
    present[v.astype(np.int64)] = True
    newid = np.cumsum(present) - 1
    V = int(present.sum())
    u = newid[u.astype(np.int64)].astype(np.uint64)
    v = newid[v.astype(np.int64)].astype(np.uint64)
    if permute and V > 1:
        pbase = mix64(np.array([seed ^ 0xA5A5F00DC0FFEE11], dtype=np.uint64))[0]
        with np.errstate(over="ignore"):
            hk = mix64(pbase + np.arange(V, dtype=np.uint64))
        order = np.lexsort((np.arange(V), hk))
        label = np.empty(V, dtype=np.uint64)
        label[order] = np.arange(V, dtype=np.uint64)
        u, v = label[u.astype(np.int64)], label[v.astype(np.int64)]
        if symmetrize:
            u, v = np.minimum(u, v), np.maximum(u, v)
        keys = np.sort((u << np.uint64(32)) | v)
        u = keys >> np.uint64(32)
        v = keys & np.uint64(0xFFFFFFFF)
    return V, u.astype(np.uint32), v.astype(np.uint32)
