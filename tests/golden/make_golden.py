"""Generate the golden fixtures under tests/golden/ from the reference's data.

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Reads the reference's fixture graphs (data/graph/*.csv) with the reference's
CSV rules (plato/graph/parsers.hpp:226-290: `src,dst[,w]` per line, fields
split on ',', parsed with strtoul so surrounding blanks are tolerated, empty
lines skipped) and writes
  fixtures.npz    edge lists (uint32) of the fixture graphs,
  kats.json       the known-answer values the reference's own tests assert on
                  those graphs, each with its file:line,
  hll_golden.npz  murmurhash3 values, HyperLogLog registers and estimates
                  computed by the reference's own plato/util/hash.hpp and
                  plato/util/hyperloglog.hpp (compiled from the reference tree
                  by oracle/build.py build_ref into oracle/_ref/),
  ref_golden.npz  the reference's own algo::pagerank, personalized_pagerank
                  (pull-only and dual-mode), breadth_first_search and trustrank
                  outputs on fixture graphs (the reference's engine path
                  compiled into oracle/_ref/libplato_ref.so by build_ref; see
                  oracle/refplato.py): ranks, epoch counts, per-epoch deltas,
                  BFS visited counts, vertices activated per level and the
                  engine's push/pull choice per level; connected_component_t
                  labels and summary and hyperanf average distances on the
                  undirected graphs; weighted_pagerank on the weighted
                  fixture and a weighted RMAT graph.
The reference tree is only needed to regenerate; tests read the outputs.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GRAPHS = ["graph_10_9.csv", "v100_e2150_ua_c3.csv", "v100_e4300_da_c3.csv", "raw_graph_7_7.csv"]
WEIGHTED_GRAPHS = ["raw_graph_10_9_weighted.csv"]  # `src,dst,w` (double_decoder, parsers.hpp:84-88)


def parse_csv(path: Path, weighted: bool = False):
    src, dst, w = [], [], []
    for line in path.read_text().splitlines():
        if not line:
            continue
        parts = line.split(",")
        if len(parts) < (3 if weighted else 2):
            continue
        src.append(int(parts[0].strip() or 0))
        dst.append(int(parts[1].strip() or 0))
        if weighted:
            w.append(float(parts[2]))
    out = (np.asarray(src, dtype=np.uint32), np.asarray(dst, dtype=np.uint32))
    return out + (np.asarray(w, dtype=np.float64),) if weighted else out


KATS = {
    "dcsc_counts": [
        {"graph": "v100_e2150_ua_c3.csv", "is_directed": False, "vertices": 100, "edges": 4300,
         "source": "plato/graph/structure/test/dcsc.cc:108-109"},
        {"graph": "graph_10_9.csv", "is_directed": True, "vertices": 9, "edges": 9,
         "source": "plato/graph/structure/test/dcsc.cc:161-162"},
    ],
    "degrees": [
        {"graph": "v100_e2150_ua_c3.csv", "is_directed": False, "kind": "out",
         "values": {"0": 19, "99": 59, "28": 19}, "source": "plato/graph/test/structure.cc:137-152"},
        {"graph": "v100_e4300_da_c3.csv", "is_directed": True, "kind": "out",
         "values": {"0": 19, "99": 59, "28": 19}, "source": "plato/graph/test/structure.cc:154-169"},
        {"graph": "v100_e2150_ua_c3.csv", "is_directed": False, "kind": "in",
         "values": {"0": 19, "99": 59, "28": 19}, "source": "plato/graph/test/structure.cc:171-186"},
        {"graph": "v100_e4300_da_c3.csv", "is_directed": True, "kind": "in",
         "values": {"0": 19, "99": 59, "28": 19}, "source": "plato/graph/test/structure.cc:188-203"},
    ],
    "neighbours": [
        {"graph": "v100_e2150_ua_c3.csv", "is_directed": True, "vertex": 0, "count": 19,
         "lo": 1, "hi": 19, "source": "plato/graph/structure/test/bcsr.cc:96-107"},
        {"graph": "v100_e2150_ua_c3.csv", "is_directed": True, "vertex": 10, "count": 9,
         "lo": 11, "hi": 19, "source": "plato/graph/structure/test/bcsr.cc:111-122"},
        {"graph": "v100_e2150_ua_c3.csv", "is_directed": True, "vertex": 98, "count": 1,
         "lo": 99, "hi": 99, "source": "plato/graph/structure/test/bcsr.cc:126-137"},
    ],
    "aggregate_message": [
        {"graph": "graph_10_9.csv", "is_directed": True, "sum": 9,
         "values": [0, 1, 1, 1, 1, 1, 1, 1, 1, 1],
         "source": "plato/graph/test/message_passing.cc:62-87"},
    ],
    # (in, out) per vertex, directed, step 1, bits 6, type both, every vertex a target
    "nstep_degrees": [
        {"graph": "raw_graph_7_7.csv", "is_directed": True, "step": 1, "bits": 6, "type": "both",
         "values": {"0": [3, 1], "4": [1, 1]},
         "source": "plato/algo/nstepdegrees/test/test_nstepdegrees.cc:41-48,87-96,104-139"},
    ],
    # |hyperanf average distance - exact average distance| <= tolerance
    "hyperanf": [
        {"graph": "raw_graph_7_7.csv", "is_directed": False, "bits": 6, "iterations": 20,
         "tolerance": 0.05, "source": "plato/algo/hyperanf/test/test_hyperanf.cc:46-52,133-217"},
    ],
    "hyperloglog": [
        {"test": "add", "bits": 6, "ids": 1000, "max_rel_error": 0.25,
         "source": "plato/util/test/test_hyperloglog.cc:29-39"},
        {"test": "merge", "bits": 12, "ids": 1000, "source": "plato/util/test/test_hyperloglog.cc:41-64"},
    ],
}


def hll_vectors(root: Path) -> dict:
    """Golden HyperLogLog vectors from the reference's own headers."""
    import ctypes as C
    sys.path.insert(0, str(HERE.parent.parent))
    from oracle.build import build_ref
    lib = C.CDLL(str(build_ref(ref_root=root)))
    lib.ref_murmur3_u32.restype = C.c_uint32
    lib.ref_murmur3_u32.argtypes = [C.c_uint32, C.c_uint32]
    lib.ref_hll_add.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64]
    lib.ref_hll_estimate.restype = C.c_double
    lib.ref_hll_estimate.argtypes = [C.c_uint32, C.c_void_p]
    rng = np.random.default_rng(20240607)
    ids = np.concatenate([np.arange(4096, dtype=np.uint32),
                          rng.integers(0, 2**32, 4096, dtype=np.uint64).astype(np.uint32)])
    out = {"hash_ids": ids,
           "hash_values": np.array([lib.ref_murmur3_u32(int(i), 0x5F61767A) for i in ids], np.uint32)}
    for P in range(4, 17):
        m = 1 << P
        rows, ests, counts = [], [], []
        for n in (1, 7, 100, 3000, 60000):  # ids 0..n-1 added to an empty row
            r = np.zeros(m, np.uint8)
            a = np.arange(n, dtype=np.uint32)
            lib.ref_hll_add(P, r.ctypes.data, a.ctypes.data, n)
            rows.append(r)
            counts.append(n)
            ests.append(lib.ref_hll_estimate(P, r.ctypes.data))
        for hi in (3, 12, 20):  # random registers: linear counting, raw and large-range branches
            r = rng.integers(0 if hi < 20 else 14, min(hi, 33 - P) + 1, m).astype(np.uint8)
            rows.append(r)
            counts.append(-1)
            ests.append(lib.ref_hll_estimate(P, r.ctypes.data))
        out[f"p{P}_rows"] = np.stack(rows)
        out[f"p{P}_ids"] = np.asarray(counts, np.int64)
        out[f"p{P}_est"] = np.asarray(ests, np.float64)
    return out


REF_GRAPHS = {
    # name: (fixture CSV or RMAT (scale, seed, symmetrise), is_directed)
    "v100u": ("v100_e2150_ua_c3.csv", False),
    "v100d": ("v100_e4300_da_c3.csv", True),
    "rmat12d": ((12, 1, False), True),
    "rmat12u": ((12, 2, True), False),
    "rmat14d": ((14, 3, False), True),
}


def ref_graph_edges(root: Path, spec):
    """Edge list of a REF_GRAPHS entry: a fixture CSV, or the oracle's seeded
    RMAT generator (equal to the product's; edgefactor 16)."""
    if isinstance(spec, str):
        return parse_csv(root / "data" / "graph" / spec)
    import oracle
    scale, seed, sym = spec
    _, s, d = oracle.rmat(scale, 16, seed, symmetrize=sym)
    return s, d


def ref_vectors(root: Path) -> dict:
    """The reference's own outputs on REF_GRAPHS (oracle/_ref/libplato_ref.so)."""
    sys.path.insert(0, str(HERE.parent.parent))
    from oracle.build import build_ref
    build_ref(ref_root=root)
    from oracle.refplato import ReferenceGraph
    out = {}
    for name, (spec, directed) in REF_GRAPHS.items():
        s, d = ref_graph_edges(root, spec)
        V = int(max(s.max(), d.max())) + 1
        g = ReferenceGraph(V, s, d, directed)
        out[f"{name}__meta"] = np.array([g.vertices, g.max_v_i, g.edges, int(directed)], np.uint64)
        r, ep, dl = g.pagerank(100, 0.85, 0.0)
        out[f"{name}__pr100"], out[f"{name}__pr100_epochs"], out[f"{name}__pr100_deltas"] = r, ep, dl
        r, ep, dl = g.pagerank(100, 0.85, 0.001)  # pagerank_opts_t defaults: early exit
        out[f"{name}__preps"], out[f"{name}__preps_epochs"] = r, ep
        deg = np.bincount(s, minlength=V) + (0 if directed else np.bincount(d, minlength=V))
        src = int(np.random.default_rng(7).choice(np.flatnonzero(deg > 0)))
        out[f"{name}__ppr_src"] = src
        for mode, pp in (("pull", False), ("pp", True)):
            r, ep = g.ppr(src, 200, 0.85, 1e-7, pp)
            out[f"{name}__ppr_{mode}"], out[f"{name}__ppr_{mode}_epochs"] = r, ep
        roots = np.random.default_rng(11).choice(np.flatnonzero(deg > 0), 3, replace=False)
        vis, acts, trs = [], [], []
        for rt in roots:
            v, a, t = g.bfs(int(rt))
            vis.append(v)
            acts.append(np.pad(a, (0, 64 - a.size)))
            trs.append(t)
        out[f"{name}__bfs_roots"] = roots.astype(np.uint32)
        out[f"{name}__bfs_visited"] = np.array(vis, np.uint64)
        out[f"{name}__bfs_actives"] = np.stack(acts)
        out[f"{name}__bfs_trace"] = np.array(trs, np.uint64)
        good = (np.arange(V) % 5 == 0).astype(np.uint8)
        out[f"{name}__good"] = good
        r, ep = g.trustrank(good, V + 1, 0, 100, 0.85, 1e-6)  # every good vertex a seed
        out[f"{name}__tr_all"], out[f"{name}__tr_all_epochs"] = r, ep
        for m in (0, 1):
            r, ep = g.trustrank(good, 20, m, 100, 0.85, 0.001)
            out[f"{name}__tr_m{m}"], out[f"{name}__tr_m{m}_epochs"] = r, ep
        if not directed:  # connected_component_t and hyperanf run on undirected graphs
            lab, comps, major, mv, me = g.connected_components()
            out[f"{name}__cc_labels"] = lab
            out[f"{name}__cc_summary"] = np.array([comps, major, mv, me], np.uint64)
            out[f"{name}__anf_avg"] = np.array([g.hyperanf(6, 20), g.hyperanf(8, 20)])
        g.close()
    # weighted PageRank: the reference's weighted fixture and a weighted RMAT s12
    from oracle.refplato import WeightedReferenceGraph
    z = np.load(HERE / "fixtures.npz")
    for name, (s, d, w) in {"w10": (z["raw_graph_10_9_weighted__src"], z["raw_graph_10_9_weighted__dst"],
                                    z["raw_graph_10_9_weighted__w"]),
                            "wrmat12": ref_graph_edges(root, (12, 1, False)) + (None,)}.items():
        if w is None:  # seeded weights, exactly representable as float32 (stored that way)
            w32 = np.random.default_rng(12).uniform(0.1, 10.0, s.size).astype(np.float32)
            out[f"{name}__w"] = w32
            w = w32.astype(np.float64)
        V = int(max(s.max(), d.max())) + 1
        wg = WeightedReferenceGraph(V, s, d, w, True)
        for tag, eps in (("100", 0.0), ("eps", 0.001)):
            r, ep = wg.weighted_pagerank(100, 0.85, eps)
            out[f"{name}__wpr{tag}"], out[f"{name}__wpr{tag}_epochs"] = r, ep
        wg.close()
    return {k: np.asarray(v) for k, v in out.items()}


def main(root: Path) -> None:
    arrays = {}
    for name in GRAPHS:
        s, d = parse_csv(root / "data" / "graph" / name)
        key = name.replace(".csv", "")
        arrays[f"{key}__src"] = s
        arrays[f"{key}__dst"] = d
    for name in WEIGHTED_GRAPHS:
        s, d, w = parse_csv(root / "data" / "graph" / name, weighted=True)
        key = name.replace(".csv", "")
        arrays[f"{key}__src"] = s
        arrays[f"{key}__dst"] = d
        arrays[f"{key}__w"] = w
    np.savez_compressed(HERE / "fixtures.npz", **arrays)
    (HERE / "kats.json").write_text(json.dumps(KATS, indent=1) + "\n")
    np.savez_compressed(HERE / "hll_golden.npz", **hll_vectors(root))
    np.savez_compressed(HERE / "ref_golden.npz", **ref_vectors(root))
    print("wrote", HERE / "fixtures.npz", HERE / "kats.json", HERE / "hll_golden.npz", HERE / "ref_golden.npz")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else
         Path(os.environ.get("PLATO_REFERENCE_ROOT", "/root/reference")))
