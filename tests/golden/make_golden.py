"""Generate the golden fixtures under tests/golden/ from the reference's data.

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Reads the reference's fixture graphs (data/graph/*.csv) with the reference's
CSV rules (plato/graph/parsers.hpp:226-290: `src,dst[,w]` per line, fields
split on ',', parsed with strtoul so surrounding blanks are tolerated, empty
lines skipped) and writes
  fixtures.npz  edge lists (uint32) of the fixture graphs,
  kats.json     the known-answer values the reference's own substrate tests
                assert on those graphs, each with its file:line.
The reference tree is only needed to regenerate; tests read the outputs.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GRAPHS = ["graph_10_9.csv", "v100_e2150_ua_c3.csv", "v100_e4300_da_c3.csv"]


def parse_csv(path: Path) -> tuple[np.ndarray, np.ndarray]:
    src, dst = [], []
    for line in path.read_text().splitlines():
        if not line:
            continue
        parts = line.split(",")
        if len(parts) < 2:
            continue
        src.append(int(parts[0].strip() or 0))
        dst.append(int(parts[1].strip() or 0))
    return np.asarray(src, dtype=np.uint32), np.asarray(dst, dtype=np.uint32)


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
}


def main(root: Path) -> None:
    arrays = {}
    for name in GRAPHS:
        s, d = parse_csv(root / "data" / "graph" / name)
        key = name.replace(".csv", "")
        arrays[f"{key}__src"] = s
        arrays[f"{key}__dst"] = d
    np.savez_compressed(HERE / "fixtures.npz", **arrays)
    (HERE / "kats.json").write_text(json.dumps(KATS, indent=1) + "\n")
    print("wrote", HERE / "fixtures.npz", HERE / "kats.json")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference"))
