import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np
    z = np.load(ROOT / "tests" / "golden" / "fixtures.npz")
    kats = json.loads((ROOT / "tests" / "golden" / "kats.json").read_text())
    graphs = {}
    for k in z.files:
        name, part = k.split("__")
        graphs.setdefault(name + ".csv", {})[part] = z[k]
    return graphs, kats
