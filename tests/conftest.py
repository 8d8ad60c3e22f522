import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")


def load_tiny_cases():
    from research_b200.ocean import HostCSR

    def mk(d, cols=None):
        return HostCSR(d["rows"], d["cols"], np.array(d["rowptr"], np.uint32), np.array(d["col"], np.uint32),
                       np.array(d["val"], np.float64))

    cases = json.loads((GOLDEN / "tiny_cases.json").read_text())["cases"]
    out = []
    for c in cases:
        A, B = mk(c["A"]), mk(c["B"])
        exp = (np.array(c["C"]["rowptr"], np.uint64), np.array(c["C"]["col"], np.uint32),
               np.array(c["C"]["val"], np.float64))
        out.append((c["name"], A, B, exp))
    return out


@pytest.fixture(scope="session")
def tiny_cases():
    return load_tiny_cases()


@pytest.fixture(scope="session")
def murmur_kat():
    d = json.loads((GOLDEN / "murmur3_kat.json").read_text())
    return np.array(d["keys"], np.uint64).astype(np.uint32), np.array(d["hashes"], np.uint64).astype(np.uint32)
