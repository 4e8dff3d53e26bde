import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN_NPZ = os.path.join(ROOT, "tests", "golden", "reference_fixtures.npz")
GOLDEN_JSON = os.path.join(ROOT, "tests", "golden", "reference_fixtures.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running CPU case")


@pytest.fixture(scope="session")
def golden():
    with np.load(GOLDEN_NPZ) as z:
        arrays = {k: z[k] for k in z.files}
    with open(GOLDEN_JSON) as f:
        meta = json.load(f)
    return arrays, meta


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def first_mismatch(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32).ravel()
    b = np.ascontiguousarray(b, dtype=np.float32).ravel()
    bad = np.nonzero(a.view(np.uint32) != b.view(np.uint32))[0]
    if bad.size == 0:
        return None
    q = int(bad[0])
    return f"{bad.size} mismatches; first at {q}: {a[q]!r} vs {b[q]!r}"
