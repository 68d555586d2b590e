import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN / "golden.npz")


@pytest.fixture(scope="session")
def golden_meta():
    return json.loads((GOLDEN / "golden.json").read_text())


@pytest.fixture(scope="session")
def orc():
    import os

    from oracle import oracle

    oracle.build()
    oracle.set_threads(os.cpu_count() or 1)
    return oracle


@pytest.fixture(scope="session")
def fold_input():
    """Regenerates the seeded input of a golden fold case (tests/golden/make_golden.py)
    and checks it against the recorded sha256."""
    import hashlib

    def make(case):
        rng = np.random.default_rng(case["seed"])
        n = case["nsamples"] * case["nchans"]
        if case["dtype"] == "uint8":
            data = rng.integers(0, 256, size=n, dtype=np.uint8)
        else:
            data = rng.normal(0.0, 1.0, size=n).astype(np.float32)
        assert hashlib.sha256(data.tobytes()).hexdigest() == case["input_sha256"]
        return data

    return make
