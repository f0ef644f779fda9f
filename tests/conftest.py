import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "qmd-progress_b200"), os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def poly512():
    import numpy as np
    path = os.path.join(GOLDEN, "poly512.npz")
    if not os.path.exists(path):
        pytest.fail("tests/golden/poly512.npz missing (run tests/golden/make_golden.py)")
    d = dict(np.load(path))
    n = int(d["n"])
    h = np.zeros((n, n))
    h[d["h_rows"], d["h_cols"]] = d["h_vals"]
    d["h"] = h
    return d


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from sp2b import _lib
    _lib.lib()
    return torch
