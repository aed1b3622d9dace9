import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: larger cases")


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def pac():
    return ge.load_package()


@pytest.fixture(scope="session")
def orc():
    o = ge.load_oracle()
    o.lib()
    return o


def golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return d["balls"], d["edges"], d["tris"], d["tets"]


def canonical(a):
    a = np.sort(np.asarray(a, dtype=np.int64), axis=1)
    if len(a) == 0:
        return a
    return a[np.lexsort(a.T[::-1])]
