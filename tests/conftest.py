import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line(
        "markers",
        "late(k): runs after every unmarked test, in increasing k; for kernels whose bodies are "
        "checked on host threads (tests/*_host.py) but have not yet run on a B200, so that a "
        "failure there under -x cannot hide the results of the kernels already validated")


def pytest_collection_modifyitems(config, items):
    def rank(item):
        m = item.get_closest_marker("late")
        return (0, 0) if m is None else (1, m.args[0] if m.args else 0)
    items[:] = sorted(items, key=rank)  # stable: file order within each rank


def golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(path):
    d = dict(np.load(path))
    for k in ("side", "howmny"):
        d[k] = str(d[k])
    d["m"] = int(d["m"])
    d["info"] = int(d["info"])
    d["name"] = os.path.basename(path)[:-4]
    return d


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
