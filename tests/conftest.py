import os
import sys

# The oracle's compiled reference maps use OpenMP; the test problems are
# small, and a parallel region per map loop across every core of a large
# host costs more than it saves.  Set before any library loads libgomp.
os.environ.setdefault("OMP_NUM_THREADS", "4")

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    """test_zz_no_alloc runs last (stable order otherwise): its entry point
    holds a fixed device array, the other tests allocate freely."""
    items.sort(key=lambda item: item.module.__name__.startswith("test_zz"))


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(ROOT, "tests", "golden", "v2rdm_maps.npz")
    data = np.load(path)
    cases = {}
    for key in data.files:
        name, field = key.split("/", 1)
        cases.setdefault(name, {})[field] = data[key]
    return cases


def case_kwargs(case):
    """keyword arguments that rebuild a golden case's problem"""
    n, na, nb, spin, sz, hub = [int(v) for v in case["spec"]]
    kw = dict(n=n, na=na, nb=nb, positivity=str(case["positivity"]), constrain_spin=bool(spin),
              constrain_sz=bool(sz))
    if hub > 0:
        kw["hubbard"] = tuple(float(v) for v in case["hubbard"])
    else:
        kw["h"] = case["h"]
        kw["g"] = case["g"]
    return kw


@pytest.fixture(scope="session")
def cuda_device():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
