"""pytest configuration: the ``gpu`` marker selects the parity tests that
need a B200 (run with ``-m gpu``); everything else runs on the CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and libmpsgpu.so")


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def kernels_npz():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "kernels.npz"))


@pytest.fixture(scope="session")
def mpo_npz():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "mpo_tensors.npz"))


@pytest.fixture(scope="session")
def trunc_npz():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "truncation.npz"))


@pytest.fixture(scope="session")
def ctx():
    """One library context on cuda:0 for the GPU tests (fails loudly when the
    library or the GPU is missing: there is no fallback)."""
    from mpsdyn_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()
