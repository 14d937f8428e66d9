import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
from oracle.build import REF_SRC as REFERENCE  # the reference checkout, located by the build recipe


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built():
    from oracle.build import build_oracle
    build_oracle()
    from internship_b200.build import build
    build()
    yield


def golden(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip("golden fixture %s not generated" % name)
    import numpy as np
    return np.load(p)


def reference_file(rel):
    p = os.path.join(REFERENCE, rel)
    if not os.path.exists(p):
        pytest.skip("reference checkout not available (%s)" % rel)
    return p
