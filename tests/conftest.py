import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the sm_100a kernels")


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    """The C restatement is a few-second gcc build; make sure it exists."""
    from oracle import build_oracle
    build_oracle.build_restatement()


def golden(name):
    import json
    import numpy as np
    d = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    meta = json.loads(str(d["meta"]))
    return d, meta
