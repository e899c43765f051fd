import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the sm_100a kernels")
    config.addinivalue_line("markers", "sets_guards: a GPU test that makes the device guards fire on purpose")


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


@pytest.fixture(autouse=True)
def _device_guards_clear(request):
    """After every GPU test: no kernel guard fired (a bounded wait that ran
    out, or a dropped batched work item) -- ndlgpu_device_status reads 0."""
    yield
    if request.node.get_closest_marker("gpu") is None or request.node.get_closest_marker("sets_guards"):
        return
    import torch
    if not torch.cuda.is_available():
        return
    import ctypes
    from ndl_b200 import abi
    code = ctypes.c_int32(-1)
    abi.check(abi.load().ndlgpu_device_status(None, ctypes.byref(code)))
    assert code.value == 0, "device guard word %d after the test" % code.value
