"""The C++ drop-in overloads (include/ndlgpu_dropin.h) against the reference's
own ndl::gaussian_blur / ndl::convolve: runs oracle/_ref/dropin_check, which
oracle/build_oracle.py compiled from tests/cpp/dropin_check.cpp."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "dropin_check")


@pytest.mark.skipif(not os.path.exists(BIN), reason="dropin_check not built (needs the ndl source tree)")
def test_cpp_dropin_against_reference():
    res = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "DROPIN OK" in res.stdout
