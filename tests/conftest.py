"""Test configuration: the `gpu` marker and import paths.

Tests marked gpu run the CUDA library on a B200 through the C ABI; the rest
run on the CPU (the oracle against the golden vectors, host logic, and the
library's exported symbols without any compute call).
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "lgpsf-hessian_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def cuda_device():
    """Fail (not skip) when a gpu test runs without a device."""
    import ctypes
    try:
        rt = ctypes.CDLL("libcudart.so.12")
    except OSError:
        import torch  # noqa: F401  (brings its bundled runtime)
        import torch.cuda
        assert torch.cuda.is_available(), "gpu test without a CUDA device"
        return 0
    n = ctypes.c_int(0)
    rc = rt.cudaGetDeviceCount(ctypes.byref(n))
    assert rc == 0 and n.value > 0, "gpu test without a CUDA device"
    return 0
