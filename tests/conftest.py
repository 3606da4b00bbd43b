import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "viennashe-dev_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def gpu_ctx():
    from vshe import gpu
    ctx = gpu.Context(0)
    yield ctx
    ctx.close()
