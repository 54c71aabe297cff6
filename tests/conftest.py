import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda_ctx():
    import torch
    from qumasun_b200 import Context
    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    torch.cuda.init()
    ctx = Context(0)
    ctx.use_torch_stream()
    yield ctx
    ctx.close()
