import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100a) and the built libdarray_b200.so")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    """One db200 context on cuda:0 bound to torch's current stream (GPU tests only)."""
    if not _have_gpu():
        pytest.skip("no GPU in this environment")
    import torch
    from darray_optimizer_b200._lib import Context
    torch.cuda.init()
    ctx = Context(0, torch.cuda.current_stream().cuda_stream)
    yield ctx
    ctx.close()
