import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle(threads=1)


@pytest.fixture(scope="session")
def gpu_ctx():
    if not cuda_available():
        pytest.fail("GPU test collected on a machine without CUDA: run with -m 'not gpu'")
    from haissinskijulia_b200 import Context
    from haissinskijulia_b200 import build as _b
    _b.build()
    return Context(0)


@pytest.fixture(scope="session")
def gpu_buffers(gpu_ctx):
    from haissinskijulia_b200 import create_simulation_buffers
    return create_simulation_buffers(1, 1, ctx=gpu_ctx)
