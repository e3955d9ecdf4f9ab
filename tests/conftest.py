import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _built():
    import oracle_api
    oracle_api.build()
    from poker_trainer_b200 import build
    if os.path.exists(build.NVCC):
        # With a compiler present a failed build is an error: testing a stale
        # library would hide it.
        build.build()
    elif not os.path.exists(build.LIB):
        pytest.fail(f"libdcfr.so is not built and {build.NVCC} is absent")
    # Without nvcc the prebuilt library that travels with the tree is used.
    yield


@pytest.fixture(scope="session")
def gpu():
    if not gpu_available():
        pytest.fail("GPU test on a machine without a CUDA device")
    return True
