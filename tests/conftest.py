import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a B200; runs the CUDA path through the C ABI")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_GPU = _cuda_available()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build(ref=True)
    return oracle


@pytest.fixture(scope="session")
def lib():
    from mgpu_old_b200 import api, build
    build.build()
    return api.load_library()


@pytest.fixture(scope="session")
def engine(lib):
    if not HAVE_GPU:
        pytest.skip("no GPU")
    import torch
    torch.cuda.init()
    torch.zeros(1, device="cuda")  # make the primary context current
    from mgpu_old_b200 import api
    e = api.MgpuSort()
    yield e
    e.release()
