import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.build()
    return o


@pytest.fixture(scope="session")
def nmlib():
    """The CUDA library's ctypes handle (built in-tree)."""
    from num_b200 import build, _lib
    build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def kspmv():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from num_b200 import build
    build.build()
    from num_b200 import kokkos_spmv
    kokkos_spmv.init(0)
    return kokkos_spmv
