import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "lbm-fem_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built liblbfem_gpu.so")
    config.addinivalue_line("markers", "slow: longer-running check")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    oracle.set_threads(min(8, os.cpu_count() or 1))
    return oracle


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library on a GPU: fails loudly when either is missing (no fallback)."""
    import lbfem_gpu

    lib = lbfem_gpu.library()
    assert lbfem_gpu.device_count() > 0, "no CUDA device visible"
    return lib
