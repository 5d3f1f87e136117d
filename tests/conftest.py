import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "sph-2d_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs libsph_b200 kernels")
    config.addinivalue_line("markers", "slow: longer physics runs")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    """The CUDA library; GPU tests fail (not skip) if it cannot be built or loaded."""
    if not _have_gpu():
        pytest.skip("no CUDA device")
    import build_lib as pkg_build
    pkg_build.build()
    import sph_b200
    return sph_b200.load()


@pytest.fixture(scope="session")
def oracle():
    import oracle_api
    oracle_api.build()          # incremental: rebuilds only when a source changed
    oracle_api.load()
    return oracle_api
