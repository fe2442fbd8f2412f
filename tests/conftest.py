import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "d-core-cuda_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine's kernels")
    # build the engine library and the oracle once per session (nvcc
    # cross-compiles without a GPU)
    import build as engine_build  # d-core-cuda_b200/build.py
    from oracle import build as oracle_build
    engine_build.build()
    oracle_build.build()


def have_gpu():
    import dcore_b200 as dc
    try:
        return dc.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def dc():
    import dcore_b200
    return dcore_b200


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture(scope="session")
def gpu():
    if not have_gpu():
        pytest.fail("GPU test needs a CUDA device; run with -m 'not gpu' on CPU-only hosts")
    return True
