import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libbsgpu.so")


@pytest.fixture(scope="session", autouse=True)
def _built_libs():
    from bigstickpublick_b200 import build
    import oracle
    build.build_host()
    oracle.build()
    if os.environ.get("BSG_SKIP_GPU_BUILD") != "1":
        try:
            build.build_gpu()
        except Exception:
            pass
    yield
