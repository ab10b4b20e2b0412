import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


import pytest  # noqa: E402


@pytest.fixture(autouse=True)
def _release_device_buffers():
    """Synchronise and drop the buffers a GPU test handed to the library."""
    yield
    gu = sys.modules.get("gpu_util")
    if gu is not None and gu.KEEP:
        gu.release()
