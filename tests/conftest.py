import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def _ensure_built():
    """Build the native library and the oracle once per session (no-op when fresh)."""
    from dynamicgraphs_scc_b200 import build
    build.build()
    oracle_so = os.path.join(ROOT, "oracle", "build", "liboracle.so")
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), oracle_so], check=True, capture_output=True)


_ensure_built()


def has_gpu() -> bool:
    try:
        from dynamicgraphs_scc_b200 import device_count
        return device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    return 0
