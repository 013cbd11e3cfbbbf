import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_c():
    """ctypes handle of the C oracle (built on demand with make)."""
    lib = ROOT / "oracle" / "liboracle_c.so"
    src = ROOT / "oracle" / "oracle_c.c"
    if not lib.exists() or lib.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "-s"], check=True)
    from oracle import oracle_c as oc
    return oc.load()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oplib_b200 import _lib
    _lib.load()
    return torch.device("cuda:0")
