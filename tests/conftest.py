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


# Device memory below 4 GB of address space for the reference's kernels that read 32-bit
# device pointers (tests/test_gpu_ref_kernels.py).  It is reserved when the session's first
# GPU test starts, while that part of the address space is still free: later in a long
# session the library's and torch's allocations may occupy it.
LOW_BYTES = 96 << 20
_low = {}


def _reserve_low_memory():
    import ctypes as C
    try:
        from oracle import ref_opcuda
        if not ref_opcuda.available():
            _low["status"] = "oracle/_ref not built"
            return
        ref = ref_opcuda.load()
        p = C.c_ulonglong()
        r = ref.ref_low_alloc(LOW_BYTES, C.byref(p))
        _low["status"] = r
        if r == 0:
            _low["base"] = p.value
    except OSError as e:  # the harness library cannot be loaded here
        _low["status"] = str(e)


@pytest.fixture(scope="session")
def low_reservation():
    """(base, size) of the session's memory below 4 GB, or the reason it is missing."""
    return (_low.get("base"), LOW_BYTES, _low.get("status"))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not _low:
        _reserve_low_memory()
    from oplib_b200 import _lib
    _lib.load()
    return torch.device("cuda:0")


@pytest.fixture()
def fused_single(cuda):
    """Single-lattice solves with the row normalisation fused into the products' epilogues,
    as the batched sweep runs it (for batch-against-single comparisons); restores the
    default (fused from 4096 states, a renormalisation kernel below) afterwards."""
    from oplib_b200 import _lib
    lib = _lib.load()
    assert lib.opb_set_fused_normalisation(1 << 30) == 0
    yield
    assert lib.opb_set_fused_normalisation(-1) == 0
