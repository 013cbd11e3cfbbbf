"""ctypes binding of ``oracle/_ref/libref_opcuda.so``: the reference's own CUDA kernels
(oplib/opcuda/sck.cu, sek.cu, sdot2.cu, sgemv3.cu, sgsvg.cu, sset.cu, ssqmm.cu, sgemm4.cu,
sgemv4.cu), compiled unchanged from its sources by ``oracle/Makefile`` and launched with the
reference's launch shapes through ``oracle/ref_opcuda.cu`` and ``oracle/ref_tables.cu``; the
kernels that read 32-bit device pointers get memory below 4 GB (``oracle/ref_lowmem.cu``).  TEST INFRASTRUCTURE ONLY: the tests use it as the
checker of the drop-in entry points; nothing in ``oplib_b200`` loads it.

The library is built where the reference's sources are present and travels prebuilt;
``available()`` says whether it is there."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libref_opcuda.so"
_lib = None

vp, i32, f32, u64 = C.c_void_p, C.c_int, C.c_float, C.c_ulonglong

PROTOTYPES = {
    "ref_sck": (i32, [i32, i32, vp, vp]),
    "ref_sek": (i32, [i32, vp, f32, vp]),
    "ref_sekd": (i32, [i32, vp, f32, vp, vp]),
    "ref_sekd_lambda": (i32, [i32, vp, f32, vp, vp, vp]),
    "ref_sdot2": (i32, [vp, vp, vp, i32, i32]),
    "ref_sgemv3": (i32, [i32, i32, i32, vp, vp, vp, vp]),
    "ref_sgsvg": (i32, [vp, i32, i32, i32, vp, vp]),
    "ref_ssetall": (i32, [vp, i32, f32, i32]),
    "ref_ssetone": (i32, [vp, i32, f32, i32]),
    "ref_ssqmm": (i32, [i32, i32, u64, u64, u64]),
    "ref_sgemm4": (i32, [i32, u64]),
    "ref_sgemv4": (i32, [i32, u64]),
    "ref_low_alloc": (i32, [u64, C.POINTER(C.c_ulonglong)]),
    "ref_low_free_all": (i32, []),
    "ref_memcpy_h2d": (i32, [u64, vp, u64]),
    "ref_memcpy_d2h": (i32, [vp, u64, u64]),
}


class LowArena:
    """Device memory below 4 GB of address space (``ref_low_alloc``) for the reference's
    kernels that read 32-bit device pointers, carved in 256-byte aligned pieces."""

    def __init__(self, lib, base: int, size: int):
        self.lib, self.base, self.size, self.used = lib, base, size, 0

    def alloc(self, nbytes: int) -> int:
        off = (self.used + 255) // 256 * 256
        if off + nbytes > self.size:
            raise MemoryError("low arena exhausted")
        self.used = off + nbytes
        return self.base + off

    def put(self, a) -> int:
        import numpy as np
        a = np.ascontiguousarray(a)
        addr = self.alloc(a.nbytes)
        if self.lib.ref_memcpy_h2d(addr, a.ctypes.data, a.nbytes) != 0:
            raise RuntimeError("ref_memcpy_h2d failed")
        return addr

    def get(self, addr: int, shape, dtype):
        import numpy as np
        out = np.empty(shape, dtype=dtype)
        if self.lib.ref_memcpy_d2h(out.ctypes.data, addr, out.nbytes) != 0:
            raise RuntimeError("ref_memcpy_d2h failed")
        return out


def available() -> bool:
    return LIB.exists()


def load():
    global _lib
    if _lib is not None:
        return _lib
    lib = C.CDLL(str(LIB))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
