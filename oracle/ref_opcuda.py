"""ctypes binding of ``oracle/_ref/libref_opcuda.so``: the reference's own CUDA kernels
(oplib/opcuda/sck.cu, sek.cu, sdot2.cu, sgemv3.cu, sgsvg.cu, sset.cu), compiled unchanged
from its sources by ``oracle/Makefile`` and launched with the reference's launch shapes
through ``oracle/ref_opcuda.cu``.  TEST INFRASTRUCTURE ONLY: the tests use it as the
checker of the drop-in entry points; nothing in ``oplib_b200`` loads it.

The library is built where the reference's sources are present and travels prebuilt;
``available()`` says whether it is there."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libref_opcuda.so"
_lib = None

vp, i32, f32 = C.c_void_p, C.c_int, C.c_float

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
}


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
