"""ctypes binding of the CPU restatement of the reference's ``opc`` library
(``oracle/opc.c``, declared in ``oracle/opc.h``).  TEST INFRASTRUCTURE ONLY.

The prototypes follow the reference's P/Invoke declarations of the same functions
(``oplib/opmodel/types/CRangen.cs:43-47,111-146``, ``oplib/opmodel/types/S1DGrid.cs:74-76``,
``oplib/opmodel/models/CModel Host Double.cs:47-61``, ``benchmarks/csgemm/Program.cs:46``,
``benchmarks/gsgemv4/Program.cs:77``, ``benchmarks/cmt/Program.cs:44-45``)."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "libopc.so"
_lib = None

vp, i32, f32, f64 = C.c_void_p, C.c_int, C.c_float, C.c_double

PROTOTYPES = {
    "opc_sgemv": (None, [i32, i32, f32, vp, i32, vp, i32, f32, vp, i32]),
    "opc_dgemv": (None, [i32, i32, f64, vp, i32, vp, i32, f64, vp, i32]),
    "opc_dgesv": (i32, [i32, i32, vp, i32, i32, i32, vp, vp, i32]),
    "opc_sgesv": (i32, [i32, i32, vp, i32, i32, i32, vp, vp, i32, vp]),
    "opc_sgemm": (None, [vp, vp, vp, i32, i32, i32, i32, i32, i32]),
    "opc_dgemm": (None, [vp, vp, vp, i32, i32, i32, i32, i32, i32]),
    "opc_dcopy": (None, [i32, vp, vp]),
    "opc_rangen_init_seed": (None, [vp, i32]),
    "opc_rangen_getstatus": (i32, []),
    "opc_rangen_finalize": (None, []),
    "opc_gennor": (None, [vp, i32, f64, f64, i32]),
    "opc_genunif": (None, [vp, i32, f64, f64, i32]),
    "opc_dmc1": (i32, [vp, vp, i32, i32, i32, i32, vp, vp, vp, C.c_ulong, i32, i32]),
    "opc_mt_benchmark": (i32, [i32, vp, i32]),
    "opc_host_mc_hash": (None, [vp, i32, i32, vp, vp]),
}

# void payoff_eval(short* y_sk, int th, int batch) (oplib/opc/rangen.cpp:99-103)
PAYOFF_EVAL = C.CFUNCTYPE(None, C.POINTER(C.c_short), C.c_int, C.c_int)


def load():
    global _lib
    if _lib is not None:
        return _lib
    sources = [HERE / "opc.c", HERE / "opc.h"]
    if not LIB.exists() or LIB.stat().st_mtime < max(s.stat().st_mtime for s in sources):
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    lib = C.CDLL(str(LIB))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
