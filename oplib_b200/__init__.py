"""opcuda-b200: B200-native operator-method pricing path (OPLib's opcuda ABI on sm_100a).

The compute lives in ``libopcuda_b200.so`` (C ABI, ``include/opcuda_b200.h``);
``oplib_b200.model`` is the host-side model layer over it.
"""
from ._lib import LIB_PATH, OpcudaError, load  # noqa: F401

__all__ = ["LIB_PATH", "OpcudaError", "load"]
