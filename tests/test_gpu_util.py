"""The drop-in utility entry points the reference's CArray and device classes bind
(oplib/opmodel/types/CArray.cs:186-211, oplib/opmodel/models/CModel Device.cs:52-105):
device queries, device and pinned host memory, blocking copies, strided copies and fills,
against a numpy replay of the same operations."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_device_queries(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    assert lib.opcuda_cublas_init() == 0
    assert lib.opcuda_device_get_count() >= 1 and lib.opcuda_device_count() >= 1
    assert lib.opcuda_set_device(0) == 0 and lib.opcuda_get_device() == 0
    name = C.create_string_buffer(256)
    assert lib.opcuda_device_get_name(name, 256, 0) == 0 and b"B200" in name.value
    mem = C.c_uint64()
    assert lib.opcuda_device_total_memory(C.byref(mem), 0) == 0
    props = torch.cuda.get_device_properties(0)
    assert mem.value == props.total_memory
    assert lib.opcuda_multi_processor_count(0) == props.multi_processor_count
    assert lib.opcuda_max_threads_per_block(0) == 1024


def test_carray_lifecycle(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    nf, nb = 1000, 4000
    d1, d2, d3 = lib.opcuda_mem_alloc(nb), lib.opcuda_mem_alloc(nb), lib.opcuda_mem_alloc(nb)
    h = lib.opcuda_mem_alloc_host(nb)
    assert d1 and d2 and d3 and h
    hv = np.ctypeslib.as_array((C.c_float * nf).from_address(h))
    hv[:] = np.arange(nf, dtype=np.float32)
    assert lib.opcuda_memcpy_h2d(d1, h, nb) == 0
    assert lib.opcuda_ssetall(d2, nf, 2.5, 1) == 0
    assert lib.opcuda_ssetone(d2, nf, -1.0, 7) == 0
    assert lib.opcuda_scopy(300, d1, 3, d2 + 4 * 100, 2) == 0   # d2[100 + 2i] = d1[3i]
    assert lib.opcuda_scopy1(d1 + 4 * 500, d2, 200) == 0        # d1[500:700] = d2[0:200]
    assert lib.opcuda_memcpy_d2d(d3, d1, nb) == 0
    got2 = np.empty(nf, dtype=np.float32)
    got3 = np.empty(nf, dtype=np.float32)
    assert lib.opcuda_memcpy_d2h(d2, got2.ctypes.data, nb) == 0
    assert lib.opcuda_memcpy_d2h(d3, got3.ctypes.data, nb) == 0
    assert lib.opcuda_thread_synchronize() == 0
    r1 = np.arange(nf, dtype=np.float32)
    r2 = np.full(nf, 2.5, dtype=np.float32)
    r2[7] = -1.0
    r2[100:700:2] = r1[0:900:3]
    r1[500:700] = r2[0:200]
    assert np.array_equal(got2, r2) and np.array_equal(got3, r1)
    for d in (d1, d2, d3):
        assert lib.opcuda_mem_free_device(d) == 0
    assert lib.opcuda_mem_free_host(h) == 0
    assert lib.opcuda_shutdown() == 0
    assert lib.opcuda_get_status() == 0
