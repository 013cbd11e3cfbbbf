"""ctypes binding of ``libopcuda_b200.so`` (the C ABI declared in include/opcuda_b200.h).

This plays the role of the reference's P/Invoke declarations
(``oplib/opmodel/models/CModel Device.cs:52-105``): one typed prototype per export.
Loading fails loudly if the library has not been built -- there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libopcuda_b200.so"

i32, i64, u32, u64, f32, f64 = C.c_int, C.c_longlong, C.c_uint32, C.c_uint64, C.c_float, C.c_double
ull = C.c_ulonglong
vp, cp = C.c_void_p, C.c_char_p


class LatticeDesc(C.Structure):
    """Mirror of ``opb_lattice_desc``."""

    _fields_ = [
        ("d", i32), ("y0", i32), ("ell_width", i32),
        ("gen_cols", vp), ("gen_vals", vp), ("gen_dense", vp), ("x", vp),
        ("dt", f64), ("niter", i32), ("nmat", i32), ("period", f64), ("rate", f64),
        ("nK", i32), ("strikes", vp),
    ]


# name: (restype, [argtypes])
PROTOTYPES: dict[str, tuple] = {
    # runtime support
    "opcuda_get_status": (i32, []),
    "opcuda_cublas_init": (i32, []),
    "opcuda_shutdown": (i32, []),
    "opcuda_thread_synchronize": (i32, []),
    "opcuda_set_device": (i32, [i32]),
    "opcuda_get_device": (i32, []),
    "opcuda_device_get_count": (i32, []),
    "opcuda_device_count": (i32, []),
    "opcuda_device_get_name": (i32, [cp, i32, i32]),
    "opcuda_device_total_memory": (i32, [C.POINTER(u64), i32]),
    "opcuda_multi_processor_count": (i32, [i32]),
    "opcuda_max_threads_per_block": (i32, [i32]),
    "opcuda_mem_alloc": (u64, [u64]),
    "opcuda_mem_free_device": (i32, [u64]),
    "opcuda_mem_alloc_host": (u64, [u64]),
    "opcuda_mem_free_host": (i32, [u64]),
    "opcuda_memcpy_h2d": (i32, [u64, u64, u64]),
    "opcuda_memcpy_d2h": (i32, [u64, u64, u64]),
    "opcuda_memcpy_d2d": (i32, [u64, u64, u64]),
    "opcuda_create_timer": (None, []),
    "opcuda_reset_timer": (None, []),
    "opcuda_stop_timer": (None, []),
    "opcuda_get_timer_value": (f64, []),
    "opcuda_scopy": (i32, [i32, u64, i32, u64, i32]),
    "opcuda_scopy1": (i32, [u64, u64, u64]),
    "opcuda_ssetall": (i32, [u64, i32, f32, i32]),
    "opcuda_ssetone": (i32, [u64, i32, f32, i32]),
    "opb_set_stream": (i32, [u64]),
    "opb_get_stream": (u64, []),
    "opb_version": (cp, []),
    "opb_status_string": (cp, [i32]),
    "opb_test_fail_next_alloc": (i32, [i32]),
    # GEMM / GEMV
    "opcuda_sgemm": (i32, [i32, i32, i32, f32, u64, i32, u64, i32, f32, u64, i32]),
    "opcuda_ssqmm": (i32, [i32, i32, u64, u64, u64]),
    "opcuda_sgemm4": (i32, [i32, u64]),
    "opb_sgemm4_task_size": (i32, []),
    "opb_sgemm_batched_rm": (i32, [i32, i32, i32, vp, i64, vp, i64, vp, i64, i32]),
    "opcuda_sgemv": (i32, [i32, i32, f32, u64, i32, u64, i32, f32, u64, i32]),
    "opcuda_sgemvT": (i32, [i32, i32, f32, u64, i32, u64, i32, f32, u64, i32]),
    "opcuda_sgemv3": (i32, [i32, i32, i32, u64, u64, u64, u64]),
    "opcuda_sgemv4": (i32, [i32, u64]),
    "opb_sgemv4_task_size": (i32, []),
    "opcuda_sdot2": (i32, [u64, u64, u64, i32, i32]),
    # kernels from generators
    "opcuda_sek": (i32, [i32, u64, f32, u64]),
    "opcuda_sekd": (i32, [i32, u64, f32, u64, u64]),
    "opcuda_sekd_lambda": (i32, [i32, u64, f32, u64, u64, u64]),
    "opcuda_sglvg": (i32, [u64, i32, i32, u64, u64]),
    "opb_lv_params": (i32, [i32, f64, f64, f64, f64, f64, f64, f64, f64, vp, vp, vp]),
    "opb_lv_generator_ell": (i32, [i32, vp, vp, vp, vp, vp]),
    "opb_sv_generator_ell": (i32, [i32, i32, f64, f64, f64, f64, f64, f64, f64, f64, f64, vp, vp, vp]),
    "opb_ell_maxdiag": (i32, [i32, i32, vp, vp, vp, C.POINTER(f64)]),
    "opb_plan_interval": (i32, [f64, f64, f64, C.POINTER(i32), C.POINTER(f64)]),
    # split-BF16 GEMM
    "opb_gemm_bf16x3": (i32, [i32, i32, i32, vp, vp, i64, vp, vp, i64, f32, vp, f32, vp, i64, vp]),
    "opb_gemm_bf16x3_nparts": (i32, [i32, i32]),
    "opb_gemm_bf16x3_kn": (i32, [i32, i32, i32, vp, vp, i64, vp, vp, i64, f32, vp, f32, vp, i64, vp]),
    "opb_gemm_f16x3_kn": (i32, [i32, i32, i32, vp, vp, i64, vp, vp, i64, f32, vp, f32, vp, i64, vp]),
    "opb_set_tile_n": (i32, [i32]),
    "opb_gemm_bf16x3_ksliced": (i32, [i32, i32, i32, vp, vp, i64, vp, vp, i64, vp, i64, i32, i64, C.POINTER(i32)]),
    "opb_gemm_f16x3": (i32, [i32, i32, i32, vp, vp, i64, vp, vp, i64, f32, vp, f32, vp, i64, vp]),
    "opb_tc_error": (i32, []),
    "opb_batch_num_configs": (i32, []),
    "opb_lv_generator_ell_batched": (i32, [i32, vp, i64, f64, f64, f64, vp, vp]),
    "opb_lv_param_size": (i32, []),
    "opcuda_sgsvg": (i32, [u64, i32, i32, i32, u64, u64]),
    "opb_set_stage_k": (i32, [i32]),
    "opb_set_cta_pair": (i32, [i32]),
    "opb_set_group_m": (i32, [i32]),
    "opb_renorm_rows": (i32, [i32, vp, vp, i32, i32, vp, vp, vp, vp, i32]),
    # lattice
    "opb_lattice_workspace_size": (ull, [i32, i32, i32]),
    "opb_lattice_solve": (i32, [C.POINTER(LatticeDesc), i32, vp, ull, vp, vp]),
    "opb_lattice_kernel": (i32, [C.POINTER(LatticeDesc), i32, vp, ull, vp]),
    "opb_lattice_bermudan": (i32, [C.POINTER(LatticeDesc), i32, i32, i32, f64, vp, ull, vp]),
    "opb_set_ksplit": (i32, [i32]),
    "opb_set_lolo_levels": (i32, [i32]),
    "opb_chain_workspace_size": (ull, [i32]),
    "opb_chain_kernels": (i32, [i32, i32, vp, vp, vp, ull]),
    "opb_set_band_skip": (i32, [i32]),
    "opb_set_fused_normalisation": (i32, [i32]),
    # batched lattices
    "opb_batch_workspace_size": (ull, [vp, i32]),
    "opb_batch_plan_create": (i32, [vp, i32, vp, ull, vp]),
    "opb_batch_plan_destroy": (i32, [vp]),
    "opb_batch_set_config": (i32, [vp, i32, i32]),
    "opb_batch_execute": (i32, [vp, vp]),
    "opb_batch_execute_bermudan": (i32, [vp, i32, i32, f64, vp]),
    "opb_batch_autotune": (i32, [vp, i32, vp, vp]),
    "opb_batch_launches": (i32, [vp]),
    # surrogate MLP
    "opb_mlp_param_count": (i32, []),
    "opb_mlp_workspace_floats": (i64, [i32]),
    "opb_mlp_set_tensor_cores": (i32, [i32]),
    "opb_mlp_set_fused_inference": (i32, [i32]),
    "opb_mlp_init": (i32, [vp, ull]),
    "opb_mlp_round": (i32, [vp, vp, vp]),
    "opb_mlp_forward": (i32, [vp, vp, i32, vp, vp]),
    "opb_mlp_loss_grad": (i32, [vp, vp, vp, i32, vp, vp, vp]),
    "opb_mlp_adam": (i32, [vp, vp, vp, vp, i32, f32, f32, f32, f32, vp]),
    "opb_mlp_adam_sched": (i32, [vp, vp, vp, vp, vp, vp, f32, f32, f32, vp]),
    "opb_implied_vol": (i32, [i64, vp, vp, vp, vp, vp, vp]),
    "opb_mlp_packed_bytes": (i64, []),
    "opb_mlp_pack": (i32, [vp, vp]),
    "opb_mlp_infer_workspace_bytes": (i64, [i64, i32]),
    "opb_mlp_infer": (i32, [vp, i32, i64, vp, i64, vp, i64, vp, vp]),
    # cumulative rows / MC
    "opcuda_sck": (i32, [i32, i32, u64, u64]),
    "opb_sck_rm": (i32, [i32, i32, vp, vp]),
    "opb_guide_table": (i32, [i32, i32, i32, vp, vp]),
    "opcuda_mc_load_mt_gpu": (i32, [cp, C.c_long]),
    "opcuda_mc_nrng": (i32, []),
    "opcuda_mc_status_sz": (i32, []),
    "opcuda_mc_setseed": (i32, [u64, u64]),
    "opcuda_mc1f": (i32, [u64, i32, u64, i32, i32, i32, u64, u64, u64]),
    "opcuda_mc1f_eval": (i32, [u64, i32, u64, i32, i32, i32, u64, u64, u64, u64, u64]),
    "opcuda_mt_benchmark": (i32, [u64, u64, i32]),
    "opb_mc_scratch_blocks": (i32, [i64]),
    "opb_mc_mt19937": (i32, [vp, i64, i64, vp, i32, i32, i32, i32, u32, ull, i64, vp, vp, f64, f64, f64, vp, vp]),
    "opb_mc_mt19937_eval": (i32, [vp, i64, i64, vp, i32, i32, i32, i32, u32, ull, i64, vp, vp, vp, vp, vp, vp]),
    "opb_mc_mt19937_noalloc": (i32, [vp, i64, i64, vp, i32, i32, i32, i32, u32, ull, i64, vp, vp, f64, f64, f64,
                                     vp]),
    "opb_mt19937_raw": (i32, [u32, i64, i32, vp]),
    "opb_mt_uniforms": (i32, [u32, i64, i32, vp]),
}

_lib = None


class OpcudaError(RuntimeError):
    def __init__(self, fn: str, status: int, text: str):
        super().__init__(f"{fn} failed with status {status}: {text}")
        self.status = status


def load() -> C.CDLL:
    """Load the library (once) and attach prototypes.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("OPB_LIB", LIB_PATH))
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build it with `python -m oplib_b200.build` (nvcc, sm_100a). "
            "There is no CPU fallback.")
    lib = C.CDLL(str(path))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(fn: str, status: int) -> int:
    if status != 0:
        lib = load()
        raise OpcudaError(fn, status, lib.opb_status_string(status).decode())
    return status


def call(name: str, *args):
    """Call an int-returning export and raise on a non-zero status."""
    lib = load()
    return check(name, getattr(lib, name)(*args))
