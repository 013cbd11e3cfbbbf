"""ctypes binding of the C oracle (``oracle/oracle_c.c``).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle_c.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    lib.oracle_mt19937_outputs.argtypes = [C.c_uint32, C.c_int, C.c_void_p]
    lib.oracle_mt19937_outputs.restype = None
    lib.oracle_uniform_f32.argtypes = [C.c_uint32]
    lib.oracle_uniform_f32.restype = C.c_float
    lib.oracle_sck_f32.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_long, C.c_long, C.c_void_p]
    lib.oracle_sck_f32.restype = None
    lib.oracle_mc_paths.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_int, C.c_int, C.c_uint32, C.c_uint64,
                                    C.c_long, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                    C.c_void_p, C.c_int]
    lib.oracle_mc_paths.restype = C.c_int
    lib.oracle_mt19937_outputs_keyed.argtypes = [C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]
    lib.oracle_mt19937_outputs_keyed.restype = None
    lib.oracle_mc_paths_seeded.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_int, C.c_int, C.c_void_p, C.c_uint64,
                                           C.c_long, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                           C.c_double, C.c_void_p, C.c_int]
    lib.oracle_mc_paths_seeded.restype = C.c_int
    lib.oracle_mt_benchmark.argtypes = [C.c_long, C.c_long, C.c_int, C.c_uint32]
    lib.oracle_mt_benchmark.restype = C.c_double
    _lib = lib
    return lib


def mt_outputs(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    load().oracle_mt19937_outputs(seed & 0xFFFFFFFF, n, out.ctypes.data)
    return out


def mt_outputs_keyed(seed: int, key1: int, n: int) -> np.ndarray:
    """First n outputs of MT19937 seeded init_genrand(seed) with key1 added to mt[1]."""
    out = np.empty(n, dtype=np.uint32)
    load().oracle_mt19937_outputs_keyed(seed & 0xFFFFFFFF, key1 & 0xFFFFFFFF, n, out.ctypes.data)
    return out


def sck(P: np.ndarray) -> np.ndarray:
    """Cumulative rows of a source-major FP32 matrix (sequential FP32)."""
    P = np.ascontiguousarray(P, dtype=np.float32)
    Cm = np.empty_like(P)
    d = P.shape[1]
    load().oracle_sck_f32(P.ctypes.data, d, P.shape[0], d, 1, Cm.ctypes.data)
    return Cm


def mc_paths(Cm: np.ndarray, y0: int, seed: int, path0: int, npaths: int, nsteps: int, x=None, strike=1.0,
             barrier=0.7, disc=1.0, want_paths=True, nthreads=8):
    """Returns (paths [npaths, nsteps] int16 or None, sums [2])."""
    Cm = np.ascontiguousarray(Cm, dtype=np.float32)
    d = Cm.shape[1]
    paths = np.empty((npaths, nsteps), dtype=np.int16) if want_paths else None
    sums = np.zeros(2, dtype=np.float64)
    xx = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
    r = load().oracle_mc_paths(Cm.ctypes.data, d, 1, d, y0, seed & 0xFFFFFFFF, path0, npaths, nsteps,
                               None if paths is None else paths.ctypes.data,
                               None if xx is None else xx.ctypes.data, strike, barrier, disc, sums.ctypes.data,
                               nthreads)
    if r != 0:
        raise RuntimeError("oracle_mc_paths failed")
    return paths, sums


def mc_paths_seeded(Cm: np.ndarray, y0: int, seeds: np.ndarray, path0: int, npaths: int, nsteps: int,
                    nthreads=8) -> np.ndarray:
    """Paths [npaths, nsteps] int16 of path ids path0 .. path0+npaths-1 with generators keyed
    from the 4096-entry stream seed table: path g uses MT19937 (seeds[g % 4096], g / 4096)."""
    Cm = np.ascontiguousarray(Cm, dtype=np.float32)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
    if seeds.shape != (4096,):
        raise ValueError("seeds must hold 4096 stream seeds")
    d = Cm.shape[1]
    paths = np.empty((npaths, nsteps), dtype=np.int16)
    sums = np.zeros(2, dtype=np.float64)
    r = load().oracle_mc_paths_seeded(Cm.ctypes.data, d, 1, d, y0, seeds.ctypes.data, path0, npaths, nsteps,
                                      paths.ctypes.data, None, 1.0, 0.0, 1.0, sums.ctypes.data, nthreads)
    if r != 0:
        raise RuntimeError("oracle_mc_paths_seeded failed")
    return paths
