"""C-ABI checks that need no GPU: the library loads, exports every symbol that
include/opcuda_b200.h declares, and rejects bad arguments on the host with the
documented status codes (no device work is issued for them)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "opcuda_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"typedef struct.*?\}\s*\w+;", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b((?:opcuda|opb)_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from oplib_b200 import _lib
    return _lib.load()


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) > 60
    for must in ["opcuda_ssqmm", "opcuda_sgemm", "opcuda_mc1f", "opcuda_sck", "opcuda_sek", "opb_lattice_solve",
                 "opb_gemm_bf16x3", "opb_mc_mt19937"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from oplib_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, missing


def test_prototypes_cover_header(lib):
    from oplib_b200 import _lib
    missing = [n for n in declared_symbols() if n not in _lib.PROTOTYPES]
    assert not missing, missing


def test_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "opcuda_b200.h"\nint main(void){return OPB_OK;}\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o",
                    str(tmp_path / "t")], check=True)


def test_c_host_program_links_and_calls(tmp_path):
    """A plain C host, as a P/Invoke or cgo binding would be, links the library by name and
    calls its host-side entry points: version, status strings, the niter rule, workspace
    sizes and a host-side argument rejection read back through opcuda_get_status."""
    from oplib_b200 import _lib
    src = tmp_path / "host.c"
    src.write_text(r"""
#include <stdio.h>
#include <string.h>
#include "opcuda_b200.h"
int main(void) {
    int n = 0;
    double dt = 0.0;
    if (!strstr(opb_version(), "sm_100a")) return 1;
    if (opb_plan_interval(1108.0573710154804, 0.25, 0.00006103515625, &n, &dt) != OPB_OK || n != 12) return 2;
    if (opb_lattice_workspace_size(512, 64, 2) == 0) return 3;
    if (opb_sgemm4_task_size() != 48) return 4;
    if (opcuda_ssqmm(-3, 1, 1, 1, 1) != OPB_E_ARG || opcuda_get_status() != OPB_E_ARG) return 5;
    printf("%s|%s\n", opb_status_string(OPB_E_ARG), opb_status_string(OPB_E_NULL));
    return 0;
}
""")
    libdir = str(_lib.LIB_PATH.parent)
    exe = tmp_path / "host"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lopcuda_b200", "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out
    assert out.stdout.strip() == "invalid size or count|null pointer"


def test_version_and_status_strings(lib):
    assert b"sm_100a" in lib.opb_version()
    assert lib.opb_status_string(-1) == b"invalid size or count"
    assert lib.opb_status_string(-2) == b"null pointer"


@pytest.mark.parametrize("call,expect", [
    (lambda L: L.opcuda_sgemm(-1, 4, 4, 1.0, 1, 4, 1, 4, 0.0, 1, 4), -1),
    (lambda L: L.opcuda_sgemm(4, 4, 4, 1.0, 0, 4, 1, 4, 0.0, 1, 4), -2),
    (lambda L: L.opcuda_sgemm(4, 4, 4, 1.0, 1, 2, 1, 4, 0.0, 1, 4), -1),  # lda < m
    (lambda L: L.opcuda_ssqmm(-3, 1, 1, 1, 1), -1),
    (lambda L: L.opcuda_ssqmm(8, 1, 0, 1, 1), -2),
    (lambda L: L.opcuda_sck(-1, 1, 1, 1), -1),
    (lambda L: L.opcuda_sek(8, 0, 0.1, 1), -2),
    (lambda L: L.opcuda_mc1f(1, 0, 1, 4096, 0, 64, 1, 1, 0), -1),  # no steps
    (lambda L: L.opcuda_mc1f(1, 70, 1, 4096, 10, 64, 1, 1, 0), -1),  # y0 >= d
    (lambda L: L.opcuda_mt_benchmark(1, 1, 4097), -1),
    (lambda L: L.opb_guide_table(64, 4, 48, 1, 1), -1),  # nb not a power of two
    (lambda L: L.opb_mc_mt19937(1, 64, 1, None, 0, 64, 0, 0, 1, 0, 10, None, None, 1.0, 0.7, 1.0, None, None), -1),
    # runs past the register-only generator would grow the driver's local memory
    (lambda L: L.opb_mc_mt19937_noalloc(1, 64, 1, None, 0, 64, 0, 624, 1, 0, 10, None, None, 1.0, 0.7, 1.0, None),
     -4),
    (lambda L: L.opb_mt19937_raw(1, 4, 0, 1), -1),
    (lambda L: L.opb_mt_uniforms(1, 4, 0, 1), -1),
    (lambda L: L.opb_sv_generator_ell(2, 8, 0.05, 5.0, 0.05, 1.0, 0.03, 2.0, 0.04, 0.6, -0.7, 1, 1, None), -1),
    (lambda L: L.opb_lv_generator_ell(2, 1, 1, 1, 1, 1), -1),
    (lambda L: L.opcuda_sgemv(4, 4, 1.0, 0, 4, 1, 1, 0.0, 1, 1), -2),
    (lambda L: L.opcuda_sdot2(0, 1, 1, 4, 4), -2),
    (lambda L: L.opb_set_fused_normalisation(-2), -1),  # -1 (automatic) is the lowest value
])
def test_host_argument_errors(lib, call, expect):
    assert call(lib) == expect
    assert lib.opcuda_get_status() == expect


def test_mc_seed_table_sizes(lib):
    """The reference's callers allocate opcuda_mc_nrng() seeds and a status record of
    opcuda_mc_status_sz() int32 words (oplib/opmodel/models/CModel Device.cs:320-338)."""
    assert lib.opcuda_mc_nrng() == 4096
    assert lib.opcuda_mc_status_sz() == 4 + 4096
    assert lib.opcuda_mc_setseed(0, 1) == -2


def test_lattice_desc_rejected_on_host(lib):
    from oplib_b200._lib import LatticeDesc
    L = LatticeDesc()
    L.d, L.y0, L.niter, L.nmat, L.nK = 100, 5, 3, 1, 4
    L.dt, L.period = 1e-4, 0.25
    assert lib.opb_lattice_solve(C.byref(L), 2, 1, 1 << 40, 1, None) == -2  # no x / strikes
    L.x, L.strikes, L.ell_width, L.gen_cols, L.gen_vals = 1, 1, 3, 1, 1
    # bf16x3 takes d = 100 as a lattice padded to 128 states: its workspace is at least the
    # 128-state one, and a smaller buffer is refused before anything runs
    need = lib.opb_lattice_workspace_size(100, 4, 2)
    assert need >= lib.opb_lattice_workspace_size(128, 4, 2) > 0
    assert lib.opb_lattice_solve(C.byref(L), 2, 1, need - 1, 1, None) == -1
    assert lib.opb_lattice_solve(C.byref(L), 7, 1, 1 << 40, 1, None) == -1  # bad mode
    assert lib.opb_lattice_solve(None, 0, 1, 1, 1, None) == -2


def test_plan_interval_rule(lib):
    n = C.c_int()
    dt = C.c_double()
    # CModel Common.cs:289-307 with maxdiag 1108.06, DeltaT 0.25, dt0 2^-14 -> 12 squarings
    assert lib.opb_plan_interval(1108.0573710154804, 0.25, 2.0 ** -14, C.byref(n), C.byref(dt)) == 0
    assert n.value == 12 and dt.value == 0.25 * 2.0 ** -12
    # config 2: DeltaT = 1/252 -> 7 squarings of Delta t / 128
    assert lib.opb_plan_interval(1108.0573710154804, 1 / 252, 2.0 ** -14, C.byref(n), C.byref(dt)) == 0
    assert n.value == 7 and abs(dt.value - (1 / 252) / 128) < 1e-18
    # a stiff generator takes the 0.5/maxdiag branch
    assert lib.opb_plan_interval(1e6, 0.25, 2.0 ** -14, C.byref(n), C.byref(dt)) == 0
    assert n.value == 19


def test_workspace_sizes(lib):
    assert lib.opb_lattice_workspace_size(512, 64, 2) > 4 * 512 * 512 * 2
    assert lib.opb_lattice_workspace_size(0, 64, 2) == 0
    assert lib.opb_gemm_bf16x3_nparts(6144, 6144) == 48  # one FP64 row-sum partial per 128 columns
    assert lib.opb_gemm_bf16x3_nparts(384 * 128, 384) == 3
    assert lib.opb_sgemm4_task_size() == 48
    assert lib.opb_sgemv4_task_size() == 56


def test_wall_clock_timers(lib):
    """opcuda_create/reset/stop_timer and opcuda_get_timer_value (oplib/opmodel/types/
    CStopWatch.cs:44-54 binds them): seconds between the last reset and the last stop."""
    import time
    lib.opcuda_create_timer()
    time.sleep(0.02)
    lib.opcuda_stop_timer()
    v = lib.opcuda_get_timer_value()
    assert 0.015 < v < 5.0
    lib.opcuda_reset_timer()
    assert lib.opcuda_get_timer_value() == 0.0


def test_injected_alloc_failure(lib):
    # the hook fails the next allocation on the host side, before any CUDA call
    assert lib.opb_test_fail_next_alloc(1) == 0
    assert lib.opcuda_mem_alloc(1024) == 0
    assert lib.opcuda_get_status() == -5


def test_fused_normalisation_knob_values(lib):
    """-1 restores the automatic rule, 0 and above set a size limit; neither needs a device."""
    for v in (0, 8192, -1):
        assert lib.opb_set_fused_normalisation(v) == 0
