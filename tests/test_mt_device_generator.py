"""The device MT19937 generator's two forms (oplib_b200/csrc/mt19937.cuh) compiled for the
host and checked against the oracle's MT19937, itself pinned to libstdc++ std::mt19937:
the register-cursor form up to its 623-output limit, and the cursor/state-array form that
the kernels use for longer runs across several regenerations of the state (no GPU).  The
keyed seeding (a key added to mt[1]) of the stream-seed-table Monte Carlo is checked against
the oracle's two restatements of it (C and numpy)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from oracle import oracle_c as OC

ROOT = Path(__file__).resolve().parents[1]
HEADER_DIR = ROOT / "oplib_b200" / "csrc"

DRIVER = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include "mt19937.cuh"

int main(int argc, char **argv) {
    const unsigned seed = (unsigned)strtoul(argv[1], 0, 10);
    const int n = atoi(argv[2]);
    const bool any = strcmp(argv[3], "any") == 0;
    const unsigned key1 = argc > 4 ? (unsigned)strtoul(argv[4], 0, 10) : 0u;
    std::vector<uint32_t> out(n, 0u);
    int calls = 0;
    auto f = [&](int k, uint32_t x) { out[k] = x; calls++; };
    if (any) opb::mt19937_stream<true>(seed, key1, n, f);
    else opb::mt19937_stream<false>(seed, key1, n, f);
    if (calls != n) return 2;
    fwrite(out.data(), 4, n, stdout);
    return 0;
}
"""


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("mtgen")
    src = d / "mtgen.cpp"
    src.write_text(DRIVER)
    binary = d / "mtgen"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Wno-unknown-pragmas", "-I", str(HEADER_DIR),
                    str(src), "-o", str(binary)], check=True)
    return binary


def run(exe, seed, n, form, key1=0):
    out = subprocess.run([str(exe), str(seed), str(n), form, str(key1)], capture_output=True, check=True).stdout
    return np.frombuffer(out, dtype=np.uint32)


@pytest.mark.parametrize("seed", [0, 1, 5489, 20260, 4294967295])
def test_cursor_form_matches_mt19937(exe, seed):
    for n in (1, 226, 227, 453, 454, 623):
        assert np.array_equal(run(exe, seed, n, "first"), OC.mt_outputs(seed, n)), (seed, n)


@pytest.mark.parametrize("seed", [0, 1, 5489, 20260, 4294967295])
def test_state_array_form_matches_mt19937(exe, seed):
    # 3 * 624 + 5 outputs: three full regenerations and the words on either side of each
    n = 3 * 624 + 5
    got = run(exe, seed, n, "any")
    assert np.array_equal(got, OC.mt_outputs(seed, n)), seed
    assert np.array_equal(got[:623], run(exe, seed, 623, "first"))
    for m in (1, 622, 623, 624, 625, 1247, 1248, 1249):  # each side of the cursor/array hand-over
        assert np.array_equal(run(exe, seed, m, "any"), got[:m]), (seed, m)


def test_state_array_form_reaches_the_standard_value(exe):
    # C++11 [rand.predef]: the 10000th output of mt19937 seeded 5489 is 4123659995
    assert int(run(exe, 5489, 10000, "any")[-1]) == 4123659995


def test_zero_outputs(exe):
    assert run(exe, 7, 0, "any").size == 0
    assert run(exe, 7, 0, "first").size == 0


def test_random_seeds_and_lengths(exe):
    rng = np.random.default_rng(20260)
    for seed, n in zip(rng.integers(0, 2**32, 40), rng.integers(0, 2600, 40)):
        seed, n = int(seed), int(n)
        ref = OC.mt_outputs(seed, n) if n else np.empty(0, dtype=np.uint32)
        assert np.array_equal(run(exe, seed, n, "any"), ref), (seed, n)
        m = min(n, 623)
        assert np.array_equal(run(exe, seed, m, "first"), ref[:m]), (seed, m)


@pytest.mark.parametrize("seed,key1", [(0, 1), (5489, 1), (7, 123456), (4294967295, 4294967295), (99, 4095)])
def test_keyed_forms_match_the_oracle(exe, seed, key1):
    n = 2 * 624 + 3
    ref = OC.mt_outputs_keyed(seed, key1, n)
    assert np.array_equal(ref, O.mt19937_outputs(np.array([seed]), n, np.array([key1]))[0])
    assert not np.array_equal(ref[:8], OC.mt_outputs(seed, 8))  # the key changes the stream
    assert np.array_equal(run(exe, seed, n, "any", key1), ref)
    for m in (1, 226, 227, 453, 454, 623):
        assert np.array_equal(run(exe, seed, m, "first", key1), ref[:m]), (seed, key1, m)
