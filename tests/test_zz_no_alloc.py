"""The allocation-free Monte Carlo entry point, checked against the regular one.

opb_mc_mt19937_noalloc exists for callers that must not let the library allocate device
memory -- a host framework that owns the device-memory budget, or a loop that cannot
afford cudaMalloc's implicit synchronisation.  It keeps its payoff partial sums in a
fixed device array inside the library instead of a caller-provided scratch buffer.  This
test calls it through the C ABI twice in a row (the second call with a smaller grid, so
stale partials from the first call must not leak into it) and compares every output with
opb_mc_mt19937 on the same inputs: state paths bit-exact, payoff sums within rtol 1e-12
(the tolerance the other Monte Carlo tests use).  It is collected last so that a run
that stops at the first failure has already run every other test, and it does its own
set-up so that it passes alone in a fresh process as well.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_mc_matches_regular_entry_point_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oplib_b200 import _lib
    from oplib_b200.model import Lattice, bind_stream, cumulative_rows, guide_table

    lib = _lib.load()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    lat = Lattice.local_vol(n=512, device=dev)
    P = lat.kernel(1 / 252, 2.0 ** -14, mode="fp32")
    Cm = cumulative_rows(P)
    g = guide_table(Cm, 64)
    bind_stream(dev)
    d, nsteps, disc = 512, 504, math.exp(-0.03 * 2.0)

    for call, (npaths, seed, path0) in enumerate([(1 << 18, 5489, 0), (3000, 77, 123456)]):
        # regular entry point with a caller-provided scratch buffer
        nblk = lib.opb_mc_scratch_blocks(npaths)
        scratch = torch.empty(2 * nblk, dtype=torch.float64, device=dev)
        sums_ref = torch.empty(2, dtype=torch.float64, device=dev)
        paths_ref = torch.empty(nsteps, npaths, dtype=torch.int16, device=dev)
        assert lib.opb_mc_mt19937(Cm.data_ptr(), d, 1, g.data_ptr(), 64, d, lat.y0, nsteps, seed, path0, npaths,
                                  paths_ref.data_ptr(), lat.x.data_ptr(), 1.0, 0.7, disc, scratch.data_ptr(),
                                  sums_ref.data_ptr()) == 0
        # allocation-free entry point: same inputs and outputs, no scratch argument
        sums = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
        paths = torch.full((nsteps, npaths), -1, dtype=torch.int16, device=dev)
        assert lib.opb_mc_mt19937_noalloc(Cm.data_ptr(), d, 1, g.data_ptr(), 64, d, lat.y0, nsteps, seed, path0,
                                          npaths, paths.data_ptr(), lat.x.data_ptr(), 1.0, 0.7, disc,
                                          sums.data_ptr()) == 0, f"call {call}"
        torch.cuda.synchronize()
        assert torch.equal(paths, paths_ref), f"call {call}: state paths differ"
        s, sr = sums.cpu().numpy(), sums_ref.cpu().numpy()
        assert np.all(np.isfinite(s)) and np.allclose(s, sr, rtol=1e-12, atol=0.0), (call, s, sr)

    # once set up, a call allocates no device memory: the device's free memory is the same
    # before and after it (torch's caching allocator idle in between)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    assert lib.opb_mc_mt19937_noalloc(Cm.data_ptr(), d, 1, g.data_ptr(), 64, d, lat.y0, nsteps, 5489, 0, npaths,
                                      paths.data_ptr(), lat.x.data_ptr(), 1.0, 0.7, disc, sums.data_ptr()) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0, (free0, free1)
