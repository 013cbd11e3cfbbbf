"""The device-side Monte Carlo evaluator (a cashflow table per step and state, with optional
discrete knock-out) against the oracle's evaluator on the oracle's own paths.

The reference values paths on the host: opcuda_mc1f copies the int16 states back and the
model calls its evaluator on them (oplib/opmodel/models/CModel Device.cs:343-364).  Here the
same paths are valued inside the sampling kernel.  Per-path values are sums in step order in
FP64 on both sides, so they agree bit for bit; the all-path sums go through a block
reduction, so they agree to rtol 1e-12."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import oracle_c as OC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rows(cuda):
    from oplib_b200.model import Lattice, cumulative_rows, guide_table
    lat = Lattice.local_vol(n=512)
    P = lat.kernel(1 / 252, 2.0 ** -14, mode="fp32")
    Cm = cumulative_rows(P)
    g = guide_table(Cm, 64)
    torch.cuda.synchronize()
    return lat, Cm, g


def _eval(lib, lat, Cm, g, nsteps, seed, path0, npaths, cf, ko, cuda):
    d = lat.d
    dcf = torch.from_numpy(np.ascontiguousarray(cf)).to(cuda)
    dko = None if ko is None else torch.from_numpy(np.ascontiguousarray(ko, dtype=np.uint8)).to(cuda)
    pv = torch.empty(npaths, dtype=torch.float64, device=cuda)
    scratch = torch.empty(2 * lib.opb_mc_scratch_blocks(npaths), dtype=torch.float64, device=cuda)
    sums = torch.empty(2, dtype=torch.float64, device=cuda)
    assert lib.opb_mc_mt19937_eval(Cm.data_ptr(), d, 1, g.data_ptr(), 64, d, lat.y0, nsteps, seed, path0, npaths,
                                   None, dcf.data_ptr(), None if dko is None else dko.data_ptr(), pv.data_ptr(),
                                   scratch.data_ptr(), sums.data_ptr()) == 0
    torch.cuda.synchronize()
    return pv.cpu().numpy(), sums.cpu().numpy()


def test_vanilla_evaluator_on_the_device(rows, cuda):
    """The reference's vanilla evaluator as a table: (x - K)^+ discounted at the last step."""
    from oplib_b200 import _lib
    lib = _lib.load()
    lat, Cm, g = rows
    d, nsteps, npaths, K = lat.d, 252, 8192, 1.05
    x = lat.x.cpu().numpy()
    cf = np.zeros((nsteps, d))
    cf[-1] = math.exp(-0.03) * np.maximum(x - K, 0.0)
    pv, sums = _eval(lib, lat, Cm, g, nsteps, 5489, 0, npaths, cf, None, cuda)
    paths, _ = OC.mc_paths(Cm.cpu().numpy(), lat.y0, 5489, 0, npaths, nsteps)
    ref = O.mc_cashflow_values(paths, cf)
    assert np.array_equal(pv, ref)
    assert np.allclose(sums, [ref.sum(), (ref * ref).sum()], rtol=1e-12, atol=0.0)


def test_knockout_table_reproduces_the_fused_barrier_payoff(rows, cuda):
    """Knock-out where x <= 0.7 at every step and the call's cashflow at the last step are the
    fused down-and-out call: the same path values, so the same payoff sum."""
    from oplib_b200 import _lib
    lib = _lib.load()
    lat, Cm, g = rows
    d, nsteps, npaths = lat.d, 504, 1 << 16
    x = lat.x.cpu().numpy()
    disc = math.exp(-0.03 * 2.0)
    cf = np.zeros((nsteps, d))
    cf[-1] = disc * np.maximum(x - 1.0, 0.0)
    ko = np.broadcast_to(x <= 0.7, (nsteps, d)).astype(np.uint8)
    pv, sums = _eval(lib, lat, Cm, g, nsteps, 77, 1000, npaths, cf, ko, cuda)
    scratch = torch.empty(2 * lib.opb_mc_scratch_blocks(npaths), dtype=torch.float64, device=cuda)
    fused = torch.empty(2, dtype=torch.float64, device=cuda)
    assert lib.opb_mc_mt19937(Cm.data_ptr(), d, 1, g.data_ptr(), 64, d, lat.y0, nsteps, 77, 1000, npaths, None,
                              lat.x.data_ptr(), 1.0, 0.7, disc, scratch.data_ptr(), fused.data_ptr()) == 0
    torch.cuda.synchronize()
    assert np.allclose(sums[0], fused.cpu().numpy()[0], rtol=1e-12, atol=0.0)
    assert 0.0 < sums[0] / npaths < 0.5


@pytest.mark.parametrize("nsteps", [60, 700])
def test_cashflows_with_knockout_bit_exact(rows, cuda, nsteps):
    """Random cashflows at every step and a random knock-out set, on the register generator and
    past its 623 steps on the state-array one."""
    from oplib_b200 import _lib
    lib = _lib.load()
    lat, Cm, g = rows
    d, npaths = lat.d, 3000
    rng = np.random.default_rng(nsteps)
    cf = rng.standard_normal((nsteps, d))
    ko = (rng.random((nsteps, d)) < 0.002).astype(np.uint8)
    pv, sums = _eval(lib, lat, Cm, g, nsteps, 4321, 55, npaths, cf, ko, cuda)
    paths, _ = OC.mc_paths(Cm.cpu().numpy(), lat.y0, 4321, 55, npaths, nsteps)
    ref = O.mc_cashflow_values(paths, cf, ko)
    assert np.array_equal(pv, ref)
    assert np.allclose(sums, [ref.sum(), (ref * ref).sum()], rtol=1e-12, atol=1e-12)
    assert np.any(ref != O.mc_cashflow_values(paths, cf))  # some paths were knocked out


def test_opcuda_mc1f_eval_matches_mc1f_with_host_evaluator(cuda):
    """The drop-in pair opcuda_mc1f + host evaluator against opcuda_mc1f_eval: the same
    results per scenario over two batches that continue the same streams."""
    from oplib_b200 import _lib
    lib = _lib.load()
    cfg = O.LVLattice(n=128)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 52, cfg.dt0)
    Cr = O.cumrows_f32(O.square(O.ek(L, dt), niter))
    d, nscen, nk, y0 = 128, 4096, 40, O.nearest_node(x)
    ccm = torch.from_numpy(np.asfortranarray(Cr).ravel(order="K").copy()).to(cuda)
    mk = torch.zeros(nk, dtype=torch.int32, device=cuda)
    cf = np.zeros((nk, d))
    cf[-1] = np.maximum(x - 1.0, 0.0)  # the reference's VanillaPayoffEvaluator, strike 1
    dcf = torch.from_numpy(cf).to(cuda)
    seed = np.random.default_rng(99).integers(0, 2**31 - 1, 4096).astype(np.uint32)
    st_a = torch.zeros(lib.opcuda_mc_status_sz(), dtype=torch.int32, device=cuda)
    st_b = torch.zeros_like(st_a)
    assert lib.opcuda_mc_setseed(seed.ctypes.data, st_a.data_ptr()) == 0
    assert lib.opcuda_mc_setseed(seed.ctypes.data, st_b.data_ptr()) == 0
    yd = torch.empty(nscen * nk, dtype=torch.int16, device=cuda)
    res = torch.empty(nscen, dtype=torch.float64, device=cuda)
    for _ in range(2):
        yh = np.empty(nscen * nk, dtype=np.int16)
        assert lib.opcuda_mc1f(st_a.data_ptr(), y0, yd.data_ptr(), nscen, nk, d, ccm.data_ptr(), mk.data_ptr(),
                               yh.ctypes.data) == 0
        host = O.mc_cashflow_values(yh.reshape(nk, nscen).T, cf)
        assert lib.opcuda_mc1f_eval(st_b.data_ptr(), y0, 0, nscen, nk, d, ccm.data_ptr(), mk.data_ptr(),
                                    dcf.data_ptr(), 0, res.data_ptr()) == 0
        assert np.array_equal(res.cpu().numpy(), host)
    assert torch.equal(st_a, st_b)
