"""The reference's integration test (tests/bstest/Program.cs:11-37, OPPricer.cs:67-148)
through this library's drop-in entry points, in the order the reference's device branch
calls them: the FP32 generator from S1DGrid.pregen's inverses (opcuda_sglvg), I + dt L
(opcuda_sek), niter squarings through pointer tables (opcuda_ssqmm), cumulative rows
(opcuda_sck), seeding and the Monte Carlo with its blocking copy of the states
(opcuda_mc_setseed, opcuda_mc1f), then the vanilla payoff and discounting on the host."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_bstest_through_the_opcuda_drop_ins(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    S, K, r, sig = 100.0, 100.0, 0.05, 0.25
    T, dt0 = 365 / 365.25, 1 / 365.25
    x, y0 = O.pivot_grid(256, O.BSTEST_PIVOTS, O.BSTEST_SPACINGS, S)
    d = x.size
    L64 = O.lv_generator(x, r * x, sig * x)
    niter, dt = O.plan_niter(L64, T, dt0)  # the plan reads the host generator

    inv = O.lv_invm(x)
    invm = torch.from_numpy(
        np.stack([inv[:, 0, 0], inv[:, 1, 0], inv[:, 0, 1], inv[:, 1, 1]], axis=1).ravel().astype(np.float32)).to(cuda)
    pars = torch.from_numpy(np.concatenate([r * x, sig * x]).astype(np.float32)).to(cuda)
    gen = torch.empty(d * d, device=cuda)
    assert lib.opcuda_sglvg(gen.data_ptr(), 1, d, invm.data_ptr(), pars.data_ptr()) == 0
    bufs = [torch.empty(d * d, device=cuda), torch.empty(d * d, device=cuda)]
    assert lib.opcuda_sek(d, gen.data_ptr(), float(dt), bufs[0].data_ptr()) == 0
    tabs = [torch.tensor([b.data_ptr()], dtype=torch.int64, device=cuda) for b in bufs]
    for level in range(niter):  # ping-pong U <- U.U
        src, dst = tabs[level % 2], tabs[(level + 1) % 2]
        assert lib.opcuda_ssqmm(d, 1, src.data_ptr(), src.data_ptr(), dst.data_ptr()) == 0
    P = bufs[niter % 2]
    Cc = torch.empty(d * d, device=cuda)
    assert lib.opcuda_sck(d, 1, P.data_ptr(), Cc.data_ptr()) == 0

    nscen, nbatch = 4096 * 25, 12
    st = torch.zeros(lib.opcuda_mc_status_sz(), dtype=torch.int32, device=cuda)
    seed = np.random.default_rng(4242).integers(0, 2**31 - 1, lib.opcuda_mc_nrng()).astype(np.uint32)
    assert lib.opcuda_mc_setseed(seed.ctypes.data, st.data_ptr()) == 0
    mk = torch.zeros(1, dtype=torch.int32, device=cuda)
    yd = torch.empty(nscen, dtype=torch.int16, device=cuda)
    yh = np.empty(nscen, dtype=np.int16)
    s1 = s2 = 0.0
    for _ in range(nbatch):
        assert lib.opcuda_mc1f(st.data_ptr(), y0, yd.data_ptr(), nscen, 1, d, Cc.data_ptr(), mk.data_ptr(),
                               yh.ctypes.data) == 0
        pay = np.maximum(x[yh] - K, 0.0)  # VanillaPayoffEvaluator
        s1 += pay.sum()
        s2 += (pay * pay).sum()
    torch.cuda.synchronize()
    n = nscen * nbatch
    disc = math.exp(-r * T)
    mean = s1 / n
    se = disc * math.sqrt((s2 / n - mean * mean) / n)
    price_mc = disc * mean
    P32 = P.cpu().numpy().reshape(d, d).T.astype(np.float64)  # column-major -> [source, target]
    price_lattice32 = disc * (P32[y0] @ np.maximum(x - K, 0.0))
    price_lattice64 = disc * (O.square(O.ek(L64, dt), niter)[y0] @ np.maximum(x - K, 0.0))
    assert abs(price_mc - price_lattice32) < 4 * se, (price_mc, price_lattice32, se)
    assert abs(price_lattice32 - price_lattice64) < 0.01, (price_lattice32, price_lattice64)
    assert abs(price_lattice64 - float(O.bs_call(S, K, r, sig, T))) < 5e-3
