"""Parity at the benchmark configurations' full sizes.

- Config 1: the SV lattice (48 x 128 = 6144 states, dt0 = 2^-16, 14 squarings, 15 chain
  products, 16 maturities x 128 strikes) in bf16x3 and fp16x3 against an FP64 solve of the
  same lattice, within 1e-5 at every quote.
- Config 3: the 512-lattice calibration sweep (seed 20260) in bf16x3 and fp16x3, every
  lattice against its own FP64 solve, within 1e-5.
- Config 2: the Monte Carlo on the config-0 lattice's daily kernel, 2^20 paths x 504 steps,
  payoff sums against the C oracle's over the same paths (rtol 1e-11: the same 2^20 FP64
  path payoffs added in different orders; the paths themselves are bit-exact,
  tests/test_gpu_mc.py).

The FP64 references run on the device (torch FP64 products): the oracle's
``solve_lattice_fp64`` restated with torch, pinned to the numpy oracle on a small lattice
first."""
import math
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import oracle_c as OC

pytestmark = pytest.mark.gpu


def _dense_generator(lat):
    d = lat.d
    cols = lat.cols.view(d, -1).long()
    vals = lat.vals.view(d, -1)
    L = torch.zeros(d, d, dtype=torch.float64, device=lat.device)
    mask = cols >= 0
    rows = torch.arange(d, device=lat.device).unsqueeze(1).expand_as(cols)
    L.index_put_((rows[mask], cols[mask]), vals[mask], accumulate=True)
    return L


def fp64_quotes(lat, plan, strikes, nmat, period):
    """oracle.solve_lattice_fp64 on the device: U0 = I + dt L, niter squarings and the chain
    products each renormalised in FP64, quotes at y0."""
    P = torch.eye(lat.d, dtype=torch.float64, device=lat.device) + plan.dt * _dense_generator(lat)
    for _ in range(plan.niter):
        P = P @ P
        P /= P.sum(dim=1, keepdim=True)
    K = torch.as_tensor(np.asarray(strikes, dtype=np.float64), device=lat.device)
    G = torch.clamp(lat.x.unsqueeze(1) - K.unsqueeze(0), min=0.0)
    out, Pm = [], P
    for m in range(1, nmat + 1):
        if m > 1:
            Pm = Pm @ P
            Pm /= Pm.sum(dim=1, keepdim=True)
        out.append(math.exp(-lat.rate * period * m) * (Pm[lat.y0] @ G))
    return torch.stack(out)


def test_device_fp64_reference_is_the_oracle(cuda):
    from oplib_b200.model import Lattice
    cfg = O.LVLattice(n=256, nmat=4)
    L, x = cfg.generator()
    V, _, _ = O.solve_lattice_fp64(L, x, cfg.strikes, cfg.r, cfg.period, cfg.nmat, cfg.dt0)
    lat = Lattice.local_vol(n=256, level=cfg.level, skew=cfg.skew, width=cfg.width, rate=cfg.r)
    q = fp64_quotes(lat, lat.plan(cfg.period, cfg.dt0), cfg.strikes, cfg.nmat, cfg.period).cpu().numpy()
    assert np.allclose(q, V[:, O.nearest_node(x), :], rtol=1e-11, atol=1e-13)


@pytest.mark.timeout(900)
def test_config1_sv6144_within_1e5(cuda):
    from oplib_b200 import _lib
    from oplib_b200.model import Lattice
    lat = Lattice.stoch_vol(nx=128, nv=48)
    strikes = [0.5 + j / 127.0 for j in range(128)]
    plan = lat.plan(0.25, 2.0 ** -16)
    assert plan.niter == 14
    ref = fp64_quotes(lat, plan, strikes, 16, 0.25)
    for mode in ("bf16x3", "fp16x3"):
        q, _ = lat.solve(strikes, 16, 0.25, 2.0 ** -16, mode=mode, plan=plan)
        err = float((q - ref).abs().max().item())
        print(f"config 1 {mode}: max abs error {err:.2e}")
        assert err <= 1e-5
    assert _lib.load().opb_tc_error() == 0


@pytest.mark.timeout(900)
def test_config3_sweep_every_lattice_within_1e5(cuda):
    from oplib_b200 import _lib
    from oplib_b200.model import Batch, calibration_sweep
    lats, _ = calibration_sweep(nlat=512, device=cuda)
    strikes = [0.5 + j / 31.0 for j in range(32)]
    errs = {}
    plans = None
    for mode in ("bf16x3", "fp16x3"):
        b = Batch(lats, strikes, 8, 0.25, 2.0 ** -14, mode=mode, autotune=True)
        plans = b.plans
        q = b.execute()
        torch.cuda.synchronize()
        errs[mode] = q
        del b
    for mode, q in errs.items():
        e = torch.stack([(q[i] - fp64_quotes(lat, pl, strikes, 8, 0.25)).abs().max() for i, (lat, pl) in
                         enumerate(zip(lats, plans))]).cpu().numpy()
        print(f"config 3 {mode}: max abs error {e.max():.2e} (lattice {int(e.argmax())}), median {np.median(e):.1e}")
        assert e.max() <= 1e-5
    assert _lib.load().opb_tc_error() == 0


@pytest.mark.timeout(900)
def test_config2_mc_full_size_sums(cuda):
    from oplib_b200.model import Lattice, cumulative_rows, guide_table, mc_run
    lat = Lattice.local_vol(n=512)
    Cm = cumulative_rows(lat.kernel(1 / 252, 2.0 ** -14, mode="fp32"))
    g = guide_table(Cm)
    npaths, nsteps, disc = 1 << 20, 504, math.exp(-0.03 * 2.0)
    sums, _ = mc_run(Cm, lat.y0, nsteps, 5489, npaths, guide=g, x=lat.x, disc=disc)
    torch.cuda.synchronize()
    _, ref = OC.mc_paths(Cm.cpu().numpy(), lat.y0, 5489, 0, npaths, nsteps, x=lat.x.cpu().numpy(), disc=disc,
                         want_paths=False, nthreads=os.cpu_count() or 8)
    got = sums.cpu().numpy()
    print(f"config 2: barrier {got[0] / npaths:.6f}, Asian {got[1] / npaths:.6f} per path")
    assert np.allclose(got, ref, rtol=1e-11, atol=0.0)
