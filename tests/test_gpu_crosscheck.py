"""Two independent pricers of the same contract on the same lattice: the Monte Carlo
sampler (MT19937 paths on the cumulative rows of the daily kernel, with the down-and-out
call fused in the kernel) against the backward induction on that daily kernel
(``opb_lattice_bermudan`` with a barrier and no early exercise).  The config-0 local-vol
lattice, 504 daily steps, strike 1, barrier 0.7 monitored every day."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mc_barrier_call_matches_lattice_induction(cuda):
    import torch
    from oplib_b200.model import Lattice, cumulative_rows, guide_table, mc_run
    lat = Lattice.local_vol(n=512, device=cuda)
    day, dt0, nsteps = 1.0 / 252, 2.0 ** -14, 504
    disc = math.exp(-lat.rate * nsteps * day)
    # induction: 504 products with the daily kernel, knocked out at x <= 0.7 on every day
    v_lat = float(lat.bermudan([1.0], nsteps, day, dt0, mode="fp16x3", put=False, exercise=False,
                               barrier=0.7).cpu()[0])
    # Monte Carlo on the same daily kernel: 16 batches of 2^18 paths
    P = lat.kernel(day, dt0, mode="fp16x3")
    Cm = cumulative_rows(P)
    g = guide_table(Cm)
    nb, per = 16, 1 << 18
    means = []
    for b in range(nb):
        sums, _ = mc_run(Cm, lat.y0, nsteps, 5489, per, path0=b * per, guide=g, x=lat.x, strike=1.0, barrier=0.7,
                         disc=disc)
        means.append(float(sums[0].item()) / per)
    torch.cuda.synchronize()
    mc = float(np.mean(means))
    se = float(np.std(means, ddof=1) / math.sqrt(nb))
    print(f"barrier call: lattice {v_lat:.6f}, MC {mc:.6f} +- {se:.2e}")
    assert 0.05 < v_lat < 0.5
    assert abs(mc - v_lat) < 5 * se + 1e-5, (mc, v_lat, se)
