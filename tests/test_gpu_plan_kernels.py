"""Monte Carlo plans whose steps span generator dates, executed on the device.

The planner (oplib_b200/plan.py, the reference's make_mc_plan) gives a step that contains a
generator date a list of elementary kernels under different generators; ``mc_plan_kernels``
squares each elementary kernel under its own generator and chains each step's factors on
the device (``opb_chain_kernels``).  Checked against the oracle's FP64 execution of the same
plan, and through the Monte Carlo: opcuda_mc1f with the plan's per-step kernel index m_k
draws paths bit-exact with the oracle's sampler on the same FP32 cumulative rows."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import oracle_c as OC

pytestmark = pytest.mark.gpu

LEVELS = (0.18, 0.3, 0.24)  # one local-vol generator per interval (t_i)


@pytest.fixture(scope="module")
def plan_and_kernels(cuda):
    from oplib_b200.model import Lattice, mc_plan_kernels
    from oplib_b200.plan import make_mc_plan
    n = 256
    lats = [Lattice.local_vol(n=n, level=lv, skew=0.1 * (i - 1), width=0.5, rate=0.02) for i, lv in enumerate(LEVELS)]
    t_i, t_k = [45, 100, 150], [30, 60, 91, 120, 150]
    plan = make_mc_plan(t_k, t_i, 1, [lat.maxdiag() for lat in lats])
    K = mc_plan_kernels(plan, lats, mode="fp32")
    torch.cuda.synchronize()
    x = O.log_grid(n)
    gens = [O.lv_generator_fast(x, 0.02 * x, O.lv_sigma(x, lv, 0.1 * (i - 1), 0.5) * x) for i, lv in enumerate(LEVELS)]
    ref = O.mc_plan_kernels(plan, gens)
    return plan, lats, K, ref


def test_plan_has_steps_across_generator_dates(plan_and_kernels):
    plan, _, _, _ = plan_and_kernels
    assert max(len(f) for f in plan.jfactor_ms) >= 2
    assert len({plan.i_j[j] for f in plan.jfactor_ms for j in f}) == 3


def test_step_kernels_match_the_fp64_plan(plan_and_kernels):
    plan, _, K, ref = plan_and_kernels
    got = K.double().cpu().numpy()
    assert got.shape == (plan.nm,) + ref[0].shape
    for m in range(plan.nm):
        assert np.abs(got[m] - ref[m]).max() < 5e-6, m
        assert np.allclose(got[m].sum(axis=1), 1.0, atol=1e-6)


def test_mc1f_over_the_plan_bit_exact(plan_and_kernels, cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    plan, lats, K, _ = plan_and_kernels
    d = K.shape[1]
    nm, nk, nscen, y0, seed = plan.nm, plan.nk, 4096, lats[0].y0, 31337
    # column-major kernels (element (source y1, target y2) at y1 + d*y2) -> cumulative rows
    kcm = K.transpose(1, 2).contiguous()
    ccm = torch.empty_like(kcm)
    assert lib.opcuda_sck(d, nm, kcm.data_ptr(), ccm.data_ptr()) == 0
    mk = torch.tensor(plan.m_k, dtype=torch.int32, device=cuda)
    st = torch.zeros(lib.opcuda_mc_status_sz(), dtype=torch.int32, device=cuda)
    s = (seed + np.arange(4096)).astype(np.uint32)  # paths 0 .. 4095: init_genrand(seed + p)
    assert lib.opcuda_mc_setseed(s.ctypes.data, st.data_ptr()) == 0
    yd = torch.empty(nscen * nk, dtype=torch.int16, device=cuda)
    yh = np.empty(nscen * nk, dtype=np.int16)
    assert lib.opcuda_mc1f(st.data_ptr(), y0, yd.data_ptr(), nscen, nk, d, ccm.data_ptr(), mk.data_ptr(),
                           yh.ctypes.data) == 0
    paths = yh.reshape(nk, nscen).T
    rows = ccm.cpu().numpy().reshape(nm, d, d).transpose(0, 2, 1)  # [m][source][target]
    for p in (0, 1, 777, nscen - 1):
        u = O.uniform_f32(OC.mt_outputs(seed + p, nk))
        y = y0
        for k in range(nk):
            y = int(O.sample_next(rows[plan.m_k[k]][y][None, :], u[k:k + 1])[0])
            assert paths[p, k] == y, (p, k)
