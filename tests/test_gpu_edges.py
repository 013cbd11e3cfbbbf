"""Edge cases of the device path against the oracle: empty and single inputs, the step
counts on either side of the register-only generator's limit, ragged sizes, degenerate
guide tables and pricing grids, and the rejections that guard the supported range."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import oracle_c as OC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rows(cuda):
    from oplib_b200.model import Lattice, cumulative_rows
    lat = Lattice.local_vol(n=256)
    P = lat.kernel(1 / 252, 2.0 ** -14, mode="fp32")
    Cm = cumulative_rows(P)
    torch.cuda.synchronize()
    return lat, Cm


def test_mc_no_paths_gives_zero_sums(rows):
    from oplib_b200.model import mc_run
    lat, Cm = rows
    sums, paths = mc_run(Cm, lat.y0, 10, 1, 0, x=lat.x, want_paths=True)
    torch.cuda.synchronize()
    assert paths.numel() == 0
    assert sums.cpu().tolist() == [0.0, 0.0]


def test_mc_single_path_longest_run_bit_exact(rows):
    """One path of 623 steps, the longest run of the register-only generator (a fresh
    MT19937 state serves 623 outputs without a second regeneration)."""
    from oplib_b200.model import mc_run
    lat, Cm = rows
    disc = math.exp(-0.03)
    sums, paths = mc_run(Cm, lat.y0, 623, 4294967295, 1, x=lat.x, disc=disc, want_paths=True)
    torch.cuda.synchronize()
    ref_paths, ref_sums = OC.mc_paths(Cm.cpu().numpy(), lat.y0, 4294967295, 0, 1, 623, x=lat.x.cpu().numpy(),
                                      disc=disc)
    assert np.array_equal(paths.cpu().numpy().T, ref_paths)
    assert np.allclose(sums.cpu().numpy(), ref_sums, rtol=1e-12, atol=0)


@pytest.mark.parametrize("nb", [1, 1024])
def test_mc_ragged_paths_with_extreme_guide_tables(rows, nb):
    """1000 paths (not a multiple of the block size) through a one-bucket guide table (the
    whole row) and a 1024-bucket one (more buckets than states)."""
    from oplib_b200.model import guide_table, mc_run
    lat, Cm = rows
    g = guide_table(Cm, nb)
    _, paths = mc_run(Cm, lat.y0, 50, 77, 1000, guide=g, nb=nb, want_paths=True)
    torch.cuda.synchronize()
    ref_paths, _ = OC.mc_paths(Cm.cpu().numpy(), lat.y0, 77, 0, 1000, 50)
    assert np.array_equal(paths.cpu().numpy().T, ref_paths)


@pytest.mark.parametrize("nsteps,use_guide", [(624, False), (1400, True)])
def test_mc_long_paths_bit_exact(rows, nsteps, use_guide):
    """Runs past the register-only generator (the per-thread state-array form): 624 steps
    (the first output of the second regeneration) and 1400 (two regenerations), 300 paths
    whose seeds wrap past 2^32, with the fused payoffs."""
    from oplib_b200.model import guide_table, mc_run
    lat, Cm = rows
    g = guide_table(Cm, 64) if use_guide else None
    disc = math.exp(-0.03 * nsteps / 252)
    seed = 4294967000
    sums, paths = mc_run(Cm, lat.y0, nsteps, seed, 300, guide=g, x=lat.x, disc=disc, want_paths=True)
    torch.cuda.synchronize()
    ref_paths, ref_sums = OC.mc_paths(Cm.cpu().numpy(), lat.y0, seed, 0, 300, nsteps, x=lat.x.cpu().numpy(),
                                      disc=disc)
    assert np.array_equal(paths.cpu().numpy().T, ref_paths)
    assert np.allclose(sums.cpu().numpy(), ref_sums, rtol=1e-12, atol=0)


def test_mc_rejects_out_of_range_start_state(rows):
    from oplib_b200 import _lib
    lat, Cm = rows
    d = Cm.shape[1]
    r = _lib.load().opb_mc_mt19937(Cm.data_ptr(), d, 1, None, 0, d, d, 10, 1, 0, 16, None, None, 1.0, 0.7, 1.0,
                                   None, None)
    assert r == -1


@pytest.mark.parametrize("d", [1, 31])
def test_cumulative_rows_tiny_and_odd(cuda, d):
    from oplib_b200.model import cumulative_rows
    rng = np.random.default_rng(d)
    P = rng.random((5, d)).astype(np.float32)
    P /= P.sum(axis=1, keepdims=True)
    got = cumulative_rows(torch.from_numpy(P).to(cuda)).cpu().numpy()
    assert np.array_equal(got, OC.sck(P))
    assert np.all(got[:, -1] == np.float32(1.0))


@pytest.mark.parametrize("mode", ["bf16x3", "fp16x3", "fp32"])
def test_one_strike_one_maturity(cuda, mode):
    """The smallest pricing grid (nK = 1, one maturity) on the config-0 lattice."""
    from oplib_b200.model import Lattice
    cfg = O.LVLattice(n=512, nmat=1)
    L, x = cfg.generator()
    V, _, _ = O.solve_lattice_fp64(L, x, np.array([1.0]), cfg.r, cfg.period, 1, cfg.dt0)
    lat = Lattice.local_vol(n=512, level=cfg.level, skew=cfg.skew, width=cfg.width, rate=cfg.r)
    q, _ = lat.solve([1.0], 1, cfg.period, cfg.dt0, mode=mode)
    assert q.shape == (1, 1)
    assert abs(q.item() - V[0, O.nearest_node(x), 0]) < 1e-5


def test_fp32_path_on_a_size_not_multiple_of_64(cuda):
    """The FP32 path takes any size (here 100 states): quotes and all-state values against
    the FP64 oracle."""
    from oplib_b200.model import Lattice
    cfg = O.LVLattice(n=100, nmat=3)
    L, x = cfg.generator()
    K = cfg.strikes[::8]
    V, _, _ = O.solve_lattice_fp64(L, x, K, cfg.r, cfg.period, cfg.nmat, cfg.dt0)
    lat = Lattice.local_vol(n=100, level=cfg.level, skew=cfg.skew, width=cfg.width, rate=cfg.r)
    q, Vall = lat.solve(K, cfg.nmat, cfg.period, cfg.dt0, mode="fp32", all_states=True)
    assert np.abs(q.cpu().numpy() - V[:, O.nearest_node(x), :]).max() < 1e-5
    assert np.abs(Vall.cpu().numpy() - V).max() < 1e-5 * max(1.0, np.abs(V).max())


@pytest.mark.parametrize("mode", ["bf16x3", "fp16x3"])
@pytest.mark.parametrize("n", [100, 300])
def test_split_modes_on_sizes_off_the_tile_grid(cuda, mode, n):
    """The split modes solve a lattice whose size is no multiple of 128 as one padded with
    absorbing states: quotes, all-state values and the period kernel against the FP64
    oracle, and a Bermudan put against the oracle's induction."""
    from oplib_b200.model import Lattice
    cfg = O.LVLattice(n=n, nmat=3)
    L, x = cfg.generator()
    K = cfg.strikes[::8]
    V, niter, dt = O.solve_lattice_fp64(L, x, K, cfg.r, cfg.period, cfg.nmat, cfg.dt0)
    lat = Lattice.local_vol(n=n, level=cfg.level, skew=cfg.skew, width=cfg.width, rate=cfg.r)
    q, Vall = lat.solve(K, cfg.nmat, cfg.period, cfg.dt0, mode=mode, all_states=True)
    P = lat.kernel(cfg.period, cfg.dt0, mode=mode)
    torch.cuda.synchronize()
    assert q.shape == (cfg.nmat, K.size) and Vall.shape == (cfg.nmat, n, K.size) and P.shape == (n, n)
    assert np.abs(q.cpu().numpy() - V[:, O.nearest_node(x), :]).max() < 1e-5
    assert np.abs(Vall.cpu().numpy() - V).max() < 5e-5 * max(1.0, np.abs(V).max())
    P1 = O.square(O.ek(L, dt), niter, renorm=True)
    assert np.abs(P.cpu().numpy() - P1).max() < 2e-5
    assert np.allclose(P.double().sum(1).cpu().numpy(), 1.0, atol=1e-6)
    Vb = O.bermudan_fp64(L, x, K, cfg.r, cfg.period, cfg.nmat, cfg.dt0, put=True)
    qb = lat.bermudan(K, cfg.nmat, cfg.period, cfg.dt0, put=True, mode=mode)
    assert np.abs(qb.cpu().numpy() - Vb[O.nearest_node(x)]).max() < 1e-5


def test_batch_of_one_lattice_matches_its_single_solve(cuda, fused_single):
    from oplib_b200.model import Batch, Lattice
    lat = Lattice.local_vol(n=384, level=0.25, skew=-0.1, width=0.6, rate=0.02, floor=0.01)
    K = np.linspace(0.8, 1.2, 8)
    single, _ = lat.solve(K, 3, 0.25, 2.0 ** -14, mode="fp16x3")
    bt = Batch([lat], K, 3, 0.25, 2.0 ** -14, mode="fp16x3")
    q = bt.execute()
    assert q.shape == (1, 3, 8)
    assert (q[0] - single).abs().max().item() < 1e-6
