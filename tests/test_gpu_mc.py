"""GPU parity of the Monte Carlo path: MT19937 streams, cumulative rows and sampled
state paths are bit-exact against the C oracle given identical FP32 rows."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import oracle_c as OC

pytestmark = pytest.mark.gpu


def test_mt19937_streams_bit_exact(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    # 623: the register-only generator's longest stream; 2000: the state-array form
    for seed, n in [(5489, 623), (0, 504), (4294967200, 300), (20260, 17), (5489, 2000), (4294967200, 624)]:
        ns = 300
        out = torch.empty(ns * n, dtype=torch.int32, device=cuda)
        assert lib.opb_mt19937_raw(seed, ns, n, out.data_ptr()) == 0
        got = out.cpu().numpy().view(np.uint32).reshape(ns, n)
        for s in [0, 1, 77, ns - 1]:
            assert np.array_equal(got[s], OC.mt_outputs((seed + s) & 0xFFFFFFFF, n)), (seed, s)


def test_sck_bit_exact(cuda):
    from oplib_b200.model import cumulative_rows
    rng = np.random.default_rng(11)
    for d, rows in [(512, 512), (100, 37), (33, 70)]:
        P = rng.random((rows, d)).astype(np.float32) ** 4
        P[0, 3] = -1e-12
        P /= P.sum(axis=1, keepdims=True)
        Cg = cumulative_rows(torch.from_numpy(P).to(cuda)).cpu().numpy()
        assert np.array_equal(Cg, OC.sck(P)), d


def test_opcuda_sck_column_major_bit_exact(cuda):
    from oplib_b200 import _lib
    rng = np.random.default_rng(12)
    d, nm = 96, 2
    P = (rng.random((nm, d, d)) ** 3).astype(np.float32)
    P /= P.sum(axis=2, keepdims=True)
    cm = np.concatenate([np.asfortranarray(p).ravel(order="K") for p in P])
    dP = torch.from_numpy(cm).to(cuda)
    dC = torch.empty_like(dP)
    assert _lib.load().opcuda_sck(d, nm, dP.data_ptr(), dC.data_ptr()) == 0
    got = dC.cpu().numpy().reshape(nm, d, d).transpose(0, 2, 1)
    for m in range(nm):
        assert np.array_equal(got[m], OC.sck(P[m]))


@pytest.fixture(scope="module")
def step_rows(cuda):
    """Config-2 step kernel (dt = 1/252 via 7 squarings) from the device, its cumulative
    rows and guide table."""
    from oplib_b200.model import Lattice, cumulative_rows, guide_table
    lat = Lattice.local_vol(n=512)
    P = lat.kernel(1 / 252, 2.0 ** -14, mode="fp32")
    Cm = cumulative_rows(P)
    g = guide_table(Cm, 64)
    torch.cuda.synchronize()
    return lat, P, Cm, g


def test_guide_brackets_contain_answer(step_rows):
    lat, P, Cm, g = step_rows
    C = Cm.cpu().numpy()
    G = g.cpu().numpy().view(np.uint32).reshape(512, 64)
    rng = np.random.default_rng(0)
    for y in rng.integers(0, 512, 40):
        u = O.uniform_f32(rng.integers(0, 2**32, 2000, dtype=np.uint64).astype(np.uint32))
        ans = O.sample_next(np.broadcast_to(C[y], (u.size, 512)), u)
        b = np.minimum((u * np.float32(64)).astype(np.int64), 63)
        lb, ub = G[y, b] & 0xFFFF, G[y, b] >> 16
        assert np.all((lb <= ans) & (ans <= ub))


@pytest.mark.parametrize("use_guide", [False, True])
def test_mc_paths_bit_exact(step_rows, use_guide):
    """4096 paths x 504 steps of the config-2 workload: every state equal to the oracle's."""
    from oplib_b200.model import mc_run
    lat, P, Cm, g = step_rows
    x = lat.x
    disc = math.exp(-0.03 * 2.0)
    sums, paths = mc_run(Cm, lat.y0, 504, 5489, 4096, guide=g if use_guide else None, x=x, disc=disc,
                         want_paths=True)
    torch.cuda.synchronize()
    ref_paths, ref_sums = OC.mc_paths(Cm.cpu().numpy(), lat.y0, 5489, 0, 4096, 504, x=x.cpu().numpy(), disc=disc)
    got = paths.cpu().numpy().T  # reference layout y[p + npaths*k] -> [path, step]
    assert np.array_equal(got, ref_paths)
    assert np.allclose(sums.cpu().numpy(), ref_sums, rtol=1e-12)


def test_mc_path_offsets_are_placement_independent(step_rows):
    """Paths are a function of (seed, path id) only: a sub-range run reproduces the same
    states, which is what lets path ranges shard across GPUs."""
    from oplib_b200.model import mc_run
    lat, P, Cm, g = step_rows
    _, full = mc_run(Cm, lat.y0, 100, 99, 2048, guide=g, want_paths=True)
    _, part = mc_run(Cm, lat.y0, 100, 99, 512, path0=1000, guide=g, want_paths=True)
    assert torch.equal(full[:, 1000:1512], part)


def test_mc_golden_fixture(cuda):
    from pathlib import Path

    from oplib_b200.model import mc_run
    gold = np.load(Path(__file__).resolve().parent / "golden" / "mc_small.npz")
    Cm = torch.from_numpy(gold["C"]).to(cuda)
    sums, paths = mc_run(Cm, int(gold["y0"]), gold["paths"].shape[1], int(gold["seed"]), gold["paths"].shape[0],
                         x=torch.from_numpy(gold["x"]).to(cuda), disc=float(gold["disc"]), want_paths=True)
    assert np.array_equal(paths.cpu().numpy().T, gold["paths"])
    assert np.allclose(sums.cpu().numpy(), gold["sums"], rtol=1e-12)


def test_opcuda_mc1f_reference_layout_and_continuation(cuda):
    """Drop-in mc1f: column-major cumulative kernel, per-step kernel index, blocking copy
    to the host, and successive calls continuing with fresh paths."""
    from oplib_b200 import _lib
    lib = _lib.load()
    cfg = O.LVLattice(n=128)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 52, cfg.dt0)
    P = O.square(O.ek(L, dt), niter)
    Cr = O.cumrows_f32(P)  # source-major
    d, nscen, y0 = 128, 4096, O.nearest_node(x)
    for nk in (40, 700):  # 700: past the register-only generator's 623 steps
        _mc1f_batches(lib, cuda, Cr, d, nk, nscen, y0)


def _stream_seeds(seed):
    """4096 stream seeds as the reference's callers draw them: uniform in [0, 2^31 - 1)."""
    return np.random.default_rng(seed).integers(0, 2**31 - 1, 4096).astype(np.uint32)


def _mc1f_batches(lib, cuda, Cr, d, nk, nscen, y0):
    ccm = torch.from_numpy(np.asfortranarray(Cr).ravel(order="K").copy()).to(cuda)
    mk = torch.zeros(nk, dtype=torch.int32, device=cuda)
    assert lib.opcuda_mc_nrng() == 4096
    st = torch.zeros(lib.opcuda_mc_status_sz(), dtype=torch.int32, device=cuda)
    yd = torch.empty(nscen * nk, dtype=torch.int16, device=cuda)
    seeds = _stream_seeds(4242)
    assert lib.opcuda_mc_setseed(seeds.ctypes.data, st.data_ptr()) == 0
    for batch in range(2):
        yh = np.empty(nscen * nk, dtype=np.int16)
        assert lib.opcuda_mc1f(st.data_ptr(), y0, yd.data_ptr(), nscen, nk, d, ccm.data_ptr(), mk.data_ptr(),
                               yh.ctypes.data) == 0
        ref = OC.mc_paths_seeded(Cr, y0, seeds, batch * nscen, nscen, nk)
        assert np.array_equal(yh.reshape(nk, nscen).T, ref)


def test_opcuda_mc1f_uses_every_stream_seed(cuda):
    """Path g is path g / 4096 of stream g % 4096: changing one stream's seed changes that
    stream's paths and no other; paths 0 .. 4095 draw from init_genrand(seeds[g])."""
    from oplib_b200 import _lib
    lib = _lib.load()
    cfg = O.LVLattice(n=128)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 52, cfg.dt0)
    Cr = O.cumrows_f32(O.square(O.ek(L, dt), niter))
    d, nk, nscen, y0 = 128, 30, 3 * 4096, O.nearest_node(x)
    ccm = torch.from_numpy(np.asfortranarray(Cr).ravel(order="K").copy()).to(cuda)
    mk = torch.zeros(nk, dtype=torch.int32, device=cuda)
    yd = torch.empty(nscen * nk, dtype=torch.int16, device=cuda)
    out = []
    seeds = _stream_seeds(7)
    for change in (False, True):
        s = seeds.copy()
        if change:
            s[5] ^= 0x5A5A5A5A
        st = torch.zeros(lib.opcuda_mc_status_sz(), dtype=torch.int32, device=cuda)
        assert lib.opcuda_mc_setseed(s.ctypes.data, st.data_ptr()) == 0
        assert int(st[4 + 5].item()) & 0xFFFFFFFF == int(s[5])
        yh = np.empty(nscen * nk, dtype=np.int16)
        assert lib.opcuda_mc1f(st.data_ptr(), y0, yd.data_ptr(), nscen, nk, d, ccm.data_ptr(), mk.data_ptr(),
                               yh.ctypes.data) == 0
        out.append(yh.reshape(nk, nscen).T.copy())
        assert np.array_equal(out[-1], OC.mc_paths_seeded(Cr, y0, s, 0, nscen, nk))
    differs = np.any(out[0] != out[1], axis=1)
    stream5 = np.arange(nscen) % 4096 == 5
    assert not differs[~stream5].any()
    assert differs[stream5].all()
    # the first path of each stream is plain init_genrand(seed)
    for g in (0, 5, 4095):
        u = O.uniform_f32(OC.mt_outputs(int(seeds[g]), nk))
        y = y0
        for k in range(nk):
            y = int(O.sample_next(Cr[y][None, :], u[k:k + 1])[0])
            assert out[0][g, k] == y


@pytest.mark.parametrize("nper", [20, 700])
def test_mt_benchmark_uniforms(cuda, nper):
    from oplib_b200 import _lib
    lib = _lib.load()
    st = torch.zeros(lib.opcuda_mc_status_sz(), dtype=torch.int32, device=cuda)
    seeds = _stream_seeds(7)
    assert lib.opcuda_mc_setseed(seeds.ctypes.data, st.data_ptr()) == 0
    n = 4096 * nper
    u = torch.empty(n, device=cuda)
    assert lib.opcuda_mt_benchmark(st.data_ptr(), u.data_ptr(), n) == 0
    got = u.cpu().numpy().reshape(nper, 4096)
    for s in [0, 5, 4095]:  # stream s: init_genrand(seeds[s]), as the reference's twister s
        ref = (OC.mt_outputs(int(seeds[s]), nper).astype(np.float32) * np.float32(2.0 ** -32)).astype(np.float32)
        assert np.array_equal(got[:, s], ref)


def test_mc_paths_bit_exact_with_default_guide_width(step_rows):
    """The default guide table (two buckets per state: 1024 for 512 states) changes only
    the search bracket: the paths stay those of the oracle."""
    from oplib_b200.model import guide_buckets, guide_table, mc_run
    lat, P, Cm, _ = step_rows
    assert guide_buckets(512) == 1024 and guide_buckets(3000) == 4096 and guide_buckets(1) == 2
    g = guide_table(Cm)
    assert tuple(g.shape) == (512, 1024)
    disc = math.exp(-0.03 * 2.0)
    sums, paths = mc_run(Cm, lat.y0, 504, 5489, 2048, guide=g, x=lat.x, disc=disc, want_paths=True)
    torch.cuda.synchronize()
    ref_paths, ref_sums = OC.mc_paths(Cm.cpu().numpy(), lat.y0, 5489, 0, 2048, 504, x=lat.x.cpu().numpy(), disc=disc)
    assert np.array_equal(paths.cpu().numpy().T, ref_paths)
    assert np.allclose(sums.cpu().numpy(), ref_sums, rtol=1e-12)
