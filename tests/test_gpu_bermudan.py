"""GPU parity of the backward-induction pricer (Bermudan and discretely monitored
down-and-out options on the period kernel, ``opb_lattice_bermudan``) against the FP64
induction oracle.  Tolerance: 1e-5 absolute price error (S0 = 1), the target accuracy of
the lattice path."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5
CASES = [  # (put, exercise, barrier)
    (True, True, 0.0),    # Bermudan put
    (False, True, 0.0),   # Bermudan call
    (True, False, 0.0),   # European put by induction
    (False, False, 0.8),  # down-and-out call, barrier 0.8
    (True, True, 0.7),    # Bermudan down-and-out put
]


@pytest.mark.parametrize("mode", ["bf16x3", "fp16x3"])
def test_bermudan_lv_matches_oracle(cuda, mode):
    """The config-0 local-vol lattice (512 nodes, quarterly dates to 2 years, 64 strikes)."""
    from oplib_b200.model import Lattice
    cfg = O.LVLattice(n=512, nmat=8)
    L, x = cfg.generator()
    lat = Lattice.local_vol(n=512, level=cfg.level, skew=cfg.skew, width=cfg.width, rate=cfg.r, device=cuda)
    y0 = O.nearest_node(x)
    assert lat.y0 == y0
    for put, ex, bar in CASES:
        ref = O.bermudan_fp64(L, x, cfg.strikes, cfg.r, cfg.period, cfg.nmat, cfg.dt0, put=put, exercise=ex,
                              barrier=bar)[y0]
        q = lat.bermudan(cfg.strikes, cfg.nmat, cfg.period, cfg.dt0, mode=mode, put=put, exercise=ex, barrier=bar)
        err = np.abs(q.cpu().numpy() - ref).max()
        print(f"lv512 {mode} put={put} exercise={ex} barrier={bar}: {err:.3e}")
        assert err <= TOL, (put, ex, bar, err)


def test_european_by_induction_matches_the_chained_solve(cuda):
    """exercise = 0, barrier = 0: the induction on P1 gives the chained solve's value at the
    last maturity (two device paths through different products)."""
    from oplib_b200.model import Lattice
    cfg = O.LVLattice(n=512, nmat=8)
    lat = Lattice.local_vol(n=512, level=cfg.level, skew=cfg.skew, width=cfg.width, rate=cfg.r, device=cuda)
    q_ind = lat.bermudan(cfg.strikes, cfg.nmat, cfg.period, cfg.dt0, mode="fp16x3", put=False, exercise=False)
    q_chain, _ = lat.solve(cfg.strikes, cfg.nmat, cfg.period, cfg.dt0, mode="fp16x3")
    assert np.abs(q_ind.cpu().numpy() - q_chain[-1].cpu().numpy()).max() <= TOL


def test_bermudan_sv_matches_oracle(cuda):
    """A reduced stochastic-vol lattice (32 x 8 = 256 states), Bermudan puts."""
    from oplib_b200.model import Lattice
    spec = O.SVSpec(nx=32, nv=8)
    L, xy, _ = O.sv_generator(spec)
    strikes = 0.7 + np.arange(64) / 100
    lat = Lattice.stoch_vol(nx=32, nv=8, device=cuda)
    ref = O.bermudan_fp64(L, xy, strikes, spec.r, 0.25, 4, 2.0 ** -16, put=True, exercise=True)[lat.y0]
    for mode in ("bf16x3", "fp16x3"):
        q = lat.bermudan(strikes, 4, 0.25, 2.0 ** -16, mode=mode, put=True, exercise=True)
        err = np.abs(q.cpu().numpy() - ref).max()
        print(f"sv256 bermudan put {mode}: {err:.3e}")
        assert err <= TOL, (mode, err)


def test_bermudan_fp32_modes(cuda):
    """The FP32 SIMT induction: with the FP64 row renormalisation within the 1e-5 bar; the
    reference's plain FP32 squaring within 5e-4 (its error is what renormalisation removes)."""
    from oplib_b200.model import Lattice
    cfg = O.LVLattice(n=256, nmat=4)
    L, x = cfg.generator()
    lat = Lattice.local_vol(n=256, level=cfg.level, skew=cfg.skew, width=cfg.width, rate=cfg.r, device=cuda)
    ref = O.bermudan_fp64(L, x, cfg.strikes, cfg.r, cfg.period, cfg.nmat, cfg.dt0, put=True, exercise=True)[lat.y0]
    for mode, tol in (("fp32", TOL), ("fp32_plain", 5e-4)):
        q = lat.bermudan(cfg.strikes, cfg.nmat, cfg.period, cfg.dt0, mode=mode, put=True, exercise=True)
        err = np.abs(q.cpu().numpy() - ref).max()
        print(f"lv256 bermudan put {mode}: {err:.3e}")
        assert err <= tol, (mode, err)


def test_bermudan_rejects_bad_flags(cuda):
    from oplib_b200._lib import OpcudaError
    from oplib_b200.model import Lattice
    lat = Lattice.local_vol(n=256, device=cuda)
    with pytest.raises(OpcudaError):
        lat.bermudan([1.0], 2, 0.25, 2.0 ** -14, mode="bf16x3", barrier=-1.0)
    with pytest.raises(OpcudaError):
        lat.bermudan([1.0], 2, 0.25, 2.0 ** -14, mode="bf16x3", put=2)


def test_bermudan_ragged_strike_count(cuda):
    """Five strikes (padded to the 64-column tile inside): the padding columns stay zero and
    the five values match the oracle."""
    from oplib_b200.model import Lattice
    cfg = O.LVLattice(n=256, nmat=3)
    L, x = cfg.generator()
    K = np.array([0.8, 0.95, 1.0, 1.1, 1.3])
    lat = Lattice.local_vol(n=256, level=cfg.level, skew=cfg.skew, width=cfg.width, rate=cfg.r, device=cuda)
    ref = O.bermudan_fp64(L, x, K, cfg.r, cfg.period, cfg.nmat, cfg.dt0, put=True, exercise=True)[lat.y0]
    q = lat.bermudan(K, cfg.nmat, cfg.period, cfg.dt0, mode="bf16x3", put=True, exercise=True)
    assert q.shape == (5,)
    assert np.abs(q.cpu().numpy() - ref).max() <= TOL


@pytest.mark.parametrize("mode", ["fp16x3", "bf16x3", "fp32"])
def test_batched_bermudan_matches_single_lattices(cuda, fused_single, mode):
    """Seven uneven local-vol lattices (sizes 256..1024, three of them odd multiples of 128)
    priced together by opb_batch_execute_bermudan against one opb_lattice_bermudan per
    lattice, under every launch configuration of the squarings; and one lattice against
    the FP64 induction oracle."""
    from oplib_b200.model import Batch, Lattice
    rng = np.random.default_rng(11)
    sizes = [256, 384, 512, 640, 768, 1024, 896]
    params = [dict(level=float(rng.uniform(0.15, 0.35)), skew=float(rng.uniform(-0.2, 0.2)),
                   width=float(rng.uniform(0.3, 0.9)), rate=float(rng.uniform(0.0, 0.05))) for _ in sizes]
    lats = [Lattice.local_vol(n=n, floor=0.01, device=cuda, **p) for n, p in zip(sizes, params)]
    K = np.linspace(0.8, 1.25, 12)
    nmat, period, dt0 = 4, 0.25, 2.0 ** -14
    bt = Batch(lats, K, nmat, period, dt0, mode=mode, autotune=False)
    for put, ex, bar in ((True, True, 0.0), (False, False, 0.85)):
        single = np.stack([lat.bermudan(K, nmat, period, dt0, mode=mode, put=put, exercise=ex, barrier=bar)
                           .cpu().numpy() for lat in lats])
        for cfg in (range(8) if mode != "fp32" else [0]):
            if mode != "fp32":
                bt.set_config(cfg)
            q = bt.execute_bermudan(put=put, exercise=ex, barrier=bar).cpu().numpy()
            assert q.shape == (len(lats), len(K))
            # the single-lattice induction products run as K-slices summed in FP64, the
            # batched ones in one pass: the two differ by FP32 rounding only
            assert np.abs(q - single).max() <= 1e-6, (mode, cfg, put, np.abs(q - single).max())
    # the 512-node lattice against the oracle
    i = 2
    x = lats[i].x.cpu().numpy()
    p = params[i]
    sig = O.lv_sigma(x, p["level"], p["skew"], p["width"], 0.01)
    L = O.lv_generator_fast(x, p["rate"] * x, sig * x)
    ref = O.bermudan_fp64(L, x, K, p["rate"], period, nmat, dt0, put=True, exercise=True)[lats[i].y0]
    q = bt.execute_bermudan(put=True, exercise=True).cpu().numpy()[i]
    assert np.abs(q - ref).max() <= TOL
