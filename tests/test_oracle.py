"""CPU tests of the oracle itself: pins against independent implementations, the
reference's known-answer test and mathematical identities (no GPU)."""
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from oracle import oracle_c as OC

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden"


def _std_mt(seed, count, skip=0):
    exe = ROOT / "oracle" / "mt_std_check"
    if not exe.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "-s"], check=True)
    out = subprocess.run([str(exe), str(seed), str(count), str(skip)], capture_output=True, text=True, check=True)
    return np.array([int(v) for v in out.stdout.split()], dtype=np.uint64).astype(np.uint32)


def test_mt19937_cpp_standard_value():
    # C++11 [rand.predef]: the 10000th output of a default-constructed mt19937 is 4123659995
    assert int(OC.mt_outputs(5489, 10000)[-1]) == 4123659995
    assert int(O.mt19937_outputs(np.array([5489]), 10000)[0, -1]) == 4123659995


@pytest.mark.parametrize("seed", [0, 1, 5489, 12345, 2**32 - 1, 20260])
def test_mt19937_matches_libstdcxx_and_numpy(seed):
    std = _std_mt(seed, 1300)
    c = OC.mt_outputs(seed, 1300)
    py = O.mt19937_outputs(np.array([seed]), 1300)[0]
    g = np.random.MT19937()
    g._legacy_seeding(seed)
    npy = g.random_raw(1300).astype(np.uint32)
    assert np.array_equal(std, c)
    assert np.array_equal(std, py)
    assert np.array_equal(std, npy)


def test_mt19937_golden_fixture():
    gold = np.load(GOLD / "mt19937.npz")
    for seed, ref in zip(gold["seeds"], gold["outputs"]):
        assert np.array_equal(OC.mt_outputs(int(seed), ref.shape[0]), ref)


def test_uniform_conversion_edges():
    u = O.uniform_f32(np.array([0, 1, 2**24, 2**32 - 1, 2**31], dtype=np.uint32))
    assert u[0] == np.float32(2.0 ** -32)
    assert u[3] == np.float32(1.0)  # (float)(2^32-1) rounds to 2^32
    for x in [0, 1, 255, 2**24 + 1, 2**32 - 1, 123456789]:
        assert OC.load().oracle_uniform_f32(x) == O.uniform_f32(np.array([x], np.uint32))[0]


def test_black_scholes_closed_form():
    # tests/bstest/Program.cs:11-19: S=K=100, r=0.05, sigma=0.25, T=1
    assert abs(float(O.bs_call(100.0, 100.0, 0.05, 0.25, 1.0)) - 12.33600) < 5e-5
    iv = O.implied_vol(O.bs_call(1.0, 1.1, 0.02, 0.3, 0.7), 1.0, 1.1, 0.02, 0.7)
    assert abs(float(iv) - 0.3) < 1e-9


def test_lattice_black_scholes_known_answer():
    """The reference's KAT (tests/bstest) as a lattice price: GBM on a log grid with the
    spot on a node, FP64 squaring, price vs the closed form."""
    n, i0, s0 = 1024, 511, 100.0
    x = O.centred_log_grid(n, s0, width=8.0, i0=i0)
    r, sig = 0.05, 0.25
    L = O.lv_generator_fast(x, r * x, sig * x)
    niter, dt = O.plan_niter(L, 1.0, 2.0 ** -14)
    P = O.square(O.ek(L, dt), niter, renorm=True)
    price = math.exp(-r) * (P[i0] @ np.maximum(x - 100.0, 0.0))
    assert abs(price - 12.33600) < 2e-3 * 100 / 100  # lattice discretisation error, spot units


def test_generator_rows_and_expm():
    cfg = O.LVLattice(n=128)
    L, x = cfg.generator()
    assert np.allclose(L.sum(axis=1), 0.0, atol=1e-9)
    assert (L - np.diag(np.diag(L)) >= 0).all()
    niter, dt = O.plan_niter(L, 0.25, cfg.dt0)
    P = O.square(O.ek(L, dt), niter)
    from scipy.linalg import expm
    assert np.abs(P - expm(L * 0.25)).max() < 1e-4  # first-order splitting error of (I+dt L)^(2^n)
    assert np.abs(P.sum(axis=1) - 1).max() < 1e-12  # probability conservation


def test_lv_generator_vectorised_matches_loop():
    x = O.log_grid(64)
    sig = O.lv_sigma(x)
    assert np.allclose(O.lv_generator(x, 0.03 * x, sig * x), O.lv_generator_fast(x, 0.03 * x, sig * x),
                       rtol=1e-12, atol=1e-9)


def test_semigroup():
    cfg = O.LVLattice(n=96)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 0.25, cfg.dt0)
    P1 = O.square(O.ek(L, dt), niter)
    P2 = O.square(O.ek(L, dt), niter + 1)
    assert np.abs(P1 @ P1 - P2).max() < 1e-12


def test_sv_generator_properties():
    spec = O.SVSpec(nx=24, nv=8)
    L, xy, vy = O.sv_generator(spec)
    off = L - np.diag(np.diag(L))
    assert (off >= 0).all()
    assert np.allclose(L.sum(axis=1), 0, atol=1e-9)
    # interior spot drift is exactly r*x after the fix-up
    drift = L @ xy
    inner = [y for y in range(spec.d) if 0 < y % spec.nx < spec.nx - 1]
    assert np.allclose(drift[inner], spec.r * xy[inner], rtol=1e-9, atol=1e-12)


def test_config0_golden_quotes():
    gold = np.load(GOLD / "lattice_lv512.npz")
    cfg = O.LVLattice()
    L, x = cfg.generator()
    V, niter, dt = O.solve_lattice_fp64(L, x, cfg.strikes, cfg.r, cfg.period, cfg.nmat, cfg.dt0)
    y0 = O.nearest_node(x)
    assert niter == int(gold["niter"]) == 12
    assert np.abs(V[:, y0, :] - gold["quotes"]).max() < 1e-12


def test_sck_c_matches_numpy():
    rng = np.random.default_rng(3)
    P = rng.random((40, 77)).astype(np.float32)
    P[3, 5] = -1e-9  # rounding residue counts as zero
    P /= P.sum(axis=1, keepdims=True)
    assert np.array_equal(OC.sck(P), O.cumrows_f32(P))


def test_mc_c_matches_numpy():
    cfg = O.LVLattice(n=64)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 252, cfg.dt0)
    P = O.square(O.ek(L, dt), niter)
    Cm = O.cumrows_f32(P)
    paths_c, _ = OC.mc_paths(Cm, 32, 5489, 0, 300, 40)
    paths_py = O.mc_paths(Cm, 32, 5489, np.arange(300), 40)
    assert np.array_equal(paths_c, paths_py)


def test_mc_golden_fixture():
    gold = np.load(GOLD / "mc_small.npz")
    paths, sums = OC.mc_paths(gold["C"], int(gold["y0"]), int(gold["seed"]), 0, gold["paths"].shape[0],
                              gold["paths"].shape[1], x=gold["x"], disc=float(gold["disc"]))
    assert np.array_equal(paths, gold["paths"])
    assert np.allclose(sums, gold["sums"], rtol=1e-12)


def test_mlp_oracle_gradient_vs_finite_differences():
    from oracle import mlp_oracle as M
    _, n = M.layout()
    assert n == 199937
    rng = np.random.default_rng(0)
    theta = rng.standard_normal(n) * 0.05
    X = rng.uniform(-1, 1, (16, 8))
    t = rng.standard_normal(16) * 0.1
    _, g = M.loss_grad(theta, X, t)
    for idx in rng.choice(n, 25, replace=False).tolist() + [n - 1, 0, 2048, 2048 + 256]:
        h = 1e-6
        tp, tm = theta.copy(), theta.copy()
        tp[idx] += h
        tm[idx] -= h
        fd = (M.loss_grad(tp, X, t)[0] - M.loss_grad(tm, X, t)[0]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-5 * abs(fd), (idx, fd, g[idx])


def test_s2d_invm_solves_the_moment_equations():
    nx, nr = 6, 4
    xval = np.tile(0.5 * 2.0 ** (np.arange(nx) / 2.0), nr)
    rval = np.repeat(0.1 * 2.0 ** np.arange(nr), nx)
    invm = O.s2d_invm(xval, rval, nx, nr)
    # interior node: rates from the moments reproduce them
    y0 = 2 + nx * 1
    inv = invm[16 * y0:16 * y0 + 16].reshape(4, 4).T
    moments = np.array([0.01, 0.04, -0.02, 0.005])
    q = inv @ moments
    dxm, dxp = xval[y0 - 1] - xval[y0], xval[y0 + 1] - xval[y0]
    drm, drp = rval[y0 - nx] - rval[y0], rval[y0 + nx] - rval[y0]
    assert np.allclose([q[0] * dxm + q[1] * dxp, q[0] * dxm ** 2 + q[1] * dxp ** 2,
                        q[2] * drm + q[3] * drp, q[2] * drm ** 2 + q[3] * drp ** 2], moments, rtol=1e-12)


def test_sgsvg_oracle_row_sums_and_jumps():
    nx, nr = 10, 4
    d = nx * nr
    xval = np.tile(0.2 * 1.3 ** np.arange(nx), nr)
    rval = np.repeat(0.1 * 2.0 ** np.arange(nr), nx)
    invm = O.s2d_invm(xval, rval, nx, nr)
    G = O.sgsvg_generator(invm, xval, 0.03 * xval, rval * xval, 2.0 * (0.3 - rval), 0.5 * rval,
                          np.full(d, 0.1), np.full(d, 0.15), nx, nr)
    assert np.abs(G.sum(axis=1)).max() < 1e-12
    off = G - np.diag(np.diag(G))
    # the up-move of an interior node spreads over its next volatility level
    y0 = 5 + nx * 1
    assert np.count_nonzero(off[y0, nx * 2:nx * 3]) > 3


def test_gelu_erf_approximation_bound():
    """The tensor-core layers' GELU uses erf from Abramowitz & Stegun 7.1.26 in the kernel's
    folded form (1/sqrt 2 inside p, the halving inside the a_i, exp(-x^2) as a power of two,
    the constants rounded to FP32 as the kernel has them); the published bound 1.5e-7
    holds, so GELU is within 0.75e-7 |z| (plus the FP32 rounding of the folded constants)
    of the exact form."""
    from scipy.special import erf
    f32 = lambda v: float(np.float32(v))
    P = f32(f32(0.3275911) * f32(0.70710678118654752))
    A = [f32(0.5 * f32(a)) for a in (0.254829592, -0.284496736, 1.421413741, -1.453152027, 1.061405429)]
    z = np.linspace(-12.0, 12.0, 200001)
    t = 1.0 / (1.0 + P * np.abs(z))
    q = A[0] + t * (A[1] + t * (A[2] + t * (A[3] + t * A[4])))
    h = q * t * np.exp2(z * z * f32(-0.72134752044448170))
    g = z * np.where(z >= 0, 1.0 - h, h)
    exact = 0.5 * z * (1.0 + erf(z / math.sqrt(2.0)))
    x = np.abs(z) / math.sqrt(2.0)
    assert np.max(np.abs((1.0 - 2.0 * h) - erf(x))) <= 1.6e-7
    assert np.all(np.abs(g - exact) <= 0.8e-7 * np.abs(z) + 1e-300)


def test_bermudan_oracle_identities():
    """The induction oracle against the chained European solve and the textbook ordering
    of contract values: on a 128-node local-vol lattice (r > 0, no dividends) the European
    value by induction equals the chained solve's value at the last maturity; a Bermudan
    call is never exercised early away from the grid's upper edge (where the truncated
    lattice is no longer a martingale), so it equals the European call there; a Bermudan
    put is worth at least the European put (strictly more near the spot); a down-and-out
    call is worth less than the vanilla call (strictly less at the spot).  Exercise and the
    barrier apply at the dates m * period, m >= 1, not at time 0."""
    cfg = O.LVLattice(n=128, nmat=6)
    L, x = cfg.generator()
    K = cfg.strikes[::8]
    V, _, _ = O.solve_lattice_fp64(L, x, K, cfg.r, cfg.period, cfg.nmat, cfg.dt0)
    args = (L, x, K, cfg.r, cfg.period, cfg.nmat, cfg.dt0)
    euro_call = O.bermudan_fp64(*args, put=False, exercise=False)
    assert np.abs(euro_call - V[-1]).max() < 1e-12
    berm_call = O.bermudan_fp64(*args, put=False, exercise=True)
    inner = x <= 1.25  # the edge's influence decays inward: 2e-11 at the spot, 1.6e-5 at x = 2.2
    assert np.abs(berm_call - euro_call)[inner].max() < 1e-9
    assert np.all(berm_call >= euro_call - 1e-14)
    euro_put = O.bermudan_fp64(*args, put=True, exercise=False)
    berm_put = O.bermudan_fp64(*args, put=True, exercise=True)
    assert np.all(berm_put >= euro_put - 1e-14)
    assert berm_put.max() - (berm_put - euro_put).max() > 0 and (berm_put - euro_put).max() > 1e-4
    dao = O.bermudan_fp64(*args, put=False, exercise=False, barrier=0.8)
    assert np.all(dao <= euro_call + 1e-14)
    y0 = O.nearest_node(x)
    assert np.all(dao[y0] < euro_call[y0] - 1e-4)


def test_host_solve_stages_matches_the_fp64_solve():
    """The staged host solve (the bench's reference arm: U0, squarings, chain products and
    payoff products one product per stage) is the oracle's FP64 solve without
    renormalisation, and yields once per product with the values at the last stage."""
    import torch
    cfg = O.LVLattice(n=256, nmat=5)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, cfg.period, cfg.dt0)
    outs = list(O.host_solve_stages(torch.from_numpy(L.copy()), x, cfg.strikes, cfg.r, cfg.period, cfg.nmat,
                                    niter, dt))
    assert len(outs) == niter + cfg.nmat - 1 and all(o is None for o in outs[:-1])
    V, _, _ = O.solve_lattice_fp64(L, x, cfg.strikes, cfg.r, cfg.period, cfg.nmat, cfg.dt0, renorm=False)
    assert np.allclose(outs[-1].numpy(), V, rtol=1e-12, atol=1e-14)
    one = list(O.host_solve_stages(torch.from_numpy(L.copy()), x, cfg.strikes, cfg.r, cfg.period, 1, niter, dt))
    assert len(one) == niter and np.allclose(one[-1].numpy()[0], V[0], rtol=1e-12, atol=1e-14)


def test_mc_cashflow_values_by_hand():
    """The evaluator's rule on a two-path, three-step example: cashflows add up in step order
    until the first knocked-out state, which pays nothing from then on."""
    paths = np.array([[0, 1, 2], [1, 1, 0]], dtype=np.int16)
    cf = np.array([[1.0, 2.0, 4.0], [8.0, 16.0, 32.0], [64.0, 128.0, 256.0]])
    assert np.array_equal(O.mc_cashflow_values(paths, cf), [1.0 + 16.0 + 256.0, 2.0 + 16.0 + 64.0])
    ko = np.zeros((3, 3), dtype=np.uint8)
    ko[1, 1] = 1
    assert np.array_equal(O.mc_cashflow_values(paths, cf, ko), [1.0, 2.0])


def test_split_bf16_floor():
    """The library's BF16 split, restated: hi = bf16(a), lo = bf16(a - hi), except that an
    entry below 2^-40 in magnitude has no parts and one below 2^-30 has no lo part."""
    third = np.float32(1.0 / 3.0)
    a = np.array([third, -third, 2.0 ** -41, -(2.0 ** -41), 1.7 * 2.0 ** -31, 1.7 * 2.0 ** -29, 0.0],
                 dtype=np.float32)
    hi, lo = O.split_bf16(a)
    assert hi[0] == np.float32(0.333984375) and lo[0] == O.bf16_round(np.float32(third - np.float32(0.333984375)))
    assert hi[1] == -hi[0] and lo[1] == -lo[0]
    assert hi[2] == 0 and lo[2] == 0 and hi[3] == 0 and lo[3] == 0
    assert hi[4] == O.bf16_round(a[4:5])[0] and hi[4] != 0 and lo[4] == 0  # below 2^-30: hi only
    assert lo[5] == O.bf16_round(np.float32(a[5] - hi[5]))                # above: both parts
    assert lo[5] != 0
    assert hi[6] == 0 and lo[6] == 0
    # hi + lo carries 16 significant bits wherever the floor does not apply
    big = np.abs(a) >= 2.0 ** -30
    assert np.all(np.abs((hi + lo).astype(np.float64) - a.astype(np.float64))[big]
                  <= 2.0 ** -16 * np.abs(a[big]).astype(np.float64))
