"""GPU parity of the lattice path against the FP64 oracle.

Tolerances (absolute price error, S0 = 1):
- OPB_BF16X3 and OPB_FP32_RENORM: <= 1e-5 versus the FP64 solve (the target accuracy);
- OPB_FP32_PLAIN (the reference's FP32 semantics, no renormalisation) is reported and
  bounded by 5e-4; its error is what the FP64 renormalisation removes.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _lv(n=512, **kw):
    from oplib_b200.model import Lattice
    return Lattice.local_vol(n=n, **kw)


def test_lv_generator_matches_oracle(cuda):
    lat = _lv(300, level=0.25, skew=-0.2, width=0.4, rate=0.02)
    torch.cuda.synchronize()
    x = lat.x.cpu().numpy()
    assert np.allclose(x, O.log_grid(300), rtol=1e-14)
    ref = O.lv_generator_fast(x, 0.02 * x, O.lv_sigma(x, 0.25, -0.2, 0.4) * x)
    cols = lat.cols.cpu().numpy().reshape(-1, 3)
    vals = lat.vals.cpu().numpy().reshape(-1, 3)
    dense = np.zeros((300, 300))
    for y in range(300):
        for c, v in zip(cols[y], vals[y]):
            if c >= 0:
                dense[y, c] += v
    assert np.allclose(dense, ref, rtol=1e-12, atol=1e-9)
    assert abs(lat.maxdiag() - np.abs(np.diag(ref)).max()) < 1e-9


def test_sv_generator_matches_oracle(cuda):
    from oplib_b200.model import Lattice
    spec = O.SVSpec(nx=20, nv=9)
    lat = Lattice.stoch_vol(nx=20, nv=9)
    torch.cuda.synchronize()
    ref, xy, _ = O.sv_generator(spec)
    cols = lat.cols.cpu().numpy().reshape(-1, 7)
    vals = lat.vals.cpu().numpy().reshape(-1, 7)
    dense = np.zeros_like(ref)
    for y in range(spec.d):
        for c, v in zip(cols[y], vals[y]):
            if c >= 0:
                dense[y, c] += v
    assert np.allclose(dense, ref, rtol=1e-11, atol=1e-9)
    assert np.allclose(lat.x.cpu().numpy(), xy, rtol=1e-14)


@pytest.fixture(scope="module")
def config0_fp64():
    cfg = O.LVLattice()
    L, x = cfg.generator()
    V, niter, dt = O.solve_lattice_fp64(L, x, cfg.strikes, cfg.r, cfg.period, cfg.nmat, cfg.dt0)
    return cfg, V, O.nearest_node(x)


@pytest.mark.parametrize("mode,tol", [("bf16x3", 1e-5), ("fp16x3", 1e-5), ("fp32", 1e-5), ("fp32_plain", 5e-4)])
def test_config0_quotes_vs_fp64(cuda, config0_fp64, mode, tol):
    cfg, V, y0 = config0_fp64
    lat = _lv()
    assert lat.y0 == y0
    q, Vall = lat.solve(cfg.strikes, cfg.nmat, cfg.period, cfg.dt0, mode=mode, all_states=True)
    torch.cuda.synchronize()
    from oplib_b200 import _lib
    assert _lib.load().opb_tc_error() == 0
    err = np.abs(q.cpu().numpy() - V[:, y0, :]).max()
    print(f"config0 {mode}: max abs quote error {err:.3e}")
    assert err <= tol
    # all source states (the backward induction result): relative to the option value
    # (values reach ~4.5 at the far spot boundary)
    errall = (np.abs(Vall.cpu().numpy() - V) / np.maximum(1.0, np.abs(V))).max()
    assert errall <= 5 * tol


def test_kernel_matches_fp64_and_conserves(cuda):
    cfg = O.LVLattice(n=256)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 252, cfg.dt0)
    P64 = O.square(O.ek(L, dt), niter, renorm=True)
    lat = _lv(256)
    for mode in ["fp32", "bf16x3", "fp16x3"]:
        P = lat.kernel(1 / 252, cfg.dt0, mode=mode).cpu().numpy().astype(np.float64)
        assert np.abs(P - P64).max() < 2e-5, mode
        assert np.abs(P.sum(axis=1) - 1).max() < 1e-6, mode


def test_sv_small_bf16x3_vs_fp64(cuda):
    """A reduced stochastic-vol lattice (d = 32 x 8 = 256) in all three modes."""
    from oplib_b200.model import Lattice
    spec = O.SVSpec(nx=32, nv=8)
    L, xy, _ = O.sv_generator(spec)
    strikes = 0.7 + np.arange(64) / 100
    lat = Lattice.stoch_vol(nx=32, nv=8)
    niter, dt = O.plan_niter(L, 0.25, 2.0 ** -16)
    U = O.ek(L, dt)
    P = O.square(U, niter, renorm=True)
    Ps = O.chain(P, 4)
    Vref = O.price_from_kernels(Ps, xy, strikes, spec.r, 0.25 * np.arange(1, 5))
    for mode, tol in [("bf16x3", 1e-5), ("fp16x3", 1e-5), ("fp32", 1e-5)]:
        q, _ = lat.solve(strikes, 4, 0.25, 2.0 ** -16, mode=mode)
        err = np.abs(q.cpu().numpy() - Vref[:, lat.y0, :]).max()
        print(f"sv256 {mode}: {err:.3e}")
        assert err <= tol, (mode, err)


def test_black_scholes_lattice_on_gpu(cuda):
    """The reference's known-answer test (tests/bstest/Program.cs:11-37) through the
    device path: GBM, spot on a node, split-BF16 squaring."""
    from oplib_b200.model import Lattice
    n, i0 = 1024, 511
    x = torch.from_numpy(O.centred_log_grid(n, 100.0, 8.0, i0)).to(cuda)
    lat = Lattice.from_drift_vol(x, 0.05 * x, 0.25 * x, 0.05, s0=100.0)
    assert lat.y0 == i0
    q, _ = lat.solve([100.0], 4, 0.25, 2.0 ** -14, mode="bf16x3")  # nK = 1: padded to the tile internally
    price = q.cpu().numpy()[3, 0]
    assert abs(price - 12.33600) < 0.2  # lattice discretisation on a 1024-node grid
    q32, _ = lat.solve([100.0], 4, 0.25, 2.0 ** -14, mode="fp32")
    assert abs(price - q32.cpu().numpy()[3, 0]) < 1e-3
    # FP16 parts with a payoff scale derived on the device from max(x) - min(K) (here ~5e3)
    q16, _ = lat.solve([100.0], 4, 0.25, 2.0 ** -14, mode="fp16x3")
    assert abs(q16.cpu().numpy()[3, 0] - q32.cpu().numpy()[3, 0]) < 1e-3


def test_workspace_too_small_is_rejected(cuda):
    from oplib_b200 import _lib
    from oplib_b200.model import BF16X3
    lat = _lv(256)
    plan = lat.plan(0.25, 2.0 ** -14)
    strikes = torch.linspace(0.5, 1.5, 64, dtype=torch.float64, device=cuda)
    L = lat.desc(plan, 0.25, 2, strikes)
    ws = torch.empty(1024, dtype=torch.uint8, device=cuda)
    q = torch.empty(2, 64, dtype=torch.float64, device=cuda)
    import ctypes as C
    assert _lib.load().opb_lattice_solve(C.byref(L), BF16X3, ws.data_ptr(), 1024, q.data_ptr(), None) == -1


@pytest.mark.gpu
@pytest.mark.parametrize("mode,f16", [(0, 0), (1, 0), (2, 0), (0, 1)])
def test_renorm_rows_bit_exact(cuda, mode, f16):
    """opb_renorm_rows against the same FP64 arithmetic on the host: sequential sum of the
    partials, one reciprocal, (x - diag * sum) * inv (+1 on the diagonal for mode 1),
    round to FP32, then the 16-bit splits (A row-major, B transposed)."""
    from oplib_b200 import _lib
    d, np_ = 192, 3
    rng = np.random.default_rng(7 + mode + 10 * f16)
    X0 = (rng.random((d, d)) * 1e-3).astype(np.float32)
    part = rng.random((np_, d)) * (1e-2 if mode != 2 else 0.5)
    X = torch.from_numpy(X0.copy()).cuda()
    P = torch.from_numpy(part).cuda()
    parts = [torch.zeros(d, d, dtype=torch.bfloat16, device="cuda") for _ in range(4)]
    _lib.call("opb_renorm_rows", d, X.data_ptr(), P.data_ptr(), np_, mode, *[t.data_ptr() for t in parts], f16)
    torch.cuda.synchronize()
    s = np.zeros(d)
    for p in range(np_):
        s = s + part[p]
    den = 1.0 + s if mode != 2 else s
    inv = 1.0 / den
    x = X0.astype(np.float64)
    if mode != 2:
        x = x - np.diag(s)
    x = x * inv[:, None]
    if mode == 1:
        x = x + np.eye(d)
    ref = x.astype(np.float32)
    got = X.cpu().numpy()
    assert np.array_equal(got, ref)
    r = torch.from_numpy(ref)
    if f16:
        rs = r * 32768.0
        hi = rs.to(torch.float16)
        lo = (rs - hi.float()).to(torch.float16)
        hi, lo = hi.view(torch.int16), lo.view(torch.int16)
    else:
        # BF16 parts with the split's absolute floor: |x| < 2^-40 -> 0, |x| < 2^-30 -> no lo part
        hi = torch.where(r.abs() < 2.0 ** -40, 0.0, r).to(torch.bfloat16)
        lo = torch.where(r.abs() < 2.0 ** -30, 0.0, r - hi.float()).to(torch.bfloat16)
        hi, lo = hi.view(torch.int16), lo.view(torch.int16)
    g = [t.view(torch.int16).cpu() for t in parts]
    assert torch.equal(g[0], hi) and torch.equal(g[1], lo)
    if mode != 2:
        assert torch.equal(g[2], hi.T.contiguous()) and torch.equal(g[3], lo.T.contiguous())
    else:
        assert not g[2].any() and not g[3].any()


@pytest.mark.gpu
def test_opcuda_sgsvg_matches_oracle(cuda):
    """The reference's two-dimensional generator with vol-level jumps (drop-in
    opcuda_sgsvg) against the FP64 restatement, two intervals of a 12 x 5 grid; moment
    inverses from the restated S2DGrid.pregen."""
    from oplib_b200 import _lib
    lib = _lib.load()
    nx, nr, ni = 12, 5, 2
    d = nx * nr
    xs = 0.05 * 100.0 ** (np.arange(nx) / (nx - 1))
    rs = 0.1 * 8.0 ** (np.arange(nr) / (nr - 1))
    xval = np.tile(xs, nr)
    rval = np.repeat(rs, nx)
    invm = O.s2d_invm(xval, rval, nx, nr).astype(np.float32)
    rng = np.random.default_rng(3)
    blocks = []
    for name in ["sdrift", "svol", "voldrift", "volvol", "jm", "jp"]:
        b = np.empty((ni, d))
        for i in range(ni):
            if name == "sdrift":
                b[i] = 0.03 * xval
            elif name == "svol":
                b[i] = rval * xval
            elif name == "voldrift":
                b[i] = 2.0 * (0.3 - rval)
            elif name == "volvol":
                b[i] = 0.5 * rval
            elif name == "jm":
                b[i] = rng.uniform(0.05, 0.2, d)
            else:
                b[i] = rng.uniform(0.05, 0.2, d)
        blocks.append(b.astype(np.float32))
    par = np.concatenate([xval.astype(np.float32)] + [b.reshape(-1) for b in blocks])
    d_par = torch.from_numpy(par).to(cuda)
    d_inv = torch.from_numpy(invm).to(cuda)
    gen = torch.zeros(ni * d * d, dtype=torch.float32, device=cuda)
    assert lib.opcuda_sgsvg(gen.data_ptr(), ni, nx, nr, d_inv.data_ptr(), d_par.data_ptr()) == 0
    torch.cuda.synchronize()
    got = gen.cpu().numpy().reshape(ni, d, d)   # [i][y1][y0]: column-major rows = source
    f64 = lambda a: np.asarray(a, dtype=np.float64)
    for i in range(ni):
        G = O.sgsvg_generator(f64(invm), f64(xval.astype(np.float32)), *[f64(b[i]) for b in blocks], nx, nr)
        dev = got[i].T.astype(np.float64)       # -> [y0][y1]
        scale = np.abs(G).max(axis=1, keepdims=True)
        assert np.all(np.abs(dev - G) <= 2e-6 * scale + 1e-12), np.max(np.abs(dev - G) / scale)
        assert np.abs(dev.sum(axis=1)).max() <= 1e-5 * scale.max()
        # jumps reached levels above the neighbour
        assert np.count_nonzero(dev) > 5 * d
    assert lib.opcuda_sgsvg(gen.data_ptr(), 0, nx, nr, d_inv.data_ptr(), d_par.data_ptr()) != 0
