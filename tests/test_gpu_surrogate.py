"""GPU tests of the surrogate pricer: the library's MLP gradient against the FP64 oracle,
tensor-core inference against the FP32 training forward, and a short end-to-end training
on lattice-generated quotes showing what the network gains over the closed-form
baseline alone (the method without it)."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def test_mlp_gradient_matches_oracle(cuda):
    from oplib_b200 import _lib
    from oplib_b200.model import bind_stream
    lib = _lib.load()
    n = lib.opb_mlp_param_count()
    B = 256
    theta = torch.empty(n, dtype=torch.float32, device=cuda)
    thb = torch.empty_like(theta)
    bind_stream(cuda)
    assert lib.opb_mlp_init(theta.data_ptr(), 42) == 0
    assert lib.opb_mlp_round(theta.data_ptr(), thb.data_ptr(), None) == 0
    rng = np.random.default_rng(1)
    X = torch.from_numpy(rng.uniform(-1, 1, (B, 8)).astype(np.float32)).to(cuda)
    t = torch.from_numpy((rng.standard_normal(B) * 0.3).astype(np.float32)).to(cuda)
    ws = torch.empty(int(lib.opb_mlp_workspace_floats(B)), dtype=torch.float32, device=cuda)
    grad = torch.empty(n, dtype=torch.float32, device=cuda)
    loss = torch.zeros(1, dtype=torch.float64, device=cuda)
    assert lib.opb_mlp_loss_grad(thb.data_ptr(), X.data_ptr(), t.data_ptr(), B, ws.data_ptr(), grad.data_ptr(),
                                 loss.data_ptr()) == 0
    torch.cuda.synchronize()
    th = thb.cpu().numpy().astype(np.float64)  # the BF16 working weights are what the kernels differentiate
    ref_loss, ref_g = M.loss_grad(th, X.cpu().numpy(), t.cpu().numpy())
    g = grad.cpu().numpy().astype(np.float64) * B  # kernels return the gradient of the mean
    assert abs(loss.item() - ref_loss) <= 1e-4 * ref_loss
    # FP32 accumulation over B rows and 256-wide layers: relative to the gradient's scale
    assert np.abs(g - ref_g).max() <= 2e-4 * np.abs(ref_g).max()
    for lo, hi in [(0, 2048), (2304, 2304 + 65536), (199937 - 257, 199937)]:
        assert np.abs(g[lo:hi] - ref_g[lo:hi]).max() <= 2e-4 * np.abs(ref_g[lo:hi]).max() + 1e-12


def test_adam_step_decreases_loss(cuda):
    from oplib_b200 import _lib
    from oplib_b200.model import bind_stream
    lib = _lib.load()
    n = lib.opb_mlp_param_count()
    B = 1024
    theta = torch.empty(n, dtype=torch.float32, device=cuda)
    thb, m, v = torch.empty_like(theta), torch.zeros_like(theta), torch.zeros_like(theta)
    bind_stream(cuda)
    lib.opb_mlp_init(theta.data_ptr(), 7)
    lib.opb_mlp_round(theta.data_ptr(), thb.data_ptr(), None)
    rng = np.random.default_rng(2)
    Xn = rng.uniform(-1, 1, (B, 8))
    X = torch.from_numpy(Xn.astype(np.float32)).to(cuda)
    t = torch.from_numpy(np.sin(2 * Xn[:, 0]) * np.cos(Xn[:, 6]).astype(np.float32)).float().to(cuda)
    ws = torch.empty(int(lib.opb_mlp_workspace_floats(B)), dtype=torch.float32, device=cuda)
    grad = torch.empty(n, dtype=torch.float32, device=cuda)
    loss = torch.zeros(1, dtype=torch.float64, device=cuda)
    losses = []
    for step in range(1, 201):
        assert lib.opb_mlp_loss_grad(thb.data_ptr(), X.data_ptr(), t.data_ptr(), B, ws.data_ptr(), grad.data_ptr(),
                                     loss.data_ptr()) == 0
        losses.append(loss.item() / B)
        assert lib.opb_mlp_adam(theta.data_ptr(), m.data_ptr(), v.data_ptr(), grad.data_ptr(), step, 1e-3, 0.9,
                                0.999, 1e-8, thb.data_ptr()) == 0
    assert losses[-1] < 0.05 * losses[0]


def test_tensor_core_inference_matches_training_forward(cuda):
    from oplib_b200.surrogate import Surrogate
    s = Surrogate(members=2, device=cuda)
    import oplib_b200._lib as L
    for m in range(2):
        L.call("opb_mlp_pack", s.theta[m].data_ptr(), s.packed[m * s.stride:].data_ptr())
    rng = np.random.default_rng(3)
    n = 1000  # not a multiple of 128: padded internally
    feat = torch.from_numpy(np.column_stack([rng.uniform(lo, hi, n) for lo, hi in
                                             [(0.1, 0.4), (-0.3, 0.3), (0.2, 1.0), (0, 0), (0, 0), (0, 0.05),
                                              (-0.7, 0.4), (0.05, 2.0)]])).to(cuda)
    base = torch.zeros(n, dtype=torch.float64, device=cuda)
    mean, spread = s.predict(feat, base)
    y0 = s.forward_simt(feat, 0).double()
    y1 = s.forward_simt(feat, 1).double()
    from oplib_b200.surrogate import TARGET_SCALE
    ref_mean = TARGET_SCALE * 0.5 * (y0 + y1)
    ref_spread = TARGET_SCALE * (y0 - y1).abs()
    # BF16 activations on the tensor-core path vs FP32 activations in training: ~1% of scale
    scale = ref_mean.abs().max().item()
    assert (mean - ref_mean).abs().max().item() <= 0.02 * scale + 1e-6
    assert (spread - ref_spread).abs().max().item() <= 0.04 * scale + 1e-6


@pytest.mark.parametrize("n,members", [(1000, 2), (128, 1), (148 * 128 * 3 + 7, 4), (1 << 18, 3)])
def test_fused_inference_is_bit_identical_to_the_layers(cuda, n, members):
    """One fused kernel per member (activations in shared memory, two tiles in flight per
    CTA) against one launch per layer: the same products, GELU and roundings, so the same
    bits -- with an odd number of tiles per CTA, fewer tiles than SMs, and padded rows."""
    from oplib_b200 import _lib as L
    from oplib_b200.surrogate import RANGES, Surrogate
    lib = L.load()
    s = Surrogate(members=members, device=cuda)
    for m in range(members):
        L.call("opb_mlp_pack", s.theta[m].data_ptr(), s.packed[m * s.stride:].data_ptr())
    rng = np.random.default_rng(n)
    feat = torch.from_numpy(np.column_stack([rng.uniform(lo, hi, n) for lo, hi in RANGES])).to(cuda)
    base = torch.zeros(n, dtype=torch.float64, device=cuda)
    out = {}
    try:
        for fused in (1, 0):
            assert lib.opb_mlp_set_fused_inference(fused) == 0
            mean, spread = s.predict(feat, base)
            torch.cuda.synchronize()
            out[fused] = (mean.clone(), spread.clone())
    finally:
        assert lib.opb_mlp_set_fused_inference(1) == 0
    assert lib.opb_tc_error() == 0
    assert torch.isfinite(out[1][0]).all()
    assert torch.equal(out[1][0], out[0][0])
    assert torch.equal(out[1][1], out[0][1])


@pytest.mark.timeout(900)
def test_surrogate_improves_on_baseline(cuda):
    """Short training on lattice quotes: the network's error is well below the closed-form
    baseline's on held-out lattices, and the ensemble spread flags the worst quotes."""
    from oplib_b200.surrogate import Surrogate, lattice_quotes
    train = lattice_quotes(128, seed=11, device=cuda)
    test = lattice_quotes(32, seed=99, device=cuda)
    s = Surrogate(members=2, device=cuda)
    s.train(train, epochs=6, batch=4096, lr=2e-3)
    iv, spread = s.predict(test.feat, test.base)
    err_net = (iv - test.iv).abs()
    err_base = (test.base - test.iv).abs()
    print(f"baseline RMS {err_base.pow(2).mean().sqrt().item()*1e4:.1f} bp, "
          f"network RMS {err_net.pow(2).mean().sqrt().item()*1e4:.1f} bp")
    assert err_net.pow(2).mean().sqrt() < 0.5 * err_base.pow(2).mean().sqrt()


def test_tensor_core_inference_matches_the_fp64_oracle(cuda):
    """Each member's tensor-core inference against the oracle's FP64 restatement of the same
    numerics (BF16 weights, inputs and stored activations, exact-erf GELU): within 0.5% of
    the output's scale (and at least 1 bp) at every quote, 0.2 bp RMS.  What is left is FP32
    accumulation order, which now and then flips an activation's BF16 rounding (one BF16 ulp,
    2^-8 relative), and the GELU's erf approximation.  The untrained networks' outputs span
    several hundred bp of implied vol, far more than trained ones."""
    from oplib_b200.surrogate import TARGET_SCALE, Surrogate, normalise
    s = Surrogate(members=2, device=cuda)
    import oplib_b200._lib as L
    for m in range(2):
        L.call("opb_mlp_pack", s.theta[m].data_ptr(), s.packed[m * s.stride:].data_ptr())
    rng = np.random.default_rng(5)
    n = 3000
    feat = torch.from_numpy(np.column_stack([rng.uniform(lo, hi, n) for lo, hi in
                                             [(0.1, 0.4), (-0.3, 0.3), (0.2, 1.0), (0, 0), (0, 0), (0, 0.05),
                                              (-0.7, 0.4), (0.05, 2.0)]])).to(cuda)
    base = torch.zeros(n, dtype=torch.float64, device=cuda)
    X = normalise(feat).cpu().numpy()
    # member 0 alone (members=1) and the two-member mean
    y0 = M.forward_inference(s.theta[0].cpu().numpy(), X)
    y1 = M.forward_inference(s.theta[1].cpu().numpy(), X)
    for nmem, ref in ((1, y0), (2, 0.5 * (y0 + y1))):
        mean, spread = s.predict(feat, base, members=nmem)
        err_bp = np.abs(mean.cpu().numpy() - TARGET_SCALE * ref) * 1e4
        scale_bp = TARGET_SCALE * np.abs(ref).max() * 1e4
        print(f"{nmem} member(s): max {err_bp.max():.3f} bp, RMS {np.sqrt((err_bp ** 2).mean()):.4f} bp, "
              f"output scale {scale_bp:.1f} bp")
        assert err_bp.max() <= max(1.0, 0.005 * scale_bp)
        assert np.sqrt((err_bp ** 2).mean()) <= 0.2
    sp_ref = TARGET_SCALE * np.abs(y0 - y1)
    assert np.abs(spread.cpu().numpy() - sp_ref).max() * 1e4 <= max(2.0, 0.01 * scale_bp)


@pytest.mark.timeout(900)
def test_surrogate_meets_the_5bp_bar_on_accepted_quotes(cuda):
    """The seeded training run of the benchmark (2600 lattices, about 2^21 quotes after the
    vega filter, four members, 40 epochs): on quotes of 128 held-out lattices, the quotes
    the ensemble accepts (spread <= 5 bp) are within 5 bp of the lattice's implied vol at
    the 99th percentile, and at most 10% of the quotes fall back to the lattice."""
    from oplib_b200.surrogate import Surrogate, lattice_quotes
    train = lattice_quotes(2600, seed=2026, device=cuda)
    test = lattice_quotes(128, seed=99, device=cuda)
    s = Surrogate(members=4, device=cuda)
    s.train(train, epochs=40, batch=4096, lr=2e-3)
    iv, spread = s.predict(test.feat, test.base)
    err = ((iv - test.iv).abs() * 1e4).cpu().numpy()
    acc = (spread * 1e4 <= 5.0).cpu().numpy()
    fb = 1.0 - acc.mean()
    p99 = float(np.quantile(err[acc], 0.99))
    print(f"train {train.feat.shape[0]} quotes, {s.train_seconds:.1f} s; test {err.size} quotes: accepted p99 "
          f"{p99:.2f} bp, RMS {np.sqrt((err[acc] ** 2).mean()):.2f} bp, fallback {100 * fb:.2f}%, all-quote p99 "
          f"{np.quantile(err, 0.99):.2f} bp")
    assert p99 <= 5.0
    assert fb <= 0.10
