"""GPU parity of the batched (ragged) lattice solve: every lattice of a small uneven batch
against the FP64 oracle (<= 1e-5 absolute, the target accuracy) and against the
single-lattice solve of the same lattice; every launch configuration of the autotuner
gives the same quotes; the whole sweep replays from a CUDA graph."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPECS = [dict(n=128, level=0.25, skew=0.1, width=0.5, rate=0.02, floor=0.01),
         dict(n=384, level=0.15, skew=-0.2, width=0.3, rate=0.04, floor=0.01),
         dict(n=256, level=0.35, skew=0.25, width=0.9, rate=0.0, floor=0.01),
         dict(n=128, level=0.1, skew=-0.3, width=0.2, rate=0.05, floor=0.01),
         dict(n=512, level=0.2, skew=0.05, width=0.6, rate=0.03, floor=0.01)]
NMAT, PERIOD, DT0 = 4, 0.25, 2.0 ** -14
STRIKES = 0.5 + np.arange(32) / 31.0


def _oracle_quotes(spec):
    x = O.log_grid(spec["n"])
    sig = O.lv_sigma(x, spec["level"], spec["skew"], spec["width"], spec["floor"])
    L = O.lv_generator_fast(x, spec["rate"] * x, sig * x)
    V, _, _ = O.solve_lattice_fp64(L, x, STRIKES, spec["rate"], PERIOD, NMAT, DT0)
    return V[:, O.nearest_node(x), :]


@pytest.fixture(scope="module")
def batch_and_refs(cuda):
    from oplib_b200.model import Batch, Lattice
    lats = [Lattice.local_vol(device=cuda, **s) for s in SPECS]
    refs = [_oracle_quotes(s) for s in SPECS]
    b = Batch(lats, STRIKES, NMAT, PERIOD, DT0, mode="bf16x3", autotune=True)
    return lats, refs, b


def test_batch_vs_fp64_and_single(batch_and_refs):
    lats, refs, b = batch_and_refs
    q = b.execute().cpu().numpy()
    torch.cuda.synchronize()
    from oplib_b200 import _lib
    lib = _lib.load()
    assert lib.opb_tc_error() == 0
    ncfg = lib.opb_batch_num_configs()
    assert ncfg == 8 and b.config in range(ncfg) and len(b.tune_ms) == ncfg
    # the batch fuses the row normalisation into the products' epilogues; the single solve
    # does too here, so the two differ only where the single solve's pricing products run as
    # K-slices summed in FP64 (too few tiles to fill the GPU) and the batch's in one pass
    assert lib.opb_set_fused_normalisation(8192) == 0
    try:
        for i, lat in enumerate(lats):
            err = np.abs(q[i] - refs[i]).max()
            print(f"lattice {i} d={lat.d}: max abs err vs FP64 {err:.2e}")
            assert err <= 1e-5, (i, err)
            qs, _ = lat.solve(STRIKES, NMAT, PERIOD, DT0, mode="bf16x3")
            assert np.abs(q[i] - qs.cpu().numpy()).max() < 1e-6
    finally:
        assert lib.opb_set_fused_normalisation(-1) == 0


def test_batch_configs_agree(batch_and_refs):
    lats, refs, b = batch_and_refs
    from oplib_b200 import _lib
    outs = []
    for cfg in range(_lib.load().opb_batch_num_configs()):
        b.set_config(cfg)
        outs.append(b.execute().cpu().numpy())
    for o in outs[1:]:
        assert np.abs(o - outs[0]).max() < 2e-7
    # 128 x 256 tiles (one CTA or a CTA pair) issue the same MMAs per element and the same
    # 128-column row-sum partials as 128 x 128 ones: bit-identical results
    assert np.array_equal(outs[4], outs[0]) and np.array_equal(outs[5], outs[2])
    assert np.array_equal(outs[6], outs[0]) and np.array_equal(outs[7], outs[2])
    for i in range(len(lats)):
        assert np.abs(outs[1][i] - refs[i]).max() <= 1e-5


def test_batch_graph_replay(batch_and_refs, cuda):
    from oplib_b200.model import bind_stream
    lats, refs, b = batch_and_refs
    q0 = b.execute()
    q = torch.empty_like(q0)
    s = torch.cuda.Stream(cuda)
    s.wait_stream(torch.cuda.current_stream(cuda))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        bind_stream(cuda)
        g.capture_begin()
        b.execute(q)
        g.capture_end()
    torch.cuda.current_stream(cuda).wait_stream(s)
    bind_stream(cuda)
    q.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(q, q0)


def test_batch_fp32_mode(cuda):
    from oplib_b200.model import Batch, Lattice
    specs = SPECS[:3]
    lats = [Lattice.local_vol(device=cuda, **s) for s in specs]
    b = Batch(lats, STRIKES, NMAT, PERIOD, DT0, mode="fp32")
    q = b.execute().cpu().numpy()
    for i, s in enumerate(specs):
        assert np.abs(q[i] - _oracle_quotes(s)).max() <= 1e-5


def test_batch_rejects_bad_sizes(cuda):
    """Sizes off the 128 grid are padded; sizes beyond the plan's tables are refused."""
    from oplib_b200.model import Batch, Lattice
    lats = [Lattice.local_vol(n=8128, device=cuda)]
    with pytest.raises(Exception):
        Batch(lats, STRIKES, NMAT, PERIOD, DT0, mode="bf16x3", autotune=False)


def test_batch_fp16x3_mode(cuda):
    from oplib_b200.model import Batch, Lattice
    lats = [Lattice.local_vol(device=cuda, **s) for s in SPECS]
    b = Batch(lats, STRIKES, NMAT, PERIOD, DT0, mode="fp16x3")
    q = b.execute().cpu().numpy()
    for i, s in enumerate(SPECS):
        err = np.abs(q[i] - _oracle_quotes(s)).max()
        print(f"fp16x3 lattice {i}: {err:.2e}")
        assert err <= 1e-5


@pytest.mark.parametrize("mode", ["bf16x3", "fp16x3"])
def test_batch_of_sizes_off_the_128_grid(cuda, fused_single, mode):
    """Split-mode plans take lattices of any size: each is solved padded to the next multiple
    of 128 with absorbing states, so its quotes match the FP64 oracle of the unpadded lattice
    and the single-lattice solve (which pads the same way)."""
    from oplib_b200.model import Batch, Lattice
    specs = [dict(n=300, level=0.25, skew=0.1, width=0.5, rate=0.02, floor=0.01),
             dict(n=200, level=0.15, skew=-0.2, width=0.3, rate=0.04, floor=0.01),
             dict(n=640, level=0.35, skew=0.25, width=0.9, rate=0.0, floor=0.01),
             dict(n=1000, level=0.2, skew=0.05, width=0.6, rate=0.03, floor=0.01)]
    lats = [Lattice.local_vol(device=cuda, **s) for s in specs]
    b = Batch(lats, STRIKES, NMAT, PERIOD, DT0, mode=mode, autotune=False)
    for cfg in (0, 6):
        b.set_config(cfg)
        q = b.execute().cpu().numpy()
        for i, (lat, spec) in enumerate(zip(lats, specs)):
            err = np.abs(q[i] - _oracle_quotes(spec)).max()
            assert err <= 1e-5, (cfg, spec["n"], err)
            qs, _ = lat.solve(STRIKES, NMAT, PERIOD, DT0, mode=mode)
            assert np.abs(q[i] - qs.cpu().numpy()).max() < 1e-6, (cfg, spec["n"])
    qb = b.execute_bermudan(put=True).cpu().numpy()
    for i, lat in enumerate(lats):
        single = lat.bermudan(STRIKES, nmat=NMAT, period=PERIOD, dt0=DT0, mode=mode, put=True).cpu().numpy()
        assert np.abs(qb[i] - single).max() < 1e-6
    from oplib_b200 import _lib
    assert _lib.load().opb_tc_error() == 0
