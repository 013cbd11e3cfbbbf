"""Row normalisation fused into the products' epilogues against the renormalisation kernel.

With fusion (``opb_set_fused_normalisation``), a squaring writes the next level's 16-bit parts
itself, and the next level applies the deferred normalisation D = diag(1/(1+s)) in its
epilogue: D [E'.E' - S E' - E' S + S^2] + 2 D (E' - S), the D between the two factors left
out; a chain product writes only its parts and the next product (and the quote's discount)
applies its row scaling.  Without it, a kernel renormalises after every product.  The two
forms differ by FP32 rounding (and the dropped D, a relative 1e-5 at most): quotes agree
within 1e-6 and both stay within 1e-5 of the FP64 oracle.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

STRIKES = 0.5 + np.arange(32) / 31.0


@pytest.fixture()
def knob(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    yield lib
    assert lib.opb_set_fused_normalisation(-1) == 0  # the default


def _lv_ref(n, nmat, dt0, **p):
    """FP64 values of every state [nmat, n, nK] and the quoted state's index."""
    x = O.log_grid(n)
    L = O.lv_generator_fast(x, p["rate"] * x, O.lv_sigma(x, p["level"], p["skew"], p["width"], p["floor"]) * x)
    V, _, _ = O.solve_lattice_fp64(L, x, STRIKES, p["rate"], 0.25, nmat, dt0)
    return V, O.nearest_node(x)


@pytest.mark.parametrize("mode", ["bf16x3", "fp16x3"])
@pytest.mark.parametrize("n", [512, 1280])
def test_fused_and_kernel_normalisation_agree_single(knob, mode, n):
    from oplib_b200.model import Lattice
    p = dict(level=0.25, skew=0.15, width=0.4, rate=0.03, floor=0.01)
    lat = Lattice.local_vol(n=n, **p)
    out = {}
    for max_d in (4096, 0):
        assert knob.opb_set_fused_normalisation(max_d) == 0
        q, V = lat.solve(STRIKES, 8, 0.25, 2.0 ** -14, mode=mode, all_states=True)
        out[max_d] = (q.cpu().numpy(), V.cpu().numpy())
    assert knob.opb_tc_error() == 0
    Vref, y0 = _lv_ref(n, 8, 2.0 ** -14, **p)
    for q, _ in out.values():
        assert np.abs(q - Vref[:, y0, :]).max() <= 1e-5
    assert np.abs(out[4096][0] - out[0][0]).max() <= 1e-6
    # every state's values (deep in the money up to 4.5, where split-BF16 reaches about
    # 1.5e-5 of the value in either form): the fused form is as close to FP64 as the kernel
    # form, relative to each value's size
    rel = {k: (np.abs(V - Vref) / np.maximum(1.0, np.abs(Vref))).max() for k, (_, V) in out.items()}
    print(f"n={n} {mode}: all-state error relative to max(1, |V|): fused {rel[4096]:.2e}, kernel {rel[0]:.2e}")
    assert rel[4096] <= 1.25 * rel[0] + 1e-6


def test_fused_normalisation_on_the_sv_lattice(knob):
    """The SV lattice of config 1 (d = 6144) in both forms."""
    from oplib_b200.model import Lattice
    lat = Lattice.stoch_vol()
    K = np.linspace(0.5, 1.5, 128)
    out = {}
    for max_d in (0, 8192):
        assert knob.opb_set_fused_normalisation(max_d) == 0
        q, _ = lat.solve(K, 16, 0.25, 2.0 ** -16, mode="bf16x3")
        torch.cuda.synchronize()
        out[max_d] = q.cpu().numpy()
    assert knob.opb_tc_error() == 0
    assert np.abs(out[8192] - out[0]).max() <= 1e-6


def test_bermudan_fused_and_kernel_agree(knob):
    from oplib_b200.model import Lattice
    lat = Lattice.local_vol(n=768, level=0.2, skew=-0.1, width=0.5, rate=0.02, floor=0.01)
    out = {}
    for max_d in (4096, 0):
        assert knob.opb_set_fused_normalisation(max_d) == 0
        out[max_d] = lat.bermudan(STRIKES, nmat=8, period=0.25, dt0=2.0 ** -14, put=True).cpu().numpy()
    assert np.abs(out[4096] - out[0]).max() <= 1e-6
