"""Error budget of the split products on the SV lattice (d = 6144, 48 vol x 128 spot states).

Every squaring and chain product is the sum of three BF16 products, hi.hi + hi.lo + lo.hi
(lo.lo added on the first 8 squarings).  Dropping a cross term would save a third of a
product.  This test measures, by an emulation of the split arithmetic (BF16 parts exact in
FP32, FP32 products with TF32 off, FP64 sums and row renormalisation, as the library
forms them), what each cross term contributes to the quote error against the exact FP64
solve:

- with all terms the emulated error is 1.8e-6 (the library's own solve: 2.5e-6);
- dropping the cross terms at one late squaring (level 5 or above, the dense ones) or the
  hi.lo term in every chain product costs 2e-5 to 7e-5, above the 1e-5 bar.

So the split form keeps all three products wherever the product is dense; only the first
band-limited levels could drop a term, and they hold about 1/3 of a dense product's work.
"""
import math

import pytest
import torch

pytestmark = pytest.mark.gpu

NMAT, PERIOD, DT0 = 16, 0.25, 2.0 ** -16


@pytest.fixture(scope="module")
def sv(cuda):
    from oplib_b200.model import Lattice
    lat = Lattice.stoch_vol()
    d, w = lat.d, lat.width
    plan = lat.plan(PERIOD, DT0)
    cols = lat.cols.view(d, w).long()
    vals = lat.vals.view(d, w)
    L = torch.zeros(d, d, dtype=torch.float64, device=cuda)
    ok = (cols >= 0) & (cols < d)
    rows = torch.arange(d, device=cuda)[:, None].expand(d, w)
    L.index_put_((rows[ok], cols[ok]), vals[ok], accumulate=True)
    strikes = torch.linspace(0.5, 1.5, 128, dtype=torch.float64, device=cuda)
    G = torch.clamp(lat.x.double()[:, None] - strikes[None, :], min=0)
    return dict(L=L, G=G, y0=lat.y0, niter=plan.niter, dt=plan.dt, rate=lat.rate, d=d)


def _split(a, floor=False):
    if floor:  # the library's absolute floor: |a| < 2^-40 -> no parts, |a| < 2^-30 -> no lo part
        h = torch.where(a.abs() < 2.0 ** -40, 0.0, a).to(torch.bfloat16).float()
        return h, torch.where(a.abs() < 2.0 ** -30, 0.0, a - h.double()).to(torch.bfloat16).float()
    h = a.to(torch.bfloat16).float()
    return h, (a - h.double()).to(torch.bfloat16).float()


def _mm(a, b, terms, floor=False):
    ah, al = _split(a, floor)
    bh, bl = _split(b, floor)
    out = torch.mm(ah, bh).double()
    if "hl" in terms:
        out += torch.mm(ah, bl).double()
    if "lh" in terms:
        out += torch.mm(al, bh).double()
    if "ll" in terms:
        out += torch.mm(al, bl).double()
    return out


def _solve(s, sq_terms=None, ch_terms=None, floor=False):
    """Quotes at the spot state for 16 maturities x 128 strikes; exact FP64 when the term
    lists are None."""
    exact = sq_terms is None
    I = torch.eye(s["d"], dtype=torch.float64, device=s["L"].device)
    E = s["dt"] * s["L"]
    for r in range(s["niter"]):
        E = 2 * E + (E @ E if exact else _mm(E, E, sq_terms[r], floor))
        P = I + E
        E = P / P.sum(1, keepdim=True) - I
    P1 = I + E
    Pk, V = P1, []
    for k in range(NMAT):
        if k > 0:
            Pk = Pk @ P1 if exact else _mm(Pk, P1, ch_terms[k], floor)
            Pk = Pk / Pk.sum(1, keepdim=True)
        Vk = Pk @ s["G"] if exact else _mm(Pk, s["G"], "hl lh", floor)
        V.append(Vk[s["y0"]] * math.exp(-s["rate"] * PERIOD * (k + 1)))
    return torch.stack(V)


@pytest.fixture()
def no_tf32():
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    yield
    torch.backends.cuda.matmul.allow_tf32 = old


def test_cross_terms_are_needed_on_dense_products(sv, no_tf32):
    ref = _solve(sv)
    n = sv["niter"]
    full_sq = ["hl lh ll" if r < 8 else "hl lh" for r in range(n)]
    full_ch = ["hl lh"] * NMAT
    err = lambda v: float((v - ref).abs().max())
    e_full = err(_solve(sv, full_sq, full_ch))
    drops = {}
    for r in (5, n - 1):
        sq = list(full_sq)
        sq[r] = ""
        drops[f"squaring {r}, both cross terms"] = err(_solve(sv, sq, full_ch))
    drops["every chain product, hi.lo"] = err(_solve(sv, full_sq, ["lh"] * NMAT))
    print(f"all terms {e_full:.2e}; " + "; ".join(f"{k} dropped {v:.2e}" for k, v in drops.items()))
    assert e_full <= 3e-6
    for k, v in drops.items():
        assert v > 1e-5, k


def test_split_floor_costs_no_accuracy(sv, no_tf32):
    """The BF16 split's absolute floor (parts of entries below 2^-40 dropped, lo parts of
    entries below 2^-30 dropped) zeroes the far tails' parts, which otherwise stay live
    bit patterns through every product.  On the SV lattice the emulated quote error with the
    floor stays that of the unfloored split, and most tail entries of the dense operands
    are affected (printed: the share of zero lo parts of P1 with and without the floor)."""
    ref = _solve(sv)
    n = sv["niter"]
    sq = ["hl lh ll" if r < 8 else "hl lh" for r in range(n)]
    ch = ["hl lh"] * NMAT
    e_plain = float((_solve(sv, sq, ch) - ref).abs().max())
    e_floor = float((_solve(sv, sq, ch, floor=True) - ref).abs().max())
    I = torch.eye(sv["d"], dtype=torch.float64, device=sv["L"].device)
    E = sv["dt"] * sv["L"]
    for r in range(n):
        E = 2 * E + E @ E
        P = I + E
        E = P / P.sum(1, keepdim=True) - I
    P1 = (I + E).float().double()
    z_plain = float((_split(P1)[1] == 0).double().mean())
    z_floor = float((_split(P1, True)[1] == 0).double().mean())
    print(f"max error: plain split {e_plain:.3e}, floored {e_floor:.3e}; "
          f"zero lo parts of P1: {z_plain:.3f} plain, {z_floor:.3f} floored")
    assert e_floor <= 3e-6
    assert abs(e_floor - e_plain) <= 2e-7
