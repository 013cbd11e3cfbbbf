"""Host-side pieces of the surrogate on the CPU: feature scaling and the closed-form
baseline the network corrects (no GPU: both are plain torch arithmetic)."""
import numpy as np
import torch

from oplib_b200.surrogate import RANGES, baseline_iv, normalise


def test_normalise_maps_the_feature_ranges_onto_the_unit_box():
    lo = torch.tensor(RANGES[:, 0], dtype=torch.float64)
    hi = torch.tensor(RANGES[:, 1], dtype=torch.float64)
    out = normalise(torch.stack([lo, hi, 0.5 * (lo + hi)]))
    assert out.dtype == torch.float32 and out.is_contiguous()
    assert torch.equal(out[0], -torch.ones(8)) and torch.equal(out[1], torch.ones(8))
    assert torch.allclose(out[2], torch.zeros(8), atol=1e-7)


def test_baseline_of_a_flat_smile_is_its_level():
    """The quadrature weights sum to one, so sigma(x) = level gives level exactly."""
    n = 50
    rng = np.random.default_rng(1)
    level = torch.tensor(rng.uniform(0.1, 0.4, n))
    lm = torch.tensor(rng.uniform(-0.7, 0.4, n))
    T = torch.tensor(rng.uniform(0.05, 2.0, n))
    iv = baseline_iv(level, torch.zeros(n), torch.full((n,), 0.5), lm, T)
    assert torch.allclose(iv, level, rtol=1e-13, atol=0)


def test_baseline_at_the_money_short_dated_is_the_spot_vol():
    level, skew, width = torch.tensor([0.2, 0.3]), torch.tensor([0.1, -0.15]), torch.tensor([0.5, 0.3])
    iv = baseline_iv(level.double(), skew.double(), width.double(), torch.zeros(2, dtype=torch.float64),
                     torch.full((2,), 1e-12, dtype=torch.float64))
    assert torch.allclose(iv, (level + skew).double(), rtol=1e-9)


def test_baseline_follows_the_skew():
    """A bump of vol centred at the spot: deep wings see less of it than the money."""
    n = 3
    lm = torch.tensor([-0.7, 0.0, 0.4], dtype=torch.float64)
    iv = baseline_iv(torch.full((n,), 0.2, dtype=torch.float64), torch.full((n,), 0.2, dtype=torch.float64),
                     torch.full((n,), 0.3, dtype=torch.float64), lm, torch.full((n,), 0.25, dtype=torch.float64))
    assert iv[1] > iv[0] and iv[1] > iv[2]
    assert torch.all(iv >= 0.2) and torch.all(iv <= 0.4)
