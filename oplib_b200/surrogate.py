"""Learned surrogate pricer over the lattice solver.

An ensemble of MLPs (8 -> 256 x 4 -> 1, GELU) maps (vol level, skew, width, kappa, rho, r,
log-moneyness, T) to implied volatility.  Training data are quotes that the batched
lattice solver (``model.Batch``) produces, converted to implied volatilities on the
device; the networks are trained by the library's own forward/backward/Adam kernels
(``opb_mlp_*``) and evaluated on the tensor cores (``opb_mlp_infer``).  A quote whose
ensemble spread exceeds the tolerance (5 bp of volatility by default) falls back to the
lattice, which is also the reference for the surrogate's error.

Local-volatility rows fix kappa = rho = 0 (the stochastic-volatility columns are inputs
of the network but constant in the local-volatility training family).

The network predicts a correction to a closed-form baseline: the implied volatility is
approximated by the root-mean-square local volatility sigma(x) over the log-spot path
from S0 to the strike (the averaging rule for local-volatility smiles), spread by a
lognormal displacement of the path at T/2; the network learns (iv - baseline) / 0.05.
The baseline alone is "the method without the network".
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import call
from .model import Batch, Lattice, bind_stream

# feature ranges -> [-1, 1]
RANGES = np.array([[0.1, 0.4], [-0.3, 0.3], [0.2, 1.0], [0.0, 4.0], [-1.0, 1.0], [0.0, 0.05], [-0.7, 0.4],
                   [0.05, 2.0]])
TARGET_SCALE = 0.05
LM = np.linspace(-0.7, 0.4, 64)          # log-moneyness grid of the training quotes
PERIOD, NMAT = 0.125, 16                 # maturities 0.125 .. 2.0
_GL_X, _GL_W = np.polynomial.legendre.leggauss(6)
_GH_X, _GH_W = np.polynomial.hermite_e.hermegauss(7)  # probabilists' Hermite: weight exp(-z^2/2)


def _ptr(t):
    return None if t is None else t.data_ptr()


def normalise(feat: torch.Tensor) -> torch.Tensor:
    lo = torch.as_tensor(RANGES[:, 0], dtype=feat.dtype, device=feat.device)
    hi = torch.as_tensor(RANGES[:, 1], dtype=feat.dtype, device=feat.device)
    return (2.0 * (feat - lo) / (hi - lo) - 1.0).to(torch.float32).contiguous()


def baseline_iv(level, skew, width, lm, T, floor=0.01):
    """sqrt of the mean of sigma(x)^2, sigma(x) = max(floor, level + skew exp(-((x-1)/width)^2)),
    over x = exp(u * lm + s z), u in [0, 1] (Gauss-Legendre), z ~ N(0, 1) (Gauss-Hermite),
    s = sigma(1) sqrt(T / 2), S0 = 1."""
    dev = lm.device
    u = torch.as_tensor((_GL_X + 1.0) / 2.0, dtype=torch.float64, device=dev)
    wu = torch.as_tensor(_GL_W / 2.0, dtype=torch.float64, device=dev)
    z = torch.as_tensor(_GH_X, dtype=torch.float64, device=dev)
    wz = torch.as_tensor(_GH_W / math.sqrt(2 * math.pi), dtype=torch.float64, device=dev)
    sig1 = torch.clamp(level + skew, min=floor)
    s = (sig1 * torch.sqrt(T / 2.0)).view(-1, 1, 1)
    logx = lm.view(-1, 1, 1) * u.view(1, -1, 1) + s * z.view(1, 1, -1)
    x = torch.exp(logx)
    sig = level.view(-1, 1, 1) + skew.view(-1, 1, 1) * torch.exp(-((x - 1.0) / width.view(-1, 1, 1)) ** 2)
    w = wu.view(1, -1, 1) * wz.view(1, 1, -1)
    return torch.sqrt((torch.clamp(sig, min=floor) ** 2 * w).sum((-1, -2)))


@dataclass
class QuoteSet:
    feat: torch.Tensor      # [n, 8] raw features (float64)
    iv: torch.Tensor        # [n] lattice implied vol (float64)
    base: torch.Tensor      # [n] baseline iv
    lattice: torch.Tensor   # [n] index of the lattice that produced the quote


def lattice_quotes(nlat: int, seed: int, device, mode: str = "fp16x3", batch: int = 512,
                   sizes=(1024,)) -> QuoteSet:
    """Quotes of seeded random local-vol lattices (the calibration-sweep family) with
    64 strikes exp(LM) and 16 maturities, as implied volatilities.  ``sizes``: lattice
    node counts drawn uniformly.  The size is not a network input, so mixing sizes adds
    their discretisation differences to the targets as noise (measured: 8.4 bp RMS over
    n in 256..1024 against 3.1 bp at n = 1024 alone, same training); the default
    trains on one resolution, the one the fallback lattice uses."""
    rng = np.random.default_rng(seed)
    strikes = np.exp(LM)
    feats, ivs, bases, lidx = [], [], [], []
    for b0 in range(0, nlat, batch):
        nb = min(batch, nlat - b0)
        n = rng.choice(np.asarray(sizes), size=nb)
        level = rng.uniform(0.1, 0.4, nb)
        skew = rng.uniform(-0.3, 0.3, nb)
        width = rng.uniform(0.2, 1.0, nb)
        r = rng.uniform(0.0, 0.05, nb)
        lats = [Lattice.local_vol(n=int(n[i]), level=float(level[i]), skew=float(skew[i]), width=float(width[i]),
                                  rate=float(r[i]), floor=0.01, device=device) for i in range(nb)]
        bt = Batch(lats, strikes, NMAT, PERIOD, 2.0 ** -14, mode=mode, autotune=False)
        q = bt.execute()  # [nb, NMAT, 64]
        T = torch.arange(1, NMAT + 1, dtype=torch.float64, device=device) * PERIOD
        Kt = torch.as_tensor(strikes, dtype=torch.float64, device=device)
        rr = torch.as_tensor(r, dtype=torch.float64, device=device)
        # the quoted state is the grid node nearest 1: its value is the spot of the quotes
        s0 = torch.stack([lat.x[lat.y0] for lat in lats])
        price = q.reshape(-1).contiguous()
        Kf = Kt.repeat(nb * NMAT)
        Tf = T.repeat_interleave(64).repeat(nb)
        rf = rr.repeat_interleave(NMAT * 64)
        s0f = s0.repeat_interleave(NMAT * 64).contiguous()
        iv = torch.empty_like(price)
        bind_stream(device)
        call("opb_implied_vol", price.numel(), price.data_ptr(), Kf.data_ptr(), Tf.data_ptr(), rf.data_ptr(),
             s0f.data_ptr(), iv.data_ptr())
        lm = torch.log(Kf / s0f)
        P = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device).repeat_interleave(NMAT * 64)
        lev, sk, wd = P(level), P(skew), P(width)
        feat = torch.stack([lev, sk, wd, torch.zeros_like(lev), torch.zeros_like(lev), rf, lm, Tf], dim=1)
        # keep quotes whose implied vol is resolvable: time value well above the lattice
        # price accuracy (1e-6) -- vega * 5bp > 2e-7
        sq = iv * torch.sqrt(Tf)
        d1 = (-lm + (rf + 0.5 * iv * iv) * Tf) / sq
        vega = torch.exp(-0.5 * d1 * d1) / math.sqrt(2 * math.pi) * torch.sqrt(Tf)
        ok = torch.isfinite(iv) & (vega * 5e-4 > 2e-7)
        feats.append(feat[ok])
        ivs.append(iv[ok])
        bases.append(baseline_iv(lev[ok], sk[ok], wd[ok], lm[ok], Tf[ok]))
        lidx.append((torch.arange(nb, device=device) + b0).repeat_interleave(NMAT * 64)[ok])
        del bt
    return QuoteSet(torch.cat(feats), torch.cat(ivs), torch.cat(bases), torch.cat(lidx))


class Surrogate:
    """Ensemble of MLPs trained by the library's kernels."""

    def __init__(self, members: int = 4, device="cuda"):
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.nparam = self.lib.opb_mlp_param_count()
        self.members = members
        self.theta = torch.empty(members, self.nparam, dtype=torch.float32, device=self.device)
        self.pack_bytes = int(self.lib.opb_mlp_packed_bytes())
        self.stride = (self.pack_bytes + 255) // 256 * 256
        self.packed = torch.zeros(members * self.stride, dtype=torch.uint8, device=self.device)
        bind_stream(self.device)
        for m in range(members):
            call("opb_mlp_init", self.theta[m].data_ptr(), 1234 + 7919 * m)
        self.history = []

    def train(self, data: QuoteSet, epochs: int = 10, batch: int = 4096, lr: float = 1e-3, seed: int = 0,
              lr_final: float = 1e-5):
        """Adam with a cosine learning-rate decay from lr to lr_final over all steps; each
        member draws its own batch order (seed + 101 m).  One epoch of a member (batch
        gathers, opb_mlp_loss_grad, opb_mlp_adam_sched) is captured once in a CUDA graph
        and replayed every epoch after a fresh permutation, the members' graphs on their own
        streams so that their small kernels overlap."""
        X = normalise(data.feat)
        t = ((data.iv - data.base) / TARGET_SCALE).to(torch.float32).contiguous()
        n = X.shape[0]
        steps = n // batch
        if steps < 1:
            raise ValueError("fewer quotes than one batch")
        total = epochs * steps
        k = torch.arange(1, total + 1, dtype=torch.float64)
        lr_tab = (lr_final + 0.5 * (lr - lr_final) * (1 + torch.cos(math.pi * k / total))).float().to(self.device)
        t0 = time.perf_counter()
        dev = self.device
        main = torch.cuda.current_stream(dev)
        members = []
        for m in range(self.members):
            st = dict(
                theta=self.theta[m], thb=torch.empty_like(self.theta[m]), mom=torch.zeros_like(self.theta[m]),
                var=torch.zeros_like(self.theta[m]), step=torch.zeros(1, dtype=torch.int32, device=dev),
                perm=torch.empty(n, dtype=torch.int64, device=dev),
                xb=torch.empty(batch, X.shape[1], dtype=torch.float32, device=dev),
                tb=torch.empty(batch, dtype=torch.float32, device=dev),
                ws=torch.empty(int(self.lib.opb_mlp_workspace_floats(batch)), dtype=torch.float32, device=dev),
                grad=torch.empty(self.nparam, dtype=torch.float32, device=dev),
                loss=torch.zeros(1, dtype=torch.float64, device=dev),
                ep_loss=torch.zeros(1, dtype=torch.float64, device=dev),
                gen=torch.Generator(device=dev), stream=torch.cuda.Stream(dev))
            st["gen"].manual_seed(seed + 101 * m)
            bind_stream(dev)
            call("opb_mlp_round", st["theta"].data_ptr(), st["thb"].data_ptr(), None)
            members.append(st)
        torch.cuda.synchronize(dev)

        def epoch(st):
            for s in range(steps):
                idx = st["perm"][s * batch:(s + 1) * batch]
                torch.index_select(X, 0, idx, out=st["xb"])
                torch.index_select(t, 0, idx, out=st["tb"])
                call("opb_mlp_loss_grad", st["thb"].data_ptr(), st["xb"].data_ptr(), st["tb"].data_ptr(), batch,
                     st["ws"].data_ptr(), st["grad"].data_ptr(), st["loss"].data_ptr())
                call("opb_mlp_adam_sched", st["theta"].data_ptr(), st["mom"].data_ptr(), st["var"].data_ptr(),
                     st["grad"].data_ptr(), st["step"].data_ptr(), lr_tab.data_ptr(), 0.9, 0.999, 1e-8,
                     st["thb"].data_ptr())
                st["ep_loss"].add_(st["loss"])

        # one gradient evaluation per member outside the capture (it changes no weights), so
        # that every kernel's one-time set-up has run before the capture
        for st in members:
            torch.index_select(X, 0, st["perm"][:batch].copy_(torch.arange(batch, device=dev)), out=st["xb"])
            torch.index_select(t, 0, st["perm"][:batch], out=st["tb"])
            call("opb_mlp_loss_grad", st["thb"].data_ptr(), st["xb"].data_ptr(), st["tb"].data_ptr(), batch,
                 st["ws"].data_ptr(), st["grad"].data_ptr(), st["loss"].data_ptr())
        torch.cuda.synchronize(dev)
        for st in members:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(st["stream"]):
                bind_stream(dev)
                g.capture_begin()
                epoch(st)
                g.capture_end()
            st["graph"] = g
        bind_stream(dev)
        for ep in range(epochs):
            for st in members:
                st["stream"].wait_stream(main)
                with torch.cuda.stream(st["stream"]):
                    st["perm"].copy_(torch.randperm(n, device=dev, generator=st["gen"]))
                    st["ep_loss"].zero_()
                    st["graph"].replay()
            for m, st in enumerate(members):
                main.wait_stream(st["stream"])
                self.history.append((m, ep, st["ep_loss"].clone()))
        torch.cuda.synchronize(dev)
        self.history = [(m, ep, float(v.item()) / (steps * batch)) if torch.is_tensor(v) else (m, ep, v)
                        for m, ep, v in self.history]
        bind_stream(dev)
        for m, st in enumerate(members):
            call("opb_mlp_pack", st["theta"].data_ptr(), self.packed[m * self.stride:].data_ptr())
            st["graph"].reset()
        torch.cuda.synchronize(dev)
        self.train_seconds = time.perf_counter() - t0
        return self.history

    def predict(self, feat: torch.Tensor, base: torch.Tensor, ws: torch.Tensor | None = None,
                members: int | None = None):
        """Ensemble mean implied vol and spread (max - min) on the tensor cores, over the
        first ``members`` members (default: all; at least 2 for a spread)."""
        nmem = self.members if members is None else int(members)
        if not 1 <= nmem <= self.members:
            raise ValueError("members out of range")
        X = normalise(feat)
        n = X.shape[0]
        need = int(self.lib.opb_mlp_infer_workspace_bytes(n, nmem))
        if ws is None or ws.numel() < need:
            ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        mean = torch.empty(n, dtype=torch.float32, device=self.device)
        spread = torch.empty(n, dtype=torch.float32, device=self.device)
        bind_stream(self.device)
        call("opb_mlp_infer", self.packed.data_ptr(), nmem, self.stride, X.data_ptr(), n, ws.data_ptr(),
             ws.numel(), mean.data_ptr(), spread.data_ptr())
        return base + TARGET_SCALE * mean.double(), TARGET_SCALE * spread.double()

    def forward_simt(self, feat: torch.Tensor, member: int = 0) -> torch.Tensor:
        """FP32 forward of one member with its BF16 working weights (the training path)."""
        X = normalise(feat)
        n = X.shape[0]
        thb = torch.empty(self.nparam, dtype=torch.float32, device=self.device)
        ws = torch.empty(int(self.lib.opb_mlp_workspace_floats(n)), dtype=torch.float32, device=self.device)
        y = torch.empty(n, dtype=torch.float32, device=self.device)
        bind_stream(self.device)
        call("opb_mlp_round", self.theta[member].data_ptr(), thb.data_ptr(), None)
        call("opb_mlp_forward", thb.data_ptr(), X.data_ptr(), n, ws.data_ptr(), y.data_ptr())
        return y
