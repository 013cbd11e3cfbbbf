"""Calibration of local-volatility lattices to option quotes, with the pricing on the device.

Each problem has the parameters theta = (level, skew, width) of
sigma(x) = max(floor, level + skew exp(-((x - 1) / width)^2)), on a lattice of its own
size and rate, and a block of target prices (maturities x strikes).  Many problems are
calibrated together by a damped Gauss-Newton (Levenberg-Marquardt) loop.  Every
iteration:

1. rewrites in place the device generators of every problem, at its trial point and at
   six parameter bumps for central differences (``opb_lv_params`` +
   ``opb_lv_generator_ell`` into the batch's ELL arrays);
2. prices all 7 x M lattices with one ``opb_batch_execute``, i.e. one persistent
   tensor-core launch and one renormalisation launch per squaring level;
3. per problem, on the host in FP64: accepts or rejects the trial, forms J^T J and J^T r
   from the bumped prices, and solves the damped 3 x 3 system for the next trial.

The targets are European calls (one batched ``opb_batch_execute`` per iteration) or, with
``contract="bermudan"``, Bermudan / down-and-out contracts priced by the batched backward
induction (``opb_batch_execute_bermudan``).

The reference lays out buffers for this loop but leaves it unwritten
(oplib/opmodel/types/SCalBuffers.cs:9-31: the discounted kernels at lambda = 1 +- eps,
kept for sensitivities).  Here the sensitivities come from bumped generators instead.

The batch plan (niter and dt per lattice) is fixed once, from generators at the largest
volatility the parameter box allows.  Every parameter inside the box then keeps
dt * max|L_yy| <= 1/2 (the plan rule of oplib/opmodel/models/CModel Common.cs:289-307),
and the plan stays valid as the parameters move.

``lm_calibrate`` is the host loop and takes any pricer; ``LVBatchPricer`` is the device
pricer.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import call
from .model import Batch, Lattice, bind_stream

# the record of opb_lv_generator_ell_batched
LV_PARAM = np.dtype([("n", "<i4"), ("pad", "<i4"), ("row_off", "<i8"), ("level", "<f8"), ("skew", "<f8"),
                     ("width", "<f8"), ("floor", "<f8"), ("rate", "<f8")])

# parameter box (level, skew, width) and the default bump sizes
BOX_LO = np.array([0.05, -0.4, 0.1])
BOX_HI = np.array([0.6, 0.4, 1.5])
BUMP = np.array([1e-3, 1e-3, 2e-3])


def lm_calibrate(price_fn, targets, theta0, lo=BOX_LO, hi=BOX_HI, h=BUMP, iters=30, lam0=1e-3, xtol=1e-7,
                 weights=None, max_step=0.1, central=True, ftol=0.0):
    """Levenberg-Marquardt over M independent problems of 3 parameters.

    ``price_fn(pts)`` takes pts[M, S, 3] and returns prices[M, S, K].  Slot 0 is the
    trial point.  With ``central`` (S = 7), slots 1 + 2j and 2 + 2j are the trial point
    moved up and down by h_j along parameter j, clipped to the box; otherwise (S = 4)
    slot 1 + j is moved by s_j h_j, with s_j = -1 at the upper bound.  Central differences
    matter: along the level/skew valley of wide bumps, the O(h) error of one-sided
    differences stalls the iteration.  ``targets`` is [M, K], and ``weights`` (optional,
    [M, K]) scales the residuals.  A step is limited to ``max_step`` of the box width per
    parameter, a trust region that stops flat directions (such as the width at small
    skew) from throwing the trial to the box boundary.  A problem stops when a step moves
    no parameter by more than ``xtol`` or its RMS residual falls below ``ftol`` (set
    ``ftol`` near the pricer's own noise).  Returns a dict with the fitted
    theta[M, 3], the weighted RMS residual per problem, the iterations used and the
    number of price_fn calls."""
    targets = np.asarray(targets, dtype=np.float64)
    M, K = targets.shape
    w = np.ones_like(targets) if weights is None else np.asarray(weights, dtype=np.float64)
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    h = np.asarray(h, dtype=np.float64)
    S = 7 if central else 4
    theta = np.clip(np.asarray(theta0, dtype=np.float64), lo, hi)
    trial = theta.copy()
    cost = np.full(M, np.inf)
    lam = np.full(M, lam0)
    J = np.zeros((M, 3, K))
    r = np.zeros((M, K))
    done = np.zeros(M, dtype=bool)
    calls = 0
    it = 0
    for it in range(1, iters + 1):
        pts = np.repeat(trial[:, None, :], S, axis=1)
        if central:
            up = np.minimum(trial + h, hi)
            dn = np.maximum(trial - h, lo)
            for j in range(3):
                pts[:, 1 + 2 * j, j] = up[:, j]
                pts[:, 2 + 2 * j, j] = dn[:, j]
            span = up - dn
        else:
            sgn = np.where(trial + h > hi, -1.0, 1.0)
            for j in range(3):
                pts[:, j + 1, j] += sgn[:, j] * h[j]
        q = np.asarray(price_fn(pts), dtype=np.float64).reshape(M, S, K)
        calls += 1
        r_t = w * (q[:, 0] - targets)
        cost_t = np.sum(r_t * r_t, axis=1)
        acc = (cost_t < cost) & ~done
        theta[acc] = trial[acc]
        cost[acc] = cost_t[acc]
        r[acc] = r_t[acc]
        for j in range(3):
            if central:
                J[acc, j] = w[acc] * (q[acc, 1 + 2 * j] - q[acc, 2 + 2 * j]) / span[acc, j, None]
            else:
                J[acc, j] = w[acc] * (q[acc, j + 1] - q[acc, 0]) / (sgn[acc, j, None] * h[j])
        lam = np.where(acc, lam * 0.3, np.where(done, lam, lam * 10.0))
        # next trial from the accepted point's Jacobian
        A = np.einsum("mik,mjk->mij", J, J)
        g = np.einsum("mik,mk->mi", J, r)
        dA = np.einsum("mii->mi", A)
        Ad = A + (lam[:, None] * dA + 1e-30)[:, :, None] * np.eye(3)[None]
        step = -np.linalg.solve(Ad, g[:, :, None])[:, :, 0]
        smax = max_step * (hi - lo)
        step = np.clip(step, -smax, smax)
        new = np.clip(theta + step, lo, hi)
        moved = np.max(np.abs(new - theta), axis=1)
        done |= acc & ((moved < xtol) | (np.sqrt(cost / K) < ftol))
        done |= lam > 1e12
        trial = np.where(done[:, None], theta, new)
        if done.all():
            break
    return {"theta": theta, "rms": np.sqrt(cost / K), "iterations": it, "calls": calls, "done": done}


# Starting points: the fit is not convex (at skew = 0 the width has no effect, and the
# path can settle on the width bound), so each problem starts from both skew signs.
STARTS = np.array([[0.2, 0.1, 0.5], [0.2, -0.1, 0.5]])


def multistart(targets, starts=STARTS):
    """Replicates M problems over S starts: returns (targets[S*M, K], theta0[S*M, 3]),
    start-major (problem i of start s at s*M + i)."""
    targets = np.asarray(targets, dtype=np.float64)
    M = targets.shape[0]
    S = len(starts)
    return np.tile(targets, (S, 1)), np.repeat(np.asarray(starts, dtype=np.float64), M, axis=0)


def best_of_starts(out, M: int):
    """Per problem, the start with the smallest residual: (theta[M, 3], rms[M])."""
    rms = out["rms"].reshape(-1, M)
    best = np.argmin(rms, axis=0)
    theta = out["theta"].reshape(-1, M, 3)[best, np.arange(M)]
    return theta, rms[best, np.arange(M)]


class LVBatchPricer:
    """Device pricer for ``lm_calibrate``: ``slots`` local-vol lattices per problem (the
    trial point and its bumps; 7 for central differences) in one batch whose generators
    are rewritten in place per call.  ``contract`` selects the quotes: "european" (calls
    at the nmat maturities m * period, nmat * nK per problem) or "bermudan" (one value per
    strike of the contract maturing at nmat * period: calls or puts (``put``) exercisable
    at every m * period, knocked out at or below ``barrier`` when it is positive)."""

    def __init__(self, n, rate, strikes, nmat: int, period: float, dt0: float = 2.0 ** -14, mode="fp16x3",
                 floor: float = 0.01, lo: float = 0.05, hi: float = 5.0, s0: float = 1.0, slots: int = 7,
                 device="cuda", contract: str = "european", put: bool = True, barrier: float = 0.0):
        if contract not in ("european", "bermudan"):
            raise ValueError(f"contract must be 'european' or 'bermudan', not {contract!r}")
        self.contract, self.put, self.barrier = contract, bool(put), float(barrier)
        self.n = [int(v) for v in n]
        self.rate = [float(v) for v in rate]
        self.M = len(self.n)
        self.S = int(slots)
        self.floor, self.lo, self.hi, self.s0 = floor, lo, hi, s0
        self.device = torch.device(device)
        bind_stream(self.device)
        vmax = float(BOX_HI[0] + max(BOX_HI[1], 0.0))
        # plan from the box's largest volatility: constant sigma = vmax bounds max|L_yy|
        lats = [Lattice.local_vol(n=self.n[i], level=vmax, skew=0.0, width=1.0, rate=self.rate[i], floor=floor,
                                  lo=lo, hi=hi, s0=s0, device=self.device)
                for i in range(self.M) for _ in range(self.S)]
        self.batch = Batch(lats, strikes, nmat, period, dt0, mode=mode, autotune=False)
        self.K = (nmat if contract == "european" else 1) * self.batch.nK
        # one 56-byte record per lattice for opb_lv_generator_ell_batched
        nlat = self.M * self.S
        self.rec = np.zeros(nlat, dtype=LV_PARAM)
        self.rec["n"] = np.repeat(self.n, self.S)
        self.rec["row_off"] = np.concatenate([[0], np.cumsum(self.rec["n"])[:-1]])
        self.rec["floor"] = floor
        self.rec["rate"] = np.repeat(self.rate, self.S)
        self.total_rows = int(self.rec["n"].sum())
        self.h_rec = torch.empty(nlat * LV_PARAM.itemsize, dtype=torch.uint8).pin_memory()
        self.d_rec = torch.empty(nlat * LV_PARAM.itemsize, dtype=torch.uint8, device=self.device)
        self.calls = 0

    def __call__(self, pts: np.ndarray) -> np.ndarray:
        pts = np.asarray(pts, dtype=np.float64).reshape(self.M * self.S, 3)
        bind_stream(self.device)
        self.rec["level"], self.rec["skew"], self.rec["width"] = pts[:, 0], pts[:, 1], pts[:, 2]
        torch.cuda.current_stream(self.device).synchronize()  # the pinned staging buffer is free again
        self.h_rec.numpy()[:] = self.rec.view(np.uint8)
        self.d_rec.copy_(self.h_rec, non_blocking=True)
        call("opb_lv_generator_ell_batched", self.M * self.S, self.d_rec.data_ptr(), self.total_rows, self.lo,
             self.hi, self.s0, self.batch.cols.data_ptr(), self.batch.vals.data_ptr())
        if self.contract == "european":
            q = self.batch.execute()
        else:
            q = self.batch.execute_bermudan(put=self.put, exercise=True, barrier=self.barrier)
        self.calls += 1
        return q.reshape(self.M, self.S, self.K).cpu().numpy()

    def quotes(self, theta: np.ndarray) -> np.ndarray:
        """Prices [M, K] at theta[M, 3] (all slots at the same point)."""
        pts = np.repeat(np.asarray(theta, dtype=np.float64)[:, None, :], self.S, axis=1)
        return self(pts)[:, 0]
