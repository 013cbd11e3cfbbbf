"""Host-side model API over the opcuda-b200 C ABI.

Mirrors the roles of the reference's managed model layer for this path:
``CLVModel``/``CSVModel`` build a generator (``mkgen``), ``CModel.make_mc_plan`` derives the
squaring plan, ``CModel.exe_mc_plan`` exponentiates and chains, and the Monte Carlo runs
over cumulative step kernels (``oplib/opmodel/models/CModel Common.cs:138-669``,
``CModel Device.cs:142-367``).  All arithmetic runs in the CUDA library; torch provides
device memory and streams only.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import LatticeDesc, call

FP32_PLAIN, FP32_RENORM, BF16X3, FP16X3 = 0, 1, 2, 3
MODES = {"fp32_plain": FP32_PLAIN, "fp32": FP32_RENORM, "fp32_renorm": FP32_RENORM, "bf16x3": BF16X3,
         "fp16x3": FP16X3}


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def bind_stream(device: torch.device | None = None) -> None:
    """Order library work on torch's current stream of ``device``."""
    dev = torch.device("cuda") if device is None else device
    _lib.load().opb_set_stream(_stream_handle(dev))


@dataclass
class Plan:
    niter: int
    dt: float
    maxdiag: float


class Lattice:
    """A discretised Markov generator on the device in ELL form (FP64) plus the spot
    value of every state.  Build with :meth:`local_vol` or :meth:`stoch_vol`."""

    def __init__(self, d: int, cols: torch.Tensor, vals: torch.Tensor, x: torch.Tensor, y0: int, rate: float):
        self.d, self.cols, self.vals, self.x, self.y0, self.rate = d, cols, vals, x, y0, rate
        self.width = cols.numel() // d
        self.device = x.device

    # ---------------------------------------------------------------- builders (mkgen)
    @classmethod
    def local_vol(cls, n=512, level=0.2, skew=0.1, width=0.5, rate=0.03, floor=0.0, lo=0.05, hi=5.0, s0=1.0,
                  device="cuda"):
        """Local-vol lattice on log-spaced nodes x_i = s0*lo*(hi/lo)^(i/(n-1)) with
        sigma(x) = max(floor, level + skew*exp(-((x-1)/width)^2)), drift r*x."""
        dev = torch.device(device)
        bind_stream(dev)
        x = torch.empty(n, dtype=torch.float64, device=dev)
        drift = torch.empty_like(x)
        vol = torch.empty_like(x)
        call("opb_lv_params", n, lo, hi, s0, level, skew, width, floor, rate, _ptr(x), _ptr(drift), _ptr(vol))
        return cls.from_drift_vol(x, drift, vol, rate, s0)

    @classmethod
    def from_drift_vol(cls, x: torch.Tensor, drift: torch.Tensor, vol: torch.Tensor, rate: float, s0: float = 1.0):
        """LV generator from per-node drift and vol (``CLVModel.mkgen``)."""
        n = x.numel()
        bind_stream(x.device)
        cols = torch.empty(3 * n, dtype=torch.int32, device=x.device)
        vals = torch.empty(3 * n, dtype=torch.float64, device=x.device)
        call("opb_lv_generator_ell", n, _ptr(x), _ptr(drift), _ptr(vol), _ptr(cols), _ptr(vals))
        y0 = int(torch.argmin(torch.abs(x - s0)).item())
        return cls(n, cols, vals, x.contiguous(), y0, rate)

    @classmethod
    def stoch_vol(cls, nx=128, nv=48, x_lo=0.05, x_hi=5.0, v_lo=0.05, v_hi=1.0, rate=0.03, kappa=2.0, theta=0.04,
                  xi=0.6, rho=-0.7, s0=1.0, device="cuda"):
        """2-D (spot, variance) lattice; the quoted state is the spot node nearest s0 at
        the vol state nearest sqrt(theta)."""
        dev = torch.device(device)
        bind_stream(dev)
        d = nx * nv
        cols = torch.empty(7 * d, dtype=torch.int32, device=dev)
        vals = torch.empty(7 * d, dtype=torch.float64, device=dev)
        x = torch.empty(d, dtype=torch.float64, device=dev)
        call("opb_sv_generator_ell", nx, nv, x_lo, x_hi, v_lo, v_hi, rate, kappa, theta, xi, rho, _ptr(cols),
             _ptr(vals), _ptr(x))
        ix = min(range(nx), key=lambda i: abs(x_lo * (x_hi / x_lo) ** (i / (nx - 1)) - s0))
        iv = min(range(nv), key=lambda j: abs(v_lo * (v_hi / v_lo) ** (j / (nv - 1)) - math.sqrt(theta)))
        return cls(d, cols, vals, x, ix + nx * iv, rate)

    # ---------------------------------------------------------------- plan
    def maxdiag(self) -> float:
        scratch = torch.empty(1, dtype=torch.int64, device=self.device)
        out = C.c_double()
        bind_stream(self.device)
        call("opb_ell_maxdiag", self.d, self.width, _ptr(self.cols), _ptr(self.vals), _ptr(scratch), C.byref(out))
        return out.value

    def plan(self, period: float, dt0: float, maxdiag: float | None = None) -> Plan:
        """``CModel Common.cs:289-307``: dt = min(0.5/max|L_yy|, dt0), niter = ceil(log2(period/dt))."""
        md = self.maxdiag() if maxdiag is None else maxdiag
        n = C.c_int()
        dt = C.c_double()
        call("opb_plan_interval", md, period, dt0, C.byref(n), C.byref(dt))
        return Plan(n.value, dt.value, md)

    # ---------------------------------------------------------------- solve
    def desc(self, plan: Plan, period: float, nmat: int, strikes: torch.Tensor | None) -> LatticeDesc:
        L = LatticeDesc()
        L.d, L.y0, L.ell_width = self.d, self.y0, self.width
        L.gen_cols, L.gen_vals, L.gen_dense, L.x = _ptr(self.cols), _ptr(self.vals), None, _ptr(self.x)
        L.dt, L.niter, L.nmat, L.period, L.rate = plan.dt, plan.niter, nmat, period, self.rate
        L.nK = 0 if strikes is None else strikes.numel()
        L.strikes = _ptr(strikes)
        return L

    def workspace(self, nK: int, mode: int) -> torch.Tensor:
        n = _lib.load().opb_lattice_workspace_size(self.d, nK, mode)
        return torch.empty(int(n), dtype=torch.uint8, device=self.device)

    def solve(self, strikes, nmat: int, period: float, dt0: float, mode="bf16x3", plan: Plan | None = None,
              all_states: bool = False, workspace: torch.Tensor | None = None):
        """Quotes[m, k] = exp(-r T_m) (P(T_m) G)[y0, k], T_m = m*period.  Returns
        (quotes [nmat, nK] FP64, V_all [nmat, d, nK] or None)."""
        mode = MODES[mode] if isinstance(mode, str) else mode
        strikes = torch.as_tensor(strikes, dtype=torch.float64, device=self.device)
        plan = plan or self.plan(period, dt0)
        ws = workspace if workspace is not None else self.workspace(strikes.numel(), mode)
        quotes = torch.empty(nmat, strikes.numel(), dtype=torch.float64, device=self.device)
        V = torch.empty(nmat, self.d, strikes.numel(), dtype=torch.float64, device=self.device) if all_states else None
        L = self.desc(plan, period, nmat, strikes)
        bind_stream(self.device)
        call("opb_lattice_solve", C.byref(L), mode, _ptr(ws), ws.numel(), _ptr(quotes), _ptr(V))
        return quotes, V

    def bermudan(self, strikes, nmat: int, period: float, dt0: float, mode="bf16x3", put: bool = False,
                 exercise: bool = True, barrier: float = 0.0, plan: Plan | None = None,
                 workspace: torch.Tensor | None = None) -> torch.Tensor:
        """Values at y0 [nK] (FP64) of calls or puts of maturity nmat*period by backward
        induction on P(period), exercisable at every m*period (``exercise``) and knocked
        out where the spot is at or below ``barrier`` on those dates (barrier > 0)."""
        mode = MODES[mode] if isinstance(mode, str) else mode
        strikes = torch.as_tensor(strikes, dtype=torch.float64, device=self.device)
        plan = plan or self.plan(period, dt0)
        ws = workspace if workspace is not None else self.workspace(strikes.numel(), mode)
        quotes = torch.empty(strikes.numel(), dtype=torch.float64, device=self.device)
        L = self.desc(plan, period, nmat, strikes)
        bind_stream(self.device)
        call("opb_lattice_bermudan", C.byref(L), mode, int(put), int(exercise), float(barrier), _ptr(ws), ws.numel(),
             _ptr(quotes))
        return quotes

    def kernel(self, period: float, dt0: float, mode="fp32", plan: Plan | None = None) -> torch.Tensor:
        """Transition kernel P(period) as a d x d FP32 source-major matrix."""
        mode = MODES[mode] if isinstance(mode, str) else mode
        plan = plan or self.plan(period, dt0)
        nk = 64
        ws = self.workspace(nk, mode)
        P = torch.empty(self.d, self.d, dtype=torch.float32, device=self.device)
        L = self.desc(plan, period, 1, None)
        L.nK = nk
        bind_stream(self.device)
        call("opb_lattice_kernel", C.byref(L), mode, _ptr(ws), ws.numel(), _ptr(P))
        return P


# -------------------------------------------------------------------- Monte Carlo

def cumulative_rows(P: torch.Tensor) -> torch.Tensor:
    """Cumulative normalised rows (``sck``) of a source-major FP32 kernel."""
    d = P.shape[1]
    Cm = torch.empty_like(P)
    bind_stream(P.device)
    call("opb_sck_rm", d, P.shape[0], _ptr(P), _ptr(Cm))
    return Cm


def guide_buckets(d: int) -> int:
    """Default guide-table width: the power of two nearest above 2 d, at most 4096.  Two
    buckets per state leave most brackets one or two states wide, so the inverse-CDF
    search takes about one probe (measured on the 512-state step kernel: 226.5e9
    path-steps/s at 1024 buckets against 153.0e9 at 64, with identical paths)."""
    nb = 1
    while nb < 2 * d and nb < 4096:
        nb *= 2
    return nb


def guide_table(Cm: torch.Tensor, nb: int | None = None) -> torch.Tensor:
    """Bracket table [rows, nb] of cumulative rows (``opb_guide_table``)."""
    d = Cm.shape[1]
    nb = guide_buckets(d) if nb is None else nb
    g = torch.empty(Cm.shape[0], nb, dtype=torch.int32, device=Cm.device)
    bind_stream(Cm.device)
    call("opb_guide_table", d, Cm.shape[0], nb, _ptr(Cm), _ptr(g))
    return g


def mc_run(Cm: torch.Tensor, y0: int, nsteps: int, seed: int, npaths: int, path0: int = 0,
           guide: torch.Tensor | None = None, nb: int | None = None, x: torch.Tensor | None = None, strike: float = 1.0,
           barrier: float = 0.7, disc: float = 1.0, want_paths: bool = False, scratch: torch.Tensor | None = None):
    """MT19937 Monte Carlo over ``npaths`` paths (ids path0..).  ``nb``: the guide table's
    width (default: from its shape).  Returns (sums[2] FP64 tensor or None, int16 paths
    [nsteps, npaths] or None)."""
    d = Cm.shape[1]
    if guide is not None and nb is None:
        nb = guide.shape[-1] if guide.dim() == 2 else 64
    dev = Cm.device
    ypaths = torch.empty(nsteps, npaths, dtype=torch.int16, device=dev) if want_paths else None
    sums = None
    if x is not None:
        nblk = _lib.load().opb_mc_scratch_blocks(npaths)
        if scratch is None or scratch.numel() < 2 * nblk:
            scratch = torch.empty(2 * nblk, dtype=torch.float64, device=dev)
        sums = torch.empty(2, dtype=torch.float64, device=dev)
    bind_stream(dev)
    call("opb_mc_mt19937", _ptr(Cm), d, 1, _ptr(guide), nb if guide is not None else 0, d, y0, nsteps,
         seed & 0xFFFFFFFF, path0, npaths, _ptr(ypaths), _ptr(x), strike, barrier, disc, _ptr(scratch), _ptr(sums))
    return sums, ypaths


# -------------------------------------------------------------------- batched lattices

def mc_plan_kernels(plan, lattices: list, mode="fp32") -> torch.Tensor:
    """Step kernels [nm, d, d] (FP32, source-major) of a Monte Carlo plan (``plan.McPlan``)
    on the device: each elementary kernel X_j = (I + dt_j L)^(2^niter_j) by the lattice
    solve's squarings under its generator ``lattices[plan.i_j[j]]``, then each step kernel
    the product of its elementary factors in time order (``opb_chain_kernels``), so a step
    that spans a generator date chains kernels of different generators."""
    dev = lattices[0].device
    d = lattices[0].d
    if any(lat.d != d for lat in lattices):
        raise ValueError("every generator of a plan lives on the same states")
    X = []
    for j in range(plan.nj):
        lat = lattices[plan.i_j[j]]
        delta_t = (plan.t1_j[j] - plan.t0_j[j]) / 365.25
        X.append(lat.kernel(delta_t, plan.dt_j[j], mode=mode, plan=Plan(plan.niter_j[j], plan.dt_j[j], 0.0)))
    lib = _lib.load()
    out = torch.empty(plan.nm, d, d, dtype=torch.float32, device=dev)
    ws = torch.empty(int(lib.opb_chain_workspace_size(d)), dtype=torch.uint8, device=dev)
    bind_stream(dev)
    for m, factors in enumerate(plan.jfactor_ms):
        ptrs = (C.c_void_p * len(factors))(*[X[j].data_ptr() for j in factors])
        call("opb_chain_kernels", d, len(factors), ptrs, out[m].data_ptr(), ws.data_ptr(), ws.numel())
    return out


class BatchDesc(C.Structure):
    """Mirror of ``opb_batch_desc``."""

    _fields_ = [
        ("nlat", C.c_int), ("d", C.c_void_p), ("y0", C.c_void_p), ("niter", C.c_void_p), ("dt", C.c_void_p),
        ("rate", C.c_void_p), ("ell_width", C.c_int), ("gen_cols", C.c_void_p), ("gen_vals", C.c_void_p),
        ("x", C.c_void_p), ("nmat", C.c_int), ("period", C.c_double), ("nK", C.c_int), ("strikes", C.c_void_p),
    ]


class Batch:
    """Many uneven lattices solved together (``opb_batch_*``): one persistent tensor-core
    launch per squaring level for all of them, whose epilogue writes the next level's
    operand parts and applies the deferred row normalisation.  In the split modes a lattice
    of a size off the 128 grid is solved padded with absorbing states."""

    def __init__(self, lattices: list, strikes, nmat: int, period: float, dt0: float, mode="bf16x3",
                 autotune: bool = True):
        import numpy as np
        self.mode = MODES[mode] if isinstance(mode, str) else mode
        self.lats = lattices
        dev = lattices[0].device
        self.device = dev
        self.nlat = len(lattices)
        self.nmat, self.period = nmat, period
        K = torch.as_tensor(strikes, dtype=torch.float64)
        if K.dim() == 1:
            K = K.unsqueeze(0).expand(self.nlat, -1)
        self.strikes = K.contiguous().to(dev)
        self.nK = self.strikes.shape[1]
        plans = [lat.plan(period, dt0) for lat in lattices]
        self.plans = plans
        w = lattices[0].width
        self.cols = torch.cat([lat.cols for lat in lattices])
        self.vals = torch.cat([lat.vals for lat in lattices])
        self.x = torch.cat([lat.x for lat in lattices])
        self._d = np.array([lat.d for lat in lattices], dtype=np.int32)
        self._y0 = np.array([lat.y0 for lat in lattices], dtype=np.int32)
        self._niter = np.array([p.niter for p in plans], dtype=np.int32)
        self._dt = np.array([p.dt for p in plans], dtype=np.float64)
        self._rate = np.array([lat.rate for lat in lattices], dtype=np.float64)
        bd = BatchDesc()
        bd.nlat, bd.d, bd.y0, bd.niter = self.nlat, self._d.ctypes.data, self._y0.ctypes.data, self._niter.ctypes.data
        bd.dt, bd.rate, bd.ell_width = self._dt.ctypes.data, self._rate.ctypes.data, w
        bd.gen_cols, bd.gen_vals, bd.x = _ptr(self.cols), _ptr(self.vals), _ptr(self.x)
        bd.nmat, bd.period, bd.nK, bd.strikes = nmat, period, self.nK, _ptr(self.strikes)
        self.desc = bd
        lib = _lib.load()
        n = lib.opb_batch_workspace_size(C.byref(bd), self.mode)
        if n == 0:
            raise _lib.OpcudaError("opb_batch_workspace_size", -1, "invalid batch description")
        self.ws = torch.empty(int(n), dtype=torch.uint8, device=dev)
        self.plan = C.c_void_p()
        bind_stream(dev)
        call("opb_batch_plan_create", C.byref(bd), self.mode, _ptr(self.ws), self.ws.numel(), C.byref(self.plan))
        self.tune_ms = None
        if autotune and self.mode in (BF16X3, FP16X3):
            ms = (C.c_float * lib.opb_batch_num_configs())()
            best = C.c_int()
            call("opb_batch_autotune", self.plan, 2, ms, C.byref(best))
            self.tune_ms = list(ms)
            self.config = best.value

    def set_config(self, cfg: int, grid: int = 0):
        call("opb_batch_set_config", self.plan, cfg, grid)
        self.config = cfg

    def execute(self, quotes: torch.Tensor | None = None) -> torch.Tensor:
        if quotes is None:
            quotes = torch.empty(self.nlat, self.nmat, self.nK, dtype=torch.float64, device=self.device)
        bind_stream(self.device)
        call("opb_batch_execute", self.plan, _ptr(quotes))
        return quotes

    def execute_bermudan(self, put: bool = True, exercise: bool = True, barrier: float = 0.0,
                         quotes: torch.Tensor | None = None) -> torch.Tensor:
        """Values [nlat, nK] (FP64) at each lattice's y0 of calls or puts of maturity
        nmat*period by backward induction on the period kernels, exercisable at every
        m*period (``exercise``) and knocked out at or below ``barrier`` on those dates."""
        if quotes is None:
            quotes = torch.empty(self.nlat, self.nK, dtype=torch.float64, device=self.device)
        bind_stream(self.device)
        call("opb_batch_execute_bermudan", self.plan, int(put), int(exercise), float(barrier), _ptr(quotes))
        return quotes

    def launches(self) -> int:
        return _lib.load().opb_batch_launches(self.plan)

    def __del__(self):
        try:
            if getattr(self, "plan", None) is not None and self.plan.value:
                _lib.load().opb_batch_plan_destroy(self.plan)
                self.plan = None
        except Exception:
            pass


def calibration_sweep(nlat=512, seed=20260, sizes=tuple(range(256, 2049, 128)), device="cuda", build=True):
    """Seeded local-vol lattices of the calibration sweep: n uniform over ``sizes``,
    level ~ U[0.1, 0.4], skew ~ U[-0.3, 0.3], width ~ U[0.2, 1.0], r ~ U[0, 0.05],
    sigma(x) = max(0.01, level + skew * exp(-((x - 1)/width)^2)).  build=False returns the
    parameters only (None for the lattices)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n = rng.choice(np.array(sizes), size=nlat)
    level = rng.uniform(0.1, 0.4, nlat)
    skew = rng.uniform(-0.3, 0.3, nlat)
    width = rng.uniform(0.2, 1.0, nlat)
    r = rng.uniform(0.0, 0.05, nlat)
    params = [dict(n=int(n[i]), level=float(level[i]), skew=float(skew[i]), width=float(width[i]), rate=float(r[i]),
                   floor=0.01) for i in range(nlat)]
    lats = [Lattice.local_vol(device=device, **p) for p in params] if build else None
    return lats, params
