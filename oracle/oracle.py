"""CPU FP64 oracle for the operator-method pricing path.

TEST INFRASTRUCTURE ONLY.  This module restates, in numpy (FP64), the algorithm of
OPLib's host double-precision path so that the CUDA library can be checked against it.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import it; nothing in the ``oplib_b200`` package does.

Parity status: OPLib ships no golden vectors for this path.  The pieces of this oracle
are pinned as follows (see ``tests/test_oracle.py``):

* MT19937: against libstdc++ ``std::mt19937`` (compiled from ``oracle/oracle_c.c``'s
  twin test program) and numpy's ``MT19937._legacy_seeding``; and against the C++
  standard's requirement that the 10000th output of a default-seeded (5489) engine is
  4123659995.
* Lattice pricing: against the Black-Scholes closed form (the reference's only known-
  answer test, ``tests/bstest/Program.cs:11-37``), against ``scipy.linalg.expm``, and
  by probability conservation / semigroup identities.
* The reference's own CUDA kernels for cumulative rows, kernels from generators, strided
  dot products, multi-vector induction, the jump generator and fills are compiled from its
  unchanged sources (``oracle/Makefile`` -> ``oracle/_ref``) and launched directly by
  ``oracle/ref_opcuda.cu`` (its exported wrappers pass 32-bit device pointers,
  ``oplib/opcuda/util.cu:170-175``); ``tests/test_gpu_ref_kernels.py`` compares the drop-in
  entry points with them.  The rest of the reference cannot be built here: its CPU path
  needs Intel MKL (``oplib/opc/rangen.cpp:36``) and its model layer needs .NET.

Layout convention.  The reference stores the transition element (source y1 -> target
y2) at ``y1 + d*y2`` (column-major with rows = source; ``oplib/opmodel/models/
CLVModel.cs:122,130``).  This oracle works with dense numpy matrices ``P[y1, y2]`` in
C (row-major) order, i.e. row = source; the two agree element by element.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------------
# Grids
# ---------------------------------------------------------------------------------


def log_grid(n: int, lo: float = 0.05, hi: float = 5.0, s0: float = 1.0) -> np.ndarray:
    """Log-spaced spot nodes x_i = s0*lo*(hi/lo)**(i/(n-1)), i = 0..n-1.

    The lattice configurations are defined on log-spaced nodes; the reference's own
    pivot/spacing grid (``oplib/opmodel/types/SGrid.cs:492-593``) is :func:`pivot_grid`."""
    i = np.arange(n, dtype=np.float64)
    return s0 * lo * (hi / lo) ** (i / (n - 1))


# The pivot grid of the reference's integration test (tests/bstest/OPPricer.cs:72-79).
BSTEST_PIVOTS = (1.0, 70.0, 90.0, 110.0, 140.0, 200.0, 300.0)
BSTEST_SPACINGS = (5.0, 2.5, 1.0, 2.5, 5.0, 7.5, 10.0)


def pivot_grid(nx: int, pivots, spacings, xval0: float) -> tuple[np.ndarray, int]:
    """The reference's pivot/spacing spot grid and its spot node (``SGrid.xgrid`` and
    ``grid_iterate``, ``oplib/opmodel/types/SGrid.cs:492-593``).

    Node 0 sits on the first pivot; node x adds scale * (current spacing), and the spacing
    switches to the next pivot's once a node passes that pivot.  The scale is bracketed in
    steps of 0.1 (up from 1 while the last node falls short of the last pivot, down
    otherwise), bisected 10 times, and the grid of the last bisection step is kept; the
    node nearest to ``xval0`` (first on ties) becomes the spot node x0 and the whole grid is
    scaled so that node is exactly ``xval0``.  Returns (nodes, x0)."""
    pivots = [float(p) for p in pivots]
    spacings = [float(s) for s in spacings]
    npv = len(pivots)
    if npv <= 2 or len(spacings) != npv:
        raise ValueError("pivot_grid needs more than two pivots, one spacing each")
    x = np.zeros(nx)

    def iterate(scale):
        x[0] = pivots[0]
        step, p = spacings[0], 1
        nextp = pivots[p] if p < npv else 0.0
        for i in range(1, nx):
            x[i] = x[i - 1] + scale * step
            if p < npv and x[i] > nextp:
                step = spacings[p]
                p += 1
                if p < npv:
                    nextp = pivots[p]
        return x[nx - 1]

    scale0 = scale1 = 1.0
    f0 = pivots[-1] / iterate(1.0)
    if f0 > 1:
        it = 1
        while True:
            scale0 = 1 + 0.1 * it
            if pivots[-1] / iterate(scale0) < 1:
                break
            scale1 = scale0
            it += 1
    else:
        it = 1
        while True:
            scale1 = 1 / (1 + 0.1 * it)
            if pivots[-1] / iterate(scale1) > 1:
                break
            scale0 = scale1
            it += 1
    for _ in range(10):
        mid = 0.5 * (scale0 + scale1)
        f2 = pivots[-1] / iterate(mid)
        if f2 > 1:
            scale1 = mid
        if f2 <= 1:
            scale0 = mid
    x0, best = 0, abs(x[0] - xval0)
    for i in range(1, nx):
        e = abs(x[i] - xval0)
        if e < best:
            x0, best = i, e
    return x * (xval0 / x[x0]), x0


def nearest_node(x: np.ndarray, s0: float = 1.0) -> int:
    """Index of the node nearest to the spot (the reference's ``grid.y0``)."""
    return int(np.argmin(np.abs(x - s0)))


def centred_log_grid(n: int, s0: float, width: float, i0: int) -> np.ndarray:
    """Log-spaced nodes with node ``i0`` exactly at ``s0`` (used by the Black-Scholes
    known-answer test so that the priced node is the spot itself)."""
    h = width / (n - 1)
    i = np.arange(n, dtype=np.float64)
    return s0 * np.exp((i - i0) * h)


# ---------------------------------------------------------------------------------
# Generators
# ---------------------------------------------------------------------------------


def lv_invm(x: np.ndarray) -> np.ndarray:
    """Per-node inverse of the 2x2 moment matrix [[dm, dp], [dm^2, dp^2]].

    Follows ``oplib/opmodel/types/S1DGrid.cs:78-147`` (``pregen``): dm = x[i-1]-x[i],
    dp = x[i+1]-x[i], with 1 in place of the missing spacing at either end
    (S1DGrid.cs:95-110).  The second row is [dm^2, dp^2] for every node but the first,
    which gets [0, 1]: the reference's test ``x0 > 0 && x0 < d`` (S1DGrid.cs:111) also holds
    for the last node, so the last node's row is [dm^2, 1] and the ``x0 == d - 1`` branch
    (S1DGrid.cs:123-127) is never reached.  The boundary inverses are unused: the generator
    zeroes the boundary nodes' rates (CLVModel.cs:99-114).  Returns an array (d, 2, 2) of
    inverses (row-major 2x2)."""
    d = x.shape[0]
    inv = np.zeros((d, 2, 2))
    for i in range(d):
        m = np.zeros((2, 2))
        m[0, 0] = x[i - 1] - x[i] if i > 0 else 1.0
        m[0, 1] = x[i + 1] - x[i] if i < d - 1 else 1.0
        if i > 0:
            m[1, 0] = m[0, 0] ** 2
            m[1, 1] = m[0, 1] ** 2
        else:
            m[1, 0], m[1, 1] = 0.0, 1.0
        inv[i] = np.linalg.inv(m)
    return inv


def lv_generator(x: np.ndarray, drift: np.ndarray, vol: np.ndarray) -> np.ndarray:
    """Tridiagonal birth-death generator L[y1, y2] of a local-volatility diffusion.

    Follows ``oplib/opmodel/models/CLVModel.cs:86-136`` (``host_d_gen``): per interior
    node, the down/up rates solve the moment system with right-hand side
    [drift, vol^2] (drift = r*x, vol = sigma(x)*x in spot units); the boundary nodes
    get zero rates (absorbing); the diagonal is minus the row sum."""
    d = x.shape[0]
    inv = lv_invm(x)
    L = np.zeros((d, d))
    for i in range(d):
        if 0 < i < d - 1:
            rhs = np.array([drift[i], vol[i] ** 2])
        else:
            rhs = np.zeros(2)
        p = inv[i] @ rhs
        s = 0.0
        if i > 0:
            L[i, i - 1] = p[0]
            s += p[0]
        if i < d - 1:
            L[i, i + 1] = p[1]
            s += p[1]
        L[i, i] = -s
    return L


def lv_generator_fast(x: np.ndarray, drift: np.ndarray, vol: np.ndarray) -> np.ndarray:
    """Vectorised restatement of :func:`lv_generator` (same arithmetic, closed-form 2x2
    solve), for large lattices."""
    d = x.shape[0]
    dm = np.zeros(d)
    dp = np.zeros(d)
    dm[1:] = x[:-1] - x[1:]
    dp[:-1] = x[1:] - x[:-1]
    det = dm * dp * dp - dp * dm * dm
    inner = np.zeros(d, dtype=bool)
    inner[1:-1] = True
    a = np.where(inner, drift, 0.0)
    b = np.where(inner, vol ** 2, 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        pm = np.where(inner, (dp * dp * a - dp * b) / det, 0.0)
        pp = np.where(inner, (-dm * dm * a + dm * b) / det, 0.0)
    L = np.zeros((d, d))
    idx = np.arange(d)
    L[idx[1:], idx[1:] - 1] = pm[1:]
    L[idx[:-1], idx[:-1] + 1] = pp[:-1]
    L[idx, idx] = -(pm + pp)
    return L


def lv_sigma(x: np.ndarray, level=0.2, skew=0.1, width=0.5, floor=0.0) -> np.ndarray:
    """sigma(x) = level + skew*exp(-((x-1)/width)^2), floored at ``floor``."""
    s = level + skew * np.exp(-(((x - 1.0) / width) ** 2))
    return np.maximum(s, floor)


@dataclass
class SVSpec:
    """Stochastic-volatility lattice: spot nodes x (nx) times vol states sigma_v (nv).

    State index y = ix + nx*iv, as in ``oplib/opmodel/types/S2DGrid.cs:142``."""

    nx: int = 128
    nv: int = 48
    x_lo: float = 0.05
    x_hi: float = 5.0
    v_lo: float = 0.05
    v_hi: float = 1.0
    r: float = 0.03
    kappa: float = 2.0
    theta: float = 0.04
    xi: float = 0.6
    rho: float = -0.7

    @property
    def d(self) -> int:
        return self.nx * self.nv


def sv_generator(spec: SVSpec) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """2-D (spot, variance) generator with a correlation stencil.

    Structure follows ``oplib/opmodel/types/S2DGrid.cs:123-245`` (per node, separate
    2x2 moment systems in the spot and in the vol direction, i.e. the block-diagonal
    4x4 ``invm``) and ``oplib/opmodel/models/CSVModel.cs:187-379`` (negative rates
    clamped to zero, then a drift fix-up so that the spot drift is exactly r*x).

    Project extension (the reference has no spot-vol correlation term): Heston
    dynamics in the variance V = sigma_v^2, dV = kappa(theta - V)dt + xi sqrt(V) dW2,
    d<W1, W2> = rho dt, give Cov(dx, dV) = rho*xi*V*x dt.  It is carried by two
    diagonal moves, (+x, -v) and (-x, +v) for rho < 0 (or (+,+), (-,-) for rho > 0),
    at a common rate q chosen so that the diagonal moves reproduce the covariance,
    capped so that the diagonal moves never carry more variance than the target
    variance in either direction (there the stencil cannot represent the full
    correlation; the effective correlation is reduced).  The axial rates then
    match the remaining first and second moments.  Spot-boundary nodes are absorbing
    (as in the local-vol model); vol-boundary nodes match the variance drift only
    (as S2DGrid.cs:209-224 does).

    Returns (L, x_y, v_y): dense generator and per-state spot and vol values."""
    nx, nv = spec.nx, spec.nv
    d = nx * nv
    xs = log_grid(nx, spec.x_lo, spec.x_hi)
    vs = spec.v_lo * (spec.v_hi / spec.v_lo) ** (np.arange(nv) / (nv - 1))
    V = vs ** 2
    L = np.zeros((d, d))
    sgn = -1 if spec.rho < 0 else 1

    def idx(ix, iv):
        return ix + nx * iv

    for iv in range(nv):
        for ix in range(nx):
            y = idx(ix, iv)
            if ix == 0 or ix == nx - 1:
                continue  # absorbing spot boundary
            x = xs[ix]
            v = V[iv]
            var_x = v * x * x
            var_v = spec.xi ** 2 * v
            cov = spec.rho * spec.xi * v * x
            mu_x = spec.r * x
            mu_v = spec.kappa * (spec.theta - v)
            dxm, dxp = xs[ix - 1] - x, xs[ix + 1] - x
            rates = {}
            q = 0.0
            ex = ev = ex2 = ev2 = 0.0
            if 0 < iv < nv - 1 and spec.rho != 0.0:
                dvm, dvp = V[iv - 1] - v, V[iv + 1] - v
                if sgn < 0:
                    moves = [(dxp, dvm, idx(ix + 1, iv - 1)), (dxm, dvp, idx(ix - 1, iv + 1))]
                else:
                    moves = [(dxp, dvp, idx(ix + 1, iv + 1)), (dxm, dvm, idx(ix - 1, iv - 1))]
                cx = sum(m[0] * m[1] for m in moves)
                sx2 = sum(m[0] ** 2 for m in moves)
                sv2 = sum(m[1] ** 2 for m in moves)
                q = cov / cx
                q = min(q, var_x / sx2, var_v / sv2)
                q = max(q, 0.0)
                for (ddx, ddv, t) in moves:
                    rates[t] = rates.get(t, 0.0) + q
                ex = q * sum(m[0] for m in moves)
                ev = q * sum(m[1] for m in moves)
                ex2 = q * sx2
                ev2 = q * sv2
            # spot direction: [dxm dxp; dxm^2 dxp^2] p = [mu_x - ex, var_x - ex2]
            a, b = mu_x - ex, var_x - ex2
            det = dxm * dxp * dxp - dxp * dxm * dxm
            pxm = (dxp * dxp * a - dxp * b) / det
            pxp = (-dxm * dxm * a + dxm * b) / det
            rates[idx(ix - 1, iv)] = rates.get(idx(ix - 1, iv), 0.0) + pxm
            rates[idx(ix + 1, iv)] = rates.get(idx(ix + 1, iv), 0.0) + pxp
            # vol direction
            if 0 < iv < nv - 1:
                dvm, dvp = V[iv - 1] - v, V[iv + 1] - v
                a, b = mu_v - ev, var_v - ev2
                det = dvm * dvp * dvp - dvp * dvm * dvm
                pvm = (dvp * dvp * a - dvp * b) / det
                pvp = (-dvm * dvm * a + dvm * b) / det
                rates[idx(ix, iv - 1)] = rates.get(idx(ix, iv - 1), 0.0) + pvm
                rates[idx(ix, iv + 1)] = rates.get(idx(ix, iv + 1), 0.0) + pvp
            elif iv == 0:
                dvp = V[1] - v
                rates[idx(ix, 1)] = max(mu_v, 0.0) / dvp
            else:
                dvm = V[iv - 1] - v
                rates[idx(ix, iv - 1)] = min(mu_v, 0.0) / dvm
            # clamp negatives (CSVModel.cs:342-345), then spot drift fix-up (353-373)
            drift = 0.0
            for t in list(rates):
                if rates[t] < 0.0:
                    rates[t] = 0.0
                tx = t % nx
                drift += rates[t] * (xs[tx] - x)
            if drift > mu_x:
                t = idx(ix - 1, iv)
                rates[t] += (drift - mu_x) / (x - xs[ix - 1])
            else:
                t = idx(ix + 1, iv)
                rates[t] += (mu_x - drift) / (xs[ix + 1] - x)
            tot = 0.0
            for t, rt in rates.items():
                L[y, t] += rt
                tot += rt
            L[y, y] -= tot
    x_y = np.tile(xs, nv)
    v_y = np.repeat(vs, nx)
    return L, x_y, v_y


# ---------------------------------------------------------------------------------
# Plan, kernels, squaring, chaining
# ---------------------------------------------------------------------------------


def plan_niter(L: np.ndarray, delta_t: float, dt0: float) -> tuple[int, float]:
    """Number of squarings and the elementary time step for one interval.

    ``oplib/opmodel/models/CModel Common.cs:289-307``: dt = min(0.5/max|L_yy|, dt0),
    niter = ceil(log2(DeltaT/dt)), dt_j = DeltaT * 2^-niter."""
    maxdiag = float(np.max(np.abs(np.diag(L))))
    dt = 0.5 / maxdiag if maxdiag > 0 else dt0
    if dt > dt0:
        dt = dt0
    niter = int(math.ceil(math.log(delta_t / dt) / math.log(2.0)))
    return niter, delta_t * 2.0 ** (-niter)


def ek(L: np.ndarray, dt: float) -> np.ndarray:
    """U0 = I + dt*L (``oplib/opmodel/models/CModel Host Double.cs:89-121``;
    ``oplib/opcuda/sek.cu:40-59``)."""
    U = dt * L
    U[np.diag_indices_from(U)] += 1.0
    return U


def renormalise(P: np.ndarray) -> np.ndarray:
    """Rows divided by their FP64 sums (probability conservation)."""
    s = P.sum(axis=1)
    return P / s[:, None]


def square(U: np.ndarray, niter: int, renorm: bool = False) -> np.ndarray:
    """niter repeated squarings U <- U.U in FP64 (``CModel Host Double.cs:125-197``,
    ping-pong through ``opc_dgemm``).  ``renorm`` renormalises rows after every level."""
    P = U.copy()
    for _ in range(niter):
        P = P @ P
        if renorm:
            P = renormalise(P)
    return P


def chain(P1: np.ndarray, nmat: int) -> list[np.ndarray]:
    """P(j*T) = P((j-1)*T) . P(T), j = 1..nmat (the chaining GEMMs of
    ``CModel Host Double.cs:227-277``, tpk_m <- tpk_m . xtpk_j)."""
    out = [P1]
    for _ in range(nmat - 1):
        out.append(out[-1] @ P1)
    return out


def mc_plan_kernels(plan, generators) -> list[np.ndarray]:
    """Step kernels of a Monte Carlo plan in FP64: elementary kernels
    X_j = (I + dt_j L_{i_j})^(2^niter_j) (``CModel Host Double.cs:125-197``) and step
    kernels X_{f0} . X_{f1} . ... over each step's factors in time order.  ``plan`` has the
    planner's ``i_j``, ``dt_j``, ``niter_j`` and ``jfactor_ms``; ``generators[i]`` is the
    dense generator that holds on generator interval i."""
    X = [square(ek(generators[i], dt), n) for i, dt, n in zip(plan.i_j, plan.dt_j, plan.niter_j)]
    out = []
    for factors in plan.jfactor_ms:
        P = X[factors[0]].copy()
        for j in factors[1:]:
            P = P @ X[j]
        out.append(P)
    return out


def payoff_calls(x: np.ndarray, strikes: np.ndarray) -> np.ndarray:
    """G[y, k] = (x_y - K_k)^+."""
    return np.maximum(x[:, None] - strikes[None, :], 0.0)


def price_from_kernels(Ps: list[np.ndarray], x: np.ndarray, strikes: np.ndarray,
                       r: float, mats: np.ndarray) -> np.ndarray:
    """Backward induction V_T = P_T . G for every maturity (all source states), with
    discounting exp(-r T).  Returns V[m, y, k]."""
    G = payoff_calls(x, strikes)
    return np.stack([math.exp(-r * T) * (P @ G) for P, T in zip(Ps, mats)])


def mc_cashflow_values(paths: np.ndarray, cashflow: np.ndarray, knockout: np.ndarray | None = None) -> np.ndarray:
    """Per-path values of the cashflow-table evaluator: v_p = sum_k cashflow[k, y_pk] over the
    steps k before the first one whose state is knocked out (knockout[k, y_pk] != 0), added
    in step order in FP64.  It generalises the reference's vanilla evaluator
    (``tests/bstest/OPPricer.cs:8-63``: the payoff (x_T - K)^+ of the last step's state,
    called back on host copies of the states, ``oplib/opmodel/interfaces/CMCEvaluator.cs:41-67``)
    to cashflows at every step with discrete knock-out.  paths: [npaths, nsteps] states."""
    npaths, nsteps = paths.shape
    v = np.zeros(npaths)
    alive = np.ones(npaths, dtype=bool)
    for k in range(nsteps):
        y = paths[:, k].astype(np.int64)
        if knockout is not None:
            alive &= knockout[k, y] == 0
        v = np.where(alive, v + cashflow[k, y], v)
    return v


class HostSolveFP64:
    """The reference's host FP64 solve, one product ("stage") at a time, on torch-CPU FP64
    tensors (the matrix products are MKL DGEMMs, the library family of ``opc_dgemm``,
    ``oplib/opc/linalg.c:93-101``):

    * U0 = I + dt L (``host_d_mc_ek``, ``CModel Host Double.cs:89-121``), built in stage 0;
    * stages 0..niter-1: squarings U <- U.U (``host_d_mc_sq``, ``CModel Host Double.cs:125-197``);
    * stages niter..niter+nmat-2: chaining P_m = P_{m-1}.P1, m = 2..nmat (``host_d_mc_mk``,
      ``CModel Host Double.cs:227-277``);
    * the payoff product V_m = exp(-r m period) P_m.G for every source state in the stage
      that forms P_m (the backward induction the reference exports as ``sgemv``/``sdot2``).

    No renormalisation: the reference's host path has none (row sums stay 1 to FP64
    rounding).  ``state`` holds the stage's inputs (``U``, or ``Pm`` and ``P1``) and the
    values so far; ``run`` leaves its inputs untouched, so a stage can be run again on the
    same inputs.  niter >= 1.  L: torch FP64 [d, d] (row = source)."""

    def __init__(self, L, x, strikes, r: float, period: float, nmat: int, niter: int, dt: float):
        import torch
        self.torch = torch
        self.L, self.r, self.period, self.nmat, self.niter, self.dt = L, r, period, nmat, niter, dt
        xs = torch.as_tensor(np.asarray(x, dtype=np.float64))
        K = torch.as_tensor(np.asarray(strikes, dtype=np.float64))
        self.G = torch.clamp(xs[:, None] - K[None, :], min=0.0)
        self.stages = niter + nmat - 1

    def run(self, p: int, state: dict) -> dict:
        """Stage p on the inputs in ``state``; returns the next stage's state."""
        if p < self.niter:
            if p == 0:
                U = self.L * self.dt
                U.diagonal().add_(1.0)
            else:
                U = state["U"]
            U = U @ U
            V = list(state.get("V", []))
            if p == self.niter - 1:
                V.append(math.exp(-self.r * self.period) * (U @ self.G))
                return {"Pm": U, "P1": U, "V": V}
            return {"U": U, "V": V}
        m = p - self.niter + 2
        Pm = state["Pm"] @ state["P1"]
        V = list(state["V"]) + [math.exp(-self.r * self.period * m) * (Pm @ self.G)]
        return {"Pm": Pm, "P1": state["P1"], "V": V}

    def values(self, state: dict):
        """V [nmat, d, nK] after the last stage."""
        return self.torch.stack(state["V"])


def host_solve_stages(L, x, strikes, r: float, period: float, nmat: int, niter: int, dt: float):
    """``HostSolveFP64`` as a generator that yields once per stage, niter + nmat - 1 times:
    None, and at the last stage V [nmat, d, nK]."""
    hs = HostSolveFP64(L, x, strikes, r, period, nmat, niter, dt)
    state = {}
    for p in range(hs.stages):
        state = hs.run(p, state)
        yield hs.values(state) if p == hs.stages - 1 else None


# ---------------------------------------------------------------------------------
# Lattice configurations
# ---------------------------------------------------------------------------------


@dataclass
class LVLattice:
    n: int = 512
    level: float = 0.2
    skew: float = 0.1
    width: float = 0.5
    r: float = 0.03
    floor: float = 0.0
    dt0: float = 2.0 ** -14
    period: float = 0.25
    nmat: int = 8
    strikes: np.ndarray = field(default_factory=lambda: 0.5 + np.arange(64) / 63.0)

    def grid(self):
        return log_grid(self.n)

    def generator(self):
        x = self.grid()
        sig = lv_sigma(x, self.level, self.skew, self.width, self.floor)
        return lv_generator_fast(x, self.r * x, sig * x), x

    @property
    def maturities(self):
        return self.period * np.arange(1, self.nmat + 1)


def solve_lattice_fp64(L: np.ndarray, x: np.ndarray, strikes: np.ndarray, r: float,
                       period: float, nmat: int, dt0: float, renorm: bool = True):
    """Full FP64 solve: plan, U0, squarings, chaining, pricing.  Returns
    (V[m, y, k], niter, dt)."""
    niter, dt = plan_niter(L, period, dt0)
    U0 = ek(L, dt)
    P1 = square(U0, niter, renorm=renorm)
    Ps = chain(P1, nmat)
    mats = period * np.arange(1, nmat + 1)
    return price_from_kernels(Ps, x, strikes, r, mats), niter, dt


def bermudan_fp64(L: np.ndarray, x: np.ndarray, strikes: np.ndarray, r: float, period: float, nmat: int,
                  dt0: float, put: bool = False, exercise: bool = True, barrier: float = 0.0) -> np.ndarray:
    """FP64 backward induction on the period kernel P1 = P(period) (the same plan,
    squarings and row renormalisation as ``solve_lattice_fp64``): V_nmat = e(x), then for
    m = nmat-1 .. 0, V_m = exp(-r period) P1 . V_{m+1}, set to 0 where x <= barrier
    (barrier > 0) and otherwise floored by the exercise value (exercise) at the dates
    m >= 1.  e(x) = (x - K)^+ for calls, (K - x)^+ for puts.  This is the multi-vector
    induction the reference's ``opcuda_sgemv3``/``sgemv4`` kernels perform
    (``oplib/opcuda/sgemv3.cu:92-159``), with the exercise and barrier rules of a
    Bermudan / discretely monitored down-and-out contract (no reference counterpart).
    Returns V_0[y, k]."""
    niter, dt = plan_niter(L, period, dt0)
    P1 = square(ek(L, dt), niter, renorm=True)
    K = np.asarray(strikes, dtype=np.float64)[None, :]
    xs = np.asarray(x, dtype=np.float64)[:, None]
    ex = np.maximum(K - xs, 0.0) if put else np.maximum(xs - K, 0.0)
    out = (xs <= barrier) if barrier > 0.0 else np.zeros_like(xs, dtype=bool)
    V = np.where(out, 0.0, ex)
    disc = math.exp(-r * period)
    for m in range(nmat - 1, -1, -1):
        V = disc * (P1 @ V)
        if m >= 1:
            if exercise:
                V = np.maximum(V, ex)
            V = np.where(out, 0.0, V)
    return V


# ---------------------------------------------------------------------------------
# The reference's two-dimensional generator with vol-level jumps (opcuda_sgsvg)
# ---------------------------------------------------------------------------------


def s2d_invm(xval: np.ndarray, rval: np.ndarray, nx: int, nr: int) -> np.ndarray:
    """Per-node inverses of the 4 x 4 moment matrices, ``S2DGrid.pregen``
    (``oplib/opmodel/types/S2DGrid.cs:123-245``).  Node y = x + nx*r; columns of the
    moment matrix are the moves (x-1, x+1, r-1, r+1), rows the moments (dx, dx^2, dr,
    dr^2), with identity-like rows at the boundaries.  Returns invm[16*d] with
    invm[16*y + k + 4*i] = inverse[k, i] (column-major per node)."""
    d = nx * nr
    invm = np.zeros(16 * d)
    for x0 in range(nx):
        for a0 in range(nr):
            y0 = x0 + nx * a0
            m = np.zeros((4, 4))
            m[0, 0] = xval[y0 - 1] - xval[y0] if x0 > 0 else 0.0
            m[0, 1] = xval[y0 + 1] - xval[y0] if x0 < nx - 1 else 0.0
            if 0 < x0 < nx - 1:
                m[1, 0], m[1, 1] = m[0, 0] ** 2, m[0, 1] ** 2
            elif x0 == 0:
                m[1, 0], m[1, 1] = 1.0, 0.0
            else:
                m[1, 0], m[1, 1] = 0.0, 1.0
            m[2, 2] = rval[y0 - nx] - rval[y0] if a0 > 0 else 0.0
            m[2, 3] = rval[y0 + nx] - rval[y0] if a0 < nr - 1 else 0.0
            if 0 < a0 < nr - 1:
                m[3, 2], m[3, 3] = m[2, 2] ** 2, m[2, 3] ** 2
            elif a0 == 0:
                m[3, 2] = 1.0
            else:
                m[3, 3] = 1.0
            inv = np.linalg.inv(m)
            invm[16 * y0:16 * y0 + 16] = inv.T.reshape(-1)  # column-major
    return invm


def sgsvg_generator(invm, xval, sdrift, svol, voldrift, volvol, jm, jp, nx, nr, gen0=None):
    """One interval of the two-dimensional generator with jumps across volatility levels,
    row by row as ``global_sgsvg`` (``oplib/opcuda/sgsvg.cu:40-209``) and
    ``CSVModel.host_d_gen`` (``oplib/opmodel/models/CSVModel.cs:187-379``) build it:

    1. nearest-neighbour rates = invm . (0, svol^2 [interior x], voldrift, volvol^2
       [interior r]) for the moves (x-1, x+1, r-1, r+1);
    2. for every higher level r1 > r0 whose entries of the row sum to prob > 0, the
       entries x1 < x0 - 1 and x1 > x0 of level r1 are set to prob * w / sum(w) with
       w = exp(+-(x1 - x0) / (J x0)), J = jm below and jp above (the device kernel uses
       jm on both sides, sgsvg.cu:111-112, a listed quirk not restated);
    3. negative off-diagonal rates are cleared; the drift sum_y1 q (x1 - x0) is moved
       toward sdrift through one neighbour with the reference's own formula (for drift
       above target: (drift - sdrift) / (x_{x0-1} - x0) added to the x-1 rate, as both
       reference versions do, sgsvg.cu:186-195, CSVModel.cs:343-352); the diagonal is
       minus the off-diagonal sum.

    ``gen0`` (optional [d, d]) is the buffer's prior content (the kernels add to what is
    there only through step 2's sums, so a zeroed buffer is the normal case).  Returns
    G[y0, y1] (row = source), FP64."""
    d = nx * nr
    G = np.zeros((d, d)) if gen0 is None else np.array(gen0, dtype=np.float64)
    for y0 in range(d):
        r0, x0 = divmod(y0, nx)
        rhs = np.array([0.0, svol[y0] ** 2 if 0 < x0 < nx - 1 else 0.0, voldrift[y0],
                        volvol[y0] ** 2 if 0 < r0 < nr - 1 else 0.0])
        inv = invm[16 * y0:16 * y0 + 16].reshape(4, 4).T
        q = inv @ rhs
        if x0 > 0:
            G[y0, y0 - 1] = q[0]
        if x0 < nx - 1:
            G[y0, y0 + 1] = q[1]
        if r0 > 0:
            G[y0, y0 - nx] = q[2]
        if r0 < nr - 1:
            G[y0, y0 + nx] = q[3]
        jmin, jplus = jm[y0] * xval[y0], jp[y0] * xval[y0]
        for r1 in range(r0 + 1, nr):
            base = nx * r1
            prob = G[y0, base:base + nx].sum()
            if prob <= 0:
                continue
            lo_idx = [base + x1 for x1 in range(0, x0 - 1)] if jmin > 0 else []
            hi_idx = [base + x1 for x1 in range(x0 + 1, nx)] if jplus > 0 else []
            w_lo = np.exp((xval[lo_idx] - xval[y0]) / jmin) if lo_idx else np.zeros(0)
            w_hi = np.exp(-(xval[hi_idx] - xval[y0]) / jplus) if hi_idx else np.zeros(0)
            sum0 = w_lo.sum() + w_hi.sum()
            if sum0 > 0:
                ratio = prob / sum0
                G[y0, lo_idx] = ratio * w_lo
                G[y0, hi_idx] = ratio * w_hi
        row = G[y0].copy()
        row[y0] = 0.0
        row[row < 0] = 0.0
        G[y0] = row
        drift = float(np.sum(row * (xval - xval[y0])))
        tot = float(row.sum())
        if drift > sdrift[y0]:
            if x0 > 0:
                ratio = (drift - sdrift[y0]) / (xval[y0 - 1] - xval[y0])
                G[y0, y0 - 1] += ratio
                tot += ratio
        elif x0 < nx - 1:
            ratio = (sdrift[y0] - drift) / (xval[y0 + 1] - xval[y0])
            G[y0, y0 + 1] += ratio
            tot += ratio
        G[y0, y0] = -tot
    return G


# ---------------------------------------------------------------------------------
# Cumulative rows and sampling
# ---------------------------------------------------------------------------------


def cumrows_f32(P: np.ndarray) -> np.ndarray:
    """Cumulative normalised rows in FP32, sequential left-to-right sums.

    ``oplib/opcuda/sck.cu:43-84``: C[y, 0] = P[y, 0]; C[y, z] = C[y, z-1] + P[y, z]
    (FP32 running sum); then every entry is divided by the row total and clamped at 1.
    The FP32 operations are done one at a time so that the rounding sequence is the
    one a sequential FP32 loop performs."""
    P32 = np.maximum(np.asarray(P, dtype=np.float32), np.float32(0.0))  # negatives count as 0
    d = P32.shape[1]
    C = np.empty_like(P32)
    acc = P32[:, 0].copy()
    C[:, 0] = acc
    for z in range(1, d):
        acc = (acc + P32[:, z]).astype(np.float32)
        C[:, z] = acc
    tot = acc
    C = (C / tot[:, None]).astype(np.float32)
    return np.minimum(C, np.float32(1.0))


def uniform_f32(x: np.ndarray) -> np.ndarray:
    """u = ((float)x + 1.0f) * 2^-32 in FP32 (``oplib/opcuda/smc.cu:329``), u in (0,1]."""
    f = x.astype(np.float32)
    f = (f + np.float32(1.0)).astype(np.float32)
    return (f * np.float32(2.0 ** -32)).astype(np.float32)


def sample_next(Crow: np.ndarray, u: np.ndarray) -> np.ndarray:
    """Smallest y with u < C[y], capped at d-1 (``oplib/opcuda/smc.cu:336-350``).

    ``Crow`` is (npaths, d) float32, ``u`` (npaths,) float32."""
    d = Crow.shape[1]
    cnt = (Crow <= u[:, None]).sum(axis=1)  # rows are non-decreasing
    return np.minimum(cnt, d - 1)


# ---------------------------------------------------------------------------------
# MT19937 (Matsumoto & Nishimura 1998, init_genrand of the 2002 reference code)
# ---------------------------------------------------------------------------------

_MT_N, _MT_M = 624, 397
_MT_A = np.uint32(0x9908B0DF)
_UPPER = np.uint32(0x80000000)
_LOWER = np.uint32(0x7FFFFFFF)


def mt19937_init(seeds: np.ndarray, key1: np.ndarray | None = None) -> np.ndarray:
    """init_genrand for a vector of seeds: mt[0] = s, mt[i] = 1812433253 *
    (mt[i-1] ^ (mt[i-1] >> 30)) + i (mod 2^32).  The same recurrence seeds the
    reference's twisters (``oplib/opcuda/smc.cu:127-131``).  ``key1`` (optional, one per
    seed) is added to mt[1] before the recurrence continues: the keyed generators of the
    library's stream-seed-table Monte Carlo.  Returns (nseeds, 624)."""
    seeds = np.asarray(seeds, dtype=np.uint64) & np.uint64(0xFFFFFFFF)
    mt = np.empty((seeds.shape[0], _MT_N), dtype=np.uint64)
    mt[:, 0] = seeds
    mask = np.uint64(0xFFFFFFFF)
    for i in range(1, _MT_N):
        prev = mt[:, i - 1]
        mt[:, i] = (np.uint64(1812433253) * (prev ^ (prev >> np.uint64(30))) + np.uint64(i)) & mask
        if i == 1 and key1 is not None:
            mt[:, 1] = (mt[:, 1] + (np.asarray(key1, dtype=np.uint64) & mask)) & mask
    return mt.astype(np.uint32)


def mt19937_twist(mt: np.ndarray) -> np.ndarray:
    """One full regeneration of the 624-word state (genrand_int32's refill loop)."""
    mt = mt.copy()
    n = _MT_N
    for k in range(n):
        y = (mt[:, k] & _UPPER) | (mt[:, (k + 1) % n] & _LOWER)
        mag = np.where((y & np.uint32(1)) != 0, _MT_A, np.uint32(0))
        mt[:, k] = mt[:, (k + _MT_M) % n] ^ (y >> np.uint32(1)) ^ mag
    return mt


def mt19937_temper(y: np.ndarray) -> np.ndarray:
    y = y ^ (y >> np.uint32(11))
    y = y ^ ((y << np.uint32(7)) & np.uint32(0x9D2C5680))
    y = y ^ ((y << np.uint32(15)) & np.uint32(0xEFC60000))
    y = y ^ (y >> np.uint32(18))
    return y


def mt19937_outputs(seeds: np.ndarray, count: int, key1: np.ndarray | None = None) -> np.ndarray:
    """First ``count`` genrand_int32 outputs of each seeded stream, (nseeds, count)."""
    st = mt19937_init(seeds, key1)
    outs = []
    while sum(o.shape[1] for o in outs) < count:
        st = mt19937_twist(st)
        outs.append(mt19937_temper(st))
    return np.concatenate(outs, axis=1)[:, :count]


# ---------------------------------------------------------------------------------
# Monte Carlo on a lattice (per-path MT19937 streams)
# ---------------------------------------------------------------------------------


def mc_paths(C: np.ndarray, y0: int, seed: int, path_ids: np.ndarray, nsteps: int) -> np.ndarray:
    """State paths y[p, k] (k = 1..nsteps) with path p drawing from MT19937
    init_genrand(seed + p) and consuming its outputs in order, one per step.

    The step loop follows ``oplib/opcuda/smc.cu:307-366`` (one uniform per step, inverse
    CDF over the row of the previous state)."""
    seeds = (np.uint64(seed) + path_ids.astype(np.uint64)) & np.uint64(0xFFFFFFFF)
    raw = mt19937_outputs(seeds, nsteps)
    y = np.full(path_ids.shape[0], y0, dtype=np.int64)
    out = np.empty((path_ids.shape[0], nsteps), dtype=np.int16)
    for k in range(nsteps):
        u = uniform_f32(raw[:, k])
        y = sample_next(C[y], u)
        out[:, k] = y
    return out


def mc_payoffs(paths: np.ndarray, x: np.ndarray, strike: float, barrier: float,
               r: float, T: float) -> dict:
    """Discounted barrier (down-and-out call, discretely monitored at every step) and
    arithmetic-Asian call payoffs per path, plus their means."""
    xv = x[paths.astype(np.int64)]
    disc = math.exp(-r * T)
    alive = xv.min(axis=1) > barrier
    barrier_pay = disc * np.where(alive, np.maximum(xv[:, -1] - strike, 0.0), 0.0)
    asian_pay = disc * np.maximum(xv.mean(axis=1) - strike, 0.0)
    return {"barrier": barrier_pay, "asian": asian_pay}


# ---------------------------------------------------------------------------------
# Black-Scholes (``tests/bstest/BSPricer.cs:7-65``) and implied volatility
# ---------------------------------------------------------------------------------


def norm_cdf(z):
    return 0.5 * (1.0 + np.vectorize(math.erf)(np.asarray(z) / math.sqrt(2.0)))


def bs_call(s, k, r, sigma, t):
    s, k, sigma, t = map(np.asarray, (s, k, sigma, t))
    sq = sigma * np.sqrt(t)
    d1 = (np.log(s / k) + (r + 0.5 * sigma * sigma) * t) / sq
    d2 = d1 - sq
    return s * norm_cdf(d1) - k * np.exp(-r * t) * norm_cdf(d2)


def implied_vol(price, s, k, r, t, lo=1e-4, hi=5.0, iters=100):
    """Bisection inversion of the Black-Scholes call price (vectorised)."""
    price, k, t = np.broadcast_arrays(np.asarray(price, float), np.asarray(k, float),
                                      np.asarray(t, float))
    a = np.full(price.shape, lo)
    b = np.full(price.shape, hi)
    for _ in range(iters):
        m = 0.5 * (a + b)
        too_high = bs_call(s, k, r, m, t) > price
        b = np.where(too_high, m, b)
        a = np.where(too_high, a, m)
    return 0.5 * (a + b)


# ---------------------------------------------------------------------------------
# Split-BF16 emulation (numerical model of the tensor-core squaring, for analysis)
# ---------------------------------------------------------------------------------


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (round to nearest even), returned as FP32."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    lsb = (u >> np.uint64(16)) & np.uint64(1)
    u = (u + np.uint64(0x7FFF) + lsb) & np.uint64(0xFFFF0000)
    return u.astype(np.uint32).view(np.float32)


def split_bf16(a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The library's BF16 two-part split: hi = bf16(a), lo = bf16(a - hi), with its absolute
    floor (|a| < 2^-40: both parts zero; |a| < 2^-30: no lo part)."""
    a32 = np.asarray(a, dtype=np.float32)
    mag = np.abs(a32)
    hi = bf16_round(np.where(mag < np.float32(2.0 ** -40), np.float32(0), a32))
    lo = bf16_round(np.where(mag < np.float32(2.0 ** -30), np.float32(0), (a32 - hi).astype(np.float32)))
    return hi, lo
