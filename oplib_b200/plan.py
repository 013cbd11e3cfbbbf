"""Monte Carlo step plan: which elementary kernels to exponentiate, and which of them each
step's kernel chains -- the host planner of the reference's model layer
(``oplib/opmodel/models/CModel Common.cs:163-486``, ``make_mc_plan``), restated.

Dates are whole days after today, as the reference's ``DateTime`` differences
(``.Days``) are.  Given the step dates ``t_k`` and the generator (curve) dates ``t_i`` --
generator i holds on (t_i[i-1], t_i[i]] -- the planner

* merges both into the elementary dates ``t_q`` (sorted, distinct, up to the last step);
* gives every elementary interval its generator ``i_q`` and a distinct elementary kernel
  ``j_q``: intervals of equal length under the same generator share one (the first
  interval's length counted from today);
* plans each elementary kernel by the niter rule (``opb_plan_interval``, Common.cs:289-307);
* gives every step a step kernel ``m_k``: steps of equal length that lie under one
  generator share one; and lists each step kernel's elementary factors in time order
  (``jfactor_ms``), so the step kernel is their product.

Chaining order.  A step kernel is X_j0 . X_j1 . ... over its factor list.  The reference
chains with ``jfactor_ms[m][s]`` at chain step s = 0, 1, ... after starting from factor 0
(``CModel Host Double.cs:229-270``, ``CModel Common.cs:555-616``), so a step of two or more
factors multiplies by its first factor twice, and its device branch reads past the factor
list of shorter steps when factor counts differ.  That is not restated: every step kernel
here is the product of its own factors.  The two agree for every plan whose steps each lie
under one generator (one factor per step), which is every plan the reference's own tests
and benchmarks build.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib

DAYS_PER_YEAR = 365.25  # CModel Common.cs:168,302


@dataclass
class McPlan:
    t_k: list[int]          # step dates (days after today)
    t_i: list[int]          # generator dates
    t_q: list[int]          # elementary dates
    i_q: list[int]          # generator of each elementary interval
    j_q: list[int]          # elementary kernel of each elementary interval
    t0_j: list[int]         # elementary kernel j covers (t0_j, t1_j] under generator i_j
    t1_j: list[int]
    i_j: list[int]
    niter_j: list[int]      # squarings of elementary kernel j
    dt_j: list[float]       # its elementary time step (years)
    m_k: list[int]          # step kernel of each step
    jfactor_ms: list[list[int]]  # elementary factors of each step kernel, in time order

    @property
    def nk(self) -> int:
        return len(self.t_k)

    @property
    def nq(self) -> int:
        return len(self.t_q)

    @property
    def nj(self) -> int:
        return len(self.t0_j)

    @property
    def nm(self) -> int:
        return len(self.jfactor_ms)

    @property
    def nr(self) -> int:
        """Squaring levels of the deepest elementary kernel."""
        return max(self.niter_j)

    @property
    def ns(self) -> int:
        """Chain products of the longest step kernel."""
        return max(len(f) for f in self.jfactor_ms) - 1


def _strictly_increasing(v) -> bool:
    return all(b > a for a, b in zip(v, v[1:]))


def _curve_index(t_i, t) -> int:
    """First generator date at or after t (the reference's ``for (i...) if (t_i[i] >= t)
    break``)."""
    for i, ti in enumerate(t_i):
        if ti >= t:
            return i
    return len(t_i)


def make_mc_plan(t_k, t_i, dt0_days: int, maxdiag_i) -> McPlan:
    """The plan of steps ``t_k`` over generators ending at ``t_i`` (whole days after today),
    with elementary step cap ``dt0_days`` and max |L_yy| of each generator.  Raises
    ValueError where the reference throws or indexes past its arrays."""
    t_k = [int(t) for t in t_k]
    t_i = [int(t) for t in t_i]
    if not t_k or not t_i:
        raise ValueError("a plan needs at least one step date and one generator date")
    if t_k[0] <= 0 or not _strictly_increasing(t_k):
        raise ValueError("step dates must be strictly increasing and after today")
    if t_i[0] <= 0 or not _strictly_increasing(t_i):
        raise ValueError("generator dates must be strictly increasing and after today")
    if t_i[-1] < t_k[-1]:
        raise ValueError("the last step lies past the last generator date")
    if len(maxdiag_i) != len(t_i):
        raise ValueError("one max |L_yy| per generator")
    if int(dt0_days) < 1:
        raise ValueError("dt0 is a whole number of days, at least 1")

    # elementary dates: the union, sorted, distinct, up to the last step (Common.cs:187-200)
    merged = sorted(t_k + t_i)
    t_q = [merged[0]]
    for t in merged[1:]:
        if t > t_q[-1] and t <= t_k[-1]:
            t_q.append(t)
    nq = len(t_q)

    # generator of each elementary interval (Common.cs:202-208)
    i_q, i = [], 0
    for t in t_q:
        if t > t_i[i]:
            i += 1
        i_q.append(i)

    def length(q):
        return t_q[q] - (t_q[q - 1] if q > 0 else 0)

    # distinct elementary kernels (Common.cs:210-259)
    todo_q = [True] * nq
    for q2 in range(1, nq):
        if length(q2) == length(0) and i_q[0] == i_q[q2]:
            todo_q[q2] = False
    for q1 in range(1, nq):
        for q2 in range(q1 + 1, nq):
            if length(q2) == length(q1) and i_q[q1] == i_q[q2]:
                todo_q[q2] = False
    j_q = [0] * nq
    nj = 0
    for q1 in range(nq):
        if todo_q[q1]:
            j_q[q1] = nj
            nj += 1
            for q2 in range(q1 + 1, nq):
                if i_q[q1] == i_q[q2] and length(q2) == length(q1):
                    j_q[q2] = j_q[q1]
    t0_j, t1_j, i_j = [0] * nj, [0] * nj, [0] * nj
    for q in range(nq):
        if todo_q[q]:
            j = j_q[q]
            t0_j[j] = t_q[q - 1] if q > 0 else 0
            t1_j[j] = t_q[q]
            i_j[j] = i_q[q]

    # the niter rule per elementary kernel (Common.cs:289-307)
    lib = _lib.load()
    niter_j, dt_j = [], []
    dt0 = int(dt0_days) / DAYS_PER_YEAR
    for j in range(nj):
        n, dt = C.c_int(), C.c_double()
        delta_t = (t1_j[j] - t0_j[j]) / DAYS_PER_YEAR
        r = lib.opb_plan_interval(float(maxdiag_i[i_j[j]]), delta_t, dt0, C.byref(n), C.byref(dt))
        if r != 0:
            raise ValueError(f"opb_plan_interval rejected kernel {j}: status {r}")
        niter_j.append(n.value)
        dt_j.append(dt.value)

    # step kernels: steps of equal length under one generator share one (Common.cs:323-420)
    def step_key(k):
        start = t_k[k - 1] if k > 0 else 0
        i_end = _curve_index(t_i, t_k[k])
        i_start = _curve_index(t_i, t_k[k - 1]) if k > 0 else 0
        return i_end, i_start, t_k[k] - start

    nk = len(t_k)
    todo_k = [True] * nk
    for k1 in range(nk):
        i1, ii1, dt1 = step_key(k1)
        if i1 == ii1:
            for k2 in range(k1 + 1, nk):
                i2, ii2, dt2 = step_key(k2)
                if i2 == ii2 and i1 == i2 and dt1 == dt2:
                    todo_k[k2] = False
    m_k = [0] * nk
    nm = 0
    for k in range(nk):
        if todo_k[k]:
            m_k[k] = nm
            nm += 1
    for k1 in range(nk):
        if todo_k[k1]:
            i1, ii1, dt1 = step_key(k1)
            if i1 == ii1:
                for k2 in range(k1 + 1, nk):
                    i2, ii2, dt2 = step_key(k2)
                    if i2 == ii2 and i1 == i2 and dt1 == dt2:
                        m_k[k2] = m_k[k1]

    # factor lists (Common.cs:431-475)
    jfactor_ms: list[list[int] | None] = [None] * nm
    for k in range(nk):
        t0 = t_k[k - 1] if k > 0 else 0
        t1 = t_k[k]
        factors = [j_q[q] for q in range(nq) if (t_q[q - 1] if q > 0 else 0) >= t0 and t_q[q] <= t1]
        m = m_k[k]
        if jfactor_ms[m] is None:
            jfactor_ms[m] = factors
        elif jfactor_ms[m] != factors:
            raise RuntimeError("internal error: steps sharing a kernel have different factors")
    return McPlan(t_k=t_k, t_i=t_i, t_q=t_q, i_q=i_q, j_q=j_q, t0_j=t0_j, t1_j=t1_j, i_j=i_j, niter_j=niter_j,
                  dt_j=dt_j, m_k=m_k, jfactor_ms=jfactor_ms)


def plan_years(plan: McPlan) -> list[float]:
    """Step lengths in years, for discounting (days / 365.25)."""
    return [(t - (plan.t_k[k - 1] if k > 0 else 0)) / DAYS_PER_YEAR for k, t in enumerate(plan.t_k)]
