"""The Monte Carlo step planner (oplib_b200/plan.py, the reference's make_mc_plan,
oplib/opmodel/models/CModel Common.cs:163-486) on the schedules the reference builds and on
ones with generator dates inside steps; its kernels executed in FP64 by the oracle.  No GPU:
the planner is host logic and its niter rule is the library's host-side
opb_plan_interval."""
import numpy as np
import pytest
import scipy.linalg

from oplib_b200.plan import make_mc_plan, plan_years
from oracle import oracle as O


def bstest_generator():
    x, y0 = O.pivot_grid(256, O.BSTEST_PIVOTS, O.BSTEST_SPACINGS, 100.0)
    return O.lv_generator(x, 0.05 * x, 0.25 * x)


def maxdiag(L):
    return float(np.max(np.abs(np.diag(L))))


def test_bstest_plan():
    """tests/bstest: one 365-day step, one generator date at the step, dt0 = 1 day."""
    L = bstest_generator()
    plan = make_mc_plan([365], [365], 1, [maxdiag(L)])
    assert (plan.nq, plan.nj, plan.nm, plan.ns) == (1, 1, 1, 0)
    assert plan.m_k == [0] and plan.jfactor_ms == [[0]]
    niter, dt = O.plan_niter(L, 365 / 365.25, 1 / 365.25)
    assert plan.niter_j == [niter] and plan.dt_j == [dt] and niter == 14
    assert plan_years(plan) == [365 / 365.25]


def test_equal_steps_share_one_kernel():
    """40 weekly steps under one generator (the reference's LV benchmark schedule shape):
    one elementary kernel, one step kernel."""
    t_k = [7 * (k + 1) for k in range(40)]
    plan = make_mc_plan(t_k, [t_k[-1]], 1, [1000.0])
    assert plan.nj == 1 and plan.nm == 1 and plan.m_k == [0] * 40 and plan.jfactor_ms == [[0]]
    assert plan.t_q == t_k and plan.i_q == [0] * 40


def test_uneven_steps_deduplicate_by_length():
    plan = make_mc_plan([10, 20, 35, 50, 60], [60], 1, [1000.0])
    assert plan.j_q == [0, 0, 1, 1, 0] and plan.nj == 2
    assert plan.m_k == [0, 0, 1, 1, 0] and plan.jfactor_ms == [[0], [1]]
    assert (plan.t0_j, plan.t1_j) == ([0, 20], [10, 35])


def test_generator_date_inside_a_step():
    """Steps 30/60/90 days over generators ending at 45 and 90: the middle step runs under
    both, so its kernel is the product of a 15-day kernel of each generator."""
    cfg = O.LVLattice(n=64)
    L0, x = cfg.generator()
    L1 = O.lv_generator(x, 0.03 * x, 0.35 * x)
    plan = make_mc_plan([30, 60, 90], [45, 90], 1, [maxdiag(L0), maxdiag(L1)])
    assert plan.t_q == [30, 45, 60, 90] and plan.i_q == [0, 0, 1, 1]
    assert plan.j_q == [0, 1, 2, 3] and plan.i_j == [0, 0, 1, 1]
    assert plan.m_k == [0, 1, 2] and plan.jfactor_ms == [[0], [1, 2], [3]] and plan.ns == 1
    P = O.mc_plan_kernels(plan, [L0, L1])
    X1 = O.square(O.ek(L0, plan.dt_j[1]), plan.niter_j[1])
    X2 = O.square(O.ek(L1, plan.dt_j[2]), plan.niter_j[2])
    assert np.array_equal(P[1], X1 @ X2)
    # each kernel is the exponential of its generators over its dates, to the first-order
    # error of (I + dt L)^(2^n) at a one-day elementary step (7.7e-3 here)
    exact = scipy.linalg.expm(L0 * 15 / 365.25) @ scipy.linalg.expm(L1 * 15 / 365.25)
    assert np.abs(P[1] - exact).max() < 2e-2
    for Pm in P:
        assert np.allclose(Pm.sum(axis=1), 1.0, atol=1e-12) and Pm.min() > -1e-15


def test_step_ending_on_a_generator_date_keeps_its_own_kernel():
    """A step (45, 90] lies under generator 1 but starts on generator 0's date: the
    reference does not share its kernel (its start index is 0, its end index 1)."""
    plan = make_mc_plan([45, 90, 135], [45, 135], 1, [1000.0, 1000.0])
    assert plan.m_k == [0, 1, 2]
    assert plan.jfactor_ms == [[0], [1], [1]]  # same factor, separate step kernels


@pytest.mark.parametrize("t_k,t_i,dt0", [([30, 20], [30], 1), ([0, 10], [10], 1), ([10, 20], [15], 1),
                                         ([10], [10], 0), ([10], [5, 5, 10], 1)])
def test_plan_rejections(t_k, t_i, dt0):
    with pytest.raises(ValueError):
        make_mc_plan(t_k, t_i, dt0, [1.0] * len(t_i))


def _literal_plan(t_k, t_i):
    """A line-by-line transcription of make_mc_plan's index loops
    (CModel Common.cs:187-259, 323-475), dates in days after today (= 0)."""
    nk, ni = len(t_k), len(t_i)
    t_q = sorted(t_k + t_i)
    q0 = 0
    for q in range(1, len(t_q)):
        if t_q[q] > t_q[q0] and t_q[q] <= t_k[nk - 1]:
            q0 += 1
            t_q[q0] = t_q[q]
    nq = q0 + 1
    t_q = t_q[:nq]
    i_q = [0] * nq
    i = 0
    for q in range(nq):
        if t_q[q] <= t_i[i]:
            i_q[q] = i
        else:
            i += 1
            i_q[q] = i
    todo_q = [True] * nq
    for q2 in range(1, nq):
        if t_q[q2] - t_q[q2 - 1] == t_q[0] - 0 and i_q[0] == i_q[q2]:
            todo_q[q2] = False
    for q1 in range(1, nq):
        for q2 in range(q1 + 1, nq):
            if t_q[q2] - t_q[q2 - 1] == t_q[q1] - t_q[q1 - 1] and i_q[q1] == i_q[q2]:
                todo_q[q2] = False
    j_q = [0] * nq
    nj = 0
    for q1 in range(nq):
        if todo_q[q1]:
            j_q[q1] = nj
            nj += 1
            for q2 in range(q1 + 1, nq):
                if i_q[q1] == i_q[q2]:
                    if q1 == 0:
                        if t_q[q2] - t_q[q2 - 1] == t_q[q1] - 0:
                            j_q[q2] = j_q[q1]
                    elif t_q[q2] - t_q[q2 - 1] == t_q[q1] - t_q[q1 - 1]:
                        j_q[q2] = j_q[q1]

    def first_ge(t):
        ii = 0
        while ii < ni and t_i[ii] < t:
            ii += 1
        return ii

    def key(k):
        i1 = first_ge(t_k[k])
        if k == 0:
            return i1, 0, t_k[k] - 0
        return i1, first_ge(t_k[k - 1]), t_k[k] - t_k[k - 1]

    todo_k = [True] * nk
    for k1 in range(nk):
        i1, ii1, dt1 = key(k1)
        if i1 == ii1:
            for k2 in range(k1 + 1, nk):
                i2, ii2, dt2 = key(k2)
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
            i1, ii1, dt1 = key(k1)
            if i1 == ii1:
                for k2 in range(k1 + 1, nk):
                    i2, ii2, dt2 = key(k2)
                    if i2 == ii2 and i1 == i2 and dt1 == dt2:
                        m_k[k2] = m_k[k1]
    jf = [None] * nm
    for k in range(nk):
        t0 = t_k[k - 1] if k > 0 else 0
        fs = [j_q[q] for q in range(nq) if (t_q[q - 1] if q > 0 else 0) >= t0 and t_q[q] <= t_k[k]]
        if jf[m_k[k]] is None:
            jf[m_k[k]] = fs
    return t_q, i_q, j_q, m_k, jf


def test_planner_matches_a_literal_transcription_on_random_schedules():
    rng = np.random.default_rng(20260)
    for _ in range(300):
        nk = int(rng.integers(1, 12))
        t_k = sorted(set(int(v) for v in rng.integers(1, 200, nk)))
        ni = int(rng.integers(1, 5))
        t_i = sorted(set(int(v) for v in rng.integers(1, 200, ni - 1)) | {t_k[-1] + int(rng.integers(0, 30))})
        plan = make_mc_plan(t_k, t_i, 1, [1000.0] * len(t_i))
        t_q, i_q, j_q, m_k, jf = _literal_plan(t_k, t_i)
        assert (plan.t_q, plan.i_q, plan.j_q, plan.m_k, plan.jfactor_ms) == (t_q, i_q, j_q, m_k, jf)
        # every step's factors tile its interval, and each factor lies under one generator
        for k, m in enumerate(plan.m_k):
            span = sum(plan.t1_j[j] - plan.t0_j[j] for j in plan.jfactor_ms[m])
            assert span == t_k[k] - (t_k[k - 1] if k else 0)
