"""CPU tests of the restated ``opc`` library (``oracle/opc.c``): the reference's CPU
entry points under their own names and argument order, checked against numpy/scipy, the
MT19937 pins, and the reference's own call sequences (S1DGrid.pregen's dgesv solves, the
host bracket table and opc_dmc1's sampler with its payoff callback).  No GPU."""
import ctypes as C
import math

import numpy as np
import pytest
import scipy.linalg
import scipy.special

from oracle import opc
from oracle import oracle as O
from oracle import oracle_c as OC

F32_EPS, F64_EPS = np.finfo(np.float32).eps, np.finfo(np.float64).eps


def p(a):
    return a.ctypes.data


@pytest.fixture(scope="module")
def lib():
    return opc.load()


def colmajor(m, ld):
    """Column-major buffer of m with leading dimension ld >= rows (padding = NaN, which a
    correct routine never reads)."""
    rows, cols = m.shape
    buf = np.full((cols, ld), np.nan, dtype=m.dtype)
    buf[:, :rows] = m.T
    return buf


@pytest.mark.parametrize("dt,fn", [(np.float32, "opc_sgemm"), (np.float64, "opc_dgemm")])
def test_gemm(lib, dt, fn):
    rng = np.random.default_rng(1)
    for m, n, k in [(7, 5, 3), (64, 33, 100), (1, 1, 1), (5, 4, 0)]:
        A = rng.standard_normal((m, k)).astype(dt)
        B = rng.standard_normal((k, n)).astype(dt)
        a, b = colmajor(A, m + 3), colmajor(B, k + 1)
        c = colmajor(np.full((m, n), 7, dtype=dt), m + 2)
        getattr(lib, fn)(p(a), p(b), p(c), m + 3, max(k + 1, 1), m + 2, m, n, k)
        got = c[:, :m].T
        ref = A.astype(np.float64) @ B.astype(np.float64)
        bound = (k + 1) * (F32_EPS if dt == np.float32 else F64_EPS) * (np.abs(A) @ np.abs(B)) + 1e-300
        assert np.all(np.abs(got - ref) <= bound), (m, n, k)
        assert np.isnan(c[:, m:]).all()  # nothing written past m in any column


@pytest.mark.parametrize("dt,fn", [(np.float32, "opc_sgemv"), (np.float64, "opc_dgemv")])
def test_gemv_increments_alpha_beta(lib, dt, fn):
    rng = np.random.default_rng(2)
    m, n = 37, 23
    A = rng.standard_normal((m, n)).astype(dt)
    a = colmajor(A, m + 5)
    for incx, incy, alpha, beta in [(1, 1, 1.0, 0.0), (2, -1, 0.5, 2.0), (-3, 2, -1.0, 1.0), (1, 1, 0.0, 3.0)]:
        x = rng.standard_normal(n * abs(incx)).astype(dt)
        y = rng.standard_normal(m * abs(incy)).astype(dt)
        if beta == 0.0:
            y[:] = np.nan  # BLAS: beta = 0 overwrites y without reading it
        xv = x[:: abs(incx)][:n] if incx > 0 else x[:: abs(incx)][:n][::-1]
        yv = y[:: abs(incy)][:m] if incy > 0 else y[:: abs(incy)][:m][::-1]
        ref = alpha * (A.astype(np.float64) @ xv.astype(np.float64)) + (0.0 if beta == 0.0 else beta * yv)
        getattr(lib, fn)(m, n, alpha, p(a), m + 5, p(x), incx, beta, p(y), incy)
        got = y[:: abs(incy)][:m] if incy > 0 else y[:: abs(incy)][:m][::-1]
        eps = F32_EPS if dt == np.float32 else F64_EPS
        bound = (n + 2) * eps * (abs(alpha) * (np.abs(A) @ np.abs(xv)) + abs(beta) * np.abs(np.nan_to_num(yv)))
        assert np.all(np.abs(got - ref) <= bound + 1e-300), (incx, incy, alpha, beta)


def test_dcopy(lib):
    src = np.arange(10, dtype=np.float64)
    dst = np.full(12, -1.0)
    lib.opc_dcopy(10, p(dst), p(src))
    assert np.array_equal(dst[:10], src) and np.all(dst[10:] == -1)


@pytest.mark.parametrize("n,nrhs", [(2, 2), (4, 4), (50, 3)])
def test_dgesv_matches_lapack_getrf(lib, n, nrhs):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, nrhs))
    a, b = colmajor(A, n + 1), colmajor(B, n + 2)
    ipiv = np.zeros(n, dtype=np.int32)
    assert lib.opc_dgesv(n, nrhs, p(a), n, n, n + 1, p(ipiv), p(b), n + 2) == 0
    lu, piv = scipy.linalg.lu_factor(A)
    assert np.array_equal(ipiv, piv + 1)  # 1-based LAPACK pivots
    assert np.allclose(a[:, :n].T, lu, rtol=0, atol=1e-12 * n)
    assert np.allclose(b[:, :n].T, np.linalg.solve(A, B), rtol=1e-10, atol=1e-12)


def test_sgesv_and_singular_info(lib):
    A = np.array([[2.0, 1.0, 1.0], [4.0, 2.0, 2.0], [1.0, 0.0, 3.0]], dtype=np.float32)  # rank 2
    a, b = colmajor(A, 3), colmajor(np.eye(3, dtype=np.float32), 3)
    ipiv, info = np.zeros(3, dtype=np.int32), np.zeros(1, dtype=np.int32)
    r = lib.opc_sgesv(3, 3, p(a), 3, 3, 3, p(ipiv), p(b), 3, p(info))
    assert r == info[0] == 3  # U(3,3) is exactly zero
    assert np.array_equal(b, np.eye(3, dtype=np.float32).T)  # no solve after a zero pivot
    A = np.array([[3.0, 1.0], [1.0, 2.0]], dtype=np.float32)
    a, b = colmajor(A, 2), colmajor(np.eye(2, dtype=np.float32), 2)
    assert lib.opc_sgesv(2, 2, p(a), 2, 2, 2, p(ipiv), p(b), 2, p(info)) == 0
    assert np.allclose(b.T, np.linalg.inv(A.astype(np.float64)), rtol=2e-7)
    assert lib.opc_dgesv(-1, 1, None, 0, 0, 1, None, None, 1) == -1
    assert lib.opc_dgesv(3, 1, None, 3, 3, 2, None, None, 3) == -4


def test_s1dgrid_pregen_through_dgesv_matches_oracle_invm(lib):
    """S1DGrid.pregen (oplib/opmodel/types/S1DGrid.cs:78-147) step for step: identity
    blocks in invm, the 2x2 moment matrix per node, opc_dgesv(2, 2, mat, 2, 2, 2, ipiv,
    invm + 4*x0, 2).  The branch structure is the reference's: the second row is
    [dm^2, dp^2] whenever 0 < x0 < d, so also for the last node (dp = 1 there), and the
    boundary rows [0, 1] / [1, 0] sit in the else branch, of which only x0 == 0 is ever
    taken.  The oracle's lv_invm must be the same inverses."""
    x = 0.05 * 100.0 ** (np.arange(512) / 511.0)
    d = x.size
    invm = np.zeros(4 * d)
    for xx in range(d):
        for z in range(2):
            invm[4 * xx + z + 2 * z] = 1.0
    ipiv = np.zeros(20, dtype=np.int32)
    for x0 in range(d):
        mat = np.zeros(4)
        mat[0] = x[x0 - 1] - x[x0] if x0 > 0 else 1.0
        mat[2] = x[x0 + 1] - x[x0] if x0 < d - 1 else 1.0
        if 0 < x0 < d:
            mat[1], mat[3] = mat[0] ** 2, mat[2] ** 2
        else:
            if x0 == 0:
                mat[1], mat[3] = 0.0, 1.0
            if x0 == d - 1:
                mat[1], mat[3] = 1.0, 0.0
        blk = invm[4 * x0:4 * x0 + 4].copy()
        assert lib.opc_dgesv(2, 2, p(mat), 2, 2, 2, p(ipiv), p(blk), 2) == 0
        invm[4 * x0:4 * x0 + 4] = blk
    ref = O.lv_invm(x)  # (d, 2, 2) row-major
    got = invm.reshape(d, 2, 2).transpose(0, 2, 1)  # column-major blocks
    assert np.allclose(got, ref, rtol=1e-12, atol=0)
    # the last node's moment matrix is [[dm, 1], [dm^2, 1]]
    dm = x[-2] - x[-1]
    assert np.allclose(got[-1], np.linalg.inv([[dm, 1.0], [dm * dm, 1.0]]), rtol=1e-12, atol=0)


@pytest.mark.parametrize("xs,rs", [((0.05, 5.0), (0.05, 1.0)), ((10.0, 300.0), (0.5, 40.0))])
def test_s2dgrid_pregen_through_dgesv_matches_oracle_invm(lib, xs, rs):
    """S2DGrid.pregen (oplib/opmodel/types/S2DGrid.cs:123-245) literally: identity blocks
    in invm, one 4 x 4 buffer reused for every node (opc_dgesv overwrites it with its LU
    factors and the loop never resets entries (1, 2) and (1, 3); they stay zero because
    the x and r blocks never mix), opc_dgesv(4, 4, mat, 4, 4, 4, ipiv, invm + 16*y0, 4).
    The oracle's s2d_invm must be the same inverses -- on grids with spacings below and
    above 1, so both pivot orders of the 2 x 2 blocks occur."""
    nx, nr = 12, 5
    xg = xs[0] * (xs[1] / xs[0]) ** (np.arange(nx) / (nx - 1))
    rg = rs[0] * (rs[1] / rs[0]) ** (np.arange(nr) / (nr - 1))
    d = nx * nr
    xval = np.tile(xg, nr)
    rval = np.repeat(rg, nx)
    invm = np.zeros(16 * d)
    for y in range(d):
        for i in range(4):
            invm[16 * y + i + 4 * i] = 1.0
    mat = np.zeros(16)
    ipiv = np.zeros(4, dtype=np.int32)
    ld = 4
    for x0 in range(nx):
        for a0 in range(nr):
            y0 = x0 + nx * a0
            mat[0 + ld * 0] = xval[y0 - 1] - xval[y0] if x0 > 0 else 0.0
            mat[0 + ld * 1] = xval[y0 + 1] - xval[y0] if x0 < nx - 1 else 0.0
            mat[0 + ld * 2] = mat[0 + ld * 3] = 0.0
            if 0 < x0 < nx - 1:
                mat[1 + ld * 0], mat[1 + ld * 1] = mat[0] ** 2, mat[0 + ld * 1] ** 2
            if x0 == 0:
                mat[1 + ld * 0], mat[1 + ld * 1] = 1.0, 0.0
            if x0 == nx - 1:
                mat[1 + ld * 0], mat[1 + ld * 1] = 0.0, 1.0
            mat[2 + ld * 0] = mat[2 + ld * 1] = 0.0
            mat[2 + ld * 2] = rval[y0 - nx] - rval[y0] if a0 > 0 else 0.0
            mat[2 + ld * 3] = rval[y0 + nx] - rval[y0] if a0 < nr - 1 else 0.0
            mat[3 + ld * 0] = mat[3 + ld * 1] = 0.0
            if 0 < a0 < nr - 1:
                mat[3 + ld * 2], mat[3 + ld * 3] = mat[2 + ld * 2] ** 2, mat[2 + ld * 3] ** 2
            if a0 == 0:
                mat[3 + ld * 2], mat[3 + ld * 3] = 1.0, 0.0
            if a0 == nr - 1:
                mat[3 + ld * 2], mat[3 + ld * 3] = 0.0, 1.0
            blk = invm[16 * y0:16 * y0 + 16].copy()
            assert lib.opc_dgesv(4, 4, p(mat), 4, 4, 4, p(ipiv), p(blk), 4) == 0
            invm[16 * y0:16 * y0 + 16] = blk
            assert mat[1 + ld * 2] == 0.0 and mat[1 + ld * 3] == 0.0
    assert np.allclose(invm, O.s2d_invm(xval, rval, nx, nr), rtol=1e-12, atol=1e-12 * np.abs(invm).max())


def test_rangen_streams(lib):
    seeds = np.array([5489, 7, 4294967295], dtype=np.uint32)
    lib.opc_rangen_init_seed(p(seeds), 3)
    assert lib.opc_rangen_getstatus() == 0
    r = np.empty(1000)
    lib.opc_genunif(p(r), 1000, -1.0, 3.0, 1)
    assert lib.opc_rangen_getstatus() == 0
    assert np.array_equal(r, -1.0 + 4.0 * (OC.mt_outputs(7, 1000).astype(np.float64) * 2.0 ** -32))
    # a stream continues across calls; other threads' streams are untouched
    r2 = np.empty(10)
    lib.opc_genunif(p(r2), 10, 0.0, 1.0, 1)
    assert np.array_equal(r2, OC.mt_outputs(7, 1010)[1000:] * 2.0 ** -32)
    lib.opc_genunif(p(r2), 10, 0.0, 1.0, 2)
    assert np.array_equal(r2, OC.mt_outputs(4294967295, 10) * 2.0 ** -32)
    u = np.empty(4096, dtype=np.float32)
    assert lib.opc_mt_benchmark(4096, p(u), 0) == 0
    bits = OC.mt_outputs(5489, 4096)
    assert np.array_equal(u, bits.astype(np.float32) / np.float32(2.0 ** 32))
    lib.opc_genunif(p(r2), 10, 0.0, 1.0, 3)  # no such thread
    assert lib.opc_rangen_getstatus() < 0
    lib.opc_rangen_finalize()
    lib.opc_genunif(p(r2), 10, 0.0, 1.0, 0)
    assert lib.opc_rangen_getstatus() < 0


def test_gennor_inverts_the_normal_cdf(lib):
    seeds = np.array([20260], dtype=np.uint32)
    lib.opc_rangen_init_seed(p(seeds), 1)
    n = 1 << 16
    r = np.empty(n)
    lib.opc_gennor(p(r), n, 0.25, 2.0, 0)
    u = (OC.mt_outputs(20260, n).astype(np.float64) + 0.5) * 2.0 ** -32
    z = scipy.special.ndtri(u)
    assert np.all(np.abs((r - 0.25) / 2.0 - z) <= 8 * F64_EPS * np.maximum(1.0, np.abs(z)))
    assert abs(r.mean() - 0.25) < 4 * 2.0 / np.sqrt(n) and abs(r.std() / 2.0 - 1.0) < 0.02
    lib.opc_rangen_finalize()


@pytest.fixture(scope="module")
def lv64():
    cfg = O.LVLattice(n=64)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 52, cfg.dt0)
    P = O.square(O.ek(L, dt), niter)  # source-major rows
    return P, O.nearest_node(x)


def test_host_bracket_table(lib, lv64):
    """opc_host_mc_hash against a numpy restatement of host_d_mc_hash: cumulative rows
    normalised from the second column on (the first keeps the raw entry), brackets that
    contain the inverse-CDF answer of every bucket."""
    P, _ = lv64
    d = P.shape[0]
    mats = (P, P @ P)
    tpk_cm = np.concatenate([np.asfortranarray(m).ravel(order="K") for m in mats])
    ctpk = np.empty(2 * d * d)
    hash_ = np.empty(2 * d * d, dtype=np.int32)
    lib.opc_host_mc_hash(p(tpk_cm), d, 2, p(ctpk), p(hash_))
    for m, Pm in enumerate(mats):
        cs = np.cumsum(Pm, axis=1)
        ref = np.minimum(cs / cs[:, -1:], 1.0)
        ref[:, 0] = Pm[:, 0]
        Cm = ctpk[m * d * d:(m + 1) * d * d].reshape(d, d).T  # [y1, y2]
        assert np.allclose(Cm, ref, rtol=1e-15, atol=1e-17)
        H = hash_[m * d * d:(m + 1) * d * d].reshape(d, d).T  # [y1, bucket]
        lb, ub = H & 0xFFFF, H >> 16
        assert np.all(lb <= ub) and np.all(ub < d)
        rng = np.random.default_rng(m)
        for y in rng.integers(0, d, 16):
            u = rng.random(500)
            ans = np.minimum(np.argmax(u[:, None] < Cm[y][None, :], axis=1), d - 1)
            s = (u * d).astype(np.int64)
            assert np.all((lb[y, s] <= ans) & (ans <= ub[y, s]))


def test_dmc1_sampler_and_payoff_callback(lib, lv64):
    """opc_dmc1 (oplib/opc/rangen.cpp:97-153): each state is the smallest y with
    u < C[yprev, y] on the bracket table's cumulative rows, u = x / 2^32 from the thread's
    stream (step-major), and the payoff callback sees the batch once."""
    P, y0 = lv64
    d = P.shape[0]
    tpk = np.asfortranarray(P).ravel(order="K").copy()
    ctpk = np.empty(d * d)
    hash_ = np.empty(d * d, dtype=np.int32)
    lib.opc_host_mc_hash(p(tpk), d, 1, p(ctpk), p(hash_))
    nscen, nk = 512, 30
    seeds = np.array([11, 4242], dtype=np.uint32)
    lib.opc_rangen_init_seed(p(seeds), 2)
    unif = np.empty(nscen, dtype=np.uint32)
    y_sk = np.full(nscen * nk, -1, dtype=np.int16)
    m_k = np.zeros(nk, dtype=np.int32)
    seen = []

    def cb(yp, th, b):
        seen.append((th, b, int(yp[0]), int(yp[nscen * nk - 1])))

    fn = opc.PAYOFF_EVAL(cb)
    addr = C.cast(fn, C.c_void_p).value
    assert lib.opc_dmc1(p(ctpk), p(hash_), d, nscen, nk, y0, p(unif), p(y_sk), p(m_k), addr, 1, 9) == 0
    lib.opc_rangen_finalize()
    assert seen == [(1, 9, int(y_sk[0]), int(y_sk[-1]))]
    Cm = ctpk.reshape(d, d).T
    u = OC.mt_outputs(4242, nscen * nk).reshape(nk, nscen).astype(np.float64) / 2.0 ** 32
    Y = y_sk.reshape(nk, nscen)
    prev = np.full(nscen, y0)
    for k in range(nk):
        ans = np.minimum(np.argmax(u[k][:, None] < Cm[prev], axis=1), d - 1)
        assert np.array_equal(Y[k], ans), k
        prev = Y[k].astype(np.int64)
    assert len(np.unique(Y[-1])) > 5  # the chain moved


def test_dmc1_first_state_bracket(lib):
    """Rows with heavy mass on state 0 and on the last state: the sampler's bracket-at-0
    rule (oplib/opc/rangen.cpp:131-133) and the d-1 cap still give the inverse-CDF answer."""
    rng = np.random.default_rng(5)
    d = 8
    P = rng.random((d, d)) ** 3
    P[:, 0] += 2.0
    P[:, -1] += 1.0
    P /= P.sum(axis=1, keepdims=True)
    tpk = np.asfortranarray(P).ravel(order="K").copy()
    ctpk = np.empty(d * d)
    hash_ = np.empty(d * d, dtype=np.int32)
    lib.opc_host_mc_hash(p(tpk), d, 1, p(ctpk), p(hash_))
    nscen, nk = 4096, 6
    lib.opc_rangen_init_seed(p(np.array([99], dtype=np.uint32)), 1)
    unif = np.empty(nscen, dtype=np.uint32)
    y_sk = np.empty(nscen * nk, dtype=np.int16)
    m_k = np.zeros(nk, dtype=np.int32)
    assert lib.opc_dmc1(p(ctpk), p(hash_), d, nscen, nk, 3, p(unif), p(y_sk), p(m_k), 0, 0, 0) == 0
    lib.opc_rangen_finalize()
    Cm = ctpk.reshape(d, d).T
    u = OC.mt_outputs(99, nscen * nk).reshape(nk, nscen).astype(np.float64) / 2.0 ** 32
    Y = y_sk.reshape(nk, nscen)
    prev = np.full(nscen, 3)
    for k in range(nk):
        ans = np.minimum(np.argmax(u[k][:, None] < Cm[prev], axis=1), d - 1)
        assert np.array_equal(Y[k], ans), k
        prev = Y[k].astype(np.int64)
    assert (Y == 0).mean() > 0.3 and (Y == d - 1).mean() > 0.05


def test_pivot_grid_of_bstest():
    x, y0 = O.pivot_grid(256, O.BSTEST_PIVOTS, O.BSTEST_SPACINGS, 100.0)
    dx = np.diff(x)
    assert x[y0] == 100.0 and np.all(dx > 0)
    # one common scale on the pivot spacings, the finest (1) around the spot; the last node
    # lands on the last pivot, so its spacing (10) is never used
    s = dx[y0]
    assert dx.min() == s and set(np.round(dx / s, 9)) == {1.0, 2.5, 5.0, 7.5}
    assert abs(x[-1] - 300.0) < 7.5 * s and abs(x[0] - 1.0) < 0.01


def test_bstest_through_the_restated_cpu_path(lib):
    """The reference's integration test (tests/bstest/Program.cs:11-37, OPPricer.cs:67-148)
    on its host-FP64 path, call for call: the 256-node pivot grid around S = 100,
    S1DGrid.pregen's opc_dgesv solves, the LV generator with drift r x and vol sigma x,
    one 365-day step planned by the niter rule with dt0 = 1 day, I + dt L squared niter
    times through opc_dgemm, the bracket table, opc_dmc1 with the vanilla payoff evaluator
    as its callback, and discounting over 365 / 365.25 years.  The reference prints the
    price beside the closed form and checks nothing; here the Monte Carlo price must agree
    with the lattice's own expectation within 4 standard errors, and that with the closed
    form within the grid's discretisation error."""
    S, K, r, sig = 100.0, 100.0, 0.05, 0.25
    T, dt0 = 365 / 365.25, 1 / 365.25
    x, y0 = O.pivot_grid(256, O.BSTEST_PIVOTS, O.BSTEST_SPACINGS, S)
    d = x.size
    L = O.lv_generator(x, r * x, sig * x)
    niter, dt = O.plan_niter(L, T, dt0)
    a = np.asfortranarray(O.ek(L, dt)).ravel(order="K").copy()
    c = np.empty_like(a)
    for _ in range(niter):  # host_d_mc_sq: ping-pong through opc_dgemm
        lib.opc_dgemm(p(a), p(a), p(c), d, d, d, d, d, d)
        a, c = c, a
    P = a.reshape(d, d).T
    ctpk = np.empty(d * d)
    hash_ = np.empty(d * d, dtype=np.int32)
    lib.opc_host_mc_hash(p(a), d, 1, p(ctpk), p(hash_))
    nscen, nbatch = 4096 * 25, 12
    lib.opc_rangen_init_seed(p(np.array([12345], dtype=np.uint32)), 1)
    unif = np.empty(nscen, dtype=np.uint32)
    y_sk = np.empty(nscen, dtype=np.int16)
    m_k = np.zeros(1, dtype=np.int32)
    sums = np.zeros(2)

    def evaluate(yp, th, batch):  # VanillaPayoffEvaluator.mc_eval_implementation
        pay = np.maximum(x[np.ctypeslib.as_array(yp, shape=(nscen,))] - K, 0.0)
        sums[0] += pay.sum()
        sums[1] += (pay * pay).sum()

    fn = opc.PAYOFF_EVAL(evaluate)
    addr = C.cast(fn, C.c_void_p).value
    for b in range(nbatch):
        assert lib.opc_dmc1(p(ctpk), p(hash_), d, nscen, 1, y0, p(unif), p(y_sk), p(m_k), addr, 0, b) == 0
    lib.opc_rangen_finalize()
    n = nscen * nbatch
    disc = math.exp(-r * T)
    mean = sums[0] / n
    se = disc * math.sqrt((sums[1] / n - mean * mean) / n)
    price_mc = disc * mean
    price_lattice = disc * (P[y0] @ np.maximum(x - K, 0.0))
    assert abs(price_mc - price_lattice) < 4 * se, (price_mc, price_lattice, se)
    # 12.3301 against 12.3310 (the closed form at T = 365 / 365.25; 12.33600 at T = 1)
    assert abs(price_lattice - float(O.bs_call(S, K, r, sig, T))) < 5e-3, price_lattice


def test_reference_cpu_sampler_and_device_definition_sample_the_same_law(lib, lv64):
    """The reference's CPU Monte Carlo (opc_dmc1: FP64 rows, bracket table, u = x / 2^32)
    and this project's sampling definition (FP32 cumulative rows, u = (x + 1) / 2^32, the
    device kernel's bit-exact oracle) draw from different streams, so they can only agree in
    law: the terminal-state histograms of 2^17 paths x 10 steps each pass a chi-square test
    against the lattice's exact 10-step distribution."""
    import scipy.stats
    P, y0 = lv64
    d = P.shape[0]
    nscen, nk = 1 << 17, 10
    tpk = np.asfortranarray(P).ravel(order="K").copy()
    ctpk = np.empty(d * d)
    hash_ = np.empty(d * d, dtype=np.int32)
    lib.opc_host_mc_hash(p(tpk), d, 1, p(ctpk), p(hash_))
    lib.opc_rangen_init_seed(p(np.array([777], dtype=np.uint32)), 1)
    unif = np.empty(nscen, dtype=np.uint32)
    y_sk = np.empty(nscen * nk, dtype=np.int16)
    m_k = np.zeros(nk, dtype=np.int32)
    assert lib.opc_dmc1(p(ctpk), p(hash_), d, nscen, nk, y0, p(unif), p(y_sk), p(m_k), 0, 0, 0) == 0
    lib.opc_rangen_finalize()
    ref_final = y_sk.reshape(nk, nscen)[-1]
    own_paths, _ = OC.mc_paths(O.cumrows_f32(P), y0, 777, 0, nscen, nk)
    own_final = own_paths[:, -1]
    exact = np.linalg.matrix_power(P, nk)[y0]
    keep = exact * nscen >= 20  # chi-square cells with enough expected counts
    for final in (ref_final, own_final):
        counts = np.bincount(final, minlength=d).astype(np.float64)
        obs = np.append(counts[keep], counts[~keep].sum())
        exp = np.append(exact[keep], exact[~keep].sum()) * nscen
        assert scipy.stats.chisquare(obs, exp).pvalue > 1e-4


def test_dmc1_threads_run_their_own_streams(lib, lv64):
    """host_d_mc_run1f (CModel Host Double.cs:319-377) runs opc_dmc1 on every core at once,
    thread th on stream th: four concurrent threads produce the paths that the same calls
    produce one after another."""
    import threading
    P, y0 = lv64
    d = P.shape[0]
    tpk = np.asfortranarray(P).ravel(order="K").copy()
    ctpk = np.empty(d * d)
    hash_ = np.empty(d * d, dtype=np.int32)
    lib.opc_host_mc_hash(p(tpk), d, 1, p(ctpk), p(hash_))
    nth, nscen, nk = 4, 8192, 12
    seeds = np.array([101, 202, 303, 404], dtype=np.uint32)
    m_k = np.zeros(nk, dtype=np.int32)

    def run(concurrent):
        lib.opc_rangen_init_seed(p(seeds), nth)
        unif = [np.empty(nscen, dtype=np.uint32) for _ in range(nth)]
        ys = [np.empty(nscen * nk, dtype=np.int16) for _ in range(nth)]
        rc = [None] * nth

        def work(th):
            rc[th] = lib.opc_dmc1(p(ctpk), p(hash_), d, nscen, nk, y0, p(unif[th]), p(ys[th]), p(m_k), 0, th, 0)

        if concurrent:
            workers = [threading.Thread(target=work, args=(th,)) for th in range(nth)]
            for w in workers:
                w.start()
            for w in workers:
                w.join()
        else:
            for th in range(nth):
                work(th)
        lib.opc_rangen_finalize()
        assert rc == [0] * nth
        return ys

    together, alone = run(True), run(False)
    for a, b in zip(together, alone):
        assert np.array_equal(a, b)
    assert not np.array_equal(together[0], together[1])
