"""Drop-in entry points against the reference's own CUDA kernels.

``oracle/_ref/libref_opcuda.so`` is built by ``oracle/Makefile`` from the reference's
unchanged sources (oplib/opcuda/sck.cu, sek.cu, sdot2.cu, sgemv3.cu, sgsvg.cu, sset.cu) with
its own compiler flags, and ``oracle/ref_opcuda.cu`` launches each ``__global__`` kernel with
the reference wrapper's launch shape and 64-bit pointers (the reference's exported wrappers
take 32-bit handles).  Both sides get the same device inputs; the outputs are compared:

- bit for bit where the drop-in performs the reference's FP32 operations in the reference's
  order: cumulative rows (``sck``), the kernels from generators (``sek``, ``sekd``,
  ``sekd_lambda``), the strided dot products (``sdot2``, a sequential fused sum), the
  multi-vector induction (``sgemv3``, a sequential fused sum over k per column) and the
  fills (``ssetall``, ``ssetone``);
- within FP32 rounding for the jump generator (``sgsvg``), which the drop-in forms in FP64:
  both against the FP64 restatement, and against each other, relative to each row's
  largest rate.

Sizes stay inside the reference kernels' own bounds: d % 64 == 0 and column lists padded
to 16 entries for ``sgemv3``, nx*nr % 32 == 0 for ``sgsvg``, i < 128 for ``ssetone`` (its
one-block launch, sset.cu:68-72, sets nothing beyond index 127).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import ref_opcuda

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(cuda):
    if not ref_opcuda.available():
        pytest.skip("oracle/_ref/libref_opcuda.so not built (the reference's sources were absent at build time)")
    return ref_opcuda.load()


@pytest.fixture(scope="module")
def lib(cuda):
    from oplib_b200 import _lib
    return _lib.load()


def _dev(a, cuda):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def _bits(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("d,nm", [(300, 3), (512, 2), (31, 1)])
def test_sck_bit_exact_vs_reference_kernel(lib, ref, cuda, d, nm):
    rng = np.random.default_rng(d + nm)
    P = rng.random((nm, d, d)).astype(np.float32)
    P[P < 0.3] = 0.0                      # sparse rows, as after a few squarings of a stencil
    P[:, :, 0] += 1e-3                    # every row has mass (the kernel divides by the total)
    src = _dev(P.ravel(), cuda)
    mine = torch.empty_like(src)
    theirs = torch.empty_like(src)
    assert lib.opcuda_sck(d, nm, src.data_ptr(), mine.data_ptr()) == 0
    torch.cuda.synchronize()
    assert ref.ref_sck(d, nm, src.data_ptr(), theirs.data_ptr()) == 0
    assert np.array_equal(_bits(mine), _bits(theirs))


@pytest.mark.parametrize("d", [77, 512])
def test_sek_family_bit_exact_vs_reference_kernel(lib, ref, cuda, d):
    rng = np.random.default_rng(d)
    gen = rng.standard_normal(d * d).astype(np.float32) * 40.0
    r = rng.uniform(0.0, 0.2, d).astype(np.float32)
    lam = np.array([1.37], dtype=np.float32)
    g, dr, dl = _dev(gen, cuda), _dev(r, cuda), _dev(lam, cuda)
    dt = float(np.float32(1.0 / 3000.0))
    for name, extra in [("sek", []), ("sekd", [dr]), ("sekd_lambda", [dr, dl])]:
        mine = torch.empty(d * d, device=cuda)
        theirs = torch.empty(d * d, device=cuda)
        ptrs = [t.data_ptr() for t in extra]
        assert getattr(lib, "opcuda_" + name)(d, g.data_ptr(), dt, mine.data_ptr(), *ptrs) == 0
        torch.cuda.synchronize()
        assert getattr(ref, "ref_" + name)(d, g.data_ptr(), dt, theirs.data_ptr(), *ptrs) == 0
        assert np.array_equal(_bits(mine), _bits(theirs)), name


@pytest.mark.parametrize("m,n", [(300, 517), (64, 1), (1, 2048)])
def test_sdot2_bit_exact_vs_reference_kernel(lib, ref, cuda, m, n):
    rng = np.random.default_rng(m * n)
    a = _dev(rng.standard_normal(m * n).astype(np.float32), cuda)
    b = _dev(rng.standard_normal(m * n).astype(np.float32), cuda)
    mine = torch.full((m,), np.nan, device=cuda)
    theirs = torch.full((m,), np.nan, device=cuda)
    assert lib.opcuda_sdot2(a.data_ptr(), b.data_ptr(), mine.data_ptr(), m, n) == 0
    torch.cuda.synchronize()
    assert ref.ref_sdot2(a.data_ptr(), b.data_ptr(), theirs.data_ptr(), m, n) == 0
    assert np.array_equal(_bits(mine), _bits(theirs))


@pytest.mark.parametrize("d,nz,ncol,stop", [(512, 8, 16, None), (256, 20, 32, 27), (1024, 3, 16, 2)])
def test_sgemv3_bit_exact_vs_reference_kernel(lib, ref, cuda, d, nz, ncol, stop):
    """Z holds 2*nz columns of d: inputs in the first nz, outputs in the last nz.  Entry c reads
    column c % nz and writes column nz + (c % nz); `stop` puts the 2*nz*d sentinel at entry
    `stop`, so neither kernel writes that entry or any later one in its 16-entry group."""
    rng = np.random.default_rng(d + nz + ncol)
    A = _dev(rng.standard_normal(d * d).astype(np.float32) / np.sqrt(d), cuda)
    Z0 = rng.standard_normal(2 * nz * d).astype(np.float32)
    col0 = np.array([(c % nz) * d for c in range(ncol)], dtype=np.int32)
    col1 = np.array([(nz + c % nz) * d for c in range(ncol)], dtype=np.int32)
    if stop is not None:
        col1[stop] = 2 * nz * d
    c0, c1 = _dev(col0, cuda), _dev(col1, cuda)
    mine, theirs = _dev(Z0, cuda), _dev(Z0, cuda)
    assert lib.opcuda_sgemv3(d, nz, ncol, A.data_ptr(), mine.data_ptr(), c0.data_ptr(), c1.data_ptr()) == 0
    torch.cuda.synchronize()
    assert ref.ref_sgemv3(d, nz, ncol, A.data_ptr(), theirs.data_ptr(), c0.data_ptr(), c1.data_ptr()) == 0
    assert not np.array_equal(_bits(theirs), Z0.view(np.uint32))  # the reference kernel wrote outputs
    assert np.array_equal(_bits(mine), _bits(theirs))


def test_sgsvg_vs_reference_kernel(lib, ref, cuda):
    """The jump generator on a 16 x 4 grid, two intervals.  Equal lower and upper jump sizes,
    so the reference kernel's use of the lower size on both sides (sgsvg.cu:111-112) does not
    enter the comparison."""
    nx, nr, ni = 16, 4, 2
    d = nx * nr
    xs = 0.05 * 100.0 ** (np.arange(nx) / (nx - 1))
    rs = 0.1 * 8.0 ** (np.arange(nr) / (nr - 1))
    xval, rval = np.tile(xs, nr), np.repeat(rs, nx)
    invm = O.s2d_invm(xval, rval, nx, nr).astype(np.float32)
    rng = np.random.default_rng(11)
    jump = rng.uniform(0.05, 0.2, (ni, d))
    blocks = [np.tile(0.03 * xval, (ni, 1)), np.tile(rval * xval, (ni, 1)), np.tile(2.0 * (0.3 - rval), (ni, 1)),
              np.tile(0.5 * rval, (ni, 1)), jump, jump]
    blocks = [b.astype(np.float32) for b in blocks]
    par = np.concatenate([xval.astype(np.float32)] + [b.ravel() for b in blocks])
    d_par, d_inv = _dev(par, cuda), _dev(invm, cuda)
    mine = torch.zeros(ni * d * d, device=cuda)
    theirs = torch.zeros(ni * d * d, device=cuda)
    assert lib.opcuda_sgsvg(mine.data_ptr(), ni, nx, nr, d_inv.data_ptr(), d_par.data_ptr()) == 0
    torch.cuda.synchronize()
    assert ref.ref_sgsvg(theirs.data_ptr(), ni, nx, nr, d_inv.data_ptr(), d_par.data_ptr()) == 0
    got = mine.cpu().numpy().reshape(ni, d, d).transpose(0, 2, 1).astype(np.float64)   # -> [i][source][target]
    exp = theirs.cpu().numpy().reshape(ni, d, d).transpose(0, 2, 1).astype(np.float64)
    f64 = lambda a: np.asarray(a, dtype=np.float64)
    for i in range(ni):
        G = O.sgsvg_generator(f64(invm), f64(xval.astype(np.float32)), *[f64(b[i]) for b in blocks], nx, nr)
        scale = np.abs(G).max(axis=1, keepdims=True)
        # the reference kernel's FP32 sums and expf against the FP64 restatement
        assert np.all(np.abs(exp[i] - G) <= 2e-5 * scale), np.max(np.abs(exp[i] - G) / scale)
        assert np.all(np.abs(got[i] - exp[i]) <= 2e-5 * scale), np.max(np.abs(got[i] - exp[i]) / scale)
        assert np.count_nonzero(exp[i] > 1e-30 * scale) > 4 * d  # jumps across vol levels are present


def test_sset_bit_exact_vs_reference_kernel(lib, ref, cuda):
    n = 5000
    for incx in (1, 3):
        mine = torch.zeros(n * incx, device=cuda)
        theirs = torch.zeros(n * incx, device=cuda)
        assert lib.opcuda_ssetall(mine.data_ptr(), n, 0.625, incx) == 0
        torch.cuda.synchronize()
        assert ref.ref_ssetall(theirs.data_ptr(), n, 0.625, incx) == 0
        assert np.array_equal(_bits(mine), _bits(theirs))
    for i in (0, 77, 127):
        assert lib.opcuda_ssetone(mine.data_ptr(), n, -2.5, i) == 0
        torch.cuda.synchronize()
        assert ref.ref_ssetone(theirs.data_ptr(), n, -2.5, i) == 0
    assert np.array_equal(_bits(mine), _bits(theirs))


# ---- the reference's kernels that read device tables of 32-bit pointers (ssqmm, sgemm4,
# sgemv4), run on memory placed below 4 GB of device address space

@pytest.fixture(scope="module")
def low(ref, cuda, low_reservation):
    """The session's memory below 4 GB (reserved when its first GPU test started); each
    module using it starts carving from its base."""
    base, size, status = low_reservation
    if base is None:
        pytest.skip(f"no device memory below 4 GB of address space here (ref_low_alloc: {status})")
    assert 0 < base and base + size <= 1 << 32
    return ref_opcuda.LowArena(ref, base, size)


def _colmajor(a):
    return np.asfortranarray(a).ravel(order="K").copy()


def test_ssqmm_bit_exact_vs_reference_kernel(lib, ref, low, cuda):
    """The FP32 squaring drop-in (64-bit pointer tables) against global_ssqmm (32-bit tables)
    on the same column-major matrices, three products at d = 256, one of them a square."""
    d, ni = 256, 3
    rng = np.random.default_rng(4)
    A = [rng.random((d, d)).astype(np.float32) / d for _ in range(ni)]
    B = [A[0]] + [rng.random((d, d)).astype(np.float32) / d for _ in range(ni - 1)]
    a_low = [low.put(_colmajor(a)) for a in A]
    b_low = [low.put(_colmajor(b)) for b in B]
    c_low = [low.alloc(d * d * 4) for _ in range(ni)]
    tabs = [low.put(np.array(t, dtype=np.uint32)) for t in (a_low, b_low, c_low)]
    assert ref.ref_ssqmm(d, ni, *tabs) == 0
    mine = [torch.empty(d * d, device=cuda) for _ in range(ni)]
    t64 = [torch.tensor(t, dtype=torch.int64, device=cuda) for t in (a_low, b_low, [m.data_ptr() for m in mine])]
    assert lib.opcuda_ssqmm(d, ni, *[t.data_ptr() for t in t64]) == 0
    torch.cuda.synchronize()
    for i in range(ni):
        theirs = low.get(c_low[i], d * d, np.float32)
        assert np.array_equal(mine[i].cpu().numpy().view(np.uint32), theirs.view(np.uint32)), i
        ref64 = A[i].astype(np.float64) @ B[i].astype(np.float64)
        assert np.abs(theirs.reshape(d, d).T - ref64).max() < 1e-5 * np.abs(ref64).max()


def test_sgemm4_bit_exact_vs_reference_kernel(lib, ref, low, cuda):
    """Grouped column-major products through task tables: the drop-in's widened records
    (64-bit pointers) against global_sgemm4's 9-word records (32-bit), same tiles."""
    rng = np.random.default_rng(5)
    shapes = [(128, 32, 64), (64, 48, 80), (192, 16, 128)]
    mats, ref_tasks, my_tasks, outs = [], [], [], []
    for i, (m, n, k) in enumerate(shapes):
        A = rng.standard_normal((m, k)).astype(np.float32)
        B = rng.standard_normal((k, n)).astype(np.float32)
        a, b, c = low.put(_colmajor(A)), low.put(_colmajor(B)), low.alloc(m * n * 4)
        dC = torch.zeros(m * n, device=cuda)
        mats.append((m, n, c))
        outs.append(dC)
        for bx in range(m // 64):
            for by in range(n // 16):
                ref_tasks.append([i, bx, by, m, n, k, a, b, c])
                my_tasks.append((i, bx, by, m, n, k, a, b, dC.data_ptr()))
    recs = [low.put(np.array(t, dtype=np.uint32)) for t in ref_tasks]
    assert ref.ref_sgemm4(len(recs), low.put(np.array(recs, dtype=np.uint32))) == 0
    sz = lib.opb_sgemm4_task_size()
    rec = np.zeros((len(my_tasks), sz // 8), dtype=np.int64)
    for t, (i, bx, by, m, n, k, a, b, c) in enumerate(my_tasks):
        rec[t, :3] = np.array([i, bx, by, m, n, k], dtype=np.int32).view(np.int64)
        rec[t, 3:6] = [a, b, c]
    drec = torch.from_numpy(rec.ravel()).to(cuda)
    ptrs = torch.tensor([drec.data_ptr() + t * sz for t in range(len(my_tasks))], dtype=torch.int64, device=cuda)
    assert lib.opcuda_sgemm4(len(my_tasks), ptrs.data_ptr()) == 0
    torch.cuda.synchronize()
    for (m, n, c), dC in zip(mats, outs):
        assert np.array_equal(dC.cpu().numpy().view(np.uint32), low.get(c, m * n, np.float32).view(np.uint32))


def test_sgemv4_bit_exact_vs_reference_kernel(lib, ref, low, cuda):
    """Multi-vector induction through task tables (global_sgemv4's 64-row blocks against the
    drop-in's 128-row blocks) on two matrices, with a sentinel in one column list."""
    rng = np.random.default_rng(6)
    d, nz = 256, 6
    ref_tasks, my_tasks, zs = [], [], []
    for i in range(2):
        A = (rng.standard_normal((d, d)) / np.sqrt(d)).astype(np.float32)
        Z0 = rng.standard_normal(2 * nz * d).astype(np.float32)
        col0 = np.array([(c % nz) * d for c in range(16)], dtype=np.int32)
        col1 = np.array([(nz + c % nz) * d for c in range(16)], dtype=np.int32)
        if i == 1:
            col1[9] = 2 * nz * d
        a, z, c0, c1 = low.put(_colmajor(A)), low.put(Z0), low.put(col0), low.put(col1)
        mz = torch.from_numpy(Z0.copy()).to(cuda)
        zs.append((z, mz))
        ref_tasks += [[i, bx, 0, d, nz, 16, a, z, c0, c1] for bx in range(d // 64)]
        my_tasks += [(i, bx, 0, d, nz, 16, a, mz.data_ptr(), c0, c1) for bx in range(d // 128)]
    recs = [low.put(np.array(t, dtype=np.uint32)) for t in ref_tasks]
    assert ref.ref_sgemv4(len(recs), low.put(np.array(recs, dtype=np.uint32))) == 0
    sz = lib.opb_sgemv4_task_size()
    rec = np.zeros((len(my_tasks), sz // 8), dtype=np.int64)
    for t, (i, bx, by, dd, z, ncol, a, zp, c0, c1) in enumerate(my_tasks):
        rec[t, :3] = np.array([i, bx, by, dd, z, ncol], dtype=np.int32).view(np.int64)
        rec[t, 3:7] = [a, zp, c0, c1]
    drec = torch.from_numpy(rec.ravel()).to(cuda)
    ptrs = torch.tensor([drec.data_ptr() + t * sz for t in range(len(my_tasks))], dtype=torch.int64, device=cuda)
    assert lib.opcuda_sgemv4(len(my_tasks), ptrs.data_ptr()) == 0
    torch.cuda.synchronize()
    for z, mz in zs:
        assert np.array_equal(mz.cpu().numpy().view(np.uint32), low.get(z, 2 * nz * d, np.float32).view(np.uint32))
