"""GPU parity of the GEMM / GEMV kernels behind the opcuda ABI.

Floating-point kernels are compared with FP64 references of the same operation:
- split-BF16 tcgen05 GEMM: FP64 product of the same BF16 parts.  The tensor cores
  accumulate in FP32 with truncation, about half an FP32 ulp per MMA instruction, so
  the bound is (3K/16 + 8) * 2^-24 * sum|a||b| (3 products per 16-wide K step);
- FP32 SIMT GEMM / GEMV: FP64 product of the FP32 inputs, relative 1e-5 (the reference's
  own GPU-vs-MKL checks use 2e-3 and 1e-3, benchmarks/gsgemm4/Program.cs:229-291,
  benchmarks/gsgemv4/Program.cs:329-391).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import opc
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bf16_dev(a32: np.ndarray, dev):
    u = np.ascontiguousarray(a32, dtype=np.float32).view(np.uint32) >> np.uint32(16)
    return torch.from_numpy(u.astype(np.uint16).view(np.int16)).to(dev).view(torch.bfloat16)


def _split_dev(a, dev):
    hi, lo = O.split_bf16(a)
    return _bf16_dev(hi, dev), _bf16_dev(lo, dev), hi.astype(np.float64), lo.astype(np.float64)


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (256, 128, 192), (384, 256, 512), (128, 384, 128),
                                   (512, 512, 1024)])
def test_bf16x3_gemm_matches_fp64_of_split(cuda, M, N, K):
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(M + N + K)
    A = rng.random((M, K)).astype(np.float32)
    B = rng.random((N, K)).astype(np.float32)  # K-major right operand (rows of B^T)
    Cin = rng.standard_normal((M, N)).astype(np.float32)
    Ah, Al, ah, al = _split_dev(A, cuda)
    Bh, Bl, bh, bl = _split_dev(B, cuda)
    Cd = torch.from_numpy(Cin).to(cuda)
    Cout = torch.empty_like(Cd)
    nparts = lib.opb_gemm_bf16x3_nparts(M, N)
    rs = torch.empty(nparts * M, dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    st = lib.opb_gemm_bf16x3(M, N, K, Ah.data_ptr(), Al.data_ptr(), K, Bh.data_ptr(), Bl.data_ptr(), K,
                             0.5, Cd.data_ptr(), 2.0, Cout.data_ptr(), N, rs.data_ptr())
    assert st == 0
    torch.cuda.synchronize()
    assert lib.opb_tc_error() == 0
    ref = 0.5 * (ah @ bh.T + ah @ bl.T + al @ bh.T) + 2.0 * Cin.astype(np.float64)
    got = Cout.cpu().numpy().astype(np.float64)
    scale = 0.5 * (np.abs(ah) + np.abs(al)) @ (np.abs(bh) + np.abs(bl)).T + 2 * np.abs(Cin)
    bound = (3 * K / 16 + 8) * 2.0 ** -24
    assert np.all(np.abs(got - ref) <= bound * scale + 1e-30), np.max(np.abs(got - ref) / scale)
    # FP64 row sums of the stored values, per N tile
    parts = rs.cpu().numpy().reshape(nparts, M)
    bn = N // nparts
    for t in range(nparts):
        assert np.allclose(parts[t], got[:, t * bn:(t + 1) * bn].sum(axis=1), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("M,N,K,tile,pair", [(128, 64, 64, 0, 1), (256, 128, 192, 128, 1), (384, 256, 512, 256, 1),
                                             (512, 512, 1024, 256, 1), (512, 512, 1024, 256, 0),
                                             (256, 768, 320, 256, 1), (512, 256, 640, 64, 1)])
def test_kn_operand_matches_transposed_form(cuda, M, N, K, tile, pair):
    """B given K x N row-major (read as an MN-major operand) gives the same bits as the
    K-major product on B's transpose, for every tile width and with and without CTA pairs."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(7 * M + N + K)
    A = rng.random((M, K)).astype(np.float32)
    B = rng.random((K, N)).astype(np.float32)  # K x N row-major
    Ah, Al, _, _ = _split_dev(A, cuda)
    Bh, Bl, _, _ = _split_dev(B, cuda)
    BhT, BlT = Bh.t().contiguous(), Bl.t().contiguous()
    Cd = torch.from_numpy(rng.standard_normal((M, N)).astype(np.float32)).to(cuda)
    outs = []
    try:
        assert lib.opb_set_cta_pair(pair) == 0 and lib.opb_set_tile_n(tile) == 0
        nparts = lib.opb_gemm_bf16x3_nparts(M, N)  # under the forced tile width
        for kn in (0, 1):
            Cout = torch.empty_like(Cd)
            rs = torch.empty(nparts * M, dtype=torch.float64, device=cuda)
            if kn:
                st = lib.opb_gemm_bf16x3_kn(M, N, K, Ah.data_ptr(), Al.data_ptr(), K, Bh.data_ptr(), Bl.data_ptr(), N,
                                            0.5, Cd.data_ptr(), 2.0, Cout.data_ptr(), N, rs.data_ptr())
            else:
                st = lib.opb_gemm_bf16x3(M, N, K, Ah.data_ptr(), Al.data_ptr(), K, BhT.data_ptr(), BlT.data_ptr(), K,
                                         0.5, Cd.data_ptr(), 2.0, Cout.data_ptr(), N, rs.data_ptr())
            assert st == 0
            torch.cuda.synchronize()
            outs.append((Cout.cpu(), rs.cpu()))
    finally:
        lib.opb_set_cta_pair(1)
        lib.opb_set_tile_n(0)
    assert lib.opb_tc_error() == 0
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("M,N,K", [(256, 256, 512), (384, 768, 320), (1024, 512, 2048)])
def test_stage_depth_gives_identical_results(cuda, M, N, K):
    """256-wide tiles with 32-deep (4-stage, 64-byte swizzle) and 64-deep (2-stage,
    128-byte swizzle) pipeline stages issue the same MMAs in the same order: the
    outputs and row sums are bit-identical."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(K)
    A = rng.random((M, K)).astype(np.float32)
    B = rng.random((N, K)).astype(np.float32)
    Ah, Al, _, _ = _split_dev(A, cuda)
    Bh, Bl, _, _ = _split_dev(B, cuda)
    Cd = torch.from_numpy(rng.standard_normal((M, N)).astype(np.float32)).to(cuda)
    nparts = lib.opb_gemm_bf16x3_nparts(M, N)
    outs = []
    try:
        assert lib.opb_set_cta_pair(0) == 0  # stage depth applies to the one-CTA kernel
        for bk in (32, 64):
            assert lib.opb_set_stage_k(bk) == 0
            Cout = torch.empty_like(Cd)
            rs = torch.empty(nparts * M, dtype=torch.float64, device=cuda)
            assert lib.opb_gemm_bf16x3(M, N, K, Ah.data_ptr(), Al.data_ptr(), K, Bh.data_ptr(), Bl.data_ptr(), K,
                                       1.0, Cd.data_ptr(), 1.0, Cout.data_ptr(), N, rs.data_ptr()) == 0
            torch.cuda.synchronize()
            outs.append((Cout.cpu(), rs.cpu()))
    finally:
        lib.opb_set_stage_k(64)
        lib.opb_set_cta_pair(1)
    assert lib.opb_tc_error() == 0
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    assert lib.opb_set_stage_k(48) != 0


@pytest.mark.parametrize("M,N,K", [(256, 256, 512), (512, 768, 320)])
def test_pair_stage_depth_gives_identical_results(cuda, M, N, K):
    """The CTA-pair kernel with B given K x N row-major: 32-deep (6 stages) and 64-deep (3
    stages) pipeline stages give the same bits."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(M * K)
    A = rng.random((M, K)).astype(np.float32)
    B = rng.random((K, N)).astype(np.float32)
    Ah, Al, _, _ = _split_dev(A, cuda)
    Bh, Bl, _, _ = _split_dev(B, cuda)
    Cd = torch.from_numpy(rng.standard_normal((M, N)).astype(np.float32)).to(cuda)
    outs = []
    try:
        assert lib.opb_set_tile_n(256) == 0
        nparts = lib.opb_gemm_bf16x3_nparts(M, N)
        for bk in (32, 64):
            assert lib.opb_set_stage_k(bk) == 0
            Cout = torch.empty_like(Cd)
            rs = torch.empty(nparts * M, dtype=torch.float64, device=cuda)
            assert lib.opb_gemm_bf16x3_kn(M, N, K, Ah.data_ptr(), Al.data_ptr(), K, Bh.data_ptr(), Bl.data_ptr(), N,
                                          1.0, Cd.data_ptr(), 2.0, Cout.data_ptr(), N, rs.data_ptr()) == 0
            torch.cuda.synchronize()
            outs.append((Cout.cpu(), rs.cpu()))
    finally:
        lib.opb_set_stage_k(64)
        lib.opb_set_tile_n(0)
    assert lib.opb_tc_error() == 0
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("M,N,K", [(256, 256, 128), (512, 256, 512), (768, 512, 320), (1024, 1024, 2048)])
def test_cta_pair_gemm_matches_fp64_of_split(cuda, M, N, K):
    """256 x 256 tiles on 2-CTA clusters (cta_group::2): within the same FP32 bound as the
    one-CTA kernel, and row sums of the stored values per 128 columns."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(M * 7 + K)
    A = rng.random((M, K)).astype(np.float32)
    B = rng.random((N, K)).astype(np.float32)
    Cin = rng.standard_normal((M, N)).astype(np.float32)
    Ah, Al, ah, al = _split_dev(A, cuda)
    Bh, Bl, bh, bl = _split_dev(B, cuda)
    Cd = torch.from_numpy(Cin).to(cuda)
    nparts = lib.opb_gemm_bf16x3_nparts(M, N)
    outs = []
    try:
        for pair in (1, 0):
            assert lib.opb_set_cta_pair(pair) == 0
            Cout = torch.empty_like(Cd)
            rs = torch.empty(nparts * M, dtype=torch.float64, device=cuda)
            assert lib.opb_gemm_bf16x3(M, N, K, Ah.data_ptr(), Al.data_ptr(), K, Bh.data_ptr(), Bl.data_ptr(), K,
                                       0.5, Cd.data_ptr(), 2.0, Cout.data_ptr(), N, rs.data_ptr()) == 0
            torch.cuda.synchronize()
            assert lib.opb_tc_error() == 0
            outs.append((Cout.cpu().numpy().astype(np.float64), rs.cpu().numpy().reshape(nparts, M)))
    finally:
        lib.opb_set_cta_pair(1)
    ref = 0.5 * (ah @ bh.T + ah @ bl.T + al @ bh.T) + 2.0 * Cin.astype(np.float64)
    scale = 0.5 * (np.abs(ah) + np.abs(al)) @ (np.abs(bh) + np.abs(bl)).T + 2 * np.abs(Cin)
    bound = (3 * 128 / 16 + 8) * 2.0 ** -24
    got, parts = outs[0]
    assert np.all(np.abs(got - ref) <= bound * scale + 1e-30), np.max(np.abs(got - ref) / scale)
    assert np.array_equal(got, outs[1][0])  # the same MMAs in the same order as one CTA per tile
    bn = N // nparts
    for t in range(nparts):
        assert np.allclose(parts[t], got[:, t * bn:(t + 1) * bn].sum(axis=1), rtol=1e-12, atol=1e-9)
    assert lib.opb_set_cta_pair(2) != 0


def _f16_dev(a32, dev):
    return torch.from_numpy(np.ascontiguousarray(a32, dtype=np.float16).view(np.int16)).to(dev)


@pytest.mark.parametrize("M,N,K", [(128, 64, 128), (256, 256, 512)])
def test_f16x3_gemm_matches_fp64_of_split(cuda, M, N, K):
    """FP16 parts of 2^15-scaled operands: hi = fp16(a*s), lo = fp16(a*s - hi)."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(K)
    s = np.float32(32768.0)
    A = rng.random((M, K)).astype(np.float32)
    B = rng.random((N, K)).astype(np.float32)
    ah = (A * s).astype(np.float16); al = (A * s - ah.astype(np.float32)).astype(np.float16)
    bh = (B * s).astype(np.float16); bl = (B * s - bh.astype(np.float32)).astype(np.float16)
    C = torch.empty(M, N, dtype=torch.float32, device=cuda)
    alpha = 1.0 / (32768.0 * 32768.0)
    assert lib.opb_gemm_f16x3(M, N, K, _f16_dev(ah, cuda).data_ptr(), _f16_dev(al, cuda).data_ptr(), K,
                              _f16_dev(bh, cuda).data_ptr(), _f16_dev(bl, cuda).data_ptr(), K, alpha, None, 0.0,
                              C.data_ptr(), N, None) == 0
    torch.cuda.synchronize()
    f = lambda x: x.astype(np.float64)
    ref = alpha * (f(ah) @ f(bh).T + f(ah) @ f(bl).T + f(al) @ f(bh).T)
    exact = A.astype(np.float64) @ B.astype(np.float64).T
    got = C.cpu().numpy().astype(np.float64)
    assert np.abs(got - ref).max() <= (3 * K / 16 + 8) * 2.0 ** -24 * exact.max()
    # the same parts with B given K x N row-major: identical bits
    C2 = torch.empty_like(C)
    assert lib.opb_gemm_f16x3_kn(M, N, K, _f16_dev(ah, cuda).data_ptr(), _f16_dev(al, cuda).data_ptr(), K,
                                 _f16_dev(bh.T, cuda).data_ptr(), _f16_dev(bl.T, cuda).data_ptr(), N, alpha, None,
                                 0.0, C2.data_ptr(), N, None) == 0
    torch.cuda.synchronize()
    assert lib.opb_tc_error() == 0
    assert torch.equal(C, C2)
    # 22-bit parts: the split product is within ~1e-6 relative of the exact product
    assert np.abs(ref - exact).max() <= 2e-6 * exact.max()


def test_bf16x3_gemm_in_place(cuda):
    """C may alias Cin (the E-form squaring updates E in place)."""
    from oplib_b200 import _lib
    lib = _lib.load()
    M = N = K = 256
    rng = np.random.default_rng(7)
    E = (rng.random((M, K)) * 1e-2).astype(np.float32)
    Ah, Al, ah, al = _split_dev(E, cuda)
    Bh, Bl, bh, bl = _split_dev(np.ascontiguousarray(E.T), cuda)
    X = torch.from_numpy(E).to(cuda)
    assert lib.opb_gemm_bf16x3(M, N, K, Ah.data_ptr(), Al.data_ptr(), K, Bh.data_ptr(), Bl.data_ptr(), K, 1.0,
                               X.data_ptr(), 2.0, X.data_ptr(), N, None) == 0
    torch.cuda.synchronize()
    ref = ah @ bh.T + ah @ bl.T + al @ bh.T + 2.0 * E.astype(np.float64)
    assert np.abs(X.cpu().numpy() - ref).max() < 1e-7


@pytest.mark.parametrize("M,N,K,ksplit", [(6144, 128, 6144, 0), (1024, 64, 2048, 4), (512, 128, 1024, 2),
                                          (384, 128, 512, 2)])
def test_ksliced_product_matches_fp64(cuda, M, N, K, ksplit):
    """opb_gemm_bf16x3_ksliced: the K-slices' partials sum to the FP64 product of the same
    parts (each slice within the tensor cores' FP32 bound over its own K range), and every
    slice is written."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(M + N + K)
    A = (rng.random((M, K)) * (2.0 / K)).astype(np.float32)
    B = rng.random((N, K)).astype(np.float32)
    Ah, Al, ah, al = _split_dev(A, cuda)
    Bh, Bl, bh, bl = _split_dev(B, cuda)
    used = C.c_int(0)
    Cs = torch.full((4 * M * N,), float("nan"), dtype=torch.float32, device=cuda)
    assert lib.opb_gemm_bf16x3_ksliced(M, N, K, Ah.data_ptr(), Al.data_ptr(), K, Bh.data_ptr(), Bl.data_ptr(), K,
                                       Cs.data_ptr(), N, ksplit, M * N, C.byref(used)) == 0
    torch.cuda.synchronize()
    assert lib.opb_tc_error() == 0
    assert used.value == (ksplit if ksplit else lib_split_expected(M, N, K))
    out = Cs[: used.value * M * N].cpu().numpy().reshape(used.value, M, N)
    assert np.isfinite(out).all()
    got = out.astype(np.float64).sum(axis=0)
    ref = ah @ bh.T + ah @ bl.T + al @ bh.T
    scale = (np.abs(ah) + np.abs(al)) @ (np.abs(bh) + np.abs(bl)).T
    bound = (3 * K / 16 + 8) * 2.0 ** -24
    assert np.all(np.abs(got - ref) <= bound * scale + 1e-30)


def lib_split_expected(M, N, K):
    """The automatic slice count: at most 4, dividing K / 64, the one whose items (tiles x
    slices) fill the SMs' waves best; among fills within 0.02, one that reaches every SM, then
    the fewest slices."""
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    tiles = (M // 128) * max(1, N // 128)
    best, best_fill, best_all = 1, -1.0, False
    for sp in range(1, 5):
        if (K // 64) % sp:
            continue
        items = tiles * sp
        fill = items / (-(-items // sms) * sms)
        every = items >= sms
        if fill > best_fill + 0.02 or (fill > best_fill - 0.02 and every and not best_all):
            best, best_fill, best_all = sp, fill, every
    return best


def test_bf16x3_rejects_unsupported_shapes(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    t = torch.zeros(128 * 128, dtype=torch.bfloat16, device=cuda)
    c = torch.zeros(128 * 128, dtype=torch.float32, device=cuda)
    p = t.data_ptr()
    assert lib.opb_gemm_bf16x3(100, 128, 128, p, p, 128, p, p, 128, 1.0, None, 0.0, c.data_ptr(), 128, None) == -4
    assert lib.opb_gemm_bf16x3(128, 128, 96, p, p, 128, p, p, 128, 1.0, None, 0.0, c.data_ptr(), 128, None) == -4
    assert lib.opb_gemm_bf16x3(128, 128, 128, p + 2, p, 128, p, p, 128, 1.0, None, 0.0, c.data_ptr(), 128,
                               None) == -3


@pytest.mark.parametrize("m,n,k", [(64, 64, 64), (100, 37, 129), (576, 576, 576), (7, 300, 5)])
def test_opcuda_sgemm_column_major(cuda, m, n, k):
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(m * n + k)
    A = rng.standard_normal((m, k)).astype(np.float32)
    B = rng.standard_normal((k, n)).astype(np.float32)
    C0 = rng.standard_normal((m, n)).astype(np.float32)
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="K").copy()).to(cuda)
    dB = torch.from_numpy(np.asfortranarray(B).ravel(order="K").copy()).to(cuda)
    dC = torch.from_numpy(np.asfortranarray(C0).ravel(order="K").copy()).to(cuda)
    assert lib.opcuda_sgemm(m, n, k, 1.5, dA.data_ptr(), m, dB.data_ptr(), k, -0.5, dC.data_ptr(), m) == 0
    torch.cuda.synchronize()
    got = dC.cpu().numpy().reshape(n, m).T
    ref = 1.5 * A.astype(np.float64) @ B.astype(np.float64) - 0.5 * C0
    assert np.abs(got - ref).max() <= 1e-5 * (1 + np.abs(ref).max())


def test_opcuda_ssqmm_pointer_tables(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    d, ni = 96, 3
    rng = np.random.default_rng(1)
    mats = [rng.random((d, d)).astype(np.float32) / d for _ in range(ni)]
    A = [torch.from_numpy(np.asfortranarray(m).ravel(order="K").copy()).to(cuda) for m in mats]
    Cs = [torch.empty(d * d, device=cuda) for _ in range(ni)]
    tA = torch.tensor([a.data_ptr() for a in A], dtype=torch.int64, device=cuda)
    tC = torch.tensor([c.data_ptr() for c in Cs], dtype=torch.int64, device=cuda)
    assert lib.opcuda_ssqmm(d, ni, tA.data_ptr(), tA.data_ptr(), tC.data_ptr()) == 0
    torch.cuda.synchronize()
    for m, c in zip(mats, Cs):
        got = c.cpu().numpy().reshape(d, d).T
        ref = m.astype(np.float64) @ m.astype(np.float64)
        assert np.abs(got - ref).max() < 1e-5 * np.abs(ref).max()


def test_opcuda_sgemm4_task_table(cuda):
    """40-GEMM grouped call in the shape of benchmarks/gsgemm4 (reduced sizes)."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(2)
    tasks, mats, outs = [], [], []
    for i, (m, n, k) in enumerate([(128, 32, 64), (64, 48, 80), (192, 16, 128)]):
        A = rng.standard_normal((m, k)).astype(np.float32)
        B = rng.standard_normal((k, n)).astype(np.float32)
        dA = torch.from_numpy(np.asfortranarray(A).ravel(order="K").copy()).to(cuda)
        dB = torch.from_numpy(np.asfortranarray(B).ravel(order="K").copy()).to(cuda)
        dC = torch.zeros(m * n, device=cuda)
        mats.append((A, B, dA, dB))
        outs.append(dC)
        for bx in range((m + 63) // 64):
            for by in range((n + 15) // 16):
                tasks.append((i, bx, by, m, n, k, dA.data_ptr(), dB.data_ptr(), dC.data_ptr()))
    sz = lib.opb_sgemm4_task_size()
    rec = np.zeros((len(tasks), sz // 8), dtype=np.int64)
    for t, (i, bx, by, m, n, k, a, b, c) in enumerate(tasks):
        ints = np.array([i, bx, by, m, n, k], dtype=np.int32).view(np.int64)
        rec[t, :3] = ints
        rec[t, 3:6] = [a, b, c]
    drec = torch.from_numpy(rec.ravel()).to(cuda)
    ptrs = torch.tensor([drec.data_ptr() + t * sz for t in range(len(tasks))], dtype=torch.int64, device=cuda)
    assert lib.opcuda_sgemm4(len(tasks), ptrs.data_ptr()) == 0
    torch.cuda.synchronize()
    for (A, B, _, _), dC in zip(mats, outs):
        m, n = A.shape[0], B.shape[1]
        got = dC.cpu().numpy().reshape(n, m).T
        ref = A.astype(np.float64) @ B
        assert np.abs(got - ref).max() / (1 + np.abs(ref).max()) < 2e-3 * 1e-2
    # the reference's own check (benchmarks/gsgemm4/Program.cs:229-291): the inputs come
    # back unchanged, and every C agrees with the CPU library's
    # opc_sgemm(A, B, C, m, k, m, m, n, k) within |C - C'| / (1 + |C'|) <= 2e-3
    L = opc.load()
    for (A, B, dA, dB), dC in zip(mats, outs):
        (m, k), n = A.shape, B.shape[1]
        a, b = np.asfortranarray(A).ravel(order="K").copy(), np.asfortranarray(B).ravel(order="K").copy()
        assert np.array_equal(dA.cpu().numpy(), a) and np.array_equal(dB.cpu().numpy(), b)
        c = np.empty(m * n, dtype=np.float32)
        L.opc_sgemm(a.ctypes.data, b.ctypes.data, c.ctypes.data, m, k, m, m, n, k)
        assert (np.abs(dC.cpu().numpy() - c) / (1 + np.abs(c))).max() <= 2e-3


def test_opcuda_sgemv_family(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(4)
    m, n = 300, 200
    A = rng.standard_normal((m, n)).astype(np.float32)
    x = rng.standard_normal(n).astype(np.float32)
    xt = rng.standard_normal(m).astype(np.float32)
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="K").copy()).to(cuda)
    dx, dxt = torch.from_numpy(x).to(cuda), torch.from_numpy(xt).to(cuda)
    y = torch.ones(m, device=cuda)
    yt = torch.ones(n, device=cuda)
    assert lib.opcuda_sgemv(m, n, 2.0, dA.data_ptr(), m, dx.data_ptr(), 1, 0.5, y.data_ptr(), 1) == 0
    assert lib.opcuda_sgemvT(m, n, 1.0, dA.data_ptr(), m, dxt.data_ptr(), 1, 0.0, yt.data_ptr(), 1) == 0
    torch.cuda.synchronize()
    assert np.allclose(y.cpu().numpy(), 2 * A.astype(np.float64) @ x + 0.5, rtol=1e-5, atol=1e-4)
    assert np.allclose(yt.cpu().numpy(), A.T.astype(np.float64) @ xt, rtol=1e-5, atol=1e-4)
    # sdot2: c[h] = sum_y a[h + nh*y] b[h + nh*y]
    nh, dd = 37, 91
    a = rng.standard_normal(nh * dd).astype(np.float32)
    b = rng.standard_normal(nh * dd).astype(np.float32)
    da, db, dc = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda), torch.empty(nh, device=cuda)
    assert lib.opcuda_sdot2(da.data_ptr(), db.data_ptr(), dc.data_ptr(), nh, dd) == 0
    torch.cuda.synchronize()
    ref = (a.astype(np.float64) * b).reshape(dd, nh).sum(axis=0)
    assert np.allclose(dc.cpu().numpy(), ref, rtol=1e-5, atol=1e-4)


def test_opcuda_sgemv3_columns_and_sentinel(cuda):
    """Z[:, col1] = A Z[:, col0] for a column list; untouched columns keep their values
    (the non-clobbering check of benchmarks/gsgemv4/Program.cs:345-359)."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(5)
    d, nz = 200, 10
    A = (rng.random((d, d)) / d).astype(np.float32)
    Z = rng.standard_normal((2 * nz, d)).astype(np.float32)  # column j at offset j*d
    col0 = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 0, 1, 2, 3, 4, 5, 6, 7]
    col1 = [10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 2 * nz, 2 * nz, 2 * nz, 2 * nz, 2 * nz, 2 * nz, 2 * nz, 2 * nz]
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="K").copy()).to(cuda)
    dZ = torch.from_numpy(Z.ravel().copy()).to(cuda)
    c0 = torch.tensor([c * d for c in col0], dtype=torch.int32, device=cuda)
    c1 = torch.tensor([c * d for c in col1], dtype=torch.int32, device=cuda)
    assert lib.opcuda_sgemv3(d, nz, len(col0), dA.data_ptr(), dZ.data_ptr(), c0.data_ptr(), c1.data_ptr()) == 0
    torch.cuda.synchronize()
    got = dZ.cpu().numpy().reshape(2 * nz, d)
    for j in range(nz):
        assert np.allclose(got[nz + j], A.astype(np.float64) @ Z[j], rtol=1e-5, atol=1e-5)
        assert np.array_equal(got[j], Z[j])
    # the reference's own check (benchmarks/gsgemv4/Program.cs:329-391): the same column
    # list through opc_sgemv(d, d, 1, A, d, Z + col0, 1, 0, Z + col1, 1) on the host, then
    # |Z - Z'| / (1 + |Z'|) <= 1e-3
    L = opc.load()
    ah = np.asfortranarray(A).ravel(order="K").copy()
    zh = Z.ravel().copy()
    for a0, a1 in zip(col0, col1):
        if a1 != 2 * nz:  # the sentinel entry writes nothing
            L.opc_sgemv(d, d, 1.0, ah.ctypes.data, d, zh.ctypes.data + 4 * a0 * d, 1, 0.0,
                        zh.ctypes.data + 4 * a1 * d, 1)
    assert (np.abs(got.ravel() - zh) / (1 + np.abs(zh))).max() <= 1e-3


def test_opcuda_sek_fp64_sum(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    d = 77
    rng = np.random.default_rng(6)
    gen = rng.standard_normal((d, d)).astype(np.float32)
    dg = torch.from_numpy(np.asfortranarray(gen).ravel(order="K").copy()).to(cuda)
    out = torch.empty(d * d, device=cuda)
    dt = np.float32(1e-3)
    assert lib.opcuda_sek(d, dg.data_ptr(), float(dt), out.data_ptr()) == 0
    torch.cuda.synchronize()
    ref = (np.eye(d) + np.float64(dt) * gen.astype(np.float64)).astype(np.float32)
    assert np.array_equal(out.cpu().numpy().reshape(d, d).T, ref)


def test_opcuda_sglvg_matches_oracle_generator(cuda):
    from oplib_b200 import _lib
    lib = _lib.load()
    d = 64
    x = O.log_grid(d)
    sig = O.lv_sigma(x)
    inv = O.lv_invm(x)  # row-major 2x2 inverses
    invm = np.stack([inv[:, 0, 0], inv[:, 1, 0], inv[:, 0, 1], inv[:, 1, 1]], axis=1).ravel().astype(np.float32)
    pars = np.concatenate([0.03 * x, sig * x]).astype(np.float32)
    dg = torch.empty(d * d, device=cuda)
    di, dp = torch.from_numpy(invm).to(cuda), torch.from_numpy(pars).to(cuda)
    assert lib.opcuda_sglvg(dg.data_ptr(), 1, d, di.data_ptr(), dp.data_ptr()) == 0
    torch.cuda.synchronize()
    got = dg.cpu().numpy().reshape(d, d).T  # column-major -> [source, target]
    ref = O.lv_generator(x, 0.03 * x, sig * x)
    assert np.allclose(got, ref, rtol=2e-4, atol=1e-3 * np.abs(ref).max())


@pytest.mark.parametrize("m,n,lda,incx", [(2048, 1536, 2048, 1), (301, 77, 301, 1), (300, 500, 304, 2),
                                          (6144, 6144, 6144, 1), (4, 1, 4, 1)])
def test_opcuda_sgemv_paths(cuda, m, n, lda, incx):
    """Both GEMV directions on every kernel path: float4 and scalar rows, column chunks
    with the ordered partial reduction (large n), padded leading dimension and strided x
    (scalar warp-per-column path); against FP64 within the FP32 bound."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(m + n)
    A = rng.standard_normal((lda, n)).astype(np.float32)   # column-major storage, rows >= m used
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="K").copy()).to(cuda)
    Am = A[:m].astype(np.float64)
    for trans in (False, True):
        nx, ny = (n, m) if not trans else (m, n)
        x = rng.standard_normal(nx * incx).astype(np.float32)
        y0 = rng.standard_normal(ny).astype(np.float32)
        dx, dy = torch.from_numpy(x).to(cuda), torch.from_numpy(y0.copy()).to(cuda)
        f = lib.opcuda_sgemvT if trans else lib.opcuda_sgemv
        assert f(m, n, 1.5, dA.data_ptr(), lda, dx.data_ptr(), incx, -0.5, dy.data_ptr(), 1) == 0
        torch.cuda.synchronize()
        xv = x[::incx].astype(np.float64)
        M = Am.T if trans else Am
        ref = 1.5 * (M @ xv) - 0.5 * y0
        bound = 1.5 * (np.abs(M) @ np.abs(xv)) * (M.shape[1] + 8) * 2.0 ** -24 + 0.5 * np.abs(y0) * 2.0 ** -23
        err = np.abs(dy.cpu().numpy() - ref)
        assert np.all(err <= bound + 1e-6), (trans, float((err / (bound + 1e-30)).max()))
        # deterministic: a second call gives the same bits
        dy2 = torch.from_numpy(y0.copy()).to(cuda)
        assert f(m, n, 1.5, dA.data_ptr(), lda, dx.data_ptr(), incx, -0.5, dy2.data_ptr(), 1) == 0
        torch.cuda.synchronize()
        assert torch.equal(dy, dy2)


def test_opcuda_sgemv_on_two_streams(cuda):
    """Column-major GEMVs issued back to back on two streams use separate partial buffers:
    both results match FP64."""
    from oplib_b200 import _lib
    lib = _lib.load()
    m = n = 2048
    rng = np.random.default_rng(21)
    A = rng.standard_normal((m, n)).astype(np.float32)
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="K").copy()).to(cuda)
    xs = [rng.standard_normal(n).astype(np.float32) for _ in range(2)]
    dxs = [torch.from_numpy(x).to(cuda) for x in xs]
    ys = [torch.zeros(m, device=cuda) for _ in range(2)]
    streams = [torch.cuda.Stream(cuda), torch.cuda.Stream(cuda)]
    torch.cuda.synchronize()
    try:
        for k in range(2):
            assert lib.opb_set_stream(streams[k].cuda_stream) == 0
            assert lib.opcuda_sgemv(m, n, 1.0, dA.data_ptr(), m, dxs[k].data_ptr(), 1, 0.0, ys[k].data_ptr(), 1) == 0
    finally:
        lib.opb_set_stream(torch.cuda.current_stream(cuda).cuda_stream)
    torch.cuda.synchronize()
    for k in range(2):
        ref = A.astype(np.float64) @ xs[k]
        bound = (np.abs(A) @ np.abs(xs[k])) * (n + 8) * 2.0 ** -24
        assert np.all(np.abs(ys[k].cpu().numpy() - ref) <= bound + 1e-6)


@pytest.mark.parametrize("M,N,K,batch", [(256, 384, 272, 1), (128, 128, 16, 3), (512, 256, 1024, 2)])
def test_sgemm_pipelined_bit_identical_to_tiled(cuda, M, N, K, batch):
    """Whole-tile shapes with 16-byte aligned operands take the cp.async-pipelined SIMT kernel;
    the same operands one float off alignment take the register-staged one.  Both sum each
    output's products in k order with fused multiply-adds: bit-identical results, and within
    the FP32 bound of the FP64 product."""
    from oplib_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((batch, M, K)).astype(np.float32)
    B = rng.standard_normal((batch, K, N)).astype(np.float32)
    outs = []
    for off in (0, 1):
        dA = torch.zeros(batch * M * K + 4, device=cuda)
        dB = torch.zeros(batch * K * N + 4, device=cuda)
        dC = torch.zeros(batch * M * N + 4, device=cuda)
        dA[off:off + A.size] = torch.from_numpy(A.ravel()).to(cuda)
        dB[off:off + B.size] = torch.from_numpy(B.ravel()).to(cuda)
        assert lib.opb_sgemm_batched_rm(M, N, K, dA.data_ptr() + 4 * off, M * K, dB.data_ptr() + 4 * off, K * N,
                                        dC.data_ptr() + 4 * off, M * N, batch) == 0
        torch.cuda.synchronize()
        outs.append(dC[off:off + batch * M * N].cpu().numpy().reshape(batch, M, N))
    assert np.array_equal(outs[0], outs[1])
    ref = np.einsum("bmk,bkn->bmn", A.astype(np.float64), B.astype(np.float64))
    bound = K * 2.0 ** -23 * np.einsum("bmk,bkn->bmn", np.abs(A).astype(np.float64), np.abs(B).astype(np.float64))
    assert np.all(np.abs(outs[0] - ref) <= bound)
