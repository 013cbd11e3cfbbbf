// Plain FP32 GEMM on the SIMT FMA pipes (no tensor cores, no TF32).
//
// This is the "plain FP32" path behind the drop-in entry points
//   opcuda_sgemm  (oplib/opcuda/sgemm.cu:41-44, column-major, alpha/beta),
//   opcuda_ssqmm  (oplib/opcuda/ssqmm.cu:119-179, batched d x d via device pointer tables),
//   opcuda_sgemm4 (oplib/opcuda/sgemm4.cu:84-154, ragged batch through a per-block task table).
// The reference kernels are 64x16-tile Volkov-style SIMT loops for sm_1x; here one core
// kernel computes a row-major 128x128 CTA tile with 8x8 outputs per thread, a
// double-buffered shared-memory K pipeline and float4 shared-memory fragments.
// Column-major calls are mapped onto it through C^T = B^T . A^T (a column-major matrix
// is the row-major storage of its transpose), so the kernel never transposes data.
#include "common.cuh"

namespace opb {

constexpr int SG_BM = 128, SG_BN = 128, SG_BK = 8, SG_THREADS = 256;
constexpr int SG_APAD = 4;  // keeps the transposed A tile's stores off one bank

struct SgemmArgs {
    int M, N, K;
    int lda, ldb, ldc;
    float alpha, beta;
    const float *A;
    const float *B;
    float *C;
    // batching: either pointer tables (row-major roles) or strides
    const float *const *A_tab;
    const float *const *B_tab;
    float *const *C_tab;
    long long sA, sB, sC;
};

// Row-major C[M,N] = alpha * op(A)[M,K] . op(B)[K,N] + beta * C; TA: A stored K x M
// (element (m,k) at k*lda + m), TB: B stored N x K (element (k,n) at n*ldb + k).
// grid = (ceil(N/128), ceil(M/128), batch)
template <bool TA, bool TB>
__global__ void __launch_bounds__(SG_THREADS, 2) k_sgemm_rm(SgemmArgs p) {
    __shared__ __align__(16) float As[2][SG_BK][SG_BM + SG_APAD];
    __shared__ __align__(16) float Bs[2][SG_BK][SG_BN];

    const int z = blockIdx.z;
    const float *A = p.A_tab ? p.A_tab[z] : p.A + z * p.sA;
    const float *B = p.B_tab ? p.B_tab[z] : p.B + z * p.sB;
    float *C = p.C_tab ? p.C_tab[z] : p.C + z * p.sC;

    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * SG_BM, n0 = blockIdx.x * SG_BN;

    // global -> register staging coordinates
    const int a_row = tid >> 1, a_k = (tid & 1) * 4;   // 128 rows x 8 k
    const int b_k = tid >> 5, b_col = (tid & 31) * 4;  // 8 k x 128 cols

    float ra[4], rb[4];
    auto load_tiles = [&](int k0) {
        int gr = m0 + a_row;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int gk = k0 + a_k + j;
            ra[j] = (gr < p.M && gk < p.K)
                        ? __ldg(TA ? A + (long long)gk * p.lda + gr : A + (long long)gr * p.lda + gk)
                        : 0.f;
        }
        int gk = k0 + b_k;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int gc = n0 + b_col + j;
            rb[j] = (gk < p.K && gc < p.N)
                        ? __ldg(TB ? B + (long long)gc * p.ldb + gk : B + (long long)gk * p.ldb + gc)
                        : 0.f;
        }
    };
    auto store_tiles = [&](int buf) {
#pragma unroll
        for (int j = 0; j < 4; j++) As[buf][a_k + j][a_row] = ra[j];
        *reinterpret_cast<float4 *>(&Bs[buf][b_k][b_col]) = make_float4(rb[0], rb[1], rb[2], rb[3]);
    };

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;

    const int nk = (p.K + SG_BK - 1) / SG_BK;
    load_tiles(0);
    store_tiles(0);
    __syncthreads();

    for (int t = 0; t < nk; t++) {
        const int buf = t & 1;
        if (t + 1 < nk) load_tiles((t + 1) * SG_BK);
#pragma unroll
        for (int k = 0; k < SG_BK; k++) {
            float a[8], b[8];
            float4 a0 = *reinterpret_cast<const float4 *>(&As[buf][k][ty * 4]);
            float4 a1 = *reinterpret_cast<const float4 *>(&As[buf][k][64 + ty * 4]);
            float4 b0 = *reinterpret_cast<const float4 *>(&Bs[buf][k][tx * 4]);
            float4 b1 = *reinterpret_cast<const float4 *>(&Bs[buf][k][64 + tx * 4]);
            a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
            a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
            b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
            b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (t + 1 < nk) {
            store_tiles(buf ^ 1);
        }
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < 8; i++) {
        int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (r >= p.M) continue;
        float *crow = C + (long long)r * p.ldc;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            int c = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (c >= p.N) continue;
            float v = p.alpha * acc[i][j];
            if (p.beta != 0.f) v = fmaf(p.beta, crow[c], v);
            crow[c] = v;
        }
    }
}

// ---- the pipelined form for whole tiles (row-major A and B, M and N multiples of 128, K of
// 16, 16-byte aligned rows, no pointer tables): K in steps of 16 through a 3-stage
// cp.async ring (A rows padded to 20 floats, so the two row groups of a warp fall on
// different banks), each thread 8 x 8 outputs from 128-bit shared loads of A along k and of
// B along n.  Every output still sums its products in k order, so the results are
// bit-identical to k_sgemm_rm's.
constexpr int SF_BK = 16, SF_STAGES = 3, SF_APITCH = SF_BK + 4;
constexpr int SF_A_FLOATS = SG_BM * SF_APITCH, SF_B_FLOATS = SF_BK * SG_BN;
constexpr int SF_SMEM = SF_STAGES * (SF_A_FLOATS + SF_B_FLOATS) * 4;

__device__ __forceinline__ void sf_cp16(float *dst, const float *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void sf_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void sf_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Packed FP32 (sm_100): two independent FMAs per lane and instruction, each rounded as a
// scalar fmaf, so every output still sums its products in k order with the same bits.
__device__ __forceinline__ uint64_t f2_pack(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(uint64_t v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

__global__ void __launch_bounds__(SG_THREADS, 2) k_sgemm_pipe(SgemmArgs p) {
    extern __shared__ __align__(16) float sm[];
    const int z = blockIdx.z;
    const float *A = p.A + z * p.sA;
    const float *B = p.B + z * p.sB;
    float *C = p.C + z * p.sC;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * SG_BM, n0 = blockIdx.x * SG_BN;
    const float *Ab = A + (long long)m0 * p.lda;
    const float *Bb = B + n0;

    auto issue = [&](int stage, int k0) {
        float *As = sm + stage * (SF_A_FLOATS + SF_B_FLOATS);
        float *Bs = As + SF_A_FLOATS;
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int c = tid + SG_THREADS * i;
            const int row = c >> 2, kq = (c & 3) * 4;  // 128 rows x 4 chunks of 4 floats
            sf_cp16(As + row * SF_APITCH + kq, Ab + (long long)row * p.lda + k0 + kq);
        }
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int c = tid + SG_THREADS * i;
            const int kr = c >> 5, col = (c & 31) * 4;  // 16 rows x 32 chunks of 4 floats
            sf_cp16(Bs + kr * SG_BN + col, Bb + (long long)(k0 + kr) * p.ldb + col);
        }
        sf_commit();
    };

    // acc2[i][jp] holds the outputs (row i, columns 2jp and 2jp + 1) of this thread's 8 x 8
    uint64_t acc2[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc2[i][j] = 0ull;

    const int nk = p.K / SF_BK;
#pragma unroll
    for (int st = 0; st < SF_STAGES - 1; st++) {
        if (st < nk) issue(st, st * SF_BK);
        else sf_commit();
    }
    for (int kt = 0; kt < nk; kt++) {
        sf_wait<SF_STAGES - 2>();
        __syncthreads();  // stage kt landed for every thread; stage kt - 1 is free to refill
        const int nt = kt + SF_STAGES - 1;
        if (nt < nk) issue(nt % SF_STAGES, nt * SF_BK);
        else sf_commit();
        const float *As = sm + (kt % SF_STAGES) * (SF_A_FLOATS + SF_B_FLOATS);
        const float *Bs = As + SF_A_FLOATS;
#pragma unroll
        for (int kk = 0; kk < SF_BK; kk += 4) {
            float4 a4[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int row = i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4);
                a4[i] = *reinterpret_cast<const float4 *>(As + row * SF_APITCH + kk);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float4 b0 = *reinterpret_cast<const float4 *>(Bs + (kk + u) * SG_BN + tx * 4);
                const float4 b1 = *reinterpret_cast<const float4 *>(Bs + (kk + u) * SG_BN + 64 + tx * 4);
                const uint64_t b2[4] = {f2_pack(b0.x, b0.y), f2_pack(b0.z, b0.w), f2_pack(b1.x, b1.y),
                                        f2_pack(b1.z, b1.w)};
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const float a = u == 0 ? a4[i].x : u == 1 ? a4[i].y : u == 2 ? a4[i].z : a4[i].w;
                    const uint64_t a2 = f2_pack(a, a);
#pragma unroll
                    for (int j = 0; j < 4; j++) acc2[i][j] = f2_fma(a2, b2[j], acc2[i][j]);
                }
            }
        }
    }
    sf_wait<0>();

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) f2_unpack(acc2[i][j], acc[i][2 * j], acc[i][2 * j + 1]);
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        float *crow = C + (long long)r * p.ldc + n0;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float4 *cp = reinterpret_cast<float4 *>(crow + h * 64 + tx * 4);
            float4 v = make_float4(p.alpha * acc[i][4 * h], p.alpha * acc[i][4 * h + 1], p.alpha * acc[i][4 * h + 2],
                                   p.alpha * acc[i][4 * h + 3]);
            if (p.beta != 0.f) {
                const float4 c = *cp;
                v.x = fmaf(p.beta, c.x, v.x);
                v.y = fmaf(p.beta, c.y, v.y);
                v.z = fmaf(p.beta, c.z, v.z);
                v.w = fmaf(p.beta, c.w, v.w);
            }
            *cp = v;
        }
    }
}

static bool sgemm_pipe_ok(const SgemmArgs &a, int batch) {
    auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
    return !a.A_tab && !a.B_tab && !a.C_tab && a.M % SG_BM == 0 && a.N % SG_BN == 0 && a.K % SF_BK == 0 &&
           a.K > 0 && a.lda % 4 == 0 && a.ldb % 4 == 0 && a.ldc % 4 == 0 && al(a.A) && al(a.B) && al(a.C) &&
           (batch == 1 || (a.sA % 4 == 0 && a.sB % 4 == 0 && a.sC % 4 == 0));
}

int sgemm_rowmajor(const SgemmArgs &a, int batch, cudaStream_t s, bool ta = false, bool tb = false) {
    if (a.M <= 0 || a.N <= 0 || batch <= 0) return OPB_OK;
    if (!ta && !tb && sgemm_pipe_ok(a, batch)) {
        static bool attr[64] = {false};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev >= 0 && dev < 64 && !attr[dev]) {
            cudaError_t e = cudaFuncSetAttribute(k_sgemm_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize, SF_SMEM);
            if (e != cudaSuccess) return (int)e;
            attr[dev] = true;
        }
        dim3 grid(a.N / SG_BN, a.M / SG_BM, batch);
        k_sgemm_pipe<<<grid, SG_THREADS, SF_SMEM, s>>>(a);
        return static_cast<int>(cudaGetLastError());
    }
    dim3 grid((a.N + SG_BN - 1) / SG_BN, (a.M + SG_BM - 1) / SG_BM, batch);
    if (!ta && !tb) k_sgemm_rm<false, false><<<grid, SG_THREADS, 0, s>>>(a);
    else if (ta && !tb) k_sgemm_rm<true, false><<<grid, SG_THREADS, 0, s>>>(a);
    else if (!ta && tb) k_sgemm_rm<false, true><<<grid, SG_THREADS, 0, s>>>(a);
    else k_sgemm_rm<true, true><<<grid, SG_THREADS, 0, s>>>(a);
    return static_cast<int>(cudaGetLastError());
}

// Row-major with transpose flags (see k_sgemm_rm).
int sgemm_rm_t(bool ta, bool tb, int M, int N, int K, float alpha, const float *A, int lda, const float *B, int ldb,
               float beta, float *C, int ldc, cudaStream_t s) {
    SgemmArgs a{};
    a.M = M; a.N = N; a.K = K; a.lda = lda; a.ldb = ldb; a.ldc = ldc;
    a.alpha = alpha; a.beta = beta; a.A = A; a.B = B; a.C = C;
    return sgemm_rowmajor(a, 1, s, ta, tb);
}

int sgemm_rm_strided(bool ta, bool tb, int M, int N, int K, float alpha, const float *A, int lda, long long sA,
                     const float *B, int ldb, long long sB, float beta, float *C, int ldc, long long sC, int batch,
                     cudaStream_t s) {
    SgemmArgs a{};
    a.M = M; a.N = N; a.K = K; a.lda = lda; a.ldb = ldb; a.ldc = ldc;
    a.alpha = alpha; a.beta = beta; a.A = A; a.B = B; a.C = C; a.sA = sA; a.sB = sB; a.sC = sC;
    return sgemm_rowmajor(a, batch, s, ta, tb);
}

// Convenience: row-major, unbatched.
int sgemm_rm(int M, int N, int K, float alpha, const float *A, int lda, const float *B, int ldb,
             float beta, float *C, int ldc, cudaStream_t s) {
    SgemmArgs a{};
    a.M = M; a.N = N; a.K = K; a.lda = lda; a.ldb = ldb; a.ldc = ldc;
    a.alpha = alpha; a.beta = beta; a.A = A; a.B = B; a.C = C;
    return sgemm_rowmajor(a, 1, s);
}

// ------------------------------------------------------------------ sgemm4 task tables

// One task per block, widened from the reference's 9-word record
// {i, bx, by, m, n, k, A, B, C} (oplib/opcuda/sgemm4.cu:84-102): the block computes the
// column-major C tile rows [bx*64, bx*64+64) x columns [by*16, by*16+16) of
// C = A . B with lda = m, ldb = k, ldc = m.
struct Sgemm4Task {
    int32_t i, bx, by, m, n, k;
    uint64_t A, B, C;
};

__global__ void __launch_bounds__(256) k_sgemm4(const uint64_t *argptr_bid) {
    const Sgemm4Task *tp = reinterpret_cast<const Sgemm4Task *>(argptr_bid[blockIdx.x]);
    __shared__ Sgemm4Task t;
    if (threadIdx.x == 0) t = *tp;
    __syncthreads();
    const float *A = reinterpret_cast<const float *>(t.A);
    const float *B = reinterpret_cast<const float *>(t.B);
    float *C = reinterpret_cast<float *>(t.C);
    const int row0 = t.bx * 64, col0 = t.by * 16;
    // thread -> (row, 4 columns): 64 rows x 4 column groups of 4
    const int r = threadIdx.x & 63;
    const int cg = threadIdx.x >> 6;
    __shared__ float Bs[32][16];
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    const int row = row0 + r;
    for (int k0 = 0; k0 < t.k; k0 += 32) {
        for (int e = threadIdx.x; e < 32 * 16; e += 256) {
            int kk = e & 31, cc = e >> 5;
            int gk = k0 + kk, gc = col0 + cc;
            Bs[kk][cc] = (gk < t.k && gc < t.n) ? B[(long long)gc * t.k + gk] : 0.f;
        }
        __syncthreads();
        int kmax = min(32, t.k - k0);
        if (row < t.m) {
            for (int kk = 0; kk < kmax; kk++) {
                float a = A[(long long)(k0 + kk) * t.m + row];
#pragma unroll
                for (int j = 0; j < 4; j++) acc[j] = fmaf(a, Bs[kk][cg * 4 + j], acc[j]);
            }
        }
        __syncthreads();
    }
    if (row < t.m) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int c = col0 + cg * 4 + j;
            if (c < t.n) C[(long long)c * t.m + row] = acc[j];
        }
    }
}

}  // namespace opb

using namespace opb;

// Column-major C(m x n) = alpha * A(m x k) . B(k x n) + beta * C, the semantics of
// cublasSgemm('N','N') that the reference wraps (oplib/opcuda/sgemm.cu:41-44).
OPB_API int opcuda_sgemm(int m, int n, int k, float alpha, uint64_t A, int lda, uint64_t B, int ldb,
                         float beta, uint64_t C, int ldc) {
    OPB_REQUIRE(m >= 0 && n >= 0 && k >= 0, OPB_E_ARG);
    if (m == 0 || n == 0) return set_status(OPB_OK);
    OPB_REQUIRE(C != 0 && (k == 0 || (A != 0 && B != 0)), OPB_E_NULL);
    OPB_REQUIRE(lda >= (m > 1 ? m : 1) && ldb >= (k > 1 ? k : 1) && ldc >= (m > 1 ? m : 1), OPB_E_ARG);
    // column-major C = A.B  <=>  row-major C^T(n x m) = B^T(n x k) . A^T(k x m)
    int st = sgemm_rm(n, m, k, alpha, reinterpret_cast<const float *>(B), ldb,
                      reinterpret_cast<const float *>(A), lda, beta, reinterpret_cast<float *>(C), ldc,
                      stream());
    return set_status(st);
}

// Batched C_i = A_i . B_i for ni column-major d x d matrices given as device arrays of
// 64-bit device pointers (oplib/opcuda/ssqmm.cu:174-179; A_i == B_i squares).
OPB_API int opcuda_ssqmm(int d, int ni, uint64_t A_i, uint64_t B_i, uint64_t C_i) {
    OPB_REQUIRE(d >= 0 && ni >= 0, OPB_E_ARG);
    if (d == 0 || ni == 0) return set_status(OPB_OK);
    OPB_REQUIRE(A_i != 0 && B_i != 0 && C_i != 0, OPB_E_NULL);
    SgemmArgs a{};
    a.M = d; a.N = d; a.K = d; a.lda = d; a.ldb = d; a.ldc = d;
    a.alpha = 1.f; a.beta = 0.f;
    // row-major roles: A' = B_i, B' = A_i
    a.A_tab = reinterpret_cast<const float *const *>(B_i);
    a.B_tab = reinterpret_cast<const float *const *>(A_i);
    a.C_tab = reinterpret_cast<float *const *>(C_i);
    return set_status(sgemm_rowmajor(a, ni, stream()));
}

// Strided-batch variant with typed pointers (new; row-major, ld = d).
OPB_API int opb_sgemm_batched_rm(int M, int N, int K, const float *A, long long sA, const float *B,
                                 long long sB, float *C, long long sC, int batch) {
    OPB_REQUIRE(M >= 0 && N >= 0 && K >= 0 && batch >= 0, OPB_E_ARG);
    if (M == 0 || N == 0 || batch == 0) return set_status(OPB_OK);
    OPB_REQUIRE(A && B && C, OPB_E_NULL);
    SgemmArgs a{};
    a.M = M; a.N = N; a.K = K; a.lda = K; a.ldb = N; a.ldc = N;
    a.alpha = 1.f; a.beta = 0.f; a.A = A; a.B = B; a.C = C; a.sA = sA; a.sB = sB; a.sC = sC;
    return set_status(sgemm_rowmajor(a, batch, stream()));
}

OPB_API int opcuda_sgemm4(int nblocks, uint64_t argptr_bid) {
    OPB_REQUIRE(nblocks >= 0, OPB_E_ARG);
    if (nblocks == 0) return set_status(OPB_OK);
    OPB_REQUIRE(argptr_bid != 0, OPB_E_NULL);
    k_sgemm4<<<nblocks, 256, 0, stream()>>>(reinterpret_cast<const uint64_t *>(argptr_bid));
    return launch_check();
}

OPB_API int opb_sgemm4_task_size(void) { return static_cast<int>(sizeof(Sgemm4Task)); }
