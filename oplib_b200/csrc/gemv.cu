// Matrix-vector entry points of the opcuda ABI (column-major, FP32 SIMT, HBM-bound).
//
//   opcuda_sgemv / opcuda_sgemvT : y = alpha*op(A)*x + beta*y (oplib/opcuda/sgemv.cu:44-62,
//                                  cuBLAS 'N' / 'T' in the reference)
//   opcuda_sgemv3                : multi-vector induction Z[:, col1[c]] = A . Z[:, col0[c]]
//                                  over a column list with a 2*nz*d sentinel
//                                  (oplib/opcuda/sgemv3.cu:92-176)
//   opcuda_sgemv4                : the same driven by a per-block task table
//                                  (oplib/opcuda/sgemv4.cu:90-180)
//   opcuda_sdot2                 : c[h] = sum_y a[h + nh*y] * b[h + nh*y]
//                                  (oplib/opcuda/sdot2.cu:48-83)
//   opcuda_sglvg                 : dense local-vol generator from the per-node 2x2 inverses
//                                  (oplib/opcuda/sglvg.cu:42-125)
// Each kernel reads the matrix exactly once with coalesced accesses: consecutive threads
// own consecutive rows of a column-major matrix, so every column step is one contiguous
// 128-byte segment per warp.  Column lists are processed 16 at a time from one pass.
#include <mutex>
#include <unordered_map>

#include "common.cuh"

namespace opb {

// y = alpha * A x + beta * y, column-major A (m x n).  Block = 8 warps over one tile of
// rows (128 rows, 4 per lane with float4 loads, when VEC; else 32 rows, one per lane) and
// the column chunk [j0, j1): warp w takes the columns j0 + w, j0 + w + 8, ..., so every
// warp load is one contiguous column segment; the 8 warp sums are combined in shared
// memory in warp order.  With part != nullptr the chunk's sums go to part[chunk * m + row]
// for k_sgemv_n_reduce; otherwise the block covers all columns and writes y.
template <bool VEC>
__global__ void __launch_bounds__(256) k_sgemv_n(int m, int n, int chunk, float alpha, const float *__restrict__ A,
                                                 int lda, const float *__restrict__ x, int incx, float beta,
                                                 float *__restrict__ y, int incy, float *__restrict__ part) {
    constexpr int RPL = VEC ? 4 : 1;  // rows per lane
    constexpr int TILE = 32 * RPL;
    __shared__ float red[8][TILE];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * TILE + lane * RPL;
    const int j0 = blockIdx.y * chunk, j1 = min(n, j0 + chunk);
    float acc[RPL];
#pragma unroll
    for (int r = 0; r < RPL; r++) acc[r] = 0.f;
    if (i < m) {
        int j = j0 + warp;
        if constexpr (VEC) {
            for (; j + 24 < j1; j += 32) {  // four independent column loads in flight
                float4 a[4];
                float xv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    a[u] = __ldg(reinterpret_cast<const float4 *>(A + (long long)(j + 8 * u) * lda + i));
                    xv[u] = __ldg(x + (long long)(j + 8 * u) * incx);
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    acc[0] = fmaf(a[u].x, xv[u], acc[0]);
                    acc[1] = fmaf(a[u].y, xv[u], acc[1]);
                    acc[2] = fmaf(a[u].z, xv[u], acc[2]);
                    acc[3] = fmaf(a[u].w, xv[u], acc[3]);
                }
            }
            for (; j < j1; j += 8) {
                const float4 a = __ldg(reinterpret_cast<const float4 *>(A + (long long)j * lda + i));
                const float xv = __ldg(x + (long long)j * incx);
                acc[0] = fmaf(a.x, xv, acc[0]);
                acc[1] = fmaf(a.y, xv, acc[1]);
                acc[2] = fmaf(a.z, xv, acc[2]);
                acc[3] = fmaf(a.w, xv, acc[3]);
            }
        } else {
            for (; j < j1; j += 8) acc[0] = fmaf(__ldg(A + (long long)j * lda + i), __ldg(x + (long long)j * incx), acc[0]);
        }
    }
#pragma unroll
    for (int r = 0; r < RPL; r++) red[warp][lane * RPL + r] = acc[r];
    __syncthreads();
    // combine the 8 warp sums of each row in warp order
    for (int t = threadIdx.x; t < TILE; t += blockDim.x) {
        const int row = blockIdx.x * TILE + t;
        if (row >= m) continue;
        float v = red[0][t];
#pragma unroll
        for (int w = 1; w < 8; w++) v += red[w][t];
        if (part) {
            part[(long long)blockIdx.y * m + row] = v;
        } else {
            float o = alpha * v;
            if (beta != 0.f) o = fmaf(beta, y[(long long)row * incy], o);
            y[(long long)row * incy] = o;
        }
    }
}

// y[i] = alpha * (sum over chunks in order of part[c * m + i]) + beta * y[i].
__global__ void k_sgemv_n_reduce(int m, int nchunks, float alpha, const float *__restrict__ part, float beta,
                                 float *__restrict__ y, int incy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    float acc = 0.f;
    for (int c = 0; c < nchunks; c++) acc += part[(long long)c * m + i];
    float v = alpha * acc;
    if (beta != 0.f) v = fmaf(beta, y[(long long)i * incy], v);
    y[(long long)i * incy] = v;
}

// y = alpha * A^T x + beta * y, column-major A (m x n): warp per output, i.e. per column of
// A (a contiguous run: the warp-per-row GEMV of a source-major matrix).  VEC: float4 loads
// of the column and of x, two accumulators in a fixed order.
template <bool VEC>
__global__ void __launch_bounds__(256) k_sgemv_t(int m, int n, float alpha, const float *__restrict__ A, int lda,
                                                 const float *__restrict__ x, int incx, float beta,
                                                 float *__restrict__ y, int incy) {
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // warp per column
    const int lane = threadIdx.x & 31;
    if (j >= n) return;
    const float *col = A + (long long)j * lda;
    float acc0 = 0.f, acc1 = 0.f;
    int tail = 0;
    if constexpr (VEC) {
        const int m4 = m >> 2;
        const float4 *c4 = reinterpret_cast<const float4 *>(col);
        const float4 *x4 = reinterpret_cast<const float4 *>(x);
        int q = lane;
        for (; q + 32 < m4; q += 64) {
            const float4 a0 = __ldg(c4 + q), b0 = __ldg(x4 + q);
            const float4 a1 = __ldg(c4 + q + 32), b1 = __ldg(x4 + q + 32);
            acc0 = fmaf(a0.x, b0.x, acc0); acc0 = fmaf(a0.y, b0.y, acc0);
            acc0 = fmaf(a0.z, b0.z, acc0); acc0 = fmaf(a0.w, b0.w, acc0);
            acc1 = fmaf(a1.x, b1.x, acc1); acc1 = fmaf(a1.y, b1.y, acc1);
            acc1 = fmaf(a1.z, b1.z, acc1); acc1 = fmaf(a1.w, b1.w, acc1);
        }
        if (q < m4) {
            const float4 a0 = __ldg(c4 + q), b0 = __ldg(x4 + q);
            acc0 = fmaf(a0.x, b0.x, acc0); acc0 = fmaf(a0.y, b0.y, acc0);
            acc0 = fmaf(a0.z, b0.z, acc0); acc0 = fmaf(a0.w, b0.w, acc0);
        }
        tail = m4 << 2;
    }
    for (int i = tail + lane; i < m; i += 32) acc0 = fmaf(__ldg(col + i), __ldg(x + (long long)i * incx), acc0);
    float acc = acc0 + acc1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        float v = alpha * acc;
        if (beta != 0.f) v = fmaf(beta, y[(long long)j * incy], v);
        y[(long long)j * incy] = v;
    }
}

// Buffers for the column-chunk partials of opcuda_sgemv, one per (device, stream) so that
// calls on different streams never share one (calls on one stream run in order); grown on
// demand (cudaMalloc on the first call that needs more) and kept until exit.
struct GemvKey {
    int dev;
    cudaStream_t s;
    bool operator==(const GemvKey &o) const { return dev == o.dev && s == o.s; }
};
struct GemvKeyHash {
    size_t operator()(const GemvKey &k) const {
        return std::hash<void *>()(reinterpret_cast<void *>(k.s)) ^ ((size_t)k.dev * 0x9E3779B97F4A7C15ull);
    }
};
struct GemvBuf {
    float *p = nullptr;
    size_t cap = 0;
};
static std::unordered_map<GemvKey, GemvBuf, GemvKeyHash> g_gemv_bufs;
static std::mutex g_gemv_mu;

static int gemv_part_buffer(cudaStream_t s, size_t floats, float **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return OPB_E_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_gemv_mu);
    GemvBuf &b = g_gemv_bufs[GemvKey{dev, s}];
    if (b.cap < floats) {
        if (b.p) {
            // the stream's earlier calls may still read the old buffer
            cudaStreamSynchronize(s);
            cudaFree(b.p);
        }
        b.p = nullptr;
        b.cap = 0;
        if (cudaMalloc(&b.p, floats * sizeof(float)) != cudaSuccess) return OPB_E_NOMEM;
        b.cap = floats;
    }
    *out = b.p;
    return OPB_OK;
}

// Multi-vector product for rows [row0, row0 + 128) and the 16 list entries starting at c0.
// Z columns are element offsets (col * d) into Z, as in the reference.
__device__ void sgemv_cols(int d, long long sentinel, int ncol, const float *__restrict__ A, float *__restrict__ Z,
                           const int *__restrict__ col0, const int *__restrict__ col1, int row0, int c0) {
    __shared__ int s0[16], s1[16];
    __shared__ float zs[32][17];
    __shared__ int nvalid;
    if (threadIdx.x < 16) {
        int c = c0 + threadIdx.x;
        s0[threadIdx.x] = c < ncol ? col0[c] : -1;
        s1[threadIdx.x] = c < ncol ? col1[c] : (int)sentinel;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int nv = 0;
        while (nv < 16 && (long long)s1[nv] < sentinel && s0[nv] >= 0) nv++;
        nvalid = nv;
    }
    __syncthreads();
    const int nv = nvalid;
    if (nv == 0) return;
    const int row = row0 + threadIdx.x;
    float acc[16];
#pragma unroll
    for (int c = 0; c < 16; c++) acc[c] = 0.f;
    for (int k0 = 0; k0 < d; k0 += 32) {
        for (int e = threadIdx.x; e < 32 * 16; e += blockDim.x) {
            int kk = e & 31, c = e >> 5;
            int k = k0 + kk;
            zs[kk][c] = (c < nv && k < d) ? Z[(long long)s0[c] + k] : 0.f;
        }
        __syncthreads();
        if (row < d) {
            int kmax = min(32, d - k0);
            for (int kk = 0; kk < kmax; kk++) {
                float a = A[(long long)(k0 + kk) * d + row];
#pragma unroll
                for (int c = 0; c < 16; c++) acc[c] = fmaf(a, zs[kk][c], acc[c]);
            }
        }
        __syncthreads();
    }
    if (row < d) {
#pragma unroll
        for (int c = 0; c < 16; c++)
            if (c < nv) Z[(long long)s1[c] + row] = acc[c];
    }
}

__global__ void __launch_bounds__(128) k_sgemv3(int d, int nz, int ncol, const float *A, float *Z, const int *col0,
                                                const int *col1) {
    sgemv_cols(d, 2LL * nz * d, ncol, A, Z, col0, col1, blockIdx.x * 128, blockIdx.y * 16);
}

// Widened task record of oplib/opcuda/sgemv4.cu:100-107: rows [bx*128, bx*128+128) of the
// 16 list entries starting at by*16.
struct Sgemv4Task {
    int32_t i, bx, by, d, nz, ncol;
    uint64_t A, Z, col0, col1;
};

__global__ void __launch_bounds__(128) k_sgemv4(const uint64_t *argptr_bid) {
    const Sgemv4Task *tp = reinterpret_cast<const Sgemv4Task *>(argptr_bid[blockIdx.x]);
    __shared__ Sgemv4Task t;
    if (threadIdx.x == 0) t = *tp;
    __syncthreads();
    sgemv_cols(t.d, 2LL * t.nz * t.d, t.ncol, reinterpret_cast<const float *>(t.A), reinterpret_cast<float *>(t.Z),
               reinterpret_cast<const int *>(t.col0), reinterpret_cast<const int *>(t.col1), t.bx * 128, t.by * 16);
}

__global__ void k_sdot2(const float *__restrict__ a, const float *__restrict__ b, float *__restrict__ c, int nh, int d) {
    int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    float acc = 0.f;
    for (int y = 0; y < d; y++) acc = fmaf(a[h + (long long)nh * y], b[h + (long long)nh * y], acc);
    c[h] = acc;
}

// Dense column-major FP32 LV generator for ni periods: gen[i*d*d + y0 + d*y1]
// (oplib/opmodel/models/CLVModel.cs:86-136 semantics; invm[4*y + r + 2*c] is the
// column-major 2x2 inverse of node y; pars = [drift (ni x d); vol (ni x d)]).
__global__ void k_sglvg(float *__restrict__ gen, int ni, int d, const float *__restrict__ invm,
                        const float *__restrict__ pars) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)ni * d) return;
    int i = (int)(t / d), y = (int)(t - (long long)i * d);
    float *g = gen + (long long)i * d * d;
    float r0 = 0.f, r1 = 0.f;
    if (y > 0 && y < d - 1) {
        r0 = pars[(long long)i * d + y];
        float v = pars[(long long)ni * d + (long long)i * d + y];
        r1 = v * v;
    }
    const float *im = invm + 4LL * y;
    float dn = im[0] * r0 + im[2] * r1;
    float up = im[1] * r0 + im[3] * r1;
    float sum = 0.f;
    if (y > 0) { g[y + (long long)d * (y - 1)] = dn; sum += dn; }
    if (y < d - 1) { g[y + (long long)d * (y + 1)] = up; sum += up; }
    g[y + (long long)d * y] = -sum;
}

}  // namespace opb

using namespace opb;

OPB_API int opcuda_sgemv(int m, int n, float alpha, uint64_t A, int lda, uint64_t x, int incx, float beta, uint64_t y,
                         int incy) {
    OPB_REQUIRE(m >= 0 && n >= 0, OPB_E_ARG);
    if (m == 0) return set_status(OPB_OK);
    OPB_REQUIRE(y != 0 && (n == 0 || (A != 0 && x != 0)), OPB_E_NULL);
    OPB_REQUIRE(lda >= (m > 1 ? m : 1) && incx > 0 && incy > 0, OPB_E_ARG);
    const float *pA = reinterpret_cast<const float *>(A);
    const float *px = reinterpret_cast<const float *>(x);
    float *py = reinterpret_cast<float *>(y);
    // float4 rows when every column starts 16-byte aligned and m is a multiple of 4
    const bool vec = m % 4 == 0 && lda % 4 == 0 && aligned(pA, 16);
    const int rows_per_block = vec ? 128 : 32;
    const int tiles = (m + rows_per_block - 1) / rows_per_block;
    // column chunks: about 8 blocks per SM in total
    int nch = (8 * num_sms() + tiles - 1) / tiles;
    if (nch > n) nch = n;
    if (nch < 1) nch = 1;
    const int chunk = n > 0 ? (n + nch - 1) / nch : 1;
    nch = n > 0 ? (n + chunk - 1) / chunk : 1;
    float *part = nullptr;
    if (nch > 1) {
        const int r = gemv_part_buffer(stream(), (size_t)nch * m, &part);
        if (r != OPB_OK) return set_status(r);
    }
    dim3 g(tiles, nch);
    if (vec)
        k_sgemv_n<true><<<g, 256, 0, stream()>>>(m, n, chunk, alpha, pA, lda, px, incx, beta, py, incy, part);
    else
        k_sgemv_n<false><<<g, 256, 0, stream()>>>(m, n, chunk, alpha, pA, lda, px, incx, beta, py, incy, part);
    if (part) k_sgemv_n_reduce<<<(m + 255) / 256, 256, 0, stream()>>>(m, nch, alpha, part, beta, py, incy);
    return launch_check();
}

OPB_API int opcuda_sgemvT(int m, int n, float alpha, uint64_t A, int lda, uint64_t x, int incx, float beta, uint64_t y,
                          int incy) {
    OPB_REQUIRE(m >= 0 && n >= 0, OPB_E_ARG);
    if (n == 0) return set_status(OPB_OK);
    OPB_REQUIRE(y != 0 && (m == 0 || (A != 0 && x != 0)), OPB_E_NULL);
    OPB_REQUIRE(lda >= (m > 1 ? m : 1) && incx > 0 && incy > 0, OPB_E_ARG);
    long long threads = 32LL * n;
    const float *pA = reinterpret_cast<const float *>(A);
    const float *px = reinterpret_cast<const float *>(x);
    const bool vec = lda % 4 == 0 && incx == 1 && aligned(pA, 16) && aligned(px, 16);
    if (vec)
        k_sgemv_t<true><<<(int)((threads + 255) / 256), 256, 0, stream()>>>(m, n, alpha, pA, lda, px, incx, beta,
                                                                         reinterpret_cast<float *>(y), incy);
    else
        k_sgemv_t<false><<<(int)((threads + 255) / 256), 256, 0, stream()>>>(m, n, alpha, pA, lda, px, incx, beta,
                                                                          reinterpret_cast<float *>(y), incy);
    return launch_check();
}

OPB_API int opcuda_sgemv3(int d, int nz, int ncol, uint64_t A, uint64_t B, uint64_t col0ptr, uint64_t col1ptr) {
    OPB_REQUIRE(d >= 0 && nz >= 0 && ncol >= 0, OPB_E_ARG);
    if (d == 0 || ncol == 0) return set_status(OPB_OK);
    OPB_REQUIRE(A && B && col0ptr && col1ptr, OPB_E_NULL);
    dim3 grid((d + 127) / 128, (ncol + 15) / 16);
    k_sgemv3<<<grid, 128, 0, stream()>>>(d, nz, ncol, reinterpret_cast<const float *>(A), reinterpret_cast<float *>(B),
                                         reinterpret_cast<const int *>(col0ptr), reinterpret_cast<const int *>(col1ptr));
    return launch_check();
}

OPB_API int opcuda_sgemv4(int nblocks, uint64_t argptr_bid) {
    OPB_REQUIRE(nblocks >= 0, OPB_E_ARG);
    if (nblocks == 0) return set_status(OPB_OK);
    OPB_REQUIRE(argptr_bid != 0, OPB_E_NULL);
    k_sgemv4<<<nblocks, 128, 0, stream()>>>(reinterpret_cast<const uint64_t *>(argptr_bid));
    return launch_check();
}

OPB_API int opb_sgemv4_task_size(void) { return static_cast<int>(sizeof(Sgemv4Task)); }

OPB_API int opcuda_sdot2(uint64_t aptr, uint64_t bptr, uint64_t cptr, int m, int n) {
    OPB_REQUIRE(m >= 0 && n >= 0, OPB_E_ARG);
    if (m == 0) return set_status(OPB_OK);
    OPB_REQUIRE(aptr && bptr && cptr, OPB_E_NULL);
    k_sdot2<<<(m + 255) / 256, 256, 0, stream()>>>(reinterpret_cast<const float *>(aptr),
                                                    reinterpret_cast<const float *>(bptr), reinterpret_cast<float *>(cptr),
                                                    m, n);
    return launch_check();
}

OPB_API int opcuda_sglvg(uint64_t gen_yy_i, int ni, int d, uint64_t invmat, uint64_t pars) {
    OPB_REQUIRE(ni >= 0 && d >= 2, OPB_E_ARG);
    if (ni == 0) return set_status(OPB_OK);
    OPB_REQUIRE(gen_yy_i && invmat && pars, OPB_E_NULL);
    OPB_TRY(cudaMemsetAsync(reinterpret_cast<void *>(gen_yy_i), 0, sizeof(float) * (size_t)ni * d * d, stream()));
    long long n = (long long)ni * d;
    k_sglvg<<<(int)((n + 255) / 256), 256, 0, stream()>>>(reinterpret_cast<float *>(gen_yy_i), ni, d,
                                                           reinterpret_cast<const float *>(invmat),
                                                           reinterpret_cast<const float *>(pars));
    return launch_check();
}
