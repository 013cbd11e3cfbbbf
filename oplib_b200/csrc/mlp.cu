// Learned surrogate pricer: an MLP 8 -> 256 -> 256 -> 256 -> 256 -> 1 with GELU, from
// (level, skew, width, kappa, rho, r, log-moneyness, T) to implied volatility, trained on
// quotes that the batched lattice solver produces, with the lattice as fallback and judge.
// The reference has no counterpart (its closest piece is the Black-Scholes pricer of its
// known-answer test, tests/bstest/BSPricer.cs:7-65).
//
// Parameters live in one flat FP32 master vector theta (layer l: W_l [out x in] row-major,
// then b_l [out]); training uses BF16-rounded working weights (kept as FP32 values), FP32
// activations and gradients, and Adam on the FP32 master copy.  All kernels are this
// project's: the hidden layers' products on the tensor cores (gemm_tc.cu, split-BF16 parts
// of the activations and gradients), the first and output layers on SIMT GEMMs
// (gemm_simt.cu, with transpose flags), plus the fused element-wise kernels below.  Batched inference of the trained network runs through
// opb_mlp_infer (BF16 weights and activations, FP32 accumulation).
#include <cuda_bf16.h>

#include <cmath>

#include "common.cuh"
#include "lattice.h"

namespace opb {

constexpr int MLP_IN = 8, MLP_H = 256, MLP_LAYERS = 5;  // 4 hidden + output
constexpr int MLP_NPARAM = MLP_H * MLP_IN + MLP_H + 3 * (MLP_H * MLP_H + MLP_H) + MLP_H + 1;  // 199,937

struct MlpLayout {
    int in[MLP_LAYERS], out[MLP_LAYERS];
    long long w[MLP_LAYERS], b[MLP_LAYERS];
};

__host__ __device__ inline MlpLayout mlp_layout() {
    MlpLayout L{};
    const int ins[MLP_LAYERS] = {MLP_IN, MLP_H, MLP_H, MLP_H, MLP_H};
    const int outs[MLP_LAYERS] = {MLP_H, MLP_H, MLP_H, MLP_H, 1};
    long long o = 0;
    for (int l = 0; l < MLP_LAYERS; l++) {
        L.in[l] = ins[l];
        L.out[l] = outs[l];
        L.w[l] = o;
        o += (long long)ins[l] * outs[l];
        L.b[l] = o;
        o += outs[l];
    }
    return L;
}

__device__ __forceinline__ uint32_t hash32(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return (uint32_t)x;
}

// Uniform(-a, a) weights with a = sqrt(6 / fan_in) (He-uniform), zero biases.
__global__ void k_mlp_init(float *__restrict__ theta, uint64_t seed) {
    const MlpLayout L = mlp_layout();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < MLP_NPARAM;
         i += (long long)gridDim.x * blockDim.x) {
        int l = 0;
        while (l + 1 < MLP_LAYERS && i >= L.w[l + 1]) l++;
        if (i >= L.b[l]) {
            theta[i] = 0.f;
        } else {
            const float a = sqrtf(6.f / (float)L.in[l]);
            const float u = (hash32(seed * 0x9E3779B97F4A7C15ULL + (uint64_t)i) >> 8) * (1.0f / 16777216.0f);
            theta[i] = (2.f * u - 1.f) * a;
        }
    }
}

// BF16 working copy of the master weights (as FP32 values) and the BF16 storage used by
// inference (same layout).
__global__ void k_mlp_round(const float *__restrict__ theta, float *__restrict__ theta_bf,
                            __nv_bfloat16 *__restrict__ theta_b16, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const __nv_bfloat16 b = __float2bfloat16_rn(theta[i]);
        if (theta_bf) theta_bf[i] = __bfloat162float(b);
        if (theta_b16) theta_b16[i] = b;
    }
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Z += b (per column), H = GELU(Z).  Z, H: [B x n] row-major.  H (optional) in FP32 and/or
// its BF16 parts Hhi / Hlo (optional, for the tensor-core products).
__global__ void k_bias_gelu(long long total, int n, float *__restrict__ Z, const float *__restrict__ b,
                            float *__restrict__ H, __nv_bfloat16 *__restrict__ Hhi, __nv_bfloat16 *__restrict__ Hlo) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const float z = Z[i] + b[i % n];
        Z[i] = z;
        const float h = gelu(z);
        if (H) H[i] = h;
        if (Hhi) split2(h, Hhi[i], Hlo[i]);
    }
}

// y[r] = H[r, :] . w + b0 (warp per row), and (optional) dy = 2 (y - t) / B, loss partials.
__global__ void k_out_layer(int B, const float *__restrict__ H, const float *__restrict__ w, const float *__restrict__ b,
                            float *__restrict__ y, const float *__restrict__ t, float *__restrict__ dy,
                            double *__restrict__ loss_part) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    double se = 0.0;
    if (warp < B) {
        const float *h = H + (long long)warp * MLP_H;
        float s = 0.f;
        for (int j = lane; j < MLP_H; j += 32) s = fmaf(h[j], w[j], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        const float v = s + b[0];
        if (lane == 0) {
            y[warp] = v;
            if (t) {
                const float e = v - t[warp];
                dy[warp] = 2.f * e / (float)B;
                se = (double)e * (double)e;
            }
        }
    }
    if (loss_part && lane == 0) atomicAdd(loss_part, se);
}

// dZ = dH * GELU'(Z); its BF16 parts (optional) row-major too.
__global__ void k_gelu_back(long long total, const float *__restrict__ Z, const float *__restrict__ dH,
                            float *__restrict__ dZ, __nv_bfloat16 *__restrict__ dZhi, __nv_bfloat16 *__restrict__ dZlo) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const float g = dH[i] * gelu_grad(Z[i]);
        dZ[i] = g;
        if (dZhi) split2(g, dZhi[i], dZlo[i]);
    }
}

// First-layer weight gradient dW[c][k] = sum_r dZ[r, c] X[r, k] (n columns, 8 inputs) in the
// two fixed-order passes of the column sums: block (x, y) forms the 8 sums of its rows for 32
// columns into part[(y * 8 + k) * n + c]; k_wgrad_in_fin adds the row blocks in order.
__global__ void k_wgrad_in_part(int B, int n, int rows_per, const float *__restrict__ dZ, const float *__restrict__ X,
                                float *__restrict__ part) {
    __shared__ float red[8][MLP_IN][33];
    const int lane = threadIdx.x & 31, c = blockIdx.x * 32 + lane, rg = threadIdx.x >> 5;
    const int r0 = blockIdx.y * rows_per, r1 = min(B, r0 + rows_per);
    float s[MLP_IN];
#pragma unroll
    for (int k = 0; k < MLP_IN; k++) s[k] = 0.f;
    if (c < n)
        for (int r = r0 + rg; r < r1; r += 8) {
            const float g = dZ[(long long)r * n + c];
#pragma unroll
            for (int k = 0; k < MLP_IN; k++) s[k] = fmaf(g, X[(long long)r * MLP_IN + k], s[k]);
        }
#pragma unroll
    for (int k = 0; k < MLP_IN; k++) red[rg][k][lane] = s[k];
    __syncthreads();
    if (rg == 0 && c < n) {
        for (int k = 0; k < MLP_IN; k++) {
            float t = 0.f;
            for (int i = 0; i < 8; i++) t += red[i][k][lane];
            part[((long long)blockIdx.y * MLP_IN + k) * n + c] = t;
        }
    }
}

__global__ void k_wgrad_in_fin(int nb, int n, const float *__restrict__ part, float *__restrict__ dW) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // i = c * 8 + k
    if (i >= n * MLP_IN) return;
    const int c = i / MLP_IN, k = i - c * MLP_IN;
    float t = 0.f;
    for (int b = 0; b < nb; b++) t += part[((long long)b * MLP_IN + k) * n + c];
    dW[i] = t;
}

// Weighted column sums over the batch in two fixed-order passes, so that the reduction
// spreads over many SMs: block (x, y) sums rows [y * rows_per, (y + 1) * rows_per) of 32
// columns (8 row groups, then in order) into part[y * n + c]; k_colsum_fin adds the row
// blocks in order.  w (optional): row weights.
__global__ void k_colsum_part(int B, int n, int rows_per, const float *__restrict__ M, const float *__restrict__ w,
                              float *__restrict__ part) {
    __shared__ float red[8][33];
    const int lane = threadIdx.x & 31, c = blockIdx.x * 32 + lane, rg = threadIdx.x >> 5;
    const int r0 = blockIdx.y * rows_per, r1 = min(B, r0 + rows_per);
    float s = 0.f;
    if (c < n)
        for (int r = r0 + rg; r < r1; r += 8) s = w ? fmaf(w[r], M[(long long)r * n + c], s) : s + M[(long long)r * n + c];
    red[rg][lane] = s;
    __syncthreads();
    if (rg == 0 && c < n) {
        float t = 0.f;
        for (int i = 0; i < 8; i++) t += red[i][lane];
        part[(long long)blockIdx.y * n + c] = t;
    }
}

__global__ void k_colsum_fin(int nb, int n, const float *__restrict__ part, float *__restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float t = 0.f;
    for (int b = 0; b < nb; b++) t += part[(long long)b * n + c];
    out[c] = t;
}

// dH4 = dy (outer) w5
__global__ void k_out_back(int B, const float *__restrict__ dy, const float *__restrict__ w, float *__restrict__ dH) {
    const long long total = (long long)B * MLP_H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        dH[i] = dy[i / MLP_H] * w[i % MLP_H];
}

// Adam on the FP32 master weights; refreshes the BF16 working copy.
__global__ void k_adam(int n, float *__restrict__ theta, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, float lr, float b1, float b2, float eps, float c1, float c2,
                       float *__restrict__ theta_bf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float th = theta[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        theta[i] = th;
        theta_bf[i] = __bfloat162float(__float2bfloat16_rn(th));
    }
}

// The same step with the step count and learning rate on the device: step s = *step + 1,
// lr = lr_table[s - 1] (a schedule), bias corrections 1 - b^s; a following k_step_inc
// advances *step.  A training loop of these launches can be captured in a CUDA graph once
// and replayed every epoch.
__global__ void k_adam_sched(int n, float *__restrict__ theta, float *__restrict__ m, float *__restrict__ v,
                             const float *__restrict__ g, const float *__restrict__ lr_table,
                             const int *__restrict__ step, float b1, float b2, float eps,
                             float *__restrict__ theta_bf) {
    const int s = *step + 1;
    const float c1 = 1.f - powf(b1, (float)s), c2 = 1.f - powf(b2, (float)s);
    const float lr = lr_table[s - 1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float th = theta[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        theta[i] = th;
        theta_bf[i] = __bfloat162float(__float2bfloat16_rn(th));
    }
}

__global__ void k_step_inc(int *step) { *step += 1; }

// ---- implied volatility of call prices (FP64 bisection on the Black-Scholes price)
__device__ double bs_call(double s, double k, double r, double sig, double t) {
    const double sq = sig * sqrt(t);
    const double d1 = (log(s / k) + (r + 0.5 * sig * sig) * t) / sq;
    return s * normcdf(d1) - k * exp(-r * t) * normcdf(d1 - sq);
}

__global__ void k_implied_vol(long long n, const double *__restrict__ price, const double *__restrict__ K,
                              const double *__restrict__ T, const double *__restrict__ r,
                              const double *__restrict__ S0, double *__restrict__ iv) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double p = price[i], k = K[i], t = T[i], rr = r[i], s0 = S0[i];
        const double intrinsic = fmax(s0 - k * exp(-rr * t), 0.0);
        double lo = 1e-4, hi = 4.0;
        if (!(p > intrinsic) || p >= s0) {
            iv[i] = nan("");
            continue;
        }
        for (int it = 0; it < 80; it++) {
            const double mid = 0.5 * (lo + hi);
            if (bs_call(s0, k, rr, mid, t) > p) hi = mid; else lo = mid;
        }
        iv[i] = 0.5 * (lo + hi);
    }
}

}  // namespace opb

using namespace opb;

namespace {

struct MlpWs {  // training workspace carve (floats)
    float *Z[4], *H[4], *dZ, *dH, *y, *dy, *part;
    double *loss;
    // 16-bit parts for the tensor-core products of the hidden layers 1..3 (split2, BF16):
    // Hp[l][0/1] of H[l] (l = 0..2, B x 256 row-major), dZp of dZ (B x 256), dZt of dZ^T
    // (256 x B), Wp[l][0/1] of the working weights W_{l+1} (256 x 256, exact BF16: lo = 0)
    __nv_bfloat16 *Hp[3][2], *dZp[2], *dZt[2], *Wp[3][2];
};

// Weight gradients reduce over the batch (K = B): split into at most MLP_KSPLIT chunks,
// one batched SIMT launch over the chunks, then a fixed-order sum of the partials, so
// that the reduction keeps every SM busy and stays deterministic.
constexpr int MLP_KSPLIT = 32;

int grid_ew(long long n);

MlpWs carve_mlp(float *ws, int B) {
    MlpWs w{};
    size_t o = 0;
    for (int l = 0; l < 4; l++) {
        w.Z[l] = ws + o; o += (size_t)B * MLP_H;
        w.H[l] = ws + o; o += (size_t)B * MLP_H;
    }
    w.dZ = ws + o; o += (size_t)B * MLP_H;
    w.dH = ws + o; o += (size_t)B * MLP_H;
    w.y = ws + o; o += (size_t)B;
    w.dy = ws + o; o += (size_t)B;
    o = (o + 3) & ~size_t(3);
    w.part = ws + o; o += (size_t)MLP_KSPLIT * MLP_H * MLP_H;
    o = (o + 1) & ~size_t(1);
    w.loss = reinterpret_cast<double *>(ws + o);
    o += 2;
    // parts: 64-float (256-byte) aligned pieces, each n bf16 values in n / 2 floats
    auto parts = [&](size_t n) {
        o = (o + 63) & ~size_t(63);
        __nv_bfloat16 *q = reinterpret_cast<__nv_bfloat16 *>(ws + o);
        o += n / 2;
        return q;
    };
    const size_t bh = (size_t)B * MLP_H;
    for (int l = 0; l < 3; l++)
        for (int k = 0; k < 2; k++) w.Hp[l][k] = parts(bh);
    for (int k = 0; k < 2; k++) w.dZp[k] = parts(bh);
    for (int k = 0; k < 2; k++) w.dZt[k] = parts(bh);
    for (int l = 0; l < 3; l++)
        for (int k = 0; k < 2; k++) w.Wp[l][k] = parts((size_t)MLP_H * MLP_H);
    return w;
}

// The hidden layers' products run on the tensor cores (split-BF16, three products, FP32
// accumulation) when the batch is a multiple of 128 rows; the first layer (8 inputs) and
// the output layer stay on the SIMT kernels.  opb_mlp_set_tensor_cores(0): SIMT throughout.
int g_mlp_tc = 1;
bool mlp_tc(int B) { return g_mlp_tc && B % 128 == 0; }

// C[M x N] = A[M x K] . B^T with A's parts row-major (lda) and B's parts N x K row-major
// (b_kn = 0) or K x N row-major (b_kn = 1); ksplit > 1: K-slices into C + s * M * N.
int mlp_tc_gemm(int M, int N, int K, __nv_bfloat16 *const *A, long long lda, __nv_bfloat16 *const *Bp,
                long long ldb, int b_kn, float *C, int ksplit, cudaStream_t s) {
    TcGemmArgs a{};
    a.M = M; a.N = N; a.K = K; a.Ahi = A[0]; a.Alo = A[1]; a.lda = lda; a.Bhi = Bp[0]; a.Blo = Bp[1]; a.ldb = ldb;
    a.b_kn = b_kn; a.C = C; a.ldc = N; a.alpha = 1.f; a.beta = 0.f;
    if (ksplit > 1) {
        a.ksplit = ksplit;
        a.c_slice = (long long)M * N;
    }
    return launch_tc_gemm(a, s);
}

__global__ void k_sum_parts(int nparts, long long n, const float *__restrict__ part, float *__restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int p = 0; p < nparts; p++) acc += part[p * n + i];
        out[i] = acc;
    }
}

// dW[out x in] = dZ[B x out]^T . in[B x in], split over the batch.
int mlp_weight_grad(int out, int in, int B, const float *dZ, const float *X, float *dW, float *part,
                    cudaStream_t s) {
    int nch = (B + 63) / 64;
    if (nch > MLP_KSPLIT) nch = MLP_KSPLIT;
    const int kc = (B + nch - 1) / nch;
    const int full = B / kc, rem = B - full * kc;
    const long long n = (long long)out * in;
    if (full > 0) {
        int r = sgemm_rm_strided(true, false, out, in, kc, 1.f, dZ, out, (long long)kc * out, X, in,
                                 (long long)kc * in, 0.f, part, in, n, full, s);
        if (r) return r;
    }
    if (rem > 0) {
        int r = sgemm_rm_t(true, false, out, in, rem, 1.f, dZ + (long long)full * kc * out, out,
                           X + (long long)full * kc * in, in, 0.f, part + (long long)full * n, in, s);
        if (r) return r;
    }
    const int np = full + (rem > 0 ? 1 : 0);
    k_sum_parts<<<grid_ew(n), 256, 0, s>>>(np, n, part, dW);
    return (int)cudaGetLastError();
}

// out[c] = sum_r (w[r] *) M[r, c] for c < n over B rows (part: scratch of 32 n floats).
int mlp_colsum(int B, int n, const float *M, const float *w, float *part, float *out, cudaStream_t s) {
    const int nb = B < 32 * 128 ? (B + 127) / 128 : 32;
    const int rows_per = (B + nb - 1) / nb;
    k_colsum_part<<<dim3((n + 31) / 32, nb), 256, 0, s>>>(B, n, rows_per, M, w, part);
    k_colsum_fin<<<(n + 255) / 256, 256, 0, s>>>(nb, n, part, out);
    return (int)cudaGetLastError();
}

int grid_ew(long long n) {
    long long b = (n + 255) / 256;
    long long cap = 8LL * num_sms();
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

#define MT(expr)                          \
    do {                                  \
        int _r = (expr);                  \
        if (_r) return set_status(_r);    \
    } while (0)

int mlp_forward(const float *thb, const float *X, int B, MlpWs &w, cudaStream_t s) {
    const MlpLayout L = mlp_layout();
    const bool tc = mlp_tc(B);
    if (tc)
        for (int l = 1; l < 4; l++)
            MT(launch_split(MLP_H, MLP_H, thb + L.w[l], MLP_H, w.Wp[l - 1][0], w.Wp[l - 1][1], nullptr, nullptr, 0,
                            s));
    const float *in = X;
    for (int l = 0; l < 4; l++) {
        // Z = in . W^T  (W stored out x in: the TB form)
        if (tc && l > 0)
            MT(mlp_tc_gemm(B, MLP_H, MLP_H, w.Hp[l - 1], MLP_H, w.Wp[l - 1], MLP_H, 0, w.Z[l], 1, s));
        else
            MT(sgemm_rm_t(false, true, B, L.out[l], L.in[l], 1.f, in, L.in[l], thb + L.w[l], L.in[l], 0.f, w.Z[l],
                          L.out[l], s));
        const long long tot = (long long)B * L.out[l];
        // with the tensor cores, layers 0..2 store only their activations' parts (the next
        // product's A and the weight gradient's B); the last one FP32 for the output layer
        const bool parts = tc && l < 3;
        k_bias_gelu<<<grid_ew(tot), 256, 0, s>>>(tot, L.out[l], w.Z[l], thb + L.b[l], parts ? nullptr : w.H[l],
                                                 parts ? w.Hp[l][0] : nullptr, parts ? w.Hp[l][1] : nullptr);
        in = w.H[l];
    }
    return (int)cudaGetLastError();
}

}  // namespace

OPB_API int opb_mlp_param_count(void) { return MLP_NPARAM; }

// floats of training workspace for batch B
OPB_API long long opb_mlp_workspace_floats(int B) {
    // FP32 buffers, then the tensor-core parts (5 B x 256 + 3 x 256 x 256 floats of BF16 pairs)
    // with their alignment
    return 10LL * B * MLP_H + 2LL * B + 4 + (long long)MLP_KSPLIT * MLP_H * MLP_H + 8 + 5LL * B * MLP_H +
           3LL * MLP_H * MLP_H + 14 * 64;
}

// 1 (default): the hidden layers' training products on the tensor cores (batches of a
// multiple of 128 rows); 0: SIMT FP32 throughout.
OPB_API int opb_mlp_set_tensor_cores(int on) {
    OPB_REQUIRE(on == 0 || on == 1, OPB_E_ARG);
    g_mlp_tc = on;
    return set_status(OPB_OK);
}

OPB_API int opb_mlp_init(float *theta, unsigned long long seed) {
    OPB_REQUIRE(theta, OPB_E_NULL);
    k_mlp_init<<<grid_ew(MLP_NPARAM), 256, 0, stream()>>>(theta, seed);
    return launch_check();
}

// theta_bf: BF16-rounded FP32 working copy (optional); theta_b16: BF16 storage (optional)
OPB_API int opb_mlp_round(const float *theta, float *theta_bf, void *theta_b16) {
    OPB_REQUIRE(theta, OPB_E_NULL);
    k_mlp_round<<<grid_ew(MLP_NPARAM), 256, 0, stream()>>>(theta, theta_bf, reinterpret_cast<__nv_bfloat16 *>(theta_b16),
                                                            MLP_NPARAM);
    return launch_check();
}

// Forward pass of B rows of X [B x 8] with the working weights thb; y [B].  The workspace
// keeps the pre-activations for a following opb_mlp_backward.
OPB_API int opb_mlp_forward(const float *thb, const float *X, int B, float *ws, float *y) {
    OPB_REQUIRE(thb && X && ws && y, OPB_E_NULL);
    OPB_REQUIRE(B > 0, OPB_E_ARG);
    MlpWs w = carve_mlp(ws, B);
    cudaStream_t s = stream();
    MT(mlp_forward(thb, X, B, w, s));
    const MlpLayout L = mlp_layout();
    k_out_layer<<<(B * 32 + 255) / 256, 256, 0, s>>>(B, w.H[3], thb + L.w[4], thb + L.b[4], y, nullptr, nullptr,
                                                      nullptr);
    return launch_check();
}

// Loss (mean squared error against t) and its gradient with respect to the working weights,
// written into grad [param count].  loss (device, 1 double, optional) receives the mean.
OPB_API int opb_mlp_loss_grad(const float *thb, const float *X, const float *t, int B, float *ws, float *grad,
                              double *loss) {
    OPB_REQUIRE(thb && X && t && ws && grad, OPB_E_NULL);
    OPB_REQUIRE(B > 0, OPB_E_ARG);
    MlpWs w = carve_mlp(ws, B);
    cudaStream_t s = stream();
    const MlpLayout L = mlp_layout();
    MT(mlp_forward(thb, X, B, w, s));
    MT((int)cudaMemsetAsync(w.loss, 0, sizeof(double), s));
    k_out_layer<<<(B * 32 + 255) / 256, 256, 0, s>>>(B, w.H[3], thb + L.w[4], thb + L.b[4], w.y, t, w.dy, w.loss);
    // output layer
    // (column sums over the batch in two fixed-order passes over many blocks)
    MT(mlp_colsum(B, MLP_H, w.H[3], w.dy, w.part, grad + L.w[4], s));
    MT(mlp_colsum(B, 1, w.dy, nullptr, w.part, grad + L.b[4], s));
    k_out_back<<<grid_ew((long long)B * MLP_H), 256, 0, s>>>(B, w.dy, thb + L.w[4], w.dH);
    const bool tc = mlp_tc(B);
    // weight-gradient K-slices on the tensor cores: at most MLP_KSPLIT, dividing B / 64
    int ks = B / 64 < MLP_KSPLIT ? B / 64 : MLP_KSPLIT;
    while (ks > 1 && (B / 64) % ks) ks--;
    for (int l = 3; l >= 0; l--) {
        const long long tot = (long long)B * L.out[l];
        const bool parts = tc && l > 0;
        k_gelu_back<<<grid_ew(tot), 256, 0, s>>>(tot, w.Z[l], w.dH, w.dZ, parts ? w.dZp[0] : nullptr,
                                                 parts ? w.dZp[1] : nullptr);
        const float *in = l > 0 ? w.H[l - 1] : X;
        if (parts) {
            // dZ's parts transposed (for dW; the row-major ones, for dH, came with dZ)
            MT(launch_split(B, MLP_H, w.dZ, MLP_H, nullptr, nullptr, w.dZt[0], w.dZt[1], B, s));
            // dW = dZ^T . in: A = dZ^T's parts (256 x B), B = in's parts read K x N (B x 256)
            MT(mlp_tc_gemm(MLP_H, MLP_H, B, w.dZt, B, w.Hp[l - 1], MLP_H, 1, w.part, ks, s));
            k_sum_parts<<<grid_ew((long long)MLP_H * MLP_H), 256, 0, s>>>(ks, (long long)MLP_H * MLP_H, w.part,
                                                                          grad + L.w[l]);
        } else if (l == 0) {
            // dW = dZ^T . X (8 inputs): eight weighted column sums
            const int nb = B < 32 * 128 ? (B + 127) / 128 : 32;
            const int rows_per = (B + nb - 1) / nb;
            k_wgrad_in_part<<<dim3(MLP_H / 32, nb), 256, 0, s>>>(B, MLP_H, rows_per, w.dZ, X, w.part);
            k_wgrad_in_fin<<<(MLP_H * MLP_IN + 255) / 256, 256, 0, s>>>(nb, MLP_H, w.part, grad + L.w[0]);
        } else {
            // dW = dZ^T . in  (A = dZ stored B x out: the TA form)
            MT(mlp_weight_grad(L.out[l], L.in[l], B, w.dZ, in, grad + L.w[l], w.part, s));
        }
        MT(mlp_colsum(B, L.out[l], w.dZ, nullptr, w.part, grad + L.b[l], s));
        if (l > 0) {
            // dH = dZ . W: B = W's parts read K x N (out x in)
            if (tc) MT(mlp_tc_gemm(B, MLP_H, MLP_H, w.dZp, MLP_H, w.Wp[l - 1], MLP_H, 1, w.dH, 1, s));
            else
                MT(sgemm_rm_t(false, false, B, L.in[l], L.out[l], 1.f, w.dZ, L.out[l], thb + L.w[l], L.in[l], 0.f,
                              w.dH, L.in[l], s));
        }
    }
    if (loss) {
        // mean of the squared errors
        MT((int)cudaMemcpyAsync(loss, w.loss, sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    return launch_check();
}

OPB_API int opb_mlp_adam(float *theta, float *m, float *v, const float *grad, int step, float lr, float b1, float b2,
                         float eps, float *theta_bf) {
    OPB_REQUIRE(theta && m && v && grad && theta_bf, OPB_E_NULL);
    OPB_REQUIRE(step >= 1 && lr > 0.f, OPB_E_ARG);
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<grid_ew(MLP_NPARAM), 256, 0, stream()>>>(MLP_NPARAM, theta, m, v, grad, lr, b1, b2, eps, c1, c2, theta_bf);
    return launch_check();
}

// Adam with the step counter (device int, advanced by the call) and the learning-rate
// schedule (device lr_table[step - 1]) in device memory, so that a training loop of
// opb_mlp_loss_grad / opb_mlp_adam_sched calls is the same work every epoch and can be
// captured in a CUDA graph.  Same update as opb_mlp_adam.
OPB_API int opb_mlp_adam_sched(float *theta, float *m, float *v, const float *grad, int *step, const float *lr_table,
                               float b1, float b2, float eps, float *theta_bf) {
    OPB_REQUIRE(theta && m && v && grad && step && lr_table && theta_bf, OPB_E_NULL);
    k_adam_sched<<<grid_ew(MLP_NPARAM), 256, 0, stream()>>>(MLP_NPARAM, theta, m, v, grad, lr_table, step, b1, b2,
                                                             eps, theta_bf);
    k_step_inc<<<1, 1, 0, stream()>>>(step);
    return launch_check();
}

// Implied volatilities of n call prices with spots S0[i]; NaN where the price carries no
// time value.
OPB_API int opb_implied_vol(long long n, const double *price, const double *K, const double *T, const double *r,
                            const double *S0, double *iv) {
    OPB_REQUIRE(n >= 0, OPB_E_ARG);
    if (n == 0) return set_status(OPB_OK);
    OPB_REQUIRE(price && K && T && r && S0 && iv, OPB_E_NULL);
    k_implied_vol<<<grid_ew(n), 256, 0, stream()>>>(n, price, K, T, r, S0, iv);
    return launch_check();
}

// ---------------------------------------------------------------- tensor-core inference
//
// Packed inference weights of one network (bytes): W1 padded to [256 x 64] BF16 (input
// features 8..63 zero), W2..W4 [256 x 256] BF16, then FP32 b1..b4 [4 x 256], w5 [256], b5.
namespace opb {

constexpr long long MLP_PACK_W1 = 256LL * 64 * 2, MLP_PACK_WH = 256LL * 256 * 2;
constexpr long long MLP_PACK_BYTES = MLP_PACK_W1 + 3 * MLP_PACK_WH + (4 * 256 + 256 + 1) * 4;

__global__ void k_mlp_pack(const float *__restrict__ theta, uint8_t *__restrict__ packed) {
    const MlpLayout L = mlp_layout();
    __nv_bfloat16 *w1 = reinterpret_cast<__nv_bfloat16 *>(packed);
    __nv_bfloat16 *wh = reinterpret_cast<__nv_bfloat16 *>(packed + MLP_PACK_W1);
    float *f = reinterpret_cast<float *>(packed + MLP_PACK_W1 + 3 * MLP_PACK_WH);
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nth = (long long)gridDim.x * blockDim.x;
    for (long long i = tid; i < 256 * 64; i += nth) {
        const int o = (int)(i / 64), c = (int)(i % 64);
        w1[i] = __float2bfloat16_rn(c < MLP_IN ? theta[L.w[0] + (long long)o * MLP_IN + c] : 0.f);
    }
    for (long long i = tid; i < 3LL * 256 * 256; i += nth) {
        const int l = 1 + (int)(i / (256 * 256));
        wh[i] = __float2bfloat16_rn(theta[L.w[l] + i % (256 * 256)]);
    }
    for (long long i = tid; i < 4 * 256 + 256 + 1; i += nth) {
        float v;
        if (i < 4 * 256) v = __bfloat162float(__float2bfloat16_rn(theta[L.b[i / 256] + i % 256]));
        else if (i < 4 * 256 + 256) v = __bfloat162float(__float2bfloat16_rn(theta[L.w[4] + (i - 1024)]));
        else v = __bfloat162float(__float2bfloat16_rn(theta[L.b[4]]));
        f[i] = v;
    }
}

// X [n x 8] FP32 -> Xp [n x 64] BF16 (zero padded)
__global__ void k_mlp_pad_input(long long n, const float *__restrict__ X, __nv_bfloat16 *__restrict__ Xp) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * 64;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / 64;
        const int c = (int)(i % 64);
        Xp[i] = __float2bfloat16_rn(c < MLP_IN ? X[r * MLP_IN + c] : 0.f);
    }
}

// Ensemble mean and spread (max - min): member m's output is its MLP_YPARTS column-group
// partial dots yp[(MLP_YPARTS m + g) * np + r] (from the fused last layer) plus its bias b5
// (the last float of its packed weights).
constexpr int MLP_YPARTS = 256 / TC_LAYER_CPT;
__global__ void k_mlp_ensemble(long long n, long long np, int nmem, const float *__restrict__ yp,
                               const uint8_t *__restrict__ packed, long long stride, long long b5_off,
                               float *__restrict__ mean, float *__restrict__ spread) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        float s = 0.f, lo = 3.4e38f, hi = -3.4e38f;
        for (int m = 0; m < nmem; m++) {
            const float b5 = *reinterpret_cast<const float *>(packed + (long long)m * stride + b5_off);
            float v = 0.f;
            for (int g = 0; g < MLP_YPARTS; g++) v += yp[((long long)MLP_YPARTS * m + g) * np + r];
            v += b5;
            s += v;
            lo = fminf(lo, v);
            hi = fmaxf(hi, v);
        }
        mean[r] = s / (float)nmem;
        if (spread) spread[r] = hi - lo;
    }
}

}  // namespace opb

OPB_API long long opb_mlp_packed_bytes(void) { return MLP_PACK_BYTES; }

OPB_API int opb_mlp_pack(const float *theta, void *packed) {
    OPB_REQUIRE(theta && packed, OPB_E_NULL);
    OPB_REQUIRE(aligned(packed, 16), OPB_E_ALIGN);
    k_mlp_pack<<<grid_ew(3LL * 256 * 256), 256, 0, stream()>>>(theta, reinterpret_cast<uint8_t *>(packed));
    return launch_check();
}

// Inference workspace bytes for n rows (n padded to a multiple of 128 internally).
OPB_API long long opb_mlp_infer_workspace_bytes(long long n, int nmem) {
    const long long np = (n + 127) / 128 * 128;
    return np * 64 * 2 + 2 * np * 256 * 2 + (long long)MLP_YPARTS * nmem * np * 4 + 1024;
}

// Inference form: 1 = one fused kernel per member (default), 0 = one launch per layer with
// the activations through HBM.  Both give bit-identical outputs.
static int g_mlp_fused = 1;

// Ensemble inference on the tensor cores: members m = 0..nmem-1 with packed weights at
// packed + m * member_stride bytes; X [n x 8] normalised features (FP32).  mean [n] and
// spread [n] (optional) receive the ensemble mean and max - min of the member outputs.
OPB_API int opb_mlp_infer(const void *packed, int nmem, long long member_stride, const float *X, long long n,
                          void *ws, long long ws_bytes, float *mean, float *spread) {
    OPB_NVTX("opb_mlp_infer");
    OPB_REQUIRE(packed && X && ws && mean, OPB_E_NULL);
    OPB_REQUIRE(nmem >= 1 && n >= 1 && member_stride >= MLP_PACK_BYTES, OPB_E_ARG);
    OPB_REQUIRE(ws_bytes >= opb_mlp_infer_workspace_bytes(n, nmem), OPB_E_ARG);
    OPB_REQUIRE(aligned(packed, 16) && member_stride % 16 == 0 && aligned(ws, 256), OPB_E_ALIGN);
    cudaStream_t s = stream();
    const long long np = (n + 127) / 128 * 128;
    uint8_t *w8 = reinterpret_cast<uint8_t *>(ws);
    __nv_bfloat16 *Xp = reinterpret_cast<__nv_bfloat16 *>(w8);
    __nv_bfloat16 *Ha = reinterpret_cast<__nv_bfloat16 *>(w8 + np * 64 * 2);
    __nv_bfloat16 *Hb = Ha + np * 256;
    float *ym = reinterpret_cast<float *>(reinterpret_cast<uint8_t *>(Hb + np * 256));
    MT((int)cudaMemsetAsync(Xp, 0, np * 64 * 2, s));
    k_mlp_pad_input<<<grid_ew(n * 64), 256, 0, s>>>(n, X, Xp);
    for (int m = 0; m < nmem; m++) {
        const uint8_t *pk = reinterpret_cast<const uint8_t *>(packed) + (long long)m * member_stride;
        const __nv_bfloat16 *W1 = reinterpret_cast<const __nv_bfloat16 *>(pk);
        const __nv_bfloat16 *WH = reinterpret_cast<const __nv_bfloat16 *>(pk + MLP_PACK_W1);
        const float *f = reinterpret_cast<const float *>(pk + MLP_PACK_W1 + 3 * MLP_PACK_WH);
        if (g_mlp_fused) {  // all layers in one kernel, the activations in shared memory
            MT(launch_mlp_fused(np, Xp, W1, WH, f, ym + (long long)MLP_YPARTS * m * np, s));
            continue;
        }
        MT(launch_tc_layer((int)np, 256, 64, Xp, 64, W1, 64, 1.f, f, Ha, 256, s));
        MT(launch_tc_layer((int)np, 256, 256, Ha, 256, WH, 256, 1.f, f + 256, Hb, 256, s));
        MT(launch_tc_layer((int)np, 256, 256, Hb, 256, WH + 65536, 256, 1.f, f + 512, Ha, 256, s));
        // last hidden layer with the output layer fused into its epilogue
        MT(launch_tc_layer((int)np, 256, 256, Ha, 256, WH + 2 * 65536, 256, 1.f, f + 768, nullptr, 256, s, f + 1024,
                           ym + (long long)MLP_YPARTS * m * np));
    }
    k_mlp_ensemble<<<grid_ew(n), 256, 0, s>>>(n, np, nmem, ym, reinterpret_cast<const uint8_t *>(packed),
                                              member_stride, MLP_PACK_W1 + 3 * MLP_PACK_WH + 1280LL * 4, mean, spread);
    return launch_check();
}

OPB_API int opb_mlp_set_fused_inference(int on) {
    OPB_REQUIRE(on == 0 || on == 1, OPB_E_ARG);
    g_mlp_fused = on;
    return set_status(OPB_OK);
}
