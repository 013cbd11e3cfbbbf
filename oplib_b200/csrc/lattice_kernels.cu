// Element-wise and row-wise kernels of the lattice path (all HBM-bound).
//
// Storage is source-major (row y = source state, element (y, z) at y*d + z); it is the
// transpose of the reference's (y1 + d*y2) storage, so a row here is a column there.
//
//   ek       : U0 = I + dt*L built in FP64 on the device and rounded once to FP32, or
//              its "E-form" E0 = U0 - I = dt*L (oplib/opcuda/sek.cu:40-59;
//              oplib/opmodel/models/CModel Host Double.cs:89-121).
//   renorm   : FP64 row sums, then every row divided by its sum (probability
//              conservation after each squaring; no reference counterpart).  In E-form
//              the identity is carried implicitly: with D = 2E + E.E and s = 1 + sum(D_y.),
//              E_new[y,z] = (D[y,z] - [z==y]*sum(D_y.)) / s_y, which equals
//              (I + D)/s - I exactly.  Inside a lattice solve the FP32 matrix is not
//              written back at intermediate levels: the per-row (sum, 1/s) go to a fix
//              array that the next squaring's epilogue applies to its Cin.
//   split    : a = hi + lo with hi = bf16(a), lo = bf16(a - hi), written row-major (the
//              K-major A operand, and the MN-major B operand of the lattice products);
//              the public forms can also write the transpose (a K-major B operand).
//   payoff / discount : call payoffs G[z,k] = (x_z - K_k)^+ and the FP64 discounting of
//              the backward-induction result.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "lattice.h"

namespace opb {

__global__ void k_zero_set_diag(int d, float *__restrict__ U, float v) {
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y < d) U[(long long)y * d + y] = v;
}

// ELL generator: row y holds w (col, val) pairs; col < 0 marks padding.
__global__ void k_ek_scatter_ell(int d, int w, const int *__restrict__ cols, const double *__restrict__ vals,
                                 double dt, int eform, float *__restrict__ out, long long ld) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)d * w) return;
    int y = (int)(t / w);
    int z = cols[t];
    if (z < 0 || z >= d) return;
    double v = dt * vals[t];
    if (!eform && z == y) v += 1.0;
    out[(long long)y * ld + z] = (float)v;
}

// Half-bandwidth of an ELL generator: max |col - row| over its entries (padding excluded),
// by one block.  The squarings read it to leave out the K-blocks that multiply zeros.
__global__ void __launch_bounds__(1024) k_ell_band(int d, int w, const int *__restrict__ cols, int *__restrict__ out) {
    __shared__ int wmax[32];
    int m = 0;
    const long long n = (long long)d * w;
    for (long long t = threadIdx.x; t < n; t += blockDim.x) {
        const int z = cols[t];
        if (z >= 0 && z < d) m = max(m, abs(z - (int)(t / w)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? wmax[threadIdx.x] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) *out = m;
    }
}

// Dense FP64 generator, row-major (source-major), into rows of leading dimension ld.
__global__ void k_ek_dense(int d, const double *__restrict__ L, double dt, int eform, float *__restrict__ out,
                           long long ld) {
    long long n = (long long)d * d;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int y = (int)(t / d), z = (int)(t - (long long)y * d);
        double v = dt * L[t];
        if (!eform && z == y) v += 1.0;
        out[(long long)y * ld + z] = (float)v;
    }
}

// Spot values of a lattice padded with absorbing states: xpad[i] = x[min(i, d - 1)].
__global__ void k_pad_x(int d, int dpad, const double *__restrict__ x, double *__restrict__ xpad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < dpad) xpad[i] = x[i < d ? i : d - 1];
}

// 32x32 tiles, 256 threads.  X is (rows x cols) row-major with leading dimension ld.
// Writes hi/lo of X (row-major, ld) and of X^T (cols x rows, leading dimension ldt).
__global__ void k_split_tr(int rows, int cols, const float *__restrict__ X, long long ld,
                           __nv_bfloat16 *__restrict__ Ahi, __nv_bfloat16 *__restrict__ Alo,
                           __nv_bfloat16 *__restrict__ Bhi, __nv_bfloat16 *__restrict__ Blo, long long ldt,
                           float sscale) {
    __shared__ __nv_bfloat16 th[32][34], tl[32][34];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
        int r = r0 + i, c = c0 + tx;
        __nv_bfloat16 h = __float2bfloat16_rn(0.f), l = h;
        if (r < rows && c < cols) {
            split2(X[(long long)r * ld + c], h, l, sscale);
            if (Ahi) {
                Ahi[(long long)r * ld + c] = h;
                Alo[(long long)r * ld + c] = l;
            }
        }
        th[i][tx] = h;
        tl[i][tx] = l;
    }
    if (!Bhi) return;
    __syncthreads();
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
        int c = c0 + i, r = r0 + tx;
        if (r < rows && c < cols) {
            Bhi[(long long)c * ldt + r] = th[tx][i];
            Blo[(long long)c * ldt + r] = tl[tx][i];
        }
    }
}

// FP64 row sums of an FP32 matrix, one block per row -> partial[row].
__global__ void k_rowsum(int d, const float *__restrict__ X, double *__restrict__ partial) {
    const int y = blockIdx.x;
    const float *row = X + (long long)y * d;
    double s = 0.0;
    for (int z = threadIdx.x; z < d; z += blockDim.x) s += (double)row[z];
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) partial[y] = s;
    }
}

// Row renormalisation from FP64 row-sum partials (nparts partial sums per row, laid out
// partial[p*d + y]).  In place on X; optionally emits the hi/lo split of the result
// (row-major and transposed).
__global__ void k_renorm(int d, float *__restrict__ X, const double *__restrict__ partial, int nparts, int eform,
                         __nv_bfloat16 *__restrict__ Ahi, __nv_bfloat16 *__restrict__ Alo,
                         __nv_bfloat16 *__restrict__ Bhi, __nv_bfloat16 *__restrict__ Blo, float sscale) {
    __shared__ double s_sum[32], s_inv[32];
    __shared__ __nv_bfloat16 th[32][34], tl[32][34];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    if (ty == 0) {
        double s = 0.0;
        int r = r0 + tx;
        if (r < d)
            for (int p = 0; p < nparts; p++) s += partial[(long long)p * d + r];
        s_sum[tx] = s;
        double den = eform ? 1.0 + s : s;
        s_inv[tx] = den != 0.0 ? 1.0 / den : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
        int r = r0 + i, c = c0 + tx;
        __nv_bfloat16 h = __float2bfloat16_rn(0.f), l = h;
        if (r < d && c < d) {
            long long o = (long long)r * d + c;
            double v = (double)X[o];
            if (eform && r == c) v -= s_sum[i];
            float f = (float)(v * s_inv[i]);
            X[o] = f;
            if (Ahi) {
                split2(f, h, l, sscale);
                Ahi[o] = h;
                Alo[o] = l;
            }
        }
        th[i][tx] = h;
        tl[i][tx] = l;
    }
    if (!Bhi) return;
    __syncthreads();
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
        int c = c0 + i, r = r0 + tx;
        if (r < d && c < d) {
            Bhi[(long long)c * d + r] = th[tx][i];
            Blo[(long long)c * d + r] = tl[tx][i];
        }
    }
}

// Vectorised renormalisation of 64 x 64 tiles (d % 64 == 0), 256 threads: float4 loads
// and stores of X, 8-byte stores of four 16-bit parts, and the transposed parts staged
// through shared memory so that every global access is a contiguous run per warp.
// Modes: 0 = E-form in, E-form out; 1 = E-form in, P-form out (P = I + E_new: the last
// squaring level); 2 = P-form in and out.  nparts = 0 skips the scaling (pure split).
// Each (hi, lo) pair is one 32-bit shared word; the 65-word row stride keeps both the
// row-wise stores and the column-wise reads of the transpose at most 2-way bank-conflicted.
struct RenormSmem {
    double s_sum[64], s_inv[64];
    uint32_t t[64][65];
};

// Input staging: a ring of RN_RING tiles in shared memory filled by cp.async (16 bytes per
// thread and copy), so that RN_RING - 1 tiles are in flight per block while one is
// processed.  Each thread copies and later reads back only its own four float4 of a tile,
// so the ring needs no block barrier: cp.async.wait_group orders a thread's own copies.
struct RenormRing {
    float4 v[RN_RING][4][256];
};
constexpr int RN_SMEM = (int)(sizeof(RenormSmem) + sizeof(RenormRing));

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// This thread's four 16-byte copies of the tile at (r0, c0) into ring slot s.
__device__ __forceinline__ void renorm64_issue(RenormRing &rg, int s, int d, const float *__restrict__ X, int r0,
                                               int c0) {
    const int tid = threadIdx.x, lc = (tid & 15) * 4;
#pragma unroll
    for (int pass = 0; pass < 4; pass++)
        cp_async16(&rg.v[s][pass][tid], X + (long long)(r0 + pass * 16 + (tid >> 4)) * d + c0 + lc);
}

// FP64 row sums of rows r0..r0+63 over the nparts partials, summed in part order (the
// loads are issued 8 at a time; the additions stay sequential), and their reciprocals.
__device__ __forceinline__ void renorm64_sums(RenormSmem &sm, int d, const double *__restrict__ partial, int nparts,
                                              int mode, int r0, double2 *__restrict__ fix = nullptr) {
    const int tid = threadIdx.x;
    if (tid < 64) {
        double s = 0.0;
        const double *q = partial + r0 + tid;
        int p = 0;
        for (; p + 8 <= nparts; p += 8) {
            double v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) v[j] = q[(long long)(p + j) * d];
#pragma unroll
            for (int j = 0; j < 8; j++) s += v[j];
        }
        for (; p < nparts; p++) s += q[(long long)p * d];
        sm.s_sum[tid] = s;
        const double den = nparts == 0 ? 1.0 : (mode != 2 ? 1.0 + s : s);
        const double inv = den != 0.0 ? 1.0 / den : 0.0;
        sm.s_inv[tid] = inv;
        if (fix) fix[r0 + tid] = make_double2(s, inv);
    }
}

// One tile at (r0, c0), using the sums of renorm64_sums; vin holds the tile's values
// (read back from the staging ring) and the renormalised values are stored back into X
// unless it is null.  B parts (optional) are stored transposed, or with b_rm row-major
// like the A parts.  The sums must be visible to the block (a barrier after
// renorm64_sums); the transposed form starts with its own barrier, for the shared tile
// of the previous call.
__device__ __forceinline__ void renorm64_apply(RenormSmem &sm, int d, float *__restrict__ X, int mode,
                                               __nv_bfloat16 *__restrict__ Ahi, __nv_bfloat16 *__restrict__ Alo,
                                               __nv_bfloat16 *__restrict__ Bhi, __nv_bfloat16 *__restrict__ Blo,
                                               int r0, int c0, float sscale, const float4 (&vin)[4], bool b_rm) {
    const int tid = threadIdx.x;
    const bool eform = mode != 2;
    const bool transposed = Bhi && !b_rm;
    if (transposed) __syncthreads();
    const int lc = (tid & 15) * 4;
#pragma unroll
    for (int pass = 0; pass < 4; pass++) {
        const int lr = pass * 16 + (tid >> 4);
        const int r = r0 + lr;
        const long long o = (long long)r * d + c0 + lc;
        const float4 v = vin[pass];
        const double su = sm.s_sum[lr], inv = sm.s_inv[lr];
        float f[4] = {v.x, v.y, v.z, v.w};
        __nv_bfloat16 h[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            double x = (double)f[j];
            const bool diag = (r == c0 + lc + j);
            if (eform && diag) x -= su;
            x *= inv;
            if (mode == 1 && diag) x += 1.0;
            f[j] = (float)x;
            split2(f[j], h[j], l[j], sscale);
            if (transposed) sm.t[lr][lc + j] = pack_bf16(h[j], l[j]);
        }
        if (X) *reinterpret_cast<float4 *>(X + o) = make_float4(f[0], f[1], f[2], f[3]);
        if (Ahi) {
            *reinterpret_cast<uint2 *>(Ahi + o) = make_uint2(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]));
            *reinterpret_cast<uint2 *>(Alo + o) = make_uint2(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]));
        }
        if (Bhi && b_rm) {
            *reinterpret_cast<uint2 *>(Bhi + o) = make_uint2(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]));
            *reinterpret_cast<uint2 *>(Blo + o) = make_uint2(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]));
        }
    }
    if (!Bhi || b_rm) return;
    __syncthreads();
#pragma unroll
    for (int pass = 0; pass < 4; pass++) {
        const int orow = pass * 16 + (tid >> 4);
        const long long o = (long long)(c0 + orow) * d + r0 + lc;
        const uint32_t w0 = sm.t[lc + 0][orow], w1 = sm.t[lc + 1][orow], w2 = sm.t[lc + 2][orow],
                       w3 = sm.t[lc + 3][orow];
        *reinterpret_cast<uint2 *>(Bhi + o) = make_uint2(__byte_perm(w0, w1, 0x5410), __byte_perm(w2, w3, 0x5410));
        *reinterpret_cast<uint2 *>(Blo + o) = make_uint2(__byte_perm(w0, w1, 0x7632), __byte_perm(w2, w3, 0x7632));
    }
}

// Grid (column chunks, d / 64): block (bx, by) renormalises rows 64*by.. over the column
// tiles bx, bx + gridDim.x, ...; the row sums are formed once per block.
// Column tiles first, first + step, ... of the 64-row strip at r0, through the cp.async
// ring; the row sums are formed once, while the first tiles are in flight.  Xout (may be
// null) receives the renormalised values; fix (optional) the per-row (s, inv).
__device__ __forceinline__ void renorm64_strip(RenormSmem &sm, RenormRing &rg, int d, const float *__restrict__ X,
                                               float *__restrict__ Xout, const double *__restrict__ partial,
                                               int nparts, int mode, __nv_bfloat16 *__restrict__ Ahi,
                                               __nv_bfloat16 *__restrict__ Alo, __nv_bfloat16 *__restrict__ Bhi,
                                               __nv_bfloat16 *__restrict__ Blo, int r0, int first, int step,
                                               float sscale, double2 *__restrict__ fix, bool b_rm) {
    const int nt = d / 64, tid = threadIdx.x;
    const int cnt = first < nt ? (nt - 1 - first) / step + 1 : 0;
#pragma unroll
    for (int k = 0; k < RN_RING - 1; k++) {
        if (k < cnt) renorm64_issue(rg, k, d, X, r0, (first + k * step) * 64);
        cp_async_commit();  // possibly empty: every iteration commits exactly one group
    }
    renorm64_sums(sm, d, partial, nparts, mode, r0, fix);
    __syncthreads();  // the row sums are visible to every thread
    for (int k = 0; k < cnt; k++) {
        // the slot refilled here was read (and its values used) in iteration k - 1
        const int kn = k + RN_RING - 1;
        if (kn < cnt) renorm64_issue(rg, kn % RN_RING, d, X, r0, (first + kn * step) * 64);
        cp_async_commit();
        cp_async_wait<RN_RING - 1>();  // this thread's copies of tile k have landed
        const int sl = k % RN_RING;
        const float4 v[4] = {rg.v[sl][0][tid], rg.v[sl][1][tid], rg.v[sl][2][tid], rg.v[sl][3][tid]};
        renorm64_apply(sm, d, Xout, mode, Ahi, Alo, Bhi, Blo, r0, (first + k * step) * 64, sscale, v, b_rm);
    }
}

// Grid (column chunks, d / 64): block (bx, by) renormalises rows 64*by.. over the column
// tiles bx, bx + gridDim.x, ...  write_x = 0: X is only read (its renormalised values go
// to the splits alone); fix (optional) receives the per-row (s, inv), written by the
// blocks of column chunk 0; b_rm: B parts row-major (else transposed).  Dynamic shared
// memory RN_SMEM.
__global__ void __launch_bounds__(256) k_renorm64(int d, float *__restrict__ X, const double *__restrict__ partial,
                                                  int nparts, int mode, __nv_bfloat16 *__restrict__ Ahi,
                                                  __nv_bfloat16 *__restrict__ Alo, __nv_bfloat16 *__restrict__ Bhi,
                                                  __nv_bfloat16 *__restrict__ Blo, float sscale, int write_x = 1,
                                                  double2 *__restrict__ fix = nullptr, int b_rm = 0) {
    extern __shared__ __align__(16) uint8_t rn_smem[];
    RenormSmem &sm = *reinterpret_cast<RenormSmem *>(rn_smem);
    RenormRing &rg = *reinterpret_cast<RenormRing *>(rn_smem + sizeof(RenormSmem));
    renorm64_strip(sm, rg, d, X, write_x ? X : nullptr, partial, nparts, mode, Ahi, Alo, Bhi, Blo,
                   (int)blockIdx.y * 64, (int)blockIdx.x, (int)gridDim.x, sscale, blockIdx.x == 0 ? fix : nullptr,
                   b_rm != 0);
}

// Column chunks of a k_renorm64 launch: about 8 blocks per SM in total.
static dim3 renorm64_grid(int d) {
    const int nt = d / 64;
    int chunks = (8 * num_sms() + nt - 1) / nt;
    if (chunks > nt) chunks = nt;
    if (chunks < 1) chunks = 1;
    return dim3(chunks, nt);
}

// Batched: one block per work item (problem << 16 | mode << 14 | strip << 7 | chunk): the
// column tiles chunk, chunk + renorm_chunks(d), ... of one 64-row strip; nparts of problem
// i is d_i / parts_div (0 when parts_div == 0: pure split).  X is only read: every later
// product takes its operands from the splits, and a squaring's Cin gets this
// renormalisation through the row fixes (mode-0 items, chunk 0).  Only mode-1 items (P1,
// the B operand of every chain product) write B parts, row-major; squarings read E's
// row-major A parts as their B operand.
__global__ void __launch_bounds__(256) k_renorm64_batched(const RenormProblem *__restrict__ probs,
                                                          const uint32_t *__restrict__ work, int parts_div,
                                                          float sscale) {
    extern __shared__ __align__(16) uint8_t rn_smem[];
    RenormSmem &sm = *reinterpret_cast<RenormSmem *>(rn_smem);
    RenormRing &rg = *reinterpret_cast<RenormRing *>(rn_smem + sizeof(RenormSmem));
    const uint32_t w = work[blockIdx.x];
    const RenormProblem &pr = probs[w >> 16];
    const int mode = (int)((w >> 14) & 3u);
    const int nparts = parts_div > 0 ? pr.d / parts_div : 0;
    const int r0 = (int)((w >> 7) & 127u) * 64, chunk = (int)(w & 127u);
    renorm64_strip(sm, rg, pr.d, pr.X, nullptr, pr.partial, nparts, mode, pr.Ahi, pr.Alo,
                   mode == 1 ? pr.Bhi : nullptr, mode == 1 ? pr.Blo : nullptr, r0, chunk, renorm_chunks(pr.d),
                   sscale, mode == 0 && chunk == 0 ? pr.fix : nullptr, true);
}

// Opts both renormalisation kernels into RN_SMEM bytes of dynamic shared memory (once per
// device).
static int renorm64_prepare() {
    static bool done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return OPB_E_UNSUPPORTED;
    if (!done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k_renorm64, cudaFuncAttributeMaxDynamicSharedMemorySize, RN_SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_renorm64_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, RN_SMEM);
        if (e != cudaSuccess) return (int)e;
        done[dev] = true;
    }
    return OPB_OK;
}

// Batched ELL scatter into zeroed dense E-form matrices: thread per global ELL slot
// (rows of all lattices concatenated; row_off[i] = first global row of lattice i).
__global__ void k_ek_scatter_batched(const BatchLattice *__restrict__ lats, int nlat, long long total_rows, int w,
                                     const int *__restrict__ cols, const double *__restrict__ vals) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total_rows * w) return;
    const long long grow = t / w;
    int lo = 0, hi = nlat - 1;
    while (lo < hi) {  // last lattice with row_off <= grow
        int mid = (lo + hi + 1) >> 1;
        if (lats[mid].row_off <= grow) lo = mid; else hi = mid - 1;
    }
    const BatchLattice &L = lats[lo];
    const int y = (int)(grow - L.row_off);
    const int z = cols[t];
    if (z < 0 || z >= L.d) return;
    L.E[(long long)y * L.d + z] = (float)(L.dt * vals[t]);
}

// Batched payoff splits: G^T[k][z] = (x_z - K_k)^+ for strikes k < nK of lattice i and 0
// for the padding columns nK..ldk-1.
__global__ void k_payoff_batched(const BatchLattice *__restrict__ lats, int nlat, long long total_rows, int nK, int ldk,
                                 const double *__restrict__ x, const double *__restrict__ strikes, int f16) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total_rows * ldk) return;
    const long long grow = t / ldk;
    const int k = (int)(t - grow * ldk);
    int lo = 0, hi = nlat - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (lats[mid].row_off <= grow) lo = mid; else hi = mid - 1;
    }
    const BatchLattice &L = lats[lo];
    const int z = (int)(grow - L.row_off);
    double g = k < nK ? x[grow] - strikes[(long long)lo * nK + k] : 0.0;
    float f = (float)(g > 0.0 ? g : 0.0);
    __nv_bfloat16 h, l;
    split2(f, h, l, f16 ? L.gscale[0] : 0.f);
    L.GThi[(long long)k * L.d + z] = h;
    L.GTlo[(long long)k * L.d + z] = l;
}

// quotes[(i*nmat + m-1)*nK + k] = exp(-r_i T_m) * V_i[y0_i, k]
__global__ void k_quotes_batched(const BatchLattice *__restrict__ lats, int nlat, int nK, int ldk, int m, int nmat,
                                 double *__restrict__ quotes, int f16, int rowfix) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nlat * nK) return;
    int i = t / nK, k = t - i * nK;
    const BatchLattice &L = lats[i];
    double disc = exp(-L.rate * L.period * m);
    if (f16) disc /= (double)L.gscale[0];
    if (rowfix) disc *= L.fix[L.y0].y;  // the deferred normalisation of the priced row
    quotes[((long long)i * nmat + (m - 1)) * nK + k] = disc * (double)L.V[(long long)L.y0 * ldk + k];
}

// Row fixes from FP64 row-sum partials, with the arithmetic of the renormalisation
// kernels' row sums (renorm64_sums): s = sum of the nparts partials in order; E-form inv =
// 1 / (1 + s), P-form inv = 1 / s.
__device__ __forceinline__ double2 row_fix(const double *__restrict__ partial, int d, int nparts, int row, int eform) {
    double s = 0.0;
    const double *q = partial + row;
    int p = 0;
    for (; p + 8 <= nparts; p += 8) {
        double v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) v[j] = q[(long long)(p + j) * d];
#pragma unroll
        for (int j = 0; j < 8; j++) s += v[j];
    }
    for (; p < nparts; p++) s += q[(long long)p * d];
    const double den = nparts == 0 ? 1.0 : (eform ? 1.0 + s : s);
    return make_double2(s, den != 0.0 ? 1.0 / den : 0.0);
}

__global__ void k_rowfix(int d, const double *__restrict__ partial, int nparts, int eform, double2 *__restrict__ fix) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < d) fix[r] = row_fix(partial, d, nparts, r, eform);
}

// Thread per global row of all lattices (rows concatenated); level >= 0: only the lattices
// whose next level is an intermediate squaring (niter > level + 1), E-form; level < 0: all,
// P-form.
__global__ void k_rowfix_batched(const BatchLattice *__restrict__ lats, int nlat, long long total_rows, int parts_div,
                                 int level, int eform) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total_rows) return;
    int lo = 0, hi = nlat - 1;
    while (lo < hi) {  // last lattice with row_off <= t
        int mid = (lo + hi + 1) >> 1;
        if (lats[mid].row_off <= t) lo = mid; else hi = mid - 1;
    }
    const BatchLattice &L = lats[lo];
    if (level >= 0 && L.niter <= level + 1) return;
    const int row = (int)(t - L.row_off);
    L.fix[row] = row_fix(L.partial, L.d, L.d / parts_div, row, eform);
}

// E-form -> P-form: P = I + E (in place), FP32.
__global__ void k_add_identity(int d, float *__restrict__ X) {
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y < d) {
        long long o = (long long)y * d + y;
        X[o] = (float)(1.0 + (double)X[o]);
    }
}

// G[z, k] = (x_z - K_k)^+ (FP32, d x nK row-major) and its split transpose
// G^T hi/lo (nK x d) for the tensor-core pricing GEMM.
// Strike columns nK..ldk-1 (padding to the tensor-core tile width) get zero payoffs.
__global__ void k_payoff(int d, int nK, int ldk, const double *__restrict__ x, const double *__restrict__ K,
                         float *__restrict__ G, __nv_bfloat16 *__restrict__ GThi, __nv_bfloat16 *__restrict__ GTlo,
                         const float *__restrict__ dscale) {
    const float sscale = dscale ? *dscale : 0.f;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)d * ldk) return;
    int z = (int)(t / ldk), k = (int)(t - (long long)z * ldk);
    double g = k < nK ? x[z] - K[k] : 0.0;
    float f = (float)(g > 0.0 ? g : 0.0);
    if (G) G[t] = f;
    if (GThi) {
        __nv_bfloat16 h, l;
        split2(f, h, l, sscale);
        GThi[(long long)k * d + z] = h;
        GTlo[(long long)k * d + z] = l;
    }
}

// FP64 sum of the K-slices' partial products at offset o (slice order).
__device__ __forceinline__ double sum_slices(const float *__restrict__ P, long long o, int nslice, long long stride) {
    double v = (double)P[o];
    for (int sl = 1; sl < nslice; sl++) v += (double)P[o + sl * stride];
    return v;
}

// V64[y, k] = disc * V32[y, k] / gscale (V32 leading dimension ldk >= nK, summed over its
// nslice K-slices; gscale = the payoff split scale, 1 without one); quotes[k] = V64[y0, k].
__global__ void k_discount(int d, int nK, int ldk, const float *__restrict__ V32, double disc,
                           double *__restrict__ V64, int y0, double *__restrict__ quotes, const float *__restrict__ dscale,
                           int nslice, long long slice_stride, const double2 *__restrict__ rowfix) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)d * nK) return;
    int y = (int)(t / nK), k = (int)(t - (long long)y * nK);
    if (dscale) disc /= (double)*dscale;
    double v = disc * sum_slices(V32, (long long)y * ldk + k, nslice, slice_stride);
    if (rowfix) v *= rowfix[y].y;  // the deferred row normalisation of the priced product
    if (V64) V64[t] = v;
    if (quotes && y == y0) quotes[k] = v;
}

// ------------------------------------------------------------------ backward induction
// Bermudan / barrier induction on the period kernel (an extension: the reference exposes
// only the multi-vector GEMV kernels, oplib/opcuda/sgemv3.cu and sgemv4.cu, for it).
// Values V[z, k] are FP64, d x ldk row-major; columns nK..ldk-1 are padding (zero).  The
// exercise value is (x_z - K_k)^+ for calls, (K_k - x_z)^+ for puts; with barrier > 0 a
// state with x_z <= barrier is knocked out (value 0) at every monitoring date.

__device__ __forceinline__ double berm_exercise(double x, double K, int put) {
    const double g = put ? K - x : x - K;
    return g > 0.0 ? g : 0.0;
}

// Power-of-two FP16 split scale of the option values: every value is bounded by the
// largest exercise value (max x - min K for calls, max K - min x for puts).
__global__ void k_berm_scale(int d, const double *__restrict__ x, int nK, const double *__restrict__ K, int put,
                             float *__restrict__ out) {
    __shared__ double s0[256], s1[256];
    double a = -1e300, b = 1e300;  // calls: max x, min K; puts: max K, min x
    for (int i = threadIdx.x; i < d; i += blockDim.x) {
        if (put) b = fmin(b, x[i]);
        else a = fmax(a, x[i]);
    }
    for (int i = threadIdx.x; i < nK; i += blockDim.x) {
        if (put) a = fmax(a, K[i]);
        else b = fmin(b, K[i]);
    }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s0[threadIdx.x] = fmax(s0[threadIdx.x], s0[threadIdx.x + o]);
            s1[threadIdx.x] = fmin(s1[threadIdx.x], s1[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double g = s0[0] - s1[0];
        int e = g > 0.0 ? (int)floor(log2(16384.0 / g)) : 0;
        e = e < 0 ? 0 : (e > 60 ? 60 : e);
        *out = (float)ldexp(1.0, e);
    }
}

// Terminal values V = e(x) (knocked out below the barrier) and the next induction
// product's B operand, K x N row-major: the split parts (Vhi non-null) or FP32 values (Vf).
__global__ void k_berm_init(int d, int nK, int ldk, const double *__restrict__ x, const double *__restrict__ K,
                            int put, double barrier, double *__restrict__ V, __nv_bfloat16 *__restrict__ Vhi,
                            __nv_bfloat16 *__restrict__ Vlo, float *__restrict__ Vf, const float *__restrict__ dscale) {
    const float sscale = dscale ? *dscale : 0.f;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)d * ldk) return;
    const int z = (int)(t / ldk), k = (int)(t - (long long)z * ldk);
    double v = k < nK ? berm_exercise(x[z], K[k], put) : 0.0;
    if (barrier > 0.0 && x[z] <= barrier) v = 0.0;
    V[t] = v;
    if (Vhi) {
        __nv_bfloat16 h, l;
        split2((float)v, h, l, sscale);
        Vhi[t] = h;
        Vlo[t] = l;
    }
    if (Vf) Vf[t] = (float)v;
}

// One induction date from the product C = P1 . V_next (FP32, times the split scale when
// there is one): V = disc * C, then knocked out below the barrier, or (exercise) the larger
// of it and the exercise value; the next product's operand (split parts when Vhi is
// non-null, FP32 values when Vf is) and the quotes at state y0 (quotes non-null).
__global__ void k_berm_step(int d, int nK, int ldk, const float *__restrict__ C, double disc,
                            const double *__restrict__ x, const double *__restrict__ K, int put, double barrier,
                            int exercise, double *__restrict__ V, __nv_bfloat16 *__restrict__ Vhi,
                            __nv_bfloat16 *__restrict__ Vlo, float *__restrict__ Vf, const float *__restrict__ dscale,
                            int y0, double *__restrict__ quotes, int nslice, long long slice_stride) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)d * ldk) return;
    const int z = (int)(t / ldk), k = (int)(t - (long long)z * ldk);
    const float sscale = dscale ? *dscale : 0.f;
    double v = 0.0;
    if (k < nK) {
        v = disc * sum_slices(C, t, nslice, slice_stride);
        if (dscale) v /= (double)sscale;
        if (barrier > 0.0 && x[z] <= barrier) v = 0.0;
        else if (exercise) v = fmax(v, berm_exercise(x[z], K[k], put));
    }
    V[t] = v;
    if (Vhi) {
        __nv_bfloat16 h, l;
        split2((float)v, h, l, sscale);
        Vhi[t] = h;
        Vlo[t] = l;
    }
    if (Vf) Vf[t] = (float)v;
    if (quotes && z == y0 && k < nK) quotes[k] = v;
}

// ------------------------------------------------------------------ host launchers

static inline int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

int launch_ek_ell(int d, int w, const int *cols, const double *vals, double dt, int eform, float *out,
                  cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * (size_t)d * d, s);
    if (e != cudaSuccess) return (int)e;
    if (!eform) k_zero_set_diag<<<blocks_for(d, 256), 256, 0, s>>>(d, out, 1.0f);
    long long n = (long long)d * w;
    if (n > 0) k_ek_scatter_ell<<<blocks_for(n, 256), 256, 0, s>>>(d, w, cols, vals, dt, eform, out, d);
    return (int)cudaGetLastError();
}

int launch_ell_band(int d, int w, const int *cols, int *out, cudaStream_t s) {
    k_ell_band<<<1, 1024, 0, s>>>(d, w, cols, out);
    return (int)cudaGetLastError();
}

int launch_ek_dense(int d, const double *L, double dt, int eform, float *out, cudaStream_t s) {
    long long n = (long long)d * d;
    int b = blocks_for(n, 256);
    int cap = 16 * num_sms();
    k_ek_dense<<<b < cap ? b : cap, 256, 0, s>>>(d, L, dt, eform, out, d);
    return (int)cudaGetLastError();
}

int launch_ek_padded(int d, int dpad, int w, const int *cols, const double *vals, const double *dense, double dt,
                     float *out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * (size_t)dpad * dpad, s);
    if (e != cudaSuccess) return (int)e;
    if (w > 0) {
        long long n = (long long)d * w;
        if (n > 0) k_ek_scatter_ell<<<blocks_for(n, 256), 256, 0, s>>>(d, w, cols, vals, dt, 1, out, dpad);
    } else {
        long long n = (long long)d * d;
        int b = blocks_for(n, 256), cap = 16 * num_sms();
        k_ek_dense<<<b < cap ? b : cap, 256, 0, s>>>(d, dense, dt, 1, out, dpad);
    }
    return (int)cudaGetLastError();
}

int launch_pad_x(int d, int dpad, const double *x, double *xpad, cudaStream_t s) {
    k_pad_x<<<blocks_for(dpad, 256), 256, 0, s>>>(d, dpad, x, xpad);
    return (int)cudaGetLastError();
}

int launch_split(int rows, int cols, const float *X, long long ld, __nv_bfloat16 *Ahi, __nv_bfloat16 *Alo,
                 __nv_bfloat16 *Bhi, __nv_bfloat16 *Blo, long long ldt, cudaStream_t s, float sscale) {
    dim3 g((cols + 31) / 32, (rows + 31) / 32);
    k_split_tr<<<g, 256, 0, s>>>(rows, cols, X, ld, Ahi, Alo, Bhi, Blo, ldt, sscale);
    return (int)cudaGetLastError();
}

int launch_rowsum(int d, const float *X, double *partial, cudaStream_t s) {
    k_rowsum<<<d, 256, 0, s>>>(d, X, partial);
    return (int)cudaGetLastError();
}

int launch_renorm(int d, float *X, const double *partial, int nparts, int eform, __nv_bfloat16 *Ahi,
                  __nv_bfloat16 *Alo, __nv_bfloat16 *Bhi, __nv_bfloat16 *Blo, cudaStream_t s, float sscale,
                  int write_x, double2 *fix) {
    if (d % 64 == 0 && (Ahi != nullptr) == (Alo != nullptr)) {
        if (int r = renorm64_prepare()) return r;
        k_renorm64<<<renorm64_grid(d), 256, RN_SMEM, s>>>(d, X, partial, nparts, eform ? 0 : 2, Ahi, Alo, Bhi, Blo,
                                                          sscale, write_x, eform ? fix : nullptr);
        return (int)cudaGetLastError();
    }
    if (!write_x || fix) return OPB_E_UNSUPPORTED;
    dim3 g((d + 31) / 32, (d + 31) / 32);
    k_renorm<<<g, 256, 0, s>>>(d, X, partial, nparts, eform, Ahi, Alo, Bhi, Blo, sscale);
    return (int)cudaGetLastError();
}

// E-form renorm whose output is P = I + E_new, with its splits row-major into both A and B
// (the last squaring level: P1 is the A of the first chain product and of pricing, and
// the B of every chain product).
int launch_renorm_to_p(int d, float *X, const double *partial, int nparts, __nv_bfloat16 *Ahi, __nv_bfloat16 *Alo,
                       __nv_bfloat16 *Bhi, __nv_bfloat16 *Blo, cudaStream_t s, float sscale) {
    if (d % 64) return OPB_E_UNSUPPORTED;
    if (int r = renorm64_prepare()) return r;
    k_renorm64<<<renorm64_grid(d), 256, RN_SMEM, s>>>(d, X, partial, nparts, 1, Ahi, Alo, Bhi, Blo, sscale, 1,
                                                      nullptr, 1);
    return (int)cudaGetLastError();
}

int launch_renorm_batched(const RenormProblem *probs, const uint32_t *work, int nwork, int parts_div, cudaStream_t s,
                          float sscale) {
    if (nwork <= 0) return OPB_OK;
    if (int r = renorm64_prepare()) return r;
    k_renorm64_batched<<<nwork, 256, RN_SMEM, s>>>(probs, work, parts_div, sscale);
    return (int)cudaGetLastError();
}

// Thread per padded ELL slot (row-major rows of all lattices, w slots each).
__global__ void k_pad_batched(const BatchLattice *__restrict__ lats, int nlat, long long total_rows, int w,
                              const int *__restrict__ cols_src, const double *__restrict__ vals_src,
                              const double *__restrict__ x_src, int *__restrict__ cols, double *__restrict__ vals,
                              double *__restrict__ x) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total_rows * w) return;
    const long long grow = t / w;
    const int k = (int)(t - grow * w);
    int lo = 0, hi = nlat - 1;
    while (lo < hi) {  // last lattice with row_off <= grow
        int mid = (lo + hi + 1) >> 1;
        if (lats[mid].row_off <= grow) lo = mid; else hi = mid - 1;
    }
    const BatchLattice &L = lats[lo];
    const int y = (int)(grow - L.row_off);
    if (y < L.d_src) {
        const long long src = (L.src_off + y) * w + k;
        cols[t] = cols_src[src];
        vals[t] = vals_src[src];
    } else {
        cols[t] = -1;
        vals[t] = 0.0;
    }
    if (k == 0) x[grow] = x_src[L.src_off + (y < L.d_src ? y : L.d_src - 1)];
}

int launch_pad_batched(const BatchLattice *lats, int nlat, long long total_rows, int w, const int *cols_src,
                       const double *vals_src, const double *x_src, int *cols, double *vals, double *x,
                       cudaStream_t s) {
    const long long n = total_rows * w;
    if (n <= 0) return OPB_OK;
    k_pad_batched<<<(int)((n + 255) / 256), 256, 0, s>>>(lats, nlat, total_rows, w, cols_src, vals_src, x_src, cols,
                                                          vals, x);
    return (int)cudaGetLastError();
}

int launch_ek_batched(const BatchLattice *lats, int nlat, long long total_rows, int w, const int *cols,
                      const double *vals, cudaStream_t s) {
    long long n = total_rows * w;
    if (n <= 0) return OPB_OK;
    k_ek_scatter_batched<<<(int)((n + 255) / 256), 256, 0, s>>>(lats, nlat, total_rows, w, cols, vals);
    return (int)cudaGetLastError();
}

// Per-lattice FP16 payoff scales (one block per lattice) into BatchLattice.gscale.
__global__ void k_payoff_scale_batched(const BatchLattice *__restrict__ lats, const double *__restrict__ x, int nK,
                                       const double *__restrict__ strikes) {
    const BatchLattice &L = lats[blockIdx.x];
    __shared__ double sx[256], sk[256];
    double mx = -1e300, mk = 1e300;
    for (int i = threadIdx.x; i < L.d; i += blockDim.x) mx = fmax(mx, x[L.row_off + i]);
    for (int i = threadIdx.x; i < nK; i += blockDim.x) mk = fmin(mk, strikes[(long long)blockIdx.x * nK + i]);
    sx[threadIdx.x] = mx;
    sk[threadIdx.x] = mk;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sx[threadIdx.x] = fmax(sx[threadIdx.x], sx[threadIdx.x + o]);
            sk[threadIdx.x] = fmin(sk[threadIdx.x], sk[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double g = sx[0] - sk[0];
        int e = g > 0.0 ? (int)floor(log2(16384.0 / g)) : 0;
        e = e < 0 ? 0 : (e > 60 ? 60 : e);
        L.gscale[0] = (float)ldexp(1.0, e);
    }
}

// ---- batched backward induction: lattice i's values live at rows row_off_i .. + d_i of
// the concatenated row space; V_i = Vd_i (FP64, d x ldk), its split parts in GThi/GTlo
// read as d x ldk row-major (the K x N operand of the induction product)

__device__ __forceinline__ int lattice_of_row(const BatchLattice *__restrict__ lats, int nlat, long long grow) {
    int lo = 0, hi = nlat - 1;
    while (lo < hi) {  // last lattice with row_off <= grow
        int mid = (lo + hi + 1) >> 1;
        if (lats[mid].row_off <= grow) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Per-lattice FP16 split scales of the option values (one block per lattice): a power of
// two from the largest exercise value, as k_berm_scale.
__global__ void k_berm_scale_batched(const BatchLattice *__restrict__ lats, const double *__restrict__ x, int nK,
                                     const double *__restrict__ strikes, int put) {
    const BatchLattice &L = lats[blockIdx.x];
    __shared__ double s0[256], s1[256];
    double a = -1e300, b = 1e300;  // calls: max x, min K; puts: max K, min x
    for (int i = threadIdx.x; i < L.d; i += blockDim.x) {
        if (put) b = fmin(b, x[L.row_off + i]);
        else a = fmax(a, x[L.row_off + i]);
    }
    for (int i = threadIdx.x; i < nK; i += blockDim.x) {
        const double k = strikes[(long long)blockIdx.x * nK + i];
        if (put) a = fmax(a, k);
        else b = fmin(b, k);
    }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s0[threadIdx.x] = fmax(s0[threadIdx.x], s0[threadIdx.x + o]);
            s1[threadIdx.x] = fmin(s1[threadIdx.x], s1[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double g = s0[0] - s1[0];
        int e = g > 0.0 ? (int)floor(log2(16384.0 / g)) : 0;
        e = e < 0 ? 0 : (e > 60 ? 60 : e);
        L.gscale[0] = (float)ldexp(1.0, e);
    }
}

// Terminal values of every lattice (as k_berm_init).
__global__ void k_berm_init_batched(const BatchLattice *__restrict__ lats, int nlat, long long total_rows, int nK,
                                    int ldk, const double *__restrict__ x, const double *__restrict__ strikes, int put,
                                    double barrier, int f16) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total_rows * ldk) return;
    const long long grow = t / ldk;
    const int k = (int)(t - grow * ldk);
    const int i = lattice_of_row(lats, nlat, grow);
    const BatchLattice &L = lats[i];
    const long long o = (grow - L.row_off) * ldk + k;
    double v = k < nK ? berm_exercise(x[grow], strikes[(long long)i * nK + k], put) : 0.0;
    if (barrier > 0.0 && x[grow] <= barrier) v = 0.0;
    L.Vd[o] = v;
    __nv_bfloat16 h, l;
    split2((float)v, h, l, f16 ? L.gscale[0] : 0.f);
    L.GThi[o] = h;
    L.GTlo[o] = l;
}

// One induction date of every lattice from its product C_i = P1_i . V_i in L.V (as
// k_berm_step); at the last date (t = 0) quotes[i*nK + k] = V_i[y0_i, k] and no parts.
__global__ void k_berm_step_batched(const BatchLattice *__restrict__ lats, int nlat, long long total_rows, int nK,
                                    int ldk, const double *__restrict__ x, const double *__restrict__ strikes,
                                    int put, double barrier, int exercise, int last, int f16,
                                    double *__restrict__ quotes) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total_rows * ldk) return;
    const long long grow = t / ldk;
    const int k = (int)(t - grow * ldk);
    const int i = lattice_of_row(lats, nlat, grow);
    const BatchLattice &L = lats[i];
    const int z = (int)(grow - L.row_off);
    const long long o = (long long)z * ldk + k;
    const float sscale = f16 ? L.gscale[0] : 0.f;
    double v = 0.0;
    if (k < nK) {
        v = exp(-L.rate * L.period) * (double)L.V[o];
        if (f16) v /= (double)sscale;
        if (!last) {
            if (barrier > 0.0 && x[grow] <= barrier) v = 0.0;
            else if (exercise) v = fmax(v, berm_exercise(x[grow], strikes[(long long)i * nK + k], put));
        }
    }
    L.Vd[o] = v;
    if (!last) {
        __nv_bfloat16 h, l;
        split2((float)v, h, l, sscale);
        L.GThi[o] = h;
        L.GTlo[o] = l;
    } else if (z == L.y0 && k < nK) {
        quotes[(long long)i * nK + k] = v;
    }
}

int launch_berm_batched_init(const BatchLattice *lats, int nlat, long long total_rows, int nK, int ldk,
                             const double *x, const double *strikes, int put, double barrier, int f16,
                             cudaStream_t s) {
    const long long n = total_rows * ldk;
    if (n <= 0) return OPB_OK;
    if (f16) k_berm_scale_batched<<<nlat, 256, 0, s>>>(lats, x, nK, strikes, put);
    k_berm_init_batched<<<blocks_for(n, 256), 256, 0, s>>>(lats, nlat, total_rows, nK, ldk, x, strikes, put, barrier,
                                                          f16);
    return (int)cudaGetLastError();
}

int launch_berm_batched_step(const BatchLattice *lats, int nlat, long long total_rows, int nK, int ldk,
                             const double *x, const double *strikes, int put, double barrier, int exercise,
                             int last, int f16, double *quotes, cudaStream_t s) {
    const long long n = total_rows * ldk;
    if (n <= 0) return OPB_OK;
    k_berm_step_batched<<<blocks_for(n, 256), 256, 0, s>>>(lats, nlat, total_rows, nK, ldk, x, strikes, put, barrier,
                                                          exercise, last, f16, quotes);
    return (int)cudaGetLastError();
}

int launch_payoff_batched(const BatchLattice *lats, int nlat, long long total_rows, int nK, int ldk, const double *x,
                          const double *strikes, cudaStream_t s, int f16) {
    long long n = total_rows * ldk;
    if (n <= 0) return OPB_OK;
    if (f16) k_payoff_scale_batched<<<nlat, 256, 0, s>>>(lats, x, nK, strikes);
    k_payoff_batched<<<(int)((n + 255) / 256), 256, 0, s>>>(lats, nlat, total_rows, nK, ldk, x, strikes, f16);
    return (int)cudaGetLastError();
}

int launch_quotes_batched(const BatchLattice *lats, int nlat, int nK, int ldk, int m, int nmat, double *quotes,
                          cudaStream_t s, int f16, int rowfix) {
    int n = nlat * nK;
    k_quotes_batched<<<(n + 255) / 256, 256, 0, s>>>(lats, nlat, nK, ldk, m, nmat, quotes, f16, rowfix);
    return (int)cudaGetLastError();
}

int launch_rowfix(int d, const double *partial, int nparts, int eform, double2 *fix, cudaStream_t s) {
    k_rowfix<<<blocks_for(d, 256), 256, 0, s>>>(d, partial, nparts, eform, fix);
    return (int)cudaGetLastError();
}

int launch_rowfix_batched(const BatchLattice *lats, int nlat, long long total_rows, int parts_div, int level,
                          int eform, cudaStream_t s) {
    if (parts_div <= 0) return OPB_E_ARG;
    k_rowfix_batched<<<blocks_for(total_rows, 256), 256, 0, s>>>(lats, nlat, total_rows, parts_div, level, eform);
    return (int)cudaGetLastError();
}

int launch_add_identity(int d, float *X, cudaStream_t s) {
    k_add_identity<<<blocks_for(d, 256), 256, 0, s>>>(d, X);
    return (int)cudaGetLastError();
}

// Power-of-two scale for FP16 payoff parts: 2^floor(log2(16384 / max payoff)), at least 1,
// with max payoff = max(x) - min(K) (one block).
__global__ void k_payoff_scale(int d, const double *__restrict__ x, int nK, const double *__restrict__ K,
                               float *__restrict__ out) {
    __shared__ double sx[256], sk[256];
    double mx = -1e300, mk = 1e300;
    for (int i = threadIdx.x; i < d; i += blockDim.x) mx = fmax(mx, x[i]);
    for (int i = threadIdx.x; i < nK; i += blockDim.x) mk = fmin(mk, K[i]);
    sx[threadIdx.x] = mx;
    sk[threadIdx.x] = mk;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sx[threadIdx.x] = fmax(sx[threadIdx.x], sx[threadIdx.x + o]);
            sk[threadIdx.x] = fmin(sk[threadIdx.x], sk[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double g = sx[0] - sk[0];
        int e = g > 0.0 ? (int)floor(log2(16384.0 / g)) : 0;
        e = e < 0 ? 0 : (e > 60 ? 60 : e);
        *out = (float)ldexp(1.0, e);
    }
}

int launch_payoff_scale(int d, const double *x, int nK, const double *K, float *out, cudaStream_t s) {
    k_payoff_scale<<<1, 256, 0, s>>>(d, x, nK, K, out);
    return (int)cudaGetLastError();
}

int launch_payoff(int d, int nK, int ldk, const double *x, const double *K, float *G, __nv_bfloat16 *GThi,
                  __nv_bfloat16 *GTlo, cudaStream_t s, const float *dscale) {
    long long n = (long long)d * ldk;
    k_payoff<<<blocks_for(n, 256), 256, 0, s>>>(d, nK, ldk, x, K, G, GThi, GTlo, dscale);
    return (int)cudaGetLastError();
}

int launch_berm_scale(int d, const double *x, int nK, const double *K, int put, float *out, cudaStream_t s) {
    k_berm_scale<<<1, 256, 0, s>>>(d, x, nK, K, put, out);
    return (int)cudaGetLastError();
}

int launch_berm_init(int d, int nK, int ldk, const double *x, const double *K, int put, double barrier, double *V,
                     __nv_bfloat16 *Vhi, __nv_bfloat16 *Vlo, float *Vf, const float *dscale, cudaStream_t s) {
    const long long n = (long long)d * ldk;
    k_berm_init<<<blocks_for(n, 256), 256, 0, s>>>(d, nK, ldk, x, K, put, barrier, V, Vhi, Vlo, Vf, dscale);
    return (int)cudaGetLastError();
}

int launch_berm_step(int d, int nK, int ldk, const float *C, double disc, const double *x, const double *K, int put,
                     double barrier, int exercise, double *V, __nv_bfloat16 *Vhi, __nv_bfloat16 *Vlo, float *Vf,
                     const float *dscale, int y0, double *quotes, cudaStream_t s, int nslice,
                     long long slice_stride) {
    const long long n = (long long)d * ldk;
    k_berm_step<<<blocks_for(n, 256), 256, 0, s>>>(d, nK, ldk, C, disc, x, K, put, barrier, exercise, V, Vhi, Vlo,
                                                   Vf, dscale, y0, quotes, nslice > 1 ? nslice : 1, slice_stride);
    return (int)cudaGetLastError();
}

int launch_discount(int d, int nK, int ldk, const float *V32, double disc, double *V64, int y0, double *quotes,
                    cudaStream_t s, const float *dscale, int nslice, long long slice_stride, const double2 *rowfix) {
    long long n = (long long)d * nK;
    k_discount<<<blocks_for(n, 256), 256, 0, s>>>(d, nK, ldk, V32, disc, V64, y0, quotes, dscale,
                                                  nslice > 1 ? nslice : 1, slice_stride, rowfix);
    return (int)cudaGetLastError();
}

}  // namespace opb

// ------------------------------------------------------------------ reference ek entry points

// U = I + dt*gen for a column-major d x d FP32 generator (oplib/opcuda/sek.cu:40-59,106-115),
// in the reference kernels' FP32 arithmetic so that the drop-ins reproduce them bit for bit:
// the numerator id + dt*gen is one fused multiply-add (nvcc contracts the reference's
// expression), the discount denominator 1 + dt*r[y1] (sek.cu:78) or 1 + (dt*r[y1])*lambda
// (sek.cu:100) rounds the inner product and fuses the last one, and the quotient is the
// IEEE FP32 division.  The lattice path builds its U0 in FP64 elsewhere; this is the drop-in.
__global__ void k_sek(int d, const float *__restrict__ gen, float dt, float *__restrict__ out,
                      const float *__restrict__ r, const float *__restrict__ lambda) {
    long long n = (long long)d * d;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int y1 = (int)(t % d), y2 = (int)(t / d);  // column-major: t = y1 + d*y2
        float v = __fmaf_rn(dt, gen[t], y1 == y2 ? 1.f : 0.f);
        if (r) {
            float den = lambda ? __fmaf_rn(__fmul_rn(dt, r[y1]), lambda[0], 1.f) : __fmaf_rn(dt, r[y1], 1.f);
            v = __fdiv_rn(v, den);
        }
        out[t] = v;
    }
}

static int sek_common(int d, uint64_t gen, float dt, uint64_t tpk, uint64_t r, uint64_t lambda) {
    OPB_REQUIRE(d >= 0, OPB_E_ARG);
    if (d == 0) return opb::set_status(OPB_OK);
    OPB_REQUIRE(gen != 0 && tpk != 0, OPB_E_NULL);
    long long n = (long long)d * d;
    int b = (int)((n + 255) / 256);
    int cap = 16 * opb::num_sms();
    k_sek<<<b < cap ? b : cap, 256, 0, opb::stream()>>>(d, reinterpret_cast<const float *>(gen), dt,
                                                         reinterpret_cast<float *>(tpk),
                                                         reinterpret_cast<const float *>(r),
                                                         reinterpret_cast<const float *>(lambda));
    return opb::launch_check();
}

OPB_API int opcuda_sek(int d, uint64_t genPtr, float dt, uint64_t tpkerPtr) {
    return sek_common(d, genPtr, dt, tpkerPtr, 0, 0);
}

OPB_API int opcuda_sekd(int d, uint64_t genPtr, float dt, uint64_t tpkerPtr, uint64_t rPtr) {
    OPB_REQUIRE(rPtr != 0, OPB_E_NULL);
    return sek_common(d, genPtr, dt, tpkerPtr, rPtr, 0);
}

OPB_API int opcuda_sekd_lambda(int d, uint64_t genPtr, float dt, uint64_t tpkerPtr, uint64_t rPtr,
                               uint64_t lambdaPtr) {
    OPB_REQUIRE(rPtr != 0 && lambdaPtr != 0, OPB_E_NULL);
    return sek_common(d, genPtr, dt, tpkerPtr, rPtr, lambdaPtr);
}

// Standalone FP64 row renormalisation (+ optional 16-bit splits) of a source-major d x d
// FP32 matrix from row-sum partials partial[p * d + y], p < nparts.  mode: 0 = E-form,
// 1 = E-form in / P-form out, 2 = P-form; f16: 0 BF16 parts, 1 FP16 parts of 2^15-scaled
// values.  d % 64 == 0.
OPB_API int opb_renorm_rows(int d, float *X, const double *partial, int nparts, int mode, void *Ahi, void *Alo,
                            void *Bhi, void *Blo, int f16) {
    OPB_REQUIRE(d > 0 && d % 64 == 0 && nparts >= 0 && mode >= 0 && mode <= 2, OPB_E_ARG);
    OPB_REQUIRE(X && (nparts == 0 || partial), OPB_E_NULL);
    OPB_REQUIRE((Ahi != nullptr) == (Alo != nullptr) && (Bhi != nullptr) == (Blo != nullptr), OPB_E_NULL);
    OPB_REQUIRE(opb::aligned(X, 16) && (!Ahi || (opb::aligned(Ahi, 8) && opb::aligned(Alo, 8))) &&
                    (!Bhi || (opb::aligned(Bhi, 8) && opb::aligned(Blo, 8))),
                OPB_E_ALIGN);
    if (int r = opb::renorm64_prepare()) return opb::set_status(r);
    opb::k_renorm64<<<opb::renorm64_grid(d), 256, opb::RN_SMEM, opb::stream()>>>(
        d, X, partial, nparts, mode, reinterpret_cast<__nv_bfloat16 *>(Ahi), reinterpret_cast<__nv_bfloat16 *>(Alo),
        mode == 2 ? nullptr : reinterpret_cast<__nv_bfloat16 *>(Bhi),
        mode == 2 ? nullptr : reinterpret_cast<__nv_bfloat16 *>(Blo), f16 ? 32768.f : 0.f);
    return opb::launch_check();
}
