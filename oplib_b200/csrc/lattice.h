// Internal launcher declarations shared by the library's translation units.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace opb {

// Two-part split of an FP32 value into 16-bit storage.  sscale == 0: BF16 parts,
// hi = bf16(f), lo = bf16(f - hi), with an absolute floor: |f| < 2^-40 gives hi = lo = 0
// and |f| < 2^-30 gives lo = 0 (BF16 keeps FP32's exponent range, so without the floor the
// far tails of a transition matrix, 1e-38 .. 1e-9, stay live bit patterns; FP16 parts of
// 2^15-scaled values drop them by underflow).  The floor moves an entry by at most 2^-40,
// or by its lo part, below 2^-39, so a product row over d <= 32768 entries of size <= 1 moves
// by under 2^-24 / 2^-25 in the worst case, and by far less when the
// discarded parts carry random signs.  sscale > 0 (a power of two): FP16 parts of f*sscale,
// hi = fp16(f*s), lo = fp16(f*s - hi) -- 11 + 11 significant bits instead of 8 + 8; the
// GEMM removes the scale through alpha.  The differences are exact in FP32.
constexpr float kSplitZeroBelow = 0x1p-40f, kSplitNoLoBelow = 0x1p-30f;

__device__ __forceinline__ void split2(float f, __nv_bfloat16 &hi, __nv_bfloat16 &lo, float sscale = 0.f) {
    if (sscale == 0.f) {
        const float a = fabsf(f);
        hi = __float2bfloat16_rn(a < kSplitZeroBelow ? 0.f : f);
        lo = __float2bfloat16_rn(a < kSplitNoLoBelow ? 0.f : f - __bfloat162float(hi));
    } else {
        const float fs = f * sscale;
        const __half h = __float2half_rn(fs);
        const __half l = __float2half_rn(fs - __half2float(h));
        hi = __ushort_as_bfloat16(__half_as_ushort(h));
        lo = __ushort_as_bfloat16(__half_as_ushort(l));
    }
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// split2 of two values at once with the paired conversions, the parts packed (a in the low
// half): the same parts as split2 on each.
__device__ __forceinline__ void split2x2(float a, float b, uint32_t &hi, uint32_t &lo, float sscale = 0.f) {
    if (sscale == 0.f) {
        const float aa = fabsf(a), ab = fabsf(b);
        const __nv_bfloat162 h =
            __floats2bfloat162_rn(aa < kSplitZeroBelow ? 0.f : a, ab < kSplitZeroBelow ? 0.f : b);
        const float2 hf = __bfloat1622float2(h);
        const __nv_bfloat162 l =
            __floats2bfloat162_rn(aa < kSplitNoLoBelow ? 0.f : a - hf.x, ab < kSplitNoLoBelow ? 0.f : b - hf.y);
        hi = *reinterpret_cast<const uint32_t *>(&h);
        lo = *reinterpret_cast<const uint32_t *>(&l);
    } else {
        const float as = a * sscale, bs = b * sscale;
        const __half2 h = __floats2half2_rn(as, bs);
        const float2 hf = __half22float2(h);
        const __half2 l = __floats2half2_rn(as - hf.x, bs - hf.y);
        hi = *reinterpret_cast<const uint32_t *>(&h);
        lo = *reinterpret_cast<const uint32_t *>(&l);
    }
}

// gemm_simt.cu
int sgemm_rm(int M, int N, int K, float alpha, const float *A, int lda, const float *B, int ldb, float beta,
             float *C, int ldc, cudaStream_t s);
int sgemm_rm_t(bool ta, bool tb, int M, int N, int K, float alpha, const float *A, int lda, const float *B, int ldb,
               float beta, float *C, int ldc, cudaStream_t s);
// Strided-batch form: batch entries z use A + z*sA, B + z*sB, C + z*sC (row-major roles as
// in sgemm_rm_t); grid (N/128, M/128, batch).
int sgemm_rm_strided(bool ta, bool tb, int M, int N, int K, float alpha, const float *A, int lda, long long sA,
                     const float *B, int ldb, long long sB, float beta, float *C, int ldc, long long sC, int batch,
                     cudaStream_t s);

// lattice_kernels.cu
// *out = max |col - row| over the ELL entries (the generator's half-bandwidth)
int launch_ell_band(int d, int w, const int *cols, int *out, cudaStream_t s);
int launch_ek_ell(int d, int w, const int *cols, const double *vals, double dt, int eform, float *out,
                  cudaStream_t s);
// E0 = dt L (E-form) of a d-state generator (ELL when w > 0, else dense) into a dpad x dpad
// matrix whose states d..dpad-1 are absorbing (zero rows and columns)
int launch_ek_padded(int d, int dpad, int w, const int *cols, const double *vals, const double *dense, double dt,
                     float *out, cudaStream_t s);
// xpad[i] = x[min(i, d - 1)], i < dpad
int launch_pad_x(int d, int dpad, const double *x, double *xpad, cudaStream_t s);
int launch_ek_dense(int d, const double *L, double dt, int eform, float *out, cudaStream_t s);
int launch_split(int rows, int cols, const float *X, long long ld, __nv_bfloat16 *Ahi, __nv_bfloat16 *Alo,
                 __nv_bfloat16 *Bhi, __nv_bfloat16 *Blo, long long ldt, cudaStream_t s, float sscale = 0.f);
int launch_rowsum(int d, const float *X, double *partial, cudaStream_t s);
// write_x = 0 leaves X as it is (only the splits are written; d % 64 == 0); fix (optional,
// E-form) receives the per-row (s, inv) that a following product applies to X as its Cin.
int launch_renorm(int d, float *X, const double *partial, int nparts, int eform, __nv_bfloat16 *Ahi,
                  __nv_bfloat16 *Alo, __nv_bfloat16 *Bhi, __nv_bfloat16 *Blo, cudaStream_t s, float sscale = 0.f,
                  int write_x = 1, double2 *fix = nullptr);
int launch_add_identity(int d, float *X, cudaStream_t s);
// dscale (device, optional): FP16 payoff split scale from launch_payoff_scale
int launch_payoff_scale(int d, const double *x, int nK, const double *K, float *out, cudaStream_t s);
int launch_payoff(int d, int nK, int ldk, const double *x, const double *K, float *G, __nv_bfloat16 *GThi,
                  __nv_bfloat16 *GTlo, cudaStream_t s, const float *dscale = nullptr);
// V32 may hold nslice K-slices' partial products slice_stride elements apart, summed in
// FP64 in slice order
// rowfix (optional): per-row (s, inv) of a P-form product whose normalisation was deferred;
// row y of V is multiplied by inv_y
int launch_discount(int d, int nK, int ldk, const float *V32, double disc, double *V64, int y0, double *quotes,
                    cudaStream_t s, const float *dscale = nullptr, int nslice = 1, long long slice_stride = 0,
                    const double2 *rowfix = nullptr);
// fix[row] = (s, inv) from a product's FP64 row-sum partials (nparts per row, partial[p*d +
// row]): s = the row sum; inv = 1 / (1 + s) for an E-form product (eform), 1 / s for a
// P-form one (the arithmetic of the renormalisation kernels' row sums)
int launch_rowfix(int d, const double *partial, int nparts, int eform, double2 *fix, cudaStream_t s);

// Batched lattice tables (device memory).
struct BatchLattice {
    int d, y0;
    long long row_off;    // first global row (rows of all lattices concatenated)
    double dt, rate, period;
    float *E;             // d x d FP32 (E-form, then P1)
    float *Pa;            // d x d FP32 chain product
    float *V;             // d x ldk FP32 pricing result
    __nv_bfloat16 *GThi, *GTlo;  // ldk x d payoff splits (or, in the induction, d x ldk value splits)
    float *gscale;        // device scalar: FP16 payoff split scale
    double *Vd;           // d x ldk FP64 option values of the backward induction
    int niter;            // squaring levels
    const double *partial;  // the last product's FP64 row-sum partials (partial[p*d + row])
    double2 *fix;         // per-row (s, inv) of the last product's deferred normalisation
    // split modes, lattices of a size off the 128 grid: d above is the padded size (its states
    // d_src..d-1 absorbing), d_src the caller's, src_off the lattice's first row in the
    // caller's generator and spot arrays
    int d_src;
    long long src_off;
};
// Padded copies of the caller's ELL generator (w slots per row; padding rows get column -1)
// and spot values (padding rows repeat the last state's) in the plan's padded row space.
int launch_pad_batched(const BatchLattice *lats, int nlat, long long total_rows, int w, const int *cols_src,
                       const double *vals_src, const double *x_src, int *cols, double *vals, double *x,
                       cudaStream_t s);
// Renormalisation staging: tiles in flight per block, and column tiles per batched work
// item (a batched item renormalises the tiles chunk, chunk + renorm_chunks(d), ... of one
// 64-row strip).
constexpr int RN_RING = 3;
constexpr int RN_TILES = 8;
__host__ __device__ inline int renorm_chunks(int d) { return (d / 64 + RN_TILES - 1) / RN_TILES; }
struct RenormProblem {
    int d, pad;
    float *X;  // read only
    const double *partial;
    __nv_bfloat16 *Ahi, *Alo, *Bhi, *Blo;
    double2 *fix;  // mode-0 items: per-row (s, inv) for the next product's Cin (cin_fix)
};
// Batched backward induction over all lattices of a sweep (lattice_kernels.cu): per-lattice
// split scales, terminal values and one induction date (quotes [nlat][nK] at the last)
int launch_berm_batched_init(const BatchLattice *lats, int nlat, long long total_rows, int nK, int ldk,
                             const double *x, const double *strikes, int put, double barrier, int f16,
                             cudaStream_t s);
int launch_berm_batched_step(const BatchLattice *lats, int nlat, long long total_rows, int nK, int ldk,
                             const double *x, const double *strikes, int put, double barrier, int exercise,
                             int last, int f16, double *quotes, cudaStream_t s);
// Bermudan / barrier backward induction (lattice_kernels.cu)
int launch_berm_scale(int d, const double *x, int nK, const double *K, int put, float *out, cudaStream_t s);
int launch_berm_init(int d, int nK, int ldk, const double *x, const double *K, int put, double barrier, double *V,
                     __nv_bfloat16 *Vhi, __nv_bfloat16 *Vlo, float *Vf, const float *dscale, cudaStream_t s);
int launch_berm_step(int d, int nK, int ldk, const float *C, double disc, const double *x, const double *K, int put,
                     double barrier, int exercise, double *V, __nv_bfloat16 *Vhi, __nv_bfloat16 *Vlo, float *Vf,
                     const float *dscale, int y0, double *quotes, cudaStream_t s, int nslice = 1,
                     long long slice_stride = 0);
int launch_renorm_to_p(int d, float *X, const double *partial, int nparts, __nv_bfloat16 *Ahi, __nv_bfloat16 *Alo,
                       __nv_bfloat16 *Bhi, __nv_bfloat16 *Blo, cudaStream_t s, float sscale = 0.f);
// work items: problem << 16 | mode << 14 | strip << 7 | chunk (see renorm_chunks)
int launch_renorm_batched(const RenormProblem *probs, const uint32_t *work, int nwork, int parts_div, cudaStream_t s,
                          float sscale = 0.f);
int launch_ek_batched(const BatchLattice *lats, int nlat, long long total_rows, int w, const int *cols,
                      const double *vals, cudaStream_t s);
int launch_payoff_batched(const BatchLattice *lats, int nlat, long long total_rows, int nK, int ldk, const double *x,
                          const double *strikes, cudaStream_t s, int f16 = 0);
// rowfix: scale each lattice's V row y0 by its fix (P-form products with deferred normalisation)
int launch_quotes_batched(const BatchLattice *lats, int nlat, int nK, int ldk, int m, int nmat, double *quotes,
                          cudaStream_t s, int f16 = 0, int rowfix = 0);
// BatchLattice::fix from BatchLattice::partial (parts_div columns per partial) for every
// lattice still squaring after `level` (eform, niter > level + 1), or for all (P-form,
// level < 0)
int launch_rowfix_batched(const BatchLattice *lats, int nlat, long long total_rows, int parts_div, int level,
                          int eform, cudaStream_t s);

// gemm_tc.cu -- split-BF16 tensor-core GEMM.
//   C[M,N] = alpha * (Ahi.Bhi^T + Ahi.Blo^T + Alo.Bhi^T) + beta * Cin[M,N]
// A* are M x K row-major (K-major), B* are N x K row-major (the K-major form of the
// K x N right operand).  If rowsum != nullptr the epilogue writes FP64 partial row sums
// of the stored C values: rowsum[(n-tile) * M + row].
struct TcGemmArgs {
    int M, N, K;
    const __nv_bfloat16 *Ahi, *Alo, *Bhi, *Blo;
    long long lda, ldb;   // elements
    float *C;
    long long ldc;
    const float *Cin;     // may alias C
    float alpha, beta;
    double *rowsum;       // optional
    int f16;              // 1: FP16 parts (kind::f16 with F16 inputs), 0: BF16 parts
    // optional, with Cin: per-row (s, inv) of a deferred E-form renormalisation; the
    // epilogue reads Cin[r][c] as (float)((Cin[r][c] - (r == c ? s : 0)) * inv)
    const double2 *cin_fix;
    int b_kn;  // 1: B parts stored K x N row-major (ldb >= N; read as an MN-major operand)
    // > 1: the product runs as ksplit K-slices written to C + s * c_slice (s < ksplit) for the
    // caller to sum; needs no Cin and no rowsum, (K / 64) % ksplit == 0, c_slice >= M * ldc
    int ksplit;
    long long c_slice;
    // optional (device int h0 > 0): A and B are both zero outside the band |row - col| <=
    // h0 << level.  With band_skip, each output tile issues only the K-blocks within reach
    // of its rows and columns, in whole accumulation chunks (bit-identical to the full
    // product), and a tile that no K-block reaches writes only its zero row-sum partials:
    // such tiles must be zero in C already, with C == Cin.  Single products without K-slices.
    const int *band;
    int level;
    int band_skip;
    // 1: also issue the fourth split product lo.lo (split modes); where the band is known,
    // only while the operands are banded (2 * (h0 << level) < K)
    int lolo;
    // how cin_fix applies (OPB_FIX_*; 0 = OPB_FIX_CIN when cin_fix is given)
    int fixmode;
    // optional: the epilogue also stores the two 16-bit parts (split2 with sscale) of every
    // value it stores, row-major with leading dimension ldc; C may then be null (parts only)
    __nv_bfloat16 *Shi, *Slo;
    float sscale;
};
// Deferred normalisation in the epilogue, with cin_fix[i] = (s_i, inv_i) of the operand
// rows (E-form: the row sums s of P = I + E' are 1 + s, inv = 1 / (1 + s); P-form: s the row
// sum, inv = 1 / s):
//   OPB_FIX_CIN     Cin is read as (Cin - s_i [i == j]) * inv_i (the operands are normalised)
//   OPB_FIX_SQUARE  the operands are the parts of the unnormalised E' (= Cin), E = D (E' - S)
//                   with D = diag(inv), S = diag(s); the output is
//                   D [alpha acc + (beta - s_i - s_j) E'_ij + (s_i^2 - beta s_i) [i == j]],
//                   i.e. alpha E.E + beta E with the D between the two factors left out (a
//                   relative change of |s| <= 1e-5 in the product, below its split rounding)
//   OPB_FIX_ROWSCALE the A operand is the parts of an unnormalised P-form product: the
//                   output is inv_i * alpha * acc (exact: row scaling commutes)
enum { OPB_FIX_NONE = 0, OPB_FIX_CIN = 1, OPB_FIX_SQUARE = 2, OPB_FIX_ROWSCALE = 3 };
// Split-BF16 squarings add the fourth product lo.lo on their first OPB_LOLO_LEVELS levels,
// as long as the operands are still banded (twice the band below the size; every level up
// to OPB_LOLO_LEVELS when the band is not known).  hi.hi + hi.lo + lo.hi leaves out lo.lo,
// a term of 2^-16 relative size that does not average out on the early, banded levels: on
// the 512 lattices of the calibration sweep (n up to 2048, up to 16 squarings) leaving it
// out everywhere costs up to 1.4e-5 in price, adding it on the first 8 levels brings every
// price within 2e-6 of FP64.  Those levels are banded, so the extra product costs little.
constexpr int OPB_LOLO_LEVELS = 8;
// knobs shared by the single and batched solves (opb_set_lolo_levels, opb_set_band_skip)
extern int g_lolo_levels;  // leading squaring levels with the lo.lo product (BF16 parts)
extern int g_band_skip;    // 1: squarings leave out the K-blocks outside the operands' band
// Whether the single-lattice solve fuses the row normalisation into the products'
// epilogues (which then also write the next operand's parts) or runs a renormalisation
// kernel after every product.  By default (g_fused_max_d < 0) lattices of at least
// OPB_FUSED_AUTO_MIN_D states fuse; opb_set_fused_normalisation(max_d >= 0) fuses exactly
// the lattices of at most max_d states (0: none).  A fused epilogue lengthens each tile's
// output phase, which sits on the tile's critical path: a one-wave product has no later
// tile to hide it behind (d = 2048: 2.38 ms fused against 2.25 with the kernel), while on
// larger lattices it costs less than the kernel's pass over the matrix (SV solves, CUDA-graph
// replay: 9.02 against 9.06 ms at d = 4096; 24.13 against 24.58 ms at d = 6144, alternated
// three times in one run).  The batched sweep, where the renormalisation of hundreds of
// small lattices took 19% of the time, always fuses.
constexpr int OPB_FUSED_AUTO_MIN_D = 4096;
extern int g_fused_max_d;  // opb_set_fused_normalisation; < 0: automatic
inline bool fused_single(int d) { return g_fused_max_d < 0 ? d >= OPB_FUSED_AUTO_MIN_D : d <= g_fused_max_d; }
// K-slices that fill the GPU with the tiles of a small-N product (1 = none), at most 4
int tc_gemm_split_for(int M, int N, int K);
int tc_gemm_tile_n(int N);                    // tile width chosen for N (0 if unsupported)
int tc_gemm_check(const TcGemmArgs &a);       // argument/alignment check, OPB_* code
int launch_tc_gemm(const TcGemmArgs &a, cudaStream_t s);
// Network layers: accumulator columns per epilogue thread; the fused output layer writes
// N / TC_LAYER_CPT partial dots per row.
constexpr int TC_LAYER_CPT = 64;
int launch_tc_layer(int M, int N, int K, const __nv_bfloat16 *A, long long lda, const __nv_bfloat16 *W,
                    long long ldw, float alpha, const float *bias, __nv_bfloat16 *H, long long ldh, cudaStream_t s,
                    const float *w5 = nullptr, float *ypart = nullptr);
// The four hidden layers and the output layer's partial dots of one network in one kernel
// (activations kept in shared memory); writes what the layer-by-layer launches write.
int launch_mlp_fused(long long M, const __nv_bfloat16 *Xp, const __nv_bfloat16 *W1, const __nv_bfloat16 *WH,
                     const float *vec, float *ypart, cudaStream_t s);
int tc_gemm_nparts(int M, int N);             // number of row-sum partials written

// Batched launches: problem descriptors and tensor maps live in device memory.
struct TcProblem {
    // band > 0: squaring operands zero outside |row - col| <= band << level (TcGemmArgs::band)
    int M, N, K, band;
    float *C;
    const float *Cin;
    double *rowsum;       // partials rowsum[(col/min(bn,128)) * M + row]
    long long ldc;
    float alpha, beta;
    const double2 *cin_fix;  // as TcGemmArgs::cin_fix
    __nv_bfloat16 *Shi, *Slo;  // as TcGemmArgs::Shi / Slo (optional)
};
// Four maps (Ahi, Alo, Bhi, Blo) of one problem: A with 128-row boxes; B K-major (N x K,
// bn-row boxes) or, with b_kn, K x N row-major read as an MN-major operand (64 x 64
// boxes, the same maps for every tile width).
int tc_make_maps(CUtensorMap *out4, const __nv_bfloat16 *Ahi, const __nv_bfloat16 *Alo, long long M, long long lda,
                 const __nv_bfloat16 *Bhi, const __nv_bfloat16 *Blo, long long N, long long ldb, long long K, int bn,
                 int f16 = 0, int b_kn = 0);
// work: packed (problem << 16 | m-tile << 8 | n-tile); bn in {64, 128, 256}; K-major B
// (b_kn = 0) only for bn = 64
// level, lolo: as TcGemmArgs (band per problem in TcProblem::band)
// fixmode, sscale: as TcGemmArgs (the problems' cin_fix and Shi / Slo); fuse: the epilogue
// form (0: FP32 output, OPB_FIX_CIN; 1: squaring with its output's parts, OPB_FIX_SQUARE;
// 2: parts only, OPB_FIX_ROWSCALE), MN-major B only
int launch_tc_gemm_batched(int bn, const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                           int grid, cudaStream_t s, int f16, int b_kn, int level = 0, int lolo = 0,
                           int band_skip = 0, int fixmode = 0, float sscale = 0.f, int fuse = 0);
// 256 x 256 items (256-row / 256-column units) on 2-CTA clusters, each CTA loading its
// 128 rows of A and 128 columns of B; MN-major B maps; problems with M, N multiples of 256
int launch_tc_gemm_batched_pair(const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                                cudaStream_t s, int f16, int b_kn, int level = 0,
                                int lolo = 0, int band_skip = 0, int fixmode = 0, float sscale = 0.f, int fuse = 0);

// sck.cu
int launch_sck_rm(int d, int nrows, const float *P, float *C, cudaStream_t s);
int launch_guide(int d, int nrows, int nb, const float *C, uint32_t *guide, cudaStream_t s);

}  // namespace opb
