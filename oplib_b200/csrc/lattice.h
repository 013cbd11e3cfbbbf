// Internal launcher declarations shared by the library's translation units.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace opb {

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
int launch_discount(int d, int nK, int ldk, const float *V32, double disc, double *V64, int y0, double *quotes,
                    cudaStream_t s, const float *dscale = nullptr, int nslice = 1, long long slice_stride = 0);

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
};
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
int launch_quotes_batched(const BatchLattice *lats, int nlat, int nK, int ldk, int m, int nmat, double *quotes,
                          cudaStream_t s, int f16 = 0);

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
};
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
int launch_tc_gemm_batched(int bn, const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                           int grid, cudaStream_t s, int f16, int b_kn, int level = 0, int lolo = 0,
                           int band_skip = 0);
// 256 x 256 items (256-row / 256-column units) on 2-CTA clusters, each CTA loading its
// 128 rows of A and 128 columns of B; MN-major B maps; problems with M, N multiples of 256
int launch_tc_gemm_batched_pair(const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                                cudaStream_t s, int f16, int b_kn, int level = 0,
                                int lolo = 0, int band_skip = 0);

// sck.cu
int launch_sck_rm(int d, int nrows, const float *P, float *C, cudaStream_t s);
int launch_guide(int d, int nrows, int nb, const float *C, uint32_t *guide, cudaStream_t s);

}  // namespace opb
