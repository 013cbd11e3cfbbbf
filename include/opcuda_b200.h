/*
 * opcuda-b200: B200-native (sm_100a) replacement of OPLib's opcuda C-ABI for the
 * operator-method pricing path (generator exponentiation by repeated squaring, payoff
 * backward induction, Markov-chain Monte Carlo).
 *
 * Library: libopcuda_b200.so.  Every function is extern "C".
 *
 * Differences from the reference ABI, applied uniformly:
 *   - device pointers are 64-bit (uint64_t handles or typed pointers); the reference
 *     passes them as 32-bit `unsigned` (oplib/opcuda/util.cu:209-213), which truncates
 *     addresses on a 64-bit host;
 *   - every entry point returns an int status: 0 = success, negative = argument error
 *     detected on the host (OPB_E_*), positive = cudaError_t.  The last status of the
 *     calling thread is also returned by opcuda_get_status(), which is how the
 *     reference's callers read it (oplib/opcuda/util.cu:204-207);
 *   - work is ordered on a per-thread library stream (opb_set_stream; default: the
 *     legacy default stream).  Calls that the reference makes blocking (memcpy, mc1f)
 *     stay blocking.
 * Names, argument order and column-major semantics of the opcuda_* entry points are the
 * reference's.  opb_* entry points are new B200 forms (source-major storage).
 */
#ifndef OPCUDA_B200_H
#define OPCUDA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define OPB_OK 0
#define OPB_E_ARG (-1)
#define OPB_E_NULL (-2)
#define OPB_E_ALIGN (-3)
#define OPB_E_UNSUPPORTED (-4)
#define OPB_E_NOMEM (-5)
#define OPB_E_TIMEOUT (-6)
#define OPB_E_STATE (-7)

/* precision modes of opb_lattice_solve */
#define OPB_FP32_PLAIN 0  /* FP32 SIMT products, reference semantics (no renormalisation) */
#define OPB_FP32_RENORM 1 /* FP32 SIMT products + FP64 row renormalisation */
#define OPB_BF16X3 2      /* split-BF16 tcgen05 products (E-form squaring) + FP64 renormalisation */
#define OPB_FP16X3 3      /* as OPB_BF16X3 with FP16 parts of 2^15-scaled values (11+11 bits; same cost) */

/* ------------------------------------------------------------------ runtime support */
/* replaces oplib/opcuda/util.cu:204-207 (unsigned opcuda_get_status()) */
int opcuda_get_status(void);
/* replaces oplib/opcuda/util.cu:123-126 (cuBLAS init); creates the CUDA context */
int opcuda_cublas_init(void);
/* replaces oplib/opcuda/util.cu:287-290 */
int opcuda_shutdown(void);
/* replaces oplib/opcuda/util.cu:131-133 (void) */
int opcuda_thread_synchronize(void);
/* replaces oplib/opcuda/util.cu:139-141 (void) */
int opcuda_set_device(int dev);
/* replaces oplib/opcuda/util.cu:148-153 */
int opcuda_get_device(void);
/* replaces oplib/opcuda/util.cu:156-161 */
int opcuda_device_get_count(void);
/* replaces oplib/opcuda/util.cu:240-245 */
int opcuda_device_count(void);
/* replaces oplib/opcuda/util.cu:163-170 (the reference leaves the name unset) */
int opcuda_device_get_name(char *name, int len, int dev);
/* replaces oplib/opcuda/util.cu:172-179 (unsigned *bytes; the reference leaves it unset) */
int opcuda_device_total_memory(uint64_t *bytes, int dev);
/* replaces oplib/opcuda/util.cu:248-253 */
int opcuda_multi_processor_count(int dev);
/* replaces oplib/opcuda/util.cu:255-260 */
int opcuda_max_threads_per_block(int dev);
/* replaces oplib/opcuda/util.cu:209-214 (unsigned opcuda_mem_alloc(unsigned sz)) */
uint64_t opcuda_mem_alloc(uint64_t sz);
/* replaces oplib/opcuda/util.cu:217-221 */
int opcuda_mem_free_device(uint64_t ptr);
/* replaces oplib/opcuda/util.cu:223-230 */
uint64_t opcuda_mem_alloc_host(uint64_t sz);
/* replaces oplib/opcuda/util.cu:232-236 */
int opcuda_mem_free_host(uint64_t hptr);
/* replace oplib/opcuda/util.cu:182-200 (blocking copies) */
int opcuda_memcpy_h2d(uint64_t dptr, uint64_t hptr, uint64_t sz);
int opcuda_memcpy_d2h(uint64_t dptr, uint64_t hptr, uint64_t sz);
int opcuda_memcpy_d2d(uint64_t dptr2, uint64_t dptr1, uint64_t sz);
/* replace oplib/opcuda/util.cu:62-113 (wall-clock timers) */
void opcuda_create_timer(void);
void opcuda_reset_timer(void);
void opcuda_stop_timer(void);
double opcuda_get_timer_value(void);
/* replaces oplib/opcuda/util.cu:263-282 */
int opcuda_scopy(int n, uint64_t x, int incx, uint64_t y, int incy);
/* replaces oplib/opcuda/scopy2.cu:137-143 */
int opcuda_scopy1(uint64_t destination, uint64_t source, uint64_t n);
/* replace oplib/opcuda/sset.cu:54-74 */
int opcuda_ssetall(uint64_t x, int n, float c, int incx);
int opcuda_ssetone(uint64_t x, int n, float c, int i);

/* new: library stream of the calling thread (a cudaStream_t as an integer), version,
 * status text, and a test hook making the n-th next opcuda_mem_alloc fail */
int opb_set_stream(uint64_t stream);
uint64_t opb_get_stream(void);
const char *opb_version(void);
const char *opb_status_string(int status);
int opb_test_fail_next_alloc(int n);

/* ------------------------------------------------------------------ GEMM / GEMV (FP32) */
/* replaces oplib/opcuda/sgemm.cu:41-44: column-major C = alpha*A*B + beta*C */
int opcuda_sgemm(int m, int n, int k, float alpha, uint64_t A, int lda, uint64_t B, int ldb, float beta,
                 uint64_t C, int ldc);
/* replaces oplib/opcuda/ssqmm.cu:174-179: C_i = A_i * B_i for ni column-major d x d
 * matrices; A_i, B_i, C_i are device arrays of ni 64-bit device pointers */
int opcuda_ssqmm(int d, int ni, uint64_t A_i, uint64_t B_i, uint64_t C_i);
/* replaces oplib/opcuda/sgemm4.cu:148-154: argptr_bid is a device array of nblocks
 * 64-bit pointers to task records {int32 i, bx, by, m, n, k; uint64 A, B, C}
 * (opb_sgemm4_task_size() bytes); block computes C rows [64bx, 64bx+64) x cols
 * [16by, 16by+16) of the column-major C = A*B with lda = m, ldb = k, ldc = m */
int opcuda_sgemm4(int nblocks, uint64_t argptr_bid);
int opb_sgemm4_task_size(void);
/* new: row-major strided batch C_z = A_z * B_z (M x K times K x N) */
int opb_sgemm_batched_rm(int M, int N, int K, const float *A, long long sA, const float *B, long long sB, float *C,
                         long long sC, int batch);
/* replace oplib/opcuda/sgemv.cu:44-62 */
int opcuda_sgemv(int m, int n, float alpha, uint64_t A, int lda, uint64_t x, int incx, float beta, uint64_t y,
                 int incy);
int opcuda_sgemvT(int m, int n, float alpha, uint64_t A, int lda, uint64_t x, int incx, float beta, uint64_t y,
                  int incy);
/* replaces oplib/opcuda/sgemv3.cu:163-176: Z[col1[c] + row] = sum_k A[row + d*k] Z[col0[c] + k]
 * (column offsets in elements; entries at or after the first col1 >= 2*nz*d are skipped) */
int opcuda_sgemv3(int d, int nz, int ncol, uint64_t A, uint64_t B, uint64_t col0ptr, uint64_t col1ptr);
/* replaces oplib/opcuda/sgemv4.cu:174-180: task records {int32 i, bx, by, d, nz, ncol;
 * uint64 A, Z, col0, col1} (opb_sgemv4_task_size() bytes); rows [128bx, 128bx+128) of the
 * 16 list entries starting at 16by */
int opcuda_sgemv4(int nblocks, uint64_t argptr_bid);
int opb_sgemv4_task_size(void);
/* replaces oplib/opcuda/sdot2.cu:72-83: c[h] = sum_{y<n} a[h + m*y] * b[h + m*y], h < m */
int opcuda_sdot2(uint64_t aptr, uint64_t bptr, uint64_t cptr, int m, int n);

/* ------------------------------------------------------------------ kernels from generators */
/* replace oplib/opcuda/sek.cu:106-137: column-major U = (I + dt*gen) [/(1 + dt*r*lambda)],
 * in the reference kernels' FP32 arithmetic (fused numerator, FP32 division), bit for bit */
int opcuda_sek(int d, uint64_t genPtr, float dt, uint64_t tpkerPtr);
int opcuda_sekd(int d, uint64_t genPtr, float dt, uint64_t tpkerPtr, uint64_t rPtr);
int opcuda_sekd_lambda(int d, uint64_t genPtr, float dt, uint64_t tpkerPtr, uint64_t rPtr, uint64_t lambdaPtr);
/* replaces oplib/opcuda/sglvg.cu:104-125: dense column-major LV generators for ni periods
 * from per-node column-major 2x2 inverses invm[4d] and pars = [drift (ni*d); vol (ni*d)] */
int opcuda_sglvg(uint64_t gen_yy_i, int ni, int d, uint64_t invmat, uint64_t pars);
/* new (device generator builders, FP64, ELL form: row y holds w (col, val) pairs, col -1 = empty) */
int opb_lv_params(int d, double lo, double hi, double s0, double level, double skew, double width, double floor_,
                  double r, double *x, double *drift, double *vol);
int opb_lv_generator_ell(int d, const double *x, const double *drift, const double *vol, int *cols, double *vals);
/* new: LV generators of nlat lattices in one launch into concatenated ELL arrays (calibration
 * loops); params = device array of nlat 56-byte records {int n, pad; long long row_off;
 * double level, skew, width, floor, rate}; entries bit-identical to opb_lv_params +
 * opb_lv_generator_ell per lattice (batched form of oplib/opcuda/sglvg.cu:42-99) */
int opb_lv_generator_ell_batched(int nlat, const void *params, long long total_rows, double lo, double hi, double s0,
                                 int *cols, double *vals);
int opb_lv_param_size(void);
/* oplib/opcuda/sgsvg.cu:215 (opcuda_sgsvg): two-dimensional generator with jumps across
 * volatility levels, dense column-major FP32 [ni][d][d] (d = nx*nr, caller zeroes it) from the
 * per-node 4x4 moment inverses invmat[16 d] (S2DGrid.pregen) and par = {x[d], sdrift, svol,
 * voldrift, volvol, jump_minus, jump_plus, each [ni][d]} (FP32); FP64 arithmetic; the upper
 * jump size is the upper block (the reference kernel reads the lower one for both) */
int opcuda_sgsvg(unsigned long long gen_yyi_ptr, int ni, int nx, int nr, unsigned long long invmat_ptr,
                 unsigned long long parptr);
int opb_sv_generator_ell(int nx, int nv, double x_lo, double x_hi, double v_lo, double v_hi, double r, double kappa,
                         double theta, double xi, double rho, int *cols, double *vals, double *x_y);
int opb_ell_maxdiag(int d, int w, const int *cols, const double *vals, unsigned long long *dscratch,
                    double *out_host);
/* new: the squaring plan of one interval (oplib/opmodel/models/CModel Common.cs:289-307) */
int opb_plan_interval(double maxdiag, double delta_t, double dt0, int *niter, double *dt_j);

/* ------------------------------------------------------------------ split-BF16 tensor-core GEMM */
/* new: C = alpha*(Ahi*Bhi^T + Ahi*Blo^T + Alo*Bhi^T) + beta*Cin, row-major, K-major operands
 * (A: M x K, B: N x K), M % 128 == 0, N % 64 == 0, K % 64 == 0, 16-byte aligned; rowsum
 * (optional) receives FP64 row sums of C per N tile: rowsum[t*M + row],
 * t < opb_gemm_bf16x3_nparts(M, N).  Replaces the FP32 SIMT products of oplib/opcuda/ssqmm.cu. */
typedef uint16_t opb_bf16; /* storage of one bfloat16 */
int opb_gemm_bf16x3(int M, int N, int K, const opb_bf16 *Ahi, const opb_bf16 *Alo, long long lda,
                    const opb_bf16 *Bhi, const opb_bf16 *Blo, long long ldb, float alpha, const float *Cin,
                    float beta, float *C, long long ldc, double *rowsum);
int opb_gemm_bf16x3_nparts(int M, int N);
/* new: the same product with B given K x N row-major (ldb >= N), read by the tensor cores as
 * an MN-major operand (the form of the lattice solve's squaring and chain products, whose B
 * is a row-major split); results identical to opb_gemm_bf16x3 on the transposed B */
int opb_gemm_bf16x3_kn(int M, int N, int K, const opb_bf16 *Ahi, const opb_bf16 *Alo, long long lda,
                       const opb_bf16 *Bhi, const opb_bf16 *Blo, long long ldb, float alpha, const float *Cin,
                       float beta, float *C, long long ldc, double *rowsum);
/* new: the product of a skinny B (N <= 128: payoff or option-value columns, B N x K row-major)
 * as ksplit K-slices, slice s writing its FP32 partial product to C + s * c_slice (c_slice >=
 * M * ldc) for the caller to sum; ksplit = 0 picks the count that brings the tiles to about
 * one per SM (at most 4), as the lattice solve's pricing and induction products do, and
 * returns it through ksplit_used (optional).  The memory-bound form of the product: A is read
 * from memory once. */
int opb_gemm_bf16x3_ksliced(int M, int N, int K, const opb_bf16 *Ahi, const opb_bf16 *Alo, long long lda,
                            const opb_bf16 *Bhi, const opb_bf16 *Blo, long long ldb, float *C, long long ldc,
                            int ksplit, long long c_slice, int *ksplit_used);
/* new (tuning): force the output tile width (64, 128, 256) of single products; 0 = automatic */
int opb_set_tile_n(int bn);
/* new: tuning knob, K depth of a pipeline stage of 256-wide tiles: 64 (default) or 32 (twice
 * the stages of half the size; 64-byte swizzle for A); results are identical */
int opb_set_stage_k(int bk);
/* new: tuning knob, 256 x 256 output tiles on 2-CTA clusters (cta_group::2 MMAs over both
 * CTAs' shared memory) for products with M % 256 == 0: 1 = on (default), 0 = off;
 * results are identical */
int opb_set_cta_pair(int on);
/* new: tuning knob, M-tiles per raster group of single products (L2 reuse of operand strips);
 * 0 = 8; results are identical */
int opb_set_group_m(int gm);
/* new: the same product with FP16 parts (power-of-two-scaled splits; undo the scales in alpha) */
int opb_gemm_f16x3(int M, int N, int K, const uint16_t *Ahi, const uint16_t *Alo, long long lda, const uint16_t *Bhi,
                   const uint16_t *Blo, long long ldb, float alpha, const float *Cin, float beta, float *C,
                   long long ldc, double *rowsum);
/* new: the FP16-part product with B given K x N row-major (as opb_gemm_bf16x3_kn) */
int opb_gemm_f16x3_kn(int M, int N, int K, const uint16_t *Ahi, const uint16_t *Alo, long long lda,
                      const uint16_t *Bhi, const uint16_t *Blo, long long ldb, float alpha, const float *Cin,
                      float beta, float *C, long long ldc, double *rowsum);
/* new: FP64 row renormalisation of a source-major d x d FP32 matrix from row-sum partials
 * partial[p*d + y] (p < nparts), with optional 16-bit splits (A row-major, B transposed);
 * mode 0 E-form, 1 E-form in / P-form out, 2 P-form (no B); f16: FP16 parts of 2^15-scaled
 * values instead of BF16; d % 64 == 0 (probability conservation, no reference counterpart).
 * BF16 parts: hi = bf16(x), lo = bf16(x - hi), except that |x| < 2^-40 gives no parts and
 * |x| < 2^-30 no lo part (the split every solve uses) */
int opb_renorm_rows(int d, float *X, const double *partial, int nparts, int mode, void *Ahi, void *Alo, void *Bhi,
                    void *Blo, int f16);
/* reads and clears the device error word of the tensor-core kernels (0 = none) */
int opb_tc_error(void);

/* ------------------------------------------------------------------ lattice solve */
typedef struct opb_lattice_desc {
    int d;                   /* states */
    int y0;                  /* quoted state */
    int ell_width;           /* > 0: ELL generator (gen_cols, gen_vals); 0: dense gen_dense */
    const int *gen_cols;     /* device [d*ell_width] */
    const double *gen_vals;  /* device [d*ell_width] FP64 */
    const double *gen_dense; /* device [d*d] FP64, row-major (row = source state) */
    const double *x;         /* device [d] spot per state */
    double dt;               /* elementary step = period * 2^-niter */
    int niter;               /* squarings */
    int nmat;                /* maturities T_m = m*period, m = 1..nmat */
    double period;
    double rate;             /* discount rate */
    int nK;                  /* strikes */
    const double *strikes;   /* device [nK] */
} opb_lattice_desc;
/* new: the device branch of CModel.exe_mc_plan (oplib/opmodel/models/CModel Common.cs:651-669)
 * plus payoff backward induction: quotes[(m-1)*nK + k] = exp(-rate*T_m) * (P(T_m) G)[y0, k],
 * G[z, k] = (x_z - K_k)^+; V_all (optional) receives all states [nmat][d][nK].  Any d in every
 * mode: the split modes solve a d that is no multiple of 128 as the lattice padded with
 * absorbing states up to the next multiple (the workspace size accounts for it). */
unsigned long long opb_lattice_workspace_size(int d, int nK, int mode);
int opb_lattice_solve(const opb_lattice_desc *L, int mode, void *workspace, unsigned long long ws_bytes,
                      double *quotes, double *V_all);
/* new (extension; the reference ships the induction kernels sgemv3/sgemv4 but no pricer on
 * them): calls (put = 0) or puts (put = 1) of final maturity T = nmat * period by backward
 * induction on P1 = P(period): V_nmat = e(x), V_m = exp(-rate*period) * P1 . V_{m+1},
 * knocked out where x <= barrier (barrier > 0) and, with exercise = 1, floored by the
 * exercise value, at every T_m, m = 1..nmat-1 (Bermudan / discretely monitored
 * down-and-out); exercise = 0 and barrier = 0 give the European value at T.  quotes:
 * device [nK] FP64 values at y0.  Induction products on the tensor cores in the split modes,
 * on the FP32 SIMT GEMM in the FP32 modes; workspace as for opb_lattice_solve. */
int opb_lattice_bermudan(const opb_lattice_desc *L, int mode, int put, int exercise, double barrier,
                         void *workspace, unsigned long long ws_bytes, double *quotes);
/* new: transition kernel P(period) only (device d x d FP32, source-major), e.g. the MC step
 * kernel; nmat, nK and strikes of L are ignored */
int opb_lattice_kernel(const opb_lattice_desc *L, int mode, void *workspace, unsigned long long ws_bytes,
                       float *P_out);
/* new: step kernel of a Monte Carlo step that spans several elementary intervals (a generator
 * date inside the step): out = X_0 . X_1 ... X_{nf-1} of row-major d x d FP32 kernels (factors:
 * host array of nf device pointers, in time order), FP32 products each renormalised to unit
 * row sums in FP64.  Replaces the reference's device chaining of the planned factor lists
 * (oplib/opmodel/models/CModel Device.cs:252-295 over CModel Common.cs:431-486's jfactor_ms) */
unsigned long long opb_chain_workspace_size(int d);
int opb_chain_kernels(int d, int nf, const float *const *factors, float *out, void *workspace,
                      unsigned long long ws_bytes);
/* new: issue every tensor-core product of the solve as s K-slices summed in the FP32
 * epilogue (shorter in-TMEM accumulation chains); 0 (default) = automatic */
int opb_set_ksplit(int s);
/* new: split-BF16 squarings (single and batched solves) add the fourth product lo.lo on their
 * first n levels; default 8, 0..64.  Leaving lo.lo out everywhere (n = 0) gives the plain
 * three-product form, whose error reaches 1.4e-5 on the highest-niter lattices of the
 * calibration sweep; with the default every sweep price is within 2e-6 of FP64 */
int opb_set_lolo_levels(int n);
/* new: 1 (default): squarings of an ELL generator's E_r = P(2^r dt) - I skip the K-blocks and
 * output tiles outside twice E_r's band (h0 * 2^r for the generator's half-bandwidth h0),
 * whose products are exact zeros; 0: every squaring runs the full product.  Results are
 * bit-identical either way */
int opb_set_band_skip(int on);
/* new: the split-mode solves defer each product's FP64 row normalisation into the next
 * product's epilogue, which also writes that product's 16-bit operand parts, so no
 * renormalisation kernel runs between products (squarings: the next level applies
 * D [E'.E' - S E' - E' S + S^2] + 2 D (E' - S) with D = diag(1/(1+s)), S = diag(s), the D
 * between the factors left out; chain products: the row scaling, exact).  The batched
 * sweep always does; a single-lattice solve does up to max_d states (max_d >= 0; 0: a
 * renormalisation kernel after every product).  max_d = -1 restores the default: lattices of
 * 4096 states or more fuse, smaller ones run the kernel, which is the faster form where one
 * wave of tiles leaves the longer fused output phase nothing to hide behind. */
int opb_set_fused_normalisation(int max_d);

/* ------------------------------------------------------------------ batched lattices */
typedef struct opb_batch_desc {
    int nlat;
    const int *d;            /* host [nlat], 2..8064 (split modes: solved padded to the next
                                multiple of 128 with absorbing states) */
    const int *y0;           /* host [nlat] */
    const int *niter;        /* host [nlat], >= 1 */
    const double *dt;        /* host [nlat] */
    const double *rate;      /* host [nlat] */
    int ell_width;
    const int *gen_cols;     /* device [sum(d) * ell_width], columns within the lattice */
    const double *gen_vals;  /* device [sum(d) * ell_width] */
    const double *x;         /* device [sum(d)] */
    int nmat;
    double period;
    int nK;                  /* <= 64 */
    const double *strikes;   /* device [nlat * nK] */
} opb_batch_desc;
typedef struct opb_batch_plan opb_batch_plan;
/* new: many uneven lattices in one persistent tcgen05 launch per squaring level (the
 * reference batches squarings per level through pointer tables, oplib/opmodel/models/
 * CModel Common.cs:508-545, and ragged GEMMs through task tables, oplib/opcuda/sgemm4.cu:
 * 84-154).  plan_create uploads tables into the workspace (blocking); execute issues all
 * launches asynchronously with no allocation (capturable); quotes [nlat][nmat][nK] FP64. */
unsigned long long opb_batch_workspace_size(const opb_batch_desc *b, int mode);
int opb_batch_plan_create(const opb_batch_desc *b, int mode, void *workspace, unsigned long long ws_bytes,
                          opb_batch_plan **out);
int opb_batch_plan_destroy(opb_batch_plan *plan);
/* cfg < opb_batch_num_configs(): tile width x work order (128, 64, 256-mixed or 256 on
 * CTA pairs mixed; longest first or lattice order); grid 0 = one CTA per SM */
int opb_batch_set_config(opb_batch_plan *plan, int cfg, int grid);
int opb_batch_num_configs(void);
int opb_batch_execute(opb_batch_plan *plan, double *quotes);
/* new (extension, as opb_lattice_bermudan): Bermudan or down-and-out calls/puts of maturity
 * nmat * period on every lattice of the plan by backward induction on its period kernel,
 * one batched tensor-core product per date over all lattices; quotes: device [nlat][nK]
 * FP64 values at each lattice's y0 */
int opb_batch_execute_bermudan(opb_batch_plan *plan, int put, int exercise, double barrier, double *quotes);
/* times the chain product (all lattices, dense operands) for every configuration
 * (ms_out: opb_batch_num_configs() floats) and keeps the fastest */
int opb_batch_autotune(opb_batch_plan *plan, int reps, float *ms_out, int *best_cfg);
int opb_batch_launches(const opb_batch_plan *plan);

/* ------------------------------------------------------------------ surrogate pricer */
/* new, no reference counterpart (closest: tests/bstest/BSPricer.cs:7-65): MLP 8 -> 256 x 4 -> 1
 * (GELU) from (level, skew, width, kappa, rho, r, log-moneyness, T) to implied vol.  theta: FP32
 * master parameters (layer l: W [out x in] row-major then b); training uses BF16-rounded
 * working weights thb (FP32 storage), FP32 activations, Adam on theta.  loss receives the sum
 * of squared errors.  The hidden layers' training products run on the tensor cores as
 * split-BF16 products (activations and gradients as hi + lo parts, FP32 accumulation) when
 * B is a multiple of 128; the first and output layers on SIMT kernels. */
int opb_mlp_param_count(void);
long long opb_mlp_workspace_floats(int B);
/* new: 1 (default) tensor-core training products as above, 0 SIMT FP32 throughout */
int opb_mlp_set_tensor_cores(int on);
int opb_mlp_init(float *theta, unsigned long long seed);
int opb_mlp_round(const float *theta, float *theta_bf, void *theta_b16);
int opb_mlp_forward(const float *thb, const float *X, int B, float *ws, float *y);
int opb_mlp_loss_grad(const float *thb, const float *X, const float *t, int B, float *ws, float *grad, double *loss);
int opb_mlp_adam(float *theta, float *m, float *v, const float *grad, int step, float lr, float b1, float b2,
                 float eps, float *theta_bf);
/* new: opb_mlp_adam with the step count (device int, advanced by the call) and a learning-rate
 * table (device, lr_table[step - 1]) in device memory: every epoch of a training loop is then
 * the same launches, captured once in a CUDA graph and replayed */
int opb_mlp_adam_sched(float *theta, float *m, float *v, const float *grad, int *step, const float *lr_table, float b1,
                       float b2, float eps, float *theta_bf);
/* implied volatilities of call prices with spots S0[i] (FP64 bisection); NaN without time value */
int opb_implied_vol(long long n, const double *price, const double *K, const double *T, const double *r,
                    const double *S0, double *iv);
/* tensor-core ensemble inference: packed BF16 weights (opb_mlp_pack), members at packed +
 * m * member_stride bytes; mean / spread (max - min) of the member outputs */
long long opb_mlp_packed_bytes(void);
int opb_mlp_pack(const float *theta, void *packed);
long long opb_mlp_infer_workspace_bytes(long long n, int nmem);
int opb_mlp_infer(const void *packed, int nmem, long long member_stride, const float *X, long long n, void *ws,
                  long long ws_bytes, float *mean, float *spread);
/* new: 1 (default) one kernel per member runs all layers with the activations in shared
 * memory; 0 one launch per layer, activations through device memory (bit-identical) */
int opb_mlp_set_fused_inference(int on);

/* ------------------------------------------------------------------ cumulative rows, MC */
/* replaces oplib/opcuda/sck.cu:88-93: nm column-major kernels -> cumulative normalised rows */
int opcuda_sck(int d, int nm, uint64_t tpker_yy_m, uint64_t ctpker_yy_m);
/* new: source-major cumulative rows; per-row bracket table (nb a power of two, d <= 65535),
 * the device analogue of CModel Host Double.cs:434-455 */
int opb_sck_rm(int d, int nrows, const float *P, float *C);
int opb_guide_table(int d, int nrows, int nb, const float *C, uint32_t *guide);
/* replace oplib/opcuda/smc.cu:87-106: nrng = 4096 stream seeds, status record of
 * 4 + 4096 int32 words */
int opcuda_mc_load_mt_gpu(const char *MT_stream, long sz);
int opcuda_mc_nrng(void);
int opcuda_mc_status_sz(void);
/* replaces oplib/opcuda/smc.cu:137-156: host_seedptr holds opcuda_mc_nrng() = 4096 uint32
 * stream seeds; mtptr is the device status record (opcuda_mc_status_sz() words: next path
 * id and the seeds).  Path g (counted from this call) is path g / 4096 of stream g % 4096
 * and draws from MT19937 init_genrand(seeds[g % 4096]) with g / 4096 added to mt[1]. */
int opcuda_mc_setseed(uint64_t host_seedptr, uint64_t mtptr);
/* replaces oplib/opcuda/smc.cu:610-656 (per-path MT19937 generators keyed from the stream
 * seeds; any nk >= 1, d <= 32767) */
int opcuda_mc1f(uint64_t mtptr, int y0, uint64_t y_sk, int nscen, int nk, int d, uint64_t ctpker_m_yy, uint64_t m_k,
                uint64_t yhostptr);
/* new, the device side of the reference's opcuda_mc1f + CMCEvaluator.eval pair
 * (oplib/opmodel/models/CModel Device.cs:343-364, oplib/opmodel/interfaces/CMCEvaluator.cs:41-67):
 * the paths of opcuda_mc1f (continuing the status record), each valued on the device by a
 * cashflow table -- results[p] = sum_k cashflow[k*d + y_k] over the steps before the first
 * state with knockout[k*d + y_k] != 0 (knockout optional, 0) -- so the states need not be
 * copied to the host; y_sk optional (0).  Blocking, as opcuda_mc1f. */
int opcuda_mc1f_eval(uint64_t mtptr, int y0, uint64_t y_sk, int nscen, int nk, int d, uint64_t ctpker_m_yy,
                     uint64_t m_k, uint64_t cashflow, uint64_t knockout, uint64_t results);
/* replaces oplib/opcuda/smc.cu:731-736 (nscen % 4096 == 0): stream s of the status
 * record's 4096 writes nscen/4096 uniforms from init_genrand(seeds[s]) */
int opcuda_mt_benchmark(uint64_t mtptr, uint64_t unif_ptr, int nscen);
/* new: MT19937 Monte Carlo, path p seeded init_genrand(seed + path0 + p); see mc.cu.
 * Runs of up to 623 steps keep the generator in registers; longer runs hold the
 * 624-word state in per-thread local memory (2496 bytes a thread), which the CUDA
 * driver may provision on the first such launch. */
int opb_mc_scratch_blocks(long long npaths);
int opb_mc_mt19937(const float *C, long long row_stride, long long col_stride, const uint32_t *guide, int nb, int d,
                   int y0, int nsteps, uint32_t seed, unsigned long long path0, long long npaths, short *ypaths,
                   const double *x, double strike, double barrier, double disc, double *scratch, double *sums);
/* new: opb_mc_mt19937's paths valued by a device-side evaluator instead of the fused payoffs:
 * v_p = sum_k cashflow[k*d + y_k] (FP64 [nsteps][d], discounting folded in) over the steps
 * before the first knocked-out state (knockout [nsteps][d] bytes, optional); path_values
 * (optional) [npaths]; sums[0] = sum v_p, sums[1] = sum v_p^2; scratch as opb_mc_mt19937 */
int opb_mc_mt19937_eval(const float *C, long long row_stride, long long col_stride, const uint32_t *guide, int nb,
                        int d, int y0, int nsteps, uint32_t seed, unsigned long long path0, long long npaths,
                        short *ypaths, const double *cashflow, const unsigned char *knockout, double *path_values,
                        double *scratch, double *sums);
/* new, no counterpart in the reference: opb_mc_mt19937 without the scratch argument, for
 * callers that must not let the library allocate device memory (a host framework that owns
 * the device-memory budget, or a loop that cannot afford cudaMalloc's implicit device
 * synchronisation).  The payoff partial sums use a fixed 64 KiB device array inside the
 * library (held by every GPU that loads it until exit); results are bit-identical to
 * opb_mc_mt19937.  Grids above 4096 blocks (devices with more than 512 SMs) return
 * OPB_E_UNSUPPORTED, and so do runs longer than 623 steps (they would need the driver's
 * local-memory reservation to grow).  The first call on a device, whatever its arguments, looks up
 * the array's device address (make it before any stream capture); the address is kept for the
 * process, so the entry point must not be used on a device after cudaDeviceReset.  Calls that
 * overlap on the GPU share the array and race. */
int opb_mc_mt19937_noalloc(const float *C, long long row_stride, long long col_stride, const uint32_t *guide, int nb,
                           int d, int y0, int nsteps, uint32_t seed, unsigned long long path0, long long npaths,
                           short *ypaths, const double *x, double strike, double barrier, double disc, double *sums);
int opb_mt19937_raw(uint32_t seed, long long nstreams, int n, uint32_t *out);
int opb_mt_uniforms(uint32_t seed, long long nstreams, int nper, float *unif);

#ifdef __cplusplus
}
#endif

#endif /* OPCUDA_B200_H */
