/*
 * CPU restatement of the reference's `opc` library.  TEST INFRASTRUCTURE ONLY: the CPU
 * oracle and baseline for the opc entry points, used by tests/, never by the library.
 *
 * Same exported names, argument order and column-major semantics as the reference's
 * oplib/opc/linalg.c, util.c and rangen.cpp; Intel MKL, which those files call and which
 * is absent here, is replaced by plain C (BLAS/LAPACK) and by per-thread MT19937 streams
 * (the MKL VSL MT2203 family).  The reference builds the library with `__declspec(dllexport)`
 * emptied on Linux (-DLINUX); here every entry point is plain `extern "C"` visibility.
 */
#ifndef OPC_ORACLE_H
#define OPC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* oplib/opc/linalg.c:44-50: y = alpha*A*x + beta*y, A m x n column-major ('N') */
void opc_sgemv(int m, int n, float alpha, float *a, int lda, float *x, int incx, float beta, float *y, int incy);
/* oplib/opc/linalg.c:53-58 */
void opc_dgemv(int m, int n, double alpha, double *a, int lda, double *x, int incx, double beta, double *y,
               int incy);
/* oplib/opc/linalg.c:62-70: LU solve of A X = B (ma, na unused); returns LAPACK info */
int opc_dgesv(int n, int nrhs, double *ap, int ma, int na, int lda, int *ipivp, double *bp, int ldb);
/* oplib/opc/linalg.c:73-79: as opc_dgesv in FP32; info also stored at *info */
int opc_sgesv(int n, int nrhs, float *ap, int ma, int na, int lda, int *ipivp, float *bp, int ldb, int *info);
/* oplib/opc/linalg.c:82-90: C = A*B (m x k times k x n, column-major, alpha 1, beta 0) */
void opc_sgemm(float *a, float *b, float *c, int lda, int ldb, int ldc, int m, int n, int k);
/* oplib/opc/linalg.c:94-101 */
void opc_dgemm(double *a, double *b, double *c, int lda, int ldb, int ldc, int m, int n, int k);
/* oplib/opc/util.c:48-53: destination[i] = source[i], i < n */
void opc_dcopy(int n, double *destination, double *source);

/* oplib/opc/rangen.cpp:53-65: one generator per thread th, seeded seed_th[th] */
void opc_rangen_init_seed(unsigned int *seed_th, int nth);
/* oplib/opc/rangen.cpp:68-71: 0, or a negative code after a bad call */
int opc_rangen_getstatus(void);
/* oplib/opc/rangen.cpp:74-81 */
void opc_rangen_finalize(void);
/* oplib/opc/rangen.cpp:84-87: n normal deviates by inversion of the normal CDF */
void opc_gennor(double *r, int n, double mean, double sigma, int th);
/* oplib/opc/rangen.cpp:90-93: n uniforms on [a, b) */
void opc_genunif(double *r, int n, double a, double b, int th);
/* oplib/opc/rangen.cpp:97-153: one batch of the CPU Monte Carlo on double cumulative rows
 * with the host bracket table, then payoff_eval(y_sk, th, b) */
int opc_dmc1(double *ctpker_yy_m, int *hash_ys_m, int d, int nscen_per_batch, int nk, int y0, unsigned int *unif_s,
             short *y_sk, int *m_k, unsigned long payoff_eval_ptr, int th, int b);
/* oplib/opc/rangen.cpp:157-175: nscen_per_batch uniforms (float) of thread th's stream */
int opc_mt_benchmark(int nscen_per_batch, float *unif_s, int th);

/* Not an opc export: the host side that prepares opc_dmc1's inputs, restating
 * host_d_mc_hash (oplib/opmodel/models/CModel Host Double.cs:403-458): cumulative rows
 * and the d-bucket bracket table of nm column-major kernels. */
void opc_host_mc_hash(const double *tpk_yy_m, int d, int nm, double *ctpk_yy_m, int *hash_ys_m);

#ifdef __cplusplus
}
#endif

#endif
