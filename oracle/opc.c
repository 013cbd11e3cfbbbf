/*
 * CPU restatement of the reference's `opc` library.  TEST INFRASTRUCTURE ONLY: the CPU
 * oracle and baseline for the opc entry points (declared in opc.h), used by tests/, never
 * by the library.
 *
 * The reference's opc (oplib/opc/linalg.c, util.c, rangen.cpp) is a thin layer over Intel
 * MKL, which is absent here, so each entry point restates what it asks MKL for:
 *   - opc_sgemv/dgemv, opc_sgemm/dgemm, opc_dcopy: the reference BLAS definitions of
 *     xGEMV('N'), xGEMM('N','N') with alpha = 1, beta = 0, and DCOPY (column-major, BLAS
 *     increment convention, accumulation in the operands' precision, column by column);
 *   - opc_dgesv/sgesv: LAPACK xGESV = xGETRF (LU with partial pivoting: pivot = first
 *     entry of largest magnitude, 1-based ipiv, info = first exactly zero pivot) followed by
 *     xGETRS (row interchanges, unit-lower then upper triangular solves);
 *   - the random streams: MKL VSL's MT2203 family (one parameter set per thread, whose
 *     tables are not available) is replaced by one MT19937 per thread seeded with
 *     init_genrand(seed_th[th]); uniform bits are its genrand_int32 outputs in order.
 *     opc_genunif maps x to a + (b - a) * x * 2^-32 (the 32-bit mapping of the uniform
 *     method); opc_gennor inverts the normal CDF at (x + 1/2) * 2^-32 (an open interval, so
 *     both tails stay finite) -- Acklam's rational approximation refined by two Halley steps
 *     on erfc, accurate to a few ulps;
 *   - opc_dmc1 and the bracket table it reads (opc_host_mc_hash, the host code of
 *     oplib/opmodel/models/CModel Host Double.cs:403-458) step for step, quirks included:
 *     the bracket table's first column of cumulative rows is left unnormalised, and the
 *     sampler treats a bracket starting at 0 specially (oplib/opc/rangen.cpp:131-133).
 *
 * Compiled with -O2 -ffp-contract=off.
 */
#include "opc.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ BLAS level 1-3 */

#define GEMV_N_BODY(T)                                                                     \
    if (m < 0 || n < 0 || lda < (m > 1 ? m : 1) || incx == 0 || incy == 0) return;        \
    if (m == 0 || n == 0 || (alpha == 0 && beta == 1)) return;                             \
    long kx = incx > 0 ? 0 : -(long)(n - 1) * incx;                                        \
    long ky = incy > 0 ? 0 : -(long)(m - 1) * incy;                                        \
    if (beta != 1) {                                                                       \
        long iy = ky;                                                                      \
        for (int i = 0; i < m; i++, iy += incy) y[iy] = beta == 0 ? (T)0 : beta * y[iy];    \
    }                                                                                      \
    if (alpha == 0) return;                                                                \
    long jx = kx;                                                                          \
    for (int j = 0; j < n; j++, jx += incx) {                                              \
        const T t = alpha * x[jx];                                                         \
        const T *col = a + (long)lda * j;                                                  \
        long iy = ky;                                                                      \
        for (int i = 0; i < m; i++, iy += incy) y[iy] += t * col[i];                       \
    }

void opc_sgemv(int m, int n, float alpha, float *a, int lda, float *x, int incx, float beta, float *y, int incy) {
    GEMV_N_BODY(float)
}

void opc_dgemv(int m, int n, double alpha, double *a, int lda, double *x, int incx, double beta, double *y,
               int incy) {
    GEMV_N_BODY(double)
}

#define GEMM_NN_BODY(T)                                                                    \
    if (m < 0 || n < 0 || k < 0 || lda < (m > 1 ? m : 1) || ldb < (k > 1 ? k : 1) ||      \
        ldc < (m > 1 ? m : 1))                                                             \
        return;                                                                            \
    for (int j = 0; j < n; j++) {                                                          \
        T *cj = c + (long)ldc * j;                                                         \
        for (int i = 0; i < m; i++) cj[i] = 0;                                             \
        for (int p = 0; p < k; p++) {                                                      \
            const T t = b[p + (long)ldb * j];                                              \
            const T *ap = a + (long)lda * p;                                               \
            for (int i = 0; i < m; i++) cj[i] += t * ap[i];                                \
        }                                                                                  \
    }

void opc_sgemm(float *a, float *b, float *c, int lda, int ldb, int ldc, int m, int n, int k) { GEMM_NN_BODY(float) }

void opc_dgemm(double *a, double *b, double *c, int lda, int ldb, int ldc, int m, int n, int k) {
    GEMM_NN_BODY(double)
}

void opc_dcopy(int n, double *destination, double *source) {
    for (int i = 0; i < n; i++) destination[i] = source[i];
}

/* ------------------------------------------------------------------ LAPACK xGESV */

#define GESV_BODY(T, ABS)                                                                  \
    if (n < 0) return -1;                                                                  \
    if (nrhs < 0) return -2;                                                               \
    if (lda < (n > 1 ? n : 1)) return -4;                                                  \
    if (ldb < (n > 1 ? n : 1)) return -7;                                                  \
    int info = 0;                                                                          \
    /* xGETRF: right-looking LU with partial pivoting */                                   \
    for (int j = 0; j < n; j++) {                                                          \
        int p = j;                                                                         \
        T best = ABS(ap[j + (long)lda * j]);                                               \
        for (int i = j + 1; i < n; i++) {                                                  \
            T v = ABS(ap[i + (long)lda * j]);                                              \
            if (v > best) { best = v; p = i; }                                             \
        }                                                                                  \
        ipivp[j] = p + 1;                                                                  \
        if (ap[p + (long)lda * j] != 0) {                                                  \
            if (p != j)                                                                    \
                for (int q = 0; q < n; q++) {                                              \
                    T t = ap[j + (long)lda * q];                                           \
                    ap[j + (long)lda * q] = ap[p + (long)lda * q];                         \
                    ap[p + (long)lda * q] = t;                                             \
                }                                                                          \
            const T piv = ap[j + (long)lda * j];                                           \
            for (int i = j + 1; i < n; i++) ap[i + (long)lda * j] /= piv;                  \
        } else if (info == 0) {                                                            \
            info = j + 1;                                                                  \
        }                                                                                  \
        for (int q = j + 1; q < n; q++) {                                                  \
            const T u = ap[j + (long)lda * q];                                             \
            for (int i = j + 1; i < n; i++) ap[i + (long)lda * q] -= ap[i + (long)lda * j] * u; \
        }                                                                                  \
    }                                                                                      \
    if (info != 0) return info;                                                            \
    /* xGETRS: P, then L (unit lower), then U */                                           \
    for (int r = 0; r < nrhs; r++) {                                                       \
        T *x = bp + (long)ldb * r;                                                         \
        for (int i = 0; i < n; i++) {                                                      \
            int p = ipivp[i] - 1;                                                          \
            if (p != i) { T t = x[i]; x[i] = x[p]; x[p] = t; }                             \
        }                                                                                  \
        for (int q = 0; q < n; q++)                                                        \
            for (int i = q + 1; i < n; i++) x[i] -= ap[i + (long)lda * q] * x[q];          \
        for (int q = n - 1; q >= 0; q--) {                                                 \
            x[q] /= ap[q + (long)lda * q];                                                 \
            for (int i = 0; i < q; i++) x[i] -= ap[i + (long)lda * q] * x[q];              \
        }                                                                                  \
    }                                                                                      \
    return 0;

int opc_dgesv(int n, int nrhs, double *ap, int ma, int na, int lda, int *ipivp, double *bp, int ldb) {
    (void)ma;
    (void)na;
    GESV_BODY(double, fabs)
}

static int sgesv_impl(int n, int nrhs, float *ap, int lda, int *ipivp, float *bp, int ldb) { GESV_BODY(float, fabsf) }

int opc_sgesv(int n, int nrhs, float *ap, int ma, int na, int lda, int *ipivp, float *bp, int ldb, int *info) {
    (void)ma;
    (void)na;
    *info = sgesv_impl(n, nrhs, ap, lda, ipivp, bp, ldb);
    return *info;
}

/* ------------------------------------------------------------------ random streams */

#define OPC_E_STREAM (-1) /* th outside the initialised streams */

typedef struct {
    uint32_t mt[624];
    int mti;
} opc_stream;

static opc_stream *g_streams = NULL;
static int g_nth = 0;
static int g_status = 0;

static void stream_seed(opc_stream *s, uint32_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 624; i++) s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->mti = 624;
}

static uint32_t stream_next(opc_stream *s) {
    if (s->mti >= 624) {
        for (int i = 0; i < 624; i++) {
            uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % 624] & 0x7fffffffu);
            s->mt[i] = s->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        s->mti = 0;
    }
    uint32_t y = s->mt[s->mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* Thread th's stream; like the reference's VSL calls, every call records its status. */
static opc_stream *stream_of(int th) {
    if (!g_streams || th < 0 || th >= g_nth) {
        g_status = OPC_E_STREAM;
        return NULL;
    }
    g_status = 0;
    return &g_streams[th];
}

void opc_rangen_init_seed(unsigned int *seed_th, int nth) {
    free(g_streams);
    g_streams = NULL;
    g_nth = 0;
    if (nth < 1 || !seed_th) {
        g_status = OPC_E_STREAM;
        return;
    }
    g_streams = (opc_stream *)malloc(sizeof(opc_stream) * (size_t)nth);
    if (!g_streams) {
        g_status = OPC_E_STREAM;
        return;
    }
    for (int th = 0; th < nth; th++) stream_seed(&g_streams[th], seed_th[th]);
    g_nth = nth;
    g_status = 0;
}

int opc_rangen_getstatus(void) { return g_status; }

void opc_rangen_finalize(void) {
    free(g_streams);
    g_streams = NULL;
    g_nth = 0;
    g_status = 0;
}

void opc_genunif(double *r, int n, double a, double b, int th) {
    opc_stream *s = stream_of(th);
    if (!s) return;
    for (int i = 0; i < n; i++) r[i] = a + (b - a) * ((double)stream_next(s) * 2.3283064365386963e-10);
}

/* Phi^{-1}(p) for 0 < p <= 1/2: P. J. Acklam's rational approximation (relative error
 * below 1.2e-9), then two Halley steps on Phi(z) - p with Phi(z) = erfc(-z/sqrt 2)/2. */
static double inv_norm_lower(double p) {
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                                1.383577518672690e+02,  -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                                6.680131188771972e+01,  -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                -2.549732539343734e+00, 4.374664141464968e+00,  2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                3.754408661907416e+00};
    double z;
    if (p < 0.02425) {
        double q = sqrt(-2.0 * log(p));
        z = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    } else {
        double q = p - 0.5, r = q * q;
        z = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
            (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
    }
    for (int it = 0; it < 2; it++) {
        double e = 0.5 * erfc(-z * 0.70710678118654752440) - p;
        double u = e * 2.50662827463100050242 * exp(0.5 * z * z);
        z -= u / (1.0 + 0.5 * z * u);
    }
    return z;
}

static double inv_norm(double p) { return p <= 0.5 ? inv_norm_lower(p) : -inv_norm_lower(1.0 - p); }

void opc_gennor(double *r, int n, double mean, double sigma, int th) {
    opc_stream *s = stream_of(th);
    if (!s) return;
    for (int i = 0; i < n; i++) {
        double u = ((double)stream_next(s) + 0.5) * 2.3283064365386963e-10;
        r[i] = mean + sigma * inv_norm(u);
    }
}

typedef void (*opc_payoff_eval)(short *y_sk, int th, int batch);

int opc_dmc1(double *ctpker_yy_m, int *hash_ys_m, int d, int nscen_per_batch, int nk, int y0, unsigned int *unif_s,
             short *y_sk, int *m_k, unsigned long payoff_eval_ptr, int th, int b) {
    opc_stream *s = stream_of(th);
    if (!s) return g_status;
    const int niter = (int)(log((double)d) / log(2.0)) + 1;
    const long dd = (long)d * d;
    for (int k = 0; k < nk; k++) {
        for (int i = 0; i < nscen_per_batch; i++) unif_s[i] = stream_next(s);
        const long m = m_k[k];
        short *y_s = y_sk + (long)nscen_per_batch * k;
        const int *hash_ys = hash_ys_m + dd * m;
        const double *ctpker_yy = ctpker_yy_m + dd * m;
        for (int scen = 0; scen < nscen_per_batch; scen++) {
            const double rnd = (double)unif_s[scen] / 4294967296.0;
            const int yprev = k > 0 ? y_s[scen - nscen_per_batch] : y0;
            const int bucket = (int)(rnd * d);
            const int hash = hash_ys[yprev + (long)d * bucket];
            short ub = (short)(hash >> 16);
            short lb = (short)(hash - (ub << 16));
            if (lb == 0 && rnd < ctpker_yy[yprev]) ub = 0;
            if (ub - lb > 1) {
                const double *ctp = ctpker_yy + yprev;
                for (int iter = 0; iter < niter; iter++) {
                    const short ymid = (short)((ub + lb) / 2);
                    if (rnd < ctp[(long)d * ymid]) ub = ymid;
                    else lb = ymid;
                    if (ub - lb <= 1) break;
                }
            }
            y_s[scen] = ub;
        }
    }
    if (payoff_eval_ptr) ((opc_payoff_eval)payoff_eval_ptr)(y_sk, th, b);
    return 0;
}

int opc_mt_benchmark(int nscen_per_batch, float *unif_s, int th) {
    opc_stream *s = stream_of(th);
    if (!s) return 0;
    for (int i = 0; i < nscen_per_batch; i++) {
        const uint32_t x = stream_next(s);
        unif_s[i] = (float)x / 4294967296.0f;
    }
    return 0;
}

/* ------------------------------------------------------------------ host bracket table */

void opc_host_mc_hash(const double *tpk_yy_m, int d, int nm, double *ctpk_yy_m, int *hash_ys_m) {
    const long dd = (long)d * d;
    for (int m = 0; m < nm; m++) {
        const double *tpk = tpk_yy_m + dd * m;
        double *ctpk = ctpk_yy_m + dd * m;
        int *hash = hash_ys_m + dd * m;
        for (int y1 = 0; y1 < d; y1++) {
            double rcker = tpk[y1];
            ctpk[y1] = rcker;
            for (int y2 = 1; y2 < d; y2++) {
                rcker += tpk[y1 + (long)d * y2];
                ctpk[y1 + (long)d * y2] = rcker;
            }
            for (int y2 = 1; y2 < d; y2++) {
                double r = ctpk[y1 + (long)d * y2] / rcker;
                ctpk[y1 + (long)d * y2] = r > 1.0 ? 1.0 : r; /* Math.Min: NaN stays NaN */
            }
            int lb = 0, ub = 0;
            for (int s = 0; s < d; s++) {
                const double lo = (double)((float)s / (float)d);
                const double hi = (double)((float)(s + 1) / (float)d);
                for (; lb < d; lb++)
                    if (ctpk[y1 + (long)d * lb] > lo) break;
                if (lb > 0) lb -= 1;
                for (; ub < d; ub++)
                    if (ctpk[y1 + (long)d * ub] > hi) break;
                if (ub == d) ub -= 1;
                if (ctpk[y1 + (long)d * lb] >= 1) ub = lb;
                hash[y1 + (long)d * s] = lb + (ub << 16);
            }
        }
    }
}
