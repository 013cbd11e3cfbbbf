/*
 * CPU oracle, C part.  TEST INFRASTRUCTURE ONLY: used by tests/, by the smoke check and
 * by the CPU-baseline leg of bench.py, never by the library.
 *
 * Restates, from the published algorithms and the reference's call sites:
 *   - MT19937 (Matsumoto & Nishimura 1998; init_genrand / genrand_int32 of the 2002
 *     reference code).  The seeding recurrence is the one the reference's twisters use
 *     (oplib/opcuda/smc.cu:127-131).
 *   - the uniform conversion u = ((float)x + 1.0f) * 2^-32 (oplib/opcuda/smc.cu:329);
 *   - the inverse-CDF step "smallest y with u < C[y], capped at d-1"
 *     (oplib/opcuda/smc.cu:336-350);
 *   - the per-path step loop (oplib/opcuda/smc.cu:307-366, oplib/opc/rangen.cpp:117-150);
 *   - cumulative normalised rows with a sequential FP32 running sum
 *     (oplib/opcuda/sck.cu:43-84), negative entries taken as 0;
 *   - the CPU uniform benchmark (oplib/opc/rangen.cpp:157-175), with MT19937 standing in
 *     for MKL's MT2203.
 * Multi-threaded entry points split paths across POSIX threads like the reference's
 * CJobQueue splits batches across cores (oplib/opmodel/types/CJobQueue.cs:65-98).
 *
 * Compiled with -O2 -ffp-contract=off so no FMA contraction changes FP32 rounding.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MT_N 624
#define MT_M 397
#define MT_MATRIX_A 0x9908b0dfU
#define MT_UPPER 0x80000000U
#define MT_LOWER 0x7fffffffU

typedef struct {
    uint32_t mt[MT_N];
    int mti;
} mt_state;

/* init_genrand(seed) with key1 added to mt[1] before the recurrence continues from it
 * (key1 = 0: init_genrand itself).  The keyed form seeds the per-path generators of the
 * library's reference-facing Monte Carlo: path g of a 4096-stream seed table is keyed by
 * (seeds[g % 4096], g / 4096). */
static void mt_init_keyed(mt_state *s, uint32_t seed, uint32_t key1) {
    s->mt[0] = seed;
    for (int i = 1; i < MT_N; i++) {
        s->mt[i] = 1812433253U * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
        if (i == 1) s->mt[1] += key1;
    }
    s->mti = MT_N;
}

static void mt_init(mt_state *s, uint32_t seed) { mt_init_keyed(s, seed, 0u); }

static uint32_t mt_next(mt_state *s) {
    uint32_t y;
    if (s->mti >= MT_N) {
        int kk;
        for (kk = 0; kk < MT_N - MT_M; kk++) {
            y = (s->mt[kk] & MT_UPPER) | (s->mt[kk + 1] & MT_LOWER);
            s->mt[kk] = s->mt[kk + MT_M] ^ (y >> 1) ^ ((y & 1U) ? MT_MATRIX_A : 0U);
        }
        for (; kk < MT_N - 1; kk++) {
            y = (s->mt[kk] & MT_UPPER) | (s->mt[kk + 1] & MT_LOWER);
            s->mt[kk] = s->mt[kk + (MT_M - MT_N)] ^ (y >> 1) ^ ((y & 1U) ? MT_MATRIX_A : 0U);
        }
        y = (s->mt[MT_N - 1] & MT_UPPER) | (s->mt[0] & MT_LOWER);
        s->mt[MT_N - 1] = s->mt[MT_M - 1] ^ (y >> 1) ^ ((y & 1U) ? MT_MATRIX_A : 0U);
        s->mti = 0;
    }
    y = s->mt[s->mti++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680U;
    y ^= (y << 15) & 0xefc60000U;
    y ^= (y >> 18);
    return y;
}

void oracle_mt19937_outputs(uint32_t seed, int n, uint32_t *out) {
    mt_state s;
    mt_init(&s, seed);
    for (int i = 0; i < n; i++) out[i] = mt_next(&s);
}

void oracle_mt19937_outputs_keyed(uint32_t seed, uint32_t key1, int n, uint32_t *out) {
    mt_state s;
    mt_init_keyed(&s, seed, key1);
    for (int i = 0; i < n; i++) out[i] = mt_next(&s);
}

static inline float u_from_bits(uint32_t x) {
    volatile float f = (float)x;  /* keep the two FP32 roundings separate */
    f = f + 1.0f;
    return f * 2.3283064365386963e-10f; /* 2^-32, exact scaling */
}

float oracle_uniform_f32(uint32_t x) { return u_from_bits(x); }

static inline int search_row(const float *row, long stride, int d, float u) {
    /* smallest y with u < row[y*stride], capped at d-1 */
    int lo = 0, hi = d - 1; /* answer in [lo, hi] */
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (u < row[(long)mid * stride]) hi = mid; else lo = mid + 1;
    }
    return lo;
}

void oracle_sck_f32(const float *P, int d, int nrows, long row_stride, long col_stride, float *C) {
    for (int y = 0; y < nrows; y++) {
        const float *p = P + (long)y * row_stride;
        float *c = C + (long)y * row_stride;
        /* negative entries (rounding residue) count as 0 so rows are non-decreasing */
        float p0 = p[0] > 0.0f ? p[0] : 0.0f;
        volatile float acc = p0;
        c[0] = acc;
        for (int z = 1; z < d; z++) {
            float pz = p[(long)z * col_stride];
            pz = pz > 0.0f ? pz : 0.0f;
            acc = acc + pz;
            c[(long)z * col_stride] = acc;
        }
        float tot = acc;
        for (int z = 0; z < d; z++) {
            volatile float v = c[(long)z * col_stride] / tot;
            c[(long)z * col_stride] = v < 1.0f ? v : 1.0f;
        }
    }
}

typedef struct {
    const float *C;      /* cumulative rows, element (y1,y2) at y1*rs + y2*cs */
    long rs, cs;
    int d, y0, nsteps;
    uint32_t seed;
    const uint32_t *seeds; /* optional [4096] stream seeds: path g keyed (seeds[g % 4096], g / 4096) */
    uint64_t path0;
    long p_begin, p_end; /* path range relative to path0 */
    int16_t *ypaths;     /* optional: [path][step] */
    const double *x;     /* optional: node values for payoffs */
    double strike, barrier, disc;
    double sum_barrier, sum_asian;
} mc_job;

static void *mc_worker(void *arg) {
    mc_job *j = (mc_job *)arg;
    mt_state s;
    double sb = 0.0, sa = 0.0;
    for (long p = j->p_begin; p < j->p_end; p++) {
        const uint64_t g = j->path0 + (uint64_t)p;
        if (j->seeds) mt_init_keyed(&s, j->seeds[g & 4095u], (uint32_t)(g >> 12));
        else mt_init(&s, (uint32_t)(j->seed + (uint32_t)g));
        int y = j->y0;
        double xmin = 1e300, xsum = 0.0, xv = 0.0;
        for (int k = 0; k < j->nsteps; k++) {
            float u = u_from_bits(mt_next(&s));
            y = search_row(j->C + (long)y * j->rs, j->cs, j->d, u);
            if (j->ypaths) j->ypaths[p * (long)j->nsteps + k] = (int16_t)y;
            if (j->x) {
                xv = j->x[y];
                if (xv < xmin) xmin = xv;
                xsum += xv;
            }
        }
        if (j->x) {
            double pay = xv - j->strike;
            if (xmin > j->barrier && pay > 0.0) sb += j->disc * pay;
            double a = xsum / (double)j->nsteps - j->strike;
            if (a > 0.0) sa += j->disc * a;
        }
    }
    j->sum_barrier = sb;
    j->sum_asian = sa;
    return NULL;
}

/* Runs npaths paths (ids path0 .. path0+npaths-1) over nthreads POSIX threads.
 * Returns 0 on success.  sums[0] = sum of discounted barrier payoffs, sums[1] = Asian. */
static int mc_paths_run(const float *C, long rs, long cs, int d, int y0, uint32_t seed, const uint32_t *seeds,
                        uint64_t path0, long npaths, int nsteps, int16_t *ypaths,
                        const double *x, double strike, double barrier, double disc,
                        double *sums, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 1024) nthreads = 1024;
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    mc_job *jobs = (mc_job *)calloc((size_t)nthreads, sizeof(mc_job));
    if (!th || !jobs) { free(th); free(jobs); return -1; }
    long per = (npaths + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
        mc_job *j = &jobs[t];
        j->C = C; j->rs = rs; j->cs = cs; j->d = d; j->y0 = y0; j->nsteps = nsteps;
        j->seed = seed; j->seeds = seeds; j->path0 = path0;
        j->p_begin = (long)t * per;
        j->p_end = j->p_begin + per < npaths ? j->p_begin + per : npaths;
        if (j->p_begin > j->p_end) j->p_begin = j->p_end;
        j->ypaths = ypaths; j->x = x; j->strike = strike; j->barrier = barrier; j->disc = disc;
        pthread_create(&th[t], NULL, mc_worker, j);
    }
    double sb = 0.0, sa = 0.0;
    for (int t = 0; t < nthreads; t++) {
        pthread_join(th[t], NULL);
        sb += jobs[t].sum_barrier;
        sa += jobs[t].sum_asian;
    }
    sums[0] = sb;
    sums[1] = sa;
    free(th);
    free(jobs);
    return 0;
}

int oracle_mc_paths(const float *C, long rs, long cs, int d, int y0, uint32_t seed,
                    uint64_t path0, long npaths, int nsteps, int16_t *ypaths,
                    const double *x, double strike, double barrier, double disc,
                    double *sums, int nthreads) {
    return mc_paths_run(C, rs, cs, d, y0, seed, NULL, path0, npaths, nsteps, ypaths, x, strike, barrier, disc,
                        sums, nthreads);
}

/* The same paths with generators keyed from a 4096-entry stream seed table. */
int oracle_mc_paths_seeded(const float *C, long rs, long cs, int d, int y0, const uint32_t *seeds,
                           uint64_t path0, long npaths, int nsteps, int16_t *ypaths,
                           const double *x, double strike, double barrier, double disc,
                           double *sums, int nthreads) {
    if (!seeds) return -1;
    return mc_paths_run(C, rs, cs, d, y0, 0u, seeds, path0, npaths, nsteps, ypaths, x, strike, barrier, disc,
                        sums, nthreads);
}

typedef struct {
    uint32_t seed;
    long n_per, nbatches;
    float *out;
    double checksum;
} mtb_job;

static void *mtb_worker(void *arg) {
    mtb_job *j = (mtb_job *)arg;
    mt_state s;
    mt_init(&s, j->seed);
    double cs = 0.0;
    for (long b = 0; b < j->nbatches; b++) {
        for (long i = 0; i < j->n_per; i++)
            j->out[i] = (float)mt_next(&s) * 2.3283064365386963e-10f;
        cs += j->out[j->n_per - 1];
    }
    j->checksum = cs;
    return NULL;
}

/* CPU uniform-generation benchmark: each of nthreads threads fills n_per uniforms
 * (u = x/2^32 as float, oplib/opc/rangen.cpp:167-172) nbatches times. */
double oracle_mt_benchmark(long n_per, long nbatches, int nthreads, uint32_t seed) {
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    mtb_job *jobs = (mtb_job *)calloc((size_t)nthreads, sizeof(mtb_job));
    double cs = 0.0;
    for (int t = 0; t < nthreads; t++) {
        jobs[t].seed = seed + (uint32_t)t;
        jobs[t].n_per = n_per;
        jobs[t].nbatches = nbatches;
        jobs[t].out = (float *)malloc(sizeof(float) * (size_t)n_per);
        pthread_create(&th[t], NULL, mtb_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++) {
        pthread_join(th[t], NULL);
        cs += jobs[t].checksum;
        free(jobs[t].out);
    }
    free(th);
    free(jobs);
    return cs;
}
