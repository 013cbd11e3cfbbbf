// Markov-chain Monte Carlo on a lattice, driven by one MT19937 stream per path.
//
// Path p draws its uniforms from MT19937 seeded with init_genrand(seed + p) (Matsumoto &
// Nishimura 1998; the seeding recurrence 1812433253*(x ^ x>>30) + i is the one the
// reference's twisters use, oplib/opcuda/smc.cu:127-131) and consumes the first
// genrand_int32 outputs in order, one per step.  The reference-facing entry points seed
// from a table of 4096 stream seeds instead (opcuda_mc_setseed): path p is path p / 4096 of
// stream p % 4096, its generator MT19937 keyed by (seeds[p % 4096], p / 4096)
// (mt19937.cuh).  Each step converts the output to
// u = ((float)x + 1.0f) * 2^-32 in (0, 1] (oplib/opcuda/smc.cu:329) and moves to the
// smallest state z with u < C[y, z], capped at d-1 (oplib/opcuda/smc.cu:336-350).
//
// B200 design: one thread per path with the whole generator in registers for runs of up
// to 623 steps (mt19937_first in mt19937.cuh walks the seeding recurrence with a few
// cursors, no state array); longer runs (mt19937_any) take their first 623 outputs from
// the same cursors while storing the regenerated words in a per-thread 624-word
// local-memory array, which serves every later output.  They run in a separate
// instantiation of the same kernels, so the register-only one carries no stack frame.
// The inverse-CDF search starts from the guide-table bracket of the previous state's row
// (about one probe per step) and falls back to the full row without a guide table.
// Payoffs (discretely monitored down-and-out call, arithmetic-Asian call) are reduced per
// path in registers and per block in FP64; the optional int16 state output uses the
// reference's layout y_sk[path + npaths*k] (oplib/opcuda/smc.cu:331).
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "lattice.h"
#include "mt19937.cuh"

namespace opb {

// Stream seeds the reference-facing entry points take (the reference's MT_RNG_COUNT
// twisters, oplib/opcuda/smc.cu:98-101).
constexpr int kMcStreamsLog2 = 12;
constexpr int kMcStreams = 1 << kMcStreamsLog2;
// Status record: 4 header words, then the stream seeds.
constexpr int kMcStatusHeader = 4;

__device__ __forceinline__ float mt_uniform_open0(uint32_t x) {
    float f = __uint2float_rn(x);
    f = __fadd_rn(f, 1.0f);
    return __fmul_rn(f, 2.3283064365386963e-10f);  // * 2^-32, exact
}

struct McArgs {
    const float *C;          // cumulative rows, element (y, z) at y*rs + z*cs
    long long rs, cs;
    const int *m_k;          // optional: kernel index per step (matrix stride ms)
    long long ms;
    const uint32_t *guide;   // optional [d][nb] brackets (row-major rows only)
    int nb;
    int d, y0, nsteps;
    uint32_t seed;
    const uint32_t *seeds;   // optional [kMcStreams] stream seeds (replaces seed)
    unsigned long long path0;
    long long npaths;
    short *ypaths;           // optional, y[p + npaths*k]
    const double *x;         // optional node values (payoffs)
    double strike, barrier, disc;
    double *block_sums;      // [gridDim.x * 2]
    // device-side evaluator (EVAL): path value v = sum over steps k of cf[k*d + y_k] up to,
    // not including, the first step whose state is knocked out (ko[k*d + y_k] != 0)
    const double *cf;        // [nsteps][d] cashflow per step and state (discounting folded in)
    const unsigned char *ko; // optional [nsteps][d] knock-out flags
    double *pv;              // optional [npaths] path values
};

// EVAL: block sums are (sum v, sum v^2) of the evaluator's path values instead of the
// fused barrier / Asian payoffs.
template <bool ANY_LENGTH, bool EVAL = false>
__global__ void __launch_bounds__(256) k_mc(McArgs a) {
    double s_bar = 0.0, s_asi = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const float nbf = (float)a.nb;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < a.npaths; p += stride) {
        const unsigned long long g = a.path0 + (unsigned long long)p;
        uint32_t seed = a.seed + (uint32_t)g, key1 = 0u;
        if (a.seeds) {
            seed = __ldg(a.seeds + (g & (kMcStreams - 1)));
            key1 = (uint32_t)(g >> kMcStreamsLog2);
        }
        int y = a.y0;
        double xmin = 1e300, xsum = 0.0, xlast = 0.0;
        double v = 0.0;
        bool alive = true;
        mt19937_stream<ANY_LENGTH>(seed, key1, a.nsteps, [&](int k, uint32_t bits) {
            const float u = mt_uniform_open0(bits);
            const float *row = a.C + (long long)y * a.rs + (a.m_k ? (long long)__ldg(a.m_k + k) * a.ms : 0LL);
            int lo = 0, hi = a.d - 1;
            if (a.guide) {
                int bkt = (int)__fmul_rn(u, nbf);
                bkt = bkt < a.nb ? bkt : a.nb - 1;
                uint32_t g = __ldg(a.guide + (long long)y * a.nb + bkt);
                lo = (int)(g & 0xffffu);
                hi = (int)(g >> 16);
            }
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (u < __ldg(row + (long long)mid * a.cs)) hi = mid; else lo = mid + 1;
            }
            y = lo;
            if (a.ypaths) a.ypaths[p + a.npaths * (long long)k] = (short)y;
            if constexpr (EVAL) {
                const long long o = (long long)k * a.d + y;
                if (alive) {
                    if (a.ko && __ldg(a.ko + o)) alive = false;
                    else v += __ldg(a.cf + o);
                }
            } else if (a.x) {
                double xv = __ldg(a.x + y);
                xmin = xv < xmin ? xv : xmin;
                xsum += xv;
                xlast = xv;
            }
        });
        if constexpr (EVAL) {
            if (a.pv) a.pv[p] = v;
            s_bar += v;
            s_asi += v * v;
        } else if (a.x) {
            double pay = xlast - a.strike;
            if (xmin > a.barrier && pay > 0.0) s_bar += a.disc * pay;
            double avg = xsum / (double)a.nsteps - a.strike;
            if (avg > 0.0) s_asi += a.disc * avg;
        }
    }
    if (!a.block_sums) return;
    __shared__ double red[2][8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s_bar += __shfl_xor_sync(0xffffffffu, s_bar, o);
        s_asi += __shfl_xor_sync(0xffffffffu, s_asi, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = s_bar; red[1][w] = s_asi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) { t0 += red[0][i]; t1 += red[1][i]; }
        a.block_sums[2 * blockIdx.x] = t0;
        a.block_sums[2 * blockIdx.x + 1] = t1;
    }
}

// Deterministic final reduction of the per-block sums (fixed order, one block).
__global__ void k_reduce_pairs(int n, const double *__restrict__ in, double *__restrict__ out) {
    __shared__ double r0[256], r1[256];
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) { t0 += in[2 * i]; t1 += in[2 * i + 1]; }
    r0[threadIdx.x] = t0; r1[threadIdx.x] = t1;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { r0[threadIdx.x] += r0[threadIdx.x + s]; r1[threadIdx.x] += r1[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = r0[0]; out[1] = r1[0]; }
}

// Uniform-generation throughput kernel (the gmt workload): stream s of nstreams writes
// its first nper uniforms u = x * 2^-32 (oplib/opcuda/smc.cu:711-714) to
// unif[s + nstreams*j].  Stream s is seeded seeds[s] when a seed table is given (nstreams
// <= its length), else seed + s.
template <bool ANY_LENGTH>
__global__ void __launch_bounds__(256) k_mt_bench(uint32_t seed, const uint32_t *__restrict__ seeds,
                                                  long long nstreams, int nper, float *__restrict__ unif) {
    long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= nstreams) return;
    const uint32_t sd = seeds ? __ldg(seeds + s) : seed + (uint32_t)s;
    mt19937_stream<ANY_LENGTH>(sd, 0u, nper, [&](int j, uint32_t bits) {
        unif[s + nstreams * (long long)j] = __fmul_rn(__uint2float_rn(bits), 2.3283064365386963e-10f);
    });
}

// Raw outputs, for parity tests of the generator itself: out[s*n + j].
template <bool ANY_LENGTH>
__global__ void k_mt_raw(uint32_t seed, long long nstreams, int n, uint32_t *__restrict__ out) {
    long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= nstreams) return;
    mt19937_stream<ANY_LENGTH>(seed + (uint32_t)s, 0u, n, [&](int j, uint32_t bits) { out[s * n + j] = bits; });
}

// The register-only generator up to 623 steps, the cursor/state-array one beyond; the
// evaluator form when a cashflow table is given.
void launch_mc(int grid, const McArgs &a) {
    if (a.cf) {
        if (a.nsteps <= kMtCursorMax) k_mc<false, true><<<grid, 256, 0, stream()>>>(a);
        else k_mc<true, true><<<grid, 256, 0, stream()>>>(a);
    } else if (a.nsteps <= kMtCursorMax) {
        k_mc<false><<<grid, 256, 0, stream()>>>(a);
    } else {
        k_mc<true><<<grid, 256, 0, stream()>>>(a);
    }
}
void launch_mt_bench(int grid, uint32_t seed, const uint32_t *seeds, long long nstreams, int nper, float *unif) {
    if (nper <= kMtCursorMax) k_mt_bench<false><<<grid, 256, 0, stream()>>>(seed, seeds, nstreams, nper, unif);
    else k_mt_bench<true><<<grid, 256, 0, stream()>>>(seed, seeds, nstreams, nper, unif);
}

int mc_grid(long long npaths) {
    long long b = (npaths + 255) / 256;
    long long cap = 8LL * num_sms();  // 8 x 256 threads per SM resident
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace opb

using namespace opb;

// Monte Carlo over npaths paths with ids path0 .. path0+npaths-1.  C holds cumulative
// rows with element (y, z) at y*row_stride + z*col_stride (row_stride = d, col_stride = 1
// for source-major storage; 1 and d for the reference's column-major storage).  guide
// (optional, source-major rows only) is the opb_guide_table of C with nb buckets.
// ypaths (optional) receives int16 states y[p + npaths*k].  x (optional, d doubles)
// enables the fused payoffs; sums[0] / sums[1] receive the discounted barrier / Asian
// payoff sums.  scratch must hold 2*opb_mc_scratch_blocks(npaths) doubles.
OPB_API int opb_mc_scratch_blocks(long long npaths) { return mc_grid(npaths); }

OPB_API int opb_mc_mt19937(const float *C, long long row_stride, long long col_stride, const uint32_t *guide,
                           int nb, int d, int y0, int nsteps, uint32_t seed, unsigned long long path0,
                           long long npaths, short *ypaths, const double *x, double strike, double barrier,
                           double disc, double *scratch, double *sums) {
    OPB_NVTX("opb_mc_mt19937");
    OPB_REQUIRE(d > 0 && d <= 32767 && y0 >= 0 && y0 < d, OPB_E_ARG);
    OPB_REQUIRE(nsteps >= 1 && npaths >= 0, OPB_E_ARG);
    OPB_REQUIRE(C != nullptr, OPB_E_NULL);
    if (guide) OPB_REQUIRE(nb >= 1 && nb <= 4096 && (nb & (nb - 1)) == 0 && col_stride == 1, OPB_E_ARG);
    if (x) OPB_REQUIRE(scratch != nullptr && sums != nullptr, OPB_E_NULL);
    if (npaths == 0) {  // no paths: the payoff sums are zero
        if (x) OPB_TRY(cudaMemsetAsync(sums, 0, 2 * sizeof(double), stream()));
        return set_status(OPB_OK);
    }
    McArgs a{};
    a.C = C; a.rs = row_stride; a.cs = col_stride; a.guide = guide; a.nb = nb;
    a.d = d; a.y0 = y0; a.nsteps = nsteps; a.seed = seed; a.path0 = path0; a.npaths = npaths;
    a.ypaths = ypaths; a.x = x; a.strike = strike; a.barrier = barrier; a.disc = disc;
    a.block_sums = x ? scratch : nullptr;
    int grid = mc_grid(npaths);
    launch_mc(grid, a);
    if (x) k_reduce_pairs<<<1, 256, 0, stream()>>>(grid, scratch, sums);
    return launch_check();
}

// The same paths as opb_mc_mt19937 evaluated on the device by a cashflow table instead of
// the fused payoffs: path value v_p = sum_k cashflow[k*d + y_k] over the steps before the
// first knocked-out state (knockout[k*d + y_k] != 0; knockout optional).  path_values
// (optional) receives v_p for each path, sums[0] / sums[1] the sum of v_p and of v_p^2
// (fixed-order FP64 reductions).  This replaces the host round trip of the reference's
// evaluator callback (oplib/opmodel/models/CModel Device.cs:352-364,
// oplib/opmodel/interfaces/CMCEvaluator.cs:41-67) for payoffs that are sums of per-date
// cashflows with discrete knock-out.  scratch: 2*opb_mc_scratch_blocks(npaths) doubles.
OPB_API int opb_mc_mt19937_eval(const float *C, long long row_stride, long long col_stride, const uint32_t *guide,
                                int nb, int d, int y0, int nsteps, uint32_t seed, unsigned long long path0,
                                long long npaths, short *ypaths, const double *cashflow,
                                const unsigned char *knockout, double *path_values, double *scratch, double *sums) {
    OPB_NVTX("opb_mc_mt19937_eval");
    OPB_REQUIRE(d > 0 && d <= 32767 && y0 >= 0 && y0 < d, OPB_E_ARG);
    OPB_REQUIRE(nsteps >= 1 && npaths >= 0, OPB_E_ARG);
    OPB_REQUIRE(C != nullptr && cashflow != nullptr && scratch != nullptr && sums != nullptr, OPB_E_NULL);
    if (guide) OPB_REQUIRE(nb >= 1 && nb <= 4096 && (nb & (nb - 1)) == 0 && col_stride == 1, OPB_E_ARG);
    if (npaths == 0) {
        OPB_TRY(cudaMemsetAsync(sums, 0, 2 * sizeof(double), stream()));
        return set_status(OPB_OK);
    }
    McArgs a{};
    a.C = C; a.rs = row_stride; a.cs = col_stride; a.guide = guide; a.nb = nb;
    a.d = d; a.y0 = y0; a.nsteps = nsteps; a.seed = seed; a.path0 = path0; a.npaths = npaths;
    a.ypaths = ypaths; a.cf = cashflow; a.ko = knockout; a.pv = path_values; a.block_sums = scratch;
    const int grid = mc_grid(npaths);
    launch_mc(grid, a);
    k_reduce_pairs<<<1, 256, 0, stream()>>>(grid, scratch, sums);
    return launch_check();
}

OPB_API int opb_mt19937_raw(uint32_t seed, long long nstreams, int n, uint32_t *out) {
    OPB_REQUIRE(nstreams >= 0 && n >= 1, OPB_E_ARG);
    if (nstreams == 0) return set_status(OPB_OK);
    OPB_REQUIRE(out != nullptr, OPB_E_NULL);
    const int grid = (int)((nstreams + 255) / 256);
    if (n <= kMtCursorMax) k_mt_raw<false><<<grid, 256, 0, stream()>>>(seed, nstreams, n, out);
    else k_mt_raw<true><<<grid, 256, 0, stream()>>>(seed, nstreams, n, out);
    return launch_check();
}

// ---------------------------------------------------------------- reference MC entry points
//
// The reference keeps 4096 MT607 twister states in a device buffer between calls, each
// seeded from one of 4096 host seeds (oplib/opcuda/smc.cu:118-156, 610-656); twister r
// draws its paths one after another.  Here the status buffer holds a continuation record
// and the seed table instead: word 0 = seeds[0], words 1-2 = the next path id (64-bit),
// word 3 = 0, words 4 .. 4099 = the 4096 stream seeds.  Path g (counted over all calls
// since opcuda_mc_setseed) is path g / 4096 of stream g % 4096, with its own MT19937 keyed
// by (seeds[g % 4096], g / 4096), so every path can run on its own thread; successive
// opcuda_mc1f calls continue with fresh paths, which keeps the reference's "successive
// batches continue the same streams" contract.  Paths 0 .. 4095 are init_genrand(seeds[g]).

OPB_API int opcuda_mc_nrng(void) { return kMcStreams; }                        // stream seeds setseed reads
OPB_API int opcuda_mc_status_sz(void) { return kMcStatusHeader + kMcStreams; }  // int32 words of the record

// Accepted for ABI compatibility: MT19937 needs no per-stream parameter file
// (the reference's MersenneTwister.dat, oplib/opcuda/smc.cu:87-96).
OPB_API int opcuda_mc_load_mt_gpu(const char *MT_stream, long sz) {
    (void)MT_stream;
    (void)sz;
    return set_status(OPB_OK);
}

// host_seedptr: host array of opcuda_mc_nrng() = 4096 uint32 stream seeds (the
// reference's layout).  mtptr: device status buffer of opcuda_mc_status_sz() words.
OPB_API int opcuda_mc_setseed(uint64_t host_seedptr, uint64_t mtptr) {
    OPB_REQUIRE(host_seedptr != 0 && mtptr != 0, OPB_E_NULL);
    std::vector<uint32_t> rec(kMcStatusHeader + kMcStreams, 0u);
    const uint32_t *seeds = reinterpret_cast<const uint32_t *>(host_seedptr);
    std::copy(seeds, seeds + kMcStreams, rec.begin() + kMcStatusHeader);
    rec[0] = seeds[0];
    OPB_TRY(cudaMemcpyAsync(reinterpret_cast<void *>(mtptr), rec.data(), rec.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, stream()));
    OPB_TRY(cudaStreamSynchronize(stream()));
    return set_status(OPB_OK);
}

// Semantics of oplib/opcuda/smc.cu:610-656 with per-path MT19937: nscen paths of nk
// steps from state y0 over the column-major cumulative kernels ctpker_m_yy (kernel m_k[k]
// at step k), writing int16 states y_sk[p + nscen*k] and copying them to yhostptr
// (blocking, as the reference does).  Unlike the reference (d < 1024 only,
// smc.cu:622) any d <= 32767 is accepted, and any nk >= 1.
OPB_API int opcuda_mc1f(uint64_t mtptr, int y0, uint64_t y_sk, int nscen, int nk, int d, uint64_t ctpker_m_yy,
                        uint64_t m_k, uint64_t yhostptr) {
    OPB_NVTX("opcuda_mc1f");
    OPB_REQUIRE(mtptr != 0 && y_sk != 0 && ctpker_m_yy != 0 && m_k != 0, OPB_E_NULL);
    OPB_REQUIRE(d > 0 && d <= 32767 && y0 >= 0 && y0 < d && nscen >= 0, OPB_E_ARG);
    OPB_REQUIRE(nk >= 1, OPB_E_ARG);
    uint32_t rec[4];
    OPB_TRY(cudaMemcpyAsync(rec, reinterpret_cast<const void *>(mtptr), sizeof(rec), cudaMemcpyDeviceToHost, stream()));
    OPB_TRY(cudaStreamSynchronize(stream()));
    unsigned long long path0 = (unsigned long long)rec[1] | ((unsigned long long)rec[2] << 32);
    if (nscen > 0) {
        McArgs a{};
        a.C = reinterpret_cast<const float *>(ctpker_m_yy);
        a.rs = 1; a.cs = d; a.m_k = reinterpret_cast<const int *>(m_k); a.ms = (long long)d * d;
        a.d = d; a.y0 = y0; a.nsteps = nk; a.path0 = path0; a.npaths = nscen;
        a.seeds = reinterpret_cast<const uint32_t *>(mtptr) + kMcStatusHeader;
        a.ypaths = reinterpret_cast<short *>(y_sk);
        launch_mc(mc_grid(nscen), a);
        OPB_TRY(cudaGetLastError());
    }
    path0 += (unsigned long long)nscen;
    rec[1] = (uint32_t)(path0 & 0xffffffffull);
    rec[2] = (uint32_t)(path0 >> 32);
    OPB_TRY(cudaMemcpyAsync(reinterpret_cast<void *>(mtptr), rec, sizeof(rec), cudaMemcpyHostToDevice, stream()));
    if (yhostptr != 0 && nscen > 0)
        OPB_TRY(cudaMemcpyAsync(reinterpret_cast<void *>(yhostptr), reinterpret_cast<const void *>(y_sk),
                                sizeof(short) * (size_t)nscen * nk, cudaMemcpyDeviceToHost, stream()));
    OPB_TRY(cudaStreamSynchronize(stream()));
    return set_status(OPB_OK);
}

// opcuda_mc1f with the evaluator on the device: the same paths (continuing the status
// record), each valued by the cashflow table as in opb_mc_mt19937_eval, results[p] the
// value of path p of this call.  y_sk (optional, 0 for none) still receives the states; no
// host copy of them is made.  Blocking, as opcuda_mc1f is.  It stands for the
// reference's opcuda_mc1f + evaluator.eval(y_host) pair (oplib/opmodel/models/CModel
// Device.cs:343-364): the evaluator becomes a table, the states need not leave the device.
OPB_API int opcuda_mc1f_eval(uint64_t mtptr, int y0, uint64_t y_sk, int nscen, int nk, int d, uint64_t ctpker_m_yy,
                             uint64_t m_k, uint64_t cashflow, uint64_t knockout, uint64_t results) {
    OPB_NVTX("opcuda_mc1f_eval");
    OPB_REQUIRE(mtptr != 0 && ctpker_m_yy != 0 && m_k != 0 && cashflow != 0 && results != 0, OPB_E_NULL);
    OPB_REQUIRE(d > 0 && d <= 32767 && y0 >= 0 && y0 < d && nscen >= 0, OPB_E_ARG);
    OPB_REQUIRE(nk >= 1, OPB_E_ARG);
    uint32_t rec[4];
    OPB_TRY(cudaMemcpyAsync(rec, reinterpret_cast<const void *>(mtptr), sizeof(rec), cudaMemcpyDeviceToHost, stream()));
    OPB_TRY(cudaStreamSynchronize(stream()));
    unsigned long long path0 = (unsigned long long)rec[1] | ((unsigned long long)rec[2] << 32);
    if (nscen > 0) {
        McArgs a{};
        a.C = reinterpret_cast<const float *>(ctpker_m_yy);
        a.rs = 1; a.cs = d; a.m_k = reinterpret_cast<const int *>(m_k); a.ms = (long long)d * d;
        a.d = d; a.y0 = y0; a.nsteps = nk; a.path0 = path0; a.npaths = nscen;
        a.seeds = reinterpret_cast<const uint32_t *>(mtptr) + kMcStatusHeader;
        a.ypaths = reinterpret_cast<short *>(y_sk);
        a.cf = reinterpret_cast<const double *>(cashflow);
        a.ko = reinterpret_cast<const unsigned char *>(knockout);
        a.pv = reinterpret_cast<double *>(results);
        launch_mc(mc_grid(nscen), a);
        OPB_TRY(cudaGetLastError());
    }
    path0 += (unsigned long long)nscen;
    rec[1] = (uint32_t)(path0 & 0xffffffffull);
    rec[2] = (uint32_t)(path0 >> 32);
    OPB_TRY(cudaMemcpyAsync(reinterpret_cast<void *>(mtptr), rec, sizeof(rec), cudaMemcpyHostToDevice, stream()));
    OPB_TRY(cudaStreamSynchronize(stream()));
    return set_status(OPB_OK);
}

// Uniform throughput benchmark (oplib/opcuda/smc.cu:664-736): nscen uniforms from the
// 4096 streams of the status record, nscen/4096 values each, stream s an MT19937 seeded
// init_genrand(seeds[s]) (the reference's twister s seeded seed[s]).
OPB_API int opcuda_mt_benchmark(uint64_t mtptr, uint64_t unif_ptr, int nscen) {
    OPB_REQUIRE(mtptr != 0 && unif_ptr != 0, OPB_E_NULL);
    OPB_REQUIRE(nscen >= 0 && nscen % kMcStreams == 0, OPB_E_ARG);
    int nper = nscen / kMcStreams;
    if (nper == 0) return set_status(OPB_OK);
    launch_mt_bench(kMcStreams / 256, 0u, reinterpret_cast<const uint32_t *>(mtptr) + kMcStatusHeader, kMcStreams,
                    nper, reinterpret_cast<float *>(unif_ptr));
    return launch_check();
}

// Uniform generation with typed pointers: nstreams streams (seed + s) x nper values.
OPB_API int opb_mt_uniforms(uint32_t seed, long long nstreams, int nper, float *unif) {
    OPB_REQUIRE(nstreams >= 0 && nper >= 1, OPB_E_ARG);
    if (nstreams == 0) return set_status(OPB_OK);
    OPB_REQUIRE(unif != nullptr, OPB_E_NULL);
    launch_mt_bench((int)((nstreams + 255) / 256), seed, nullptr, nstreams, nper, unif);
    return launch_check();
}

// ---------------------------------------------------------------- allocation-free variant
//
// Some callers cannot let a library allocate device memory: a host framework that owns
// the whole device-memory budget and hands libraries only the buffers it has accounted
// for (a managed P/Invoke pricing engine is the typical case), or a latency-critical
// pricing loop that cannot afford cudaMalloc's implicit device-wide synchronisation.
// opb_mc_mt19937_noalloc serves them: it is opb_mc_mt19937 without the scratch argument.
// The per-block payoff partial sums live in a fixed file-scope device array of
// OPB_MC_NOALLOC_MAX_BLOCKS x 2 doubles (64 KiB), which every GPU that loads the library
// keeps until the process exits.  The grid is the one opb_mc_mt19937 uses for the same
// npaths (at most 8 blocks per SM), so results are bit-identical to it; a grid larger than
// the array -- only possible on a device with more than 512 SMs -- is rejected with
// OPB_E_UNSUPPORTED.  Runs longer than 623 steps are rejected with OPB_E_UNSUPPORTED too:
// opb_mc_mt19937 serves them with a per-thread local-memory state array, and the CUDA
// driver may grow its local-memory reservation for that kernel on first use, an allocation
// this entry point exists to avoid.  All calls share the array and it keeps the last call's contents (each
// call overwrites the partials of the blocks it launches before reading them), so calls
// that overlap on the GPU -- concurrent streams, or several host threads -- race on it and
// must be serialised by the caller.
//
// Host code cannot use the array's name as a device address, so the device address is
// looked up with cudaGetSymbolAddress once per device, with that device current, by the
// first call made on that device (whatever its arguments); make that first call before any
// stream capture.  The address is kept for the life of the process: after cudaDeviceReset
// (a new primary context) it no longer belongs to the array, so this entry point must not
// be used on a device after that device has been reset.

#define OPB_MC_NOALLOC_MAX_BLOCKS 4096

static __device__ __align__(256) double g_mc_noalloc_scratch[2 * OPB_MC_NOALLOC_MAX_BLOCKS];

namespace {

std::mutex g_noalloc_mu;
double *g_noalloc_ptr[64] = {nullptr};

int noalloc_scratch(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= 64) return OPB_E_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_mc_noalloc_scratch);
        if (e != cudaSuccess) return (int)e;
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return OPB_OK;
}

}  // namespace

OPB_API int opb_mc_mt19937_noalloc(const float *C, long long row_stride, long long col_stride,
                                   const uint32_t *guide, int nb, int d, int y0, int nsteps, uint32_t seed,
                                   unsigned long long path0, long long npaths, short *ypaths, const double *x,
                                   double strike, double barrier, double disc, double *sums) {
    OPB_NVTX("opb_mc_mt19937_noalloc");
    OPB_REQUIRE(nsteps <= kMtCursorMax, OPB_E_UNSUPPORTED);
    OPB_REQUIRE(npaths >= 0, OPB_E_ARG);
    OPB_REQUIRE(mc_grid(npaths) <= OPB_MC_NOALLOC_MAX_BLOCKS, OPB_E_UNSUPPORTED);
    // the address is looked up on the first call on a device even when this call needs no
    // partial sums (x == NULL), so that the lookup never falls inside a later stream capture
    double *scratch = nullptr;
    int r = noalloc_scratch(&scratch);
    if (r != OPB_OK) return set_status(r);
    if (!x) scratch = nullptr;
    return opb_mc_mt19937(C, row_stride, col_stride, guide, nb, d, y0, nsteps, seed, path0, npaths, ypaths, x,
                          strike, barrier, disc, scratch, sums);
}
