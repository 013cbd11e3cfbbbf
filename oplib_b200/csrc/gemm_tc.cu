// Split-BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   C[M,N] = alpha * (Ahi.Bhi^T + Ahi.Blo^T + Alo.Bhi^T) + beta * Cin[M,N]
//
// A = Ahi + Alo and B = Bhi + Blo are FP32 matrices split into two BF16 parts
// (hi = bf16(a), lo = bf16(a - hi)); the three products carry about 16 mantissa bits per
// operand and accumulate in FP32 in tensor memory.  This replaces the FP32 SIMT squaring
// of oplib/opcuda/ssqmm.cu:119-179 on the lattice path.  A is K-major (rows contiguous);
// B is K-major (rows of B^T contiguous) or, for the lattice's squaring and chain
// products, K x N row-major and read as an MN-major operand (64-column TMA boxes), so a
// squaring reads E's own row-major parts as B.  M % 128 == 0, N % BN == 0, K % 64 == 0.
//
// Structure (persistent: one CTA per SM over 128 x BN output tiles):
//   TMA warp, one lane : 4 tiled bulk-tensor loads per K-block (Ahi, Alo, Bhi, Blo; 128B
//                        swizzle; no multicast) into a STAGES-deep ring, completion
//                        tracked by mbarrier transaction counts.
//   MMA warp, one lane : per 16-wide K step three tcgen05.mma.kind::f16 (BF16 x BF16 ->
//                        FP32) into one of two TMEM accumulators (BN columns each), one
//                        accumulator per chunk of 2 K-blocks; tcgen05.commit releases
//                        each stage and hands each finished chunk to the epilogue.
//   epilogue warps     : (4 lane quadrants x BN/128 column groups) tcgen05.ld of each
//                        finished chunk into FP32 round-to-nearest register sums; after a
//                        tile's last chunk, the alpha/beta update (with the deferred
//                        renormalisation of Cin, when given), FP32 stores staged through
//                        shared memory in 32 x 32 blocks, and FP64 row sums of the
//                        stored values (rowsum[group * M + row], one per 128 columns,
//                        used by the row renormalisation).
// CTA pairs (the default for M % 256 == 0 with 256-wide tiles): a 2-CTA cluster owns a
// 256 x 256 output tile; each CTA loads its own 128 rows of A and 128 columns of B (3-stage
// 64 KB ring per CTA, both CTAs' copies counted on the even CTA's full barrier), the even
// CTA's MMA lane issues tcgen05.mma.cta_group::2 (M = 256) over both CTAs' shared memory
// into each CTA's own TMEM, and its commits arrive on both CTAs' barriers.  Operand bytes
// through shared memory per MMA flop drop by a third against one CTA per 128 x 256 tile.
// The tensor cores truncate their FP32 accumulator (about half an ulp per MMA); chunked
// accumulation bounds that bias by 24 MMAs instead of 3K/16.
// Every mbarrier wait is bounded by a %globaltimer deadline; on expiry the kernel records
// an error code in g_tc_error, drains its outstanding copies and MMAs, frees TMEM and
// returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cstring>
#include <mutex>

#include "common.cuh"
#include "lattice.h"

namespace opb {

__device__ int g_tc_error = 0;

constexpr int TC_BM = 128;
constexpr int TC_BK = 64;  // K granularity of the operands (64 bf16 = 128 bytes = one 128B swizzle row)
constexpr unsigned long long TC_WAIT_NS = 4000000000ull;  // 4 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: true when the phase completed, false on timeout or abort.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                          unsigned long long limit_ns) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (true) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if (gtimer() - t0 > limit_ns) return false;
    }
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major swizzled UMMA shared-memory descriptor for tiles whose rows are BK bf16 wide:
// BK = 64 -> 128-byte swizzle (8-row core groups 1024 bytes apart), BK = 32 -> 64-byte
// swizzle (512 bytes apart).  LBO is unused for swizzled K-major (1); version 1 (sm_100).
template <int BK>
__device__ __forceinline__ uint64_t umma_desc_sw(uint32_t saddr) {
    static_assert(BK == 64 || BK == 32, "BK");
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;                   // LBO
    d |= (uint64_t)((8 * BK * 2) >> 4) << 32;  // SBO: 8 rows of BK * 2 bytes
    d |= (uint64_t)1 << 46;                   // version
    d |= (uint64_t)(BK == 64 ? 2 : 4) << 61;  // SWIZZLE_128B / SWIZZLE_64B
    return d;
}

// MN-major 128-byte-swizzled descriptor for a B tile stored K x N (N contiguous) as
// 64-column boxes of BK rows: each box is BK rows of 128 bytes (8-row swizzle atoms 1024
// bytes apart: SBO), and the boxes along N are BK * 128 bytes apart (LBO).
template <int BK>
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t saddr) {
    static_assert(BK == 64 || BK == 32, "BK");
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((BK * 128) >> 4) << 16;  // LBO: next 64 columns
    d |= (uint64_t)(1024 >> 4) << 32;  // SBO: next 8 rows of K
    d |= (uint64_t)1 << 46;            // version
    d |= (uint64_t)2 << 61;            // SWIZZLE_128B
    return d;
}

// kind::f16 instruction descriptor: D = F32, A = B = BF16 (format 1) or F16 (format 0),
// A K-major, B K-major or (bmn) MN-major, N, M (128 for one CTA, 256 for a CTA pair).
__host__ __device__ constexpr uint32_t umma_idesc_16(int n, bool f16, int m = TC_BM, bool bmn = false) {
    return (1u << 4) | ((f16 ? 0u : 1u) << 7) | ((f16 ? 0u : 1u) << 10) | ((bmn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// ---- CTA-pair (cta_group::2) forms: one 256 x N MMA over the shared memory of both CTAs
// of a 2-CTA cluster, issued by the even CTA; each CTA's tensor memory holds its 128 rows.
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Address of the same shared variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t map_to_rank(uint32_t saddr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Arrive without release semantics: for signals that order only tcgen05 work the arriving
// thread has already waited for (TMEM loads completed by tcgen05.wait::ld and fenced by
// tcgen05.fence::before_thread_sync), so that the arrive does not wait for the thread's
// outstanding global stores (the output phase of the previous tile).
__device__ __forceinline__ void mbar_arrive_remote_relaxed(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.relaxed.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
// Tiled load into this CTA's shared memory whose completion is counted on an mbarrier
// that may live in the peer CTA (the pair leader's).  No multicast.
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap *map, uint32_t bar_cluster, int x,
                                                 int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_cluster), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void umma_bf16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive on the mbarrier at this offset in both CTAs of the pair once the pair's MMAs
// issued so far have completed.
__device__ __forceinline__ void umma_commit_pair(uint32_t bar) {
    const uint16_t mask = 3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
        "h"(mask)
        : "memory");
}

// Bulk prefetch of bytes (a multiple of 16) at a 16-byte aligned global address into L2.
__device__ __forceinline__ void prefetch_l2(const void *ptr, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(ptr), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// GELU(z) = z Phi(z), Phi(z) = 0.5 (1 + erf(z / sqrt 2)), with erf from Abramowitz & Stegun,
// Handbook of Mathematical Functions, formula 7.1.26 (|error| <= 1.5e-7): for x >= 0,
// erf(x) = 1 - q(t) exp(-x^2), t = 1 / (1 + p x), q(t) = a1 t + ... + a5 t^5.  With
// h = q(t) exp(-x^2) / 2 at x = |z| / sqrt 2, Phi(z) = 1 - h for z >= 0 and h for z < 0 (no
// cancellation in the negative tail).  Folded for the epilogue's instruction count: 1/sqrt 2
// into p, the halving into the a_i, exp(-x^2) = 2^(z^2 (-log2(e) / 2)); one reciprocal and
// one exponential on the XU pipe, nine FMA-pipe instructions.  The error is far below the
// BF16 rounding of the stored activations.
__device__ __forceinline__ float gelu_as(float z) {
    constexpr float P = 0.3275911f * 0.70710678118654752f;
    constexpr float A1 = 0.5f * 0.254829592f, A2 = 0.5f * -0.284496736f, A3 = 0.5f * 1.421413741f,
                    A4 = 0.5f * -1.453152027f, A5 = 0.5f * 1.061405429f;
    const float t = rcp_approx(fmaf(P, fabsf(z), 1.0f));
    float q = fmaf(t, A5, A4);
    q = fmaf(t, q, A3);
    q = fmaf(t, q, A2);
    q = fmaf(t, q, A1);
    const float h = q * t * ex2_approx(z * z * -0.72134752044448170f);  // -log2(e) / 2
    return z * (z >= 0.f ? 1.f - h : h);
}

template <int BN, int STAGES, int NPROD = 3, int BK = TC_BK, bool PAIR = false, int EPIMODE = 0>
struct TcCfg {
    static constexpr int CPT_MAX = EPIMODE ? TC_LAYER_CPT : 128;
    static constexpr int A_BYTES = TC_BM * BK * 2;                  // one of Ahi/Alo
    static constexpr int B_ROWS = PAIR ? BN / 2 : BN;               // B rows held by this CTA
    static constexpr int B_BYTES = B_ROWS * BK * 2;                 // one of Bhi/Blo
    static constexpr int TILE_M = PAIR ? 2 * TC_BM : TC_BM;         // output rows per work item
    static constexpr int NPARTS = NPROD == 1 ? 1 : 2;  // parts loaded per operand
    // network layers (single products with one column tile, K <= 256): the whole B, the
    // layer's weights, stays resident in shared memory, loaded once per CTA, and the stage
    // ring carries A alone -- each 128-row tile then moves 64 KB from L2 instead of 192 KB
    static constexpr bool BRES = NPROD == 1 && EPIMODE != 0 && !PAIR;
    static constexpr int BRES_KB = BRES ? 256 / BK : 0;           // resident K-blocks of B
    static constexpr int STAGE_BYTES = BRES ? A_BYTES : NPARTS * (A_BYTES + B_BYTES);
    static constexpr int RING_BYTES = STAGES * STAGE_BYTES + BRES_KB * B_BYTES;
    static constexpr int CPT = BN < CPT_MAX ? BN : CPT_MAX;  // accumulator columns per epilogue thread
    static constexpr int HALVES = BN / CPT;                 // column groups per TMEM lane
    static constexpr int EPI_WARPS = 4 * HALVES;            // epilogue warps (4 lane quadrants x groups)
    // FP32 output: each epilogue warp transposes 32 x 32 blocks through shared memory
    // (row stride 33 words) so that Cin loads and C stores are whole 128-byte lines.
    // Network layers (EPIMODE 1): each warp stages its 32 rows x CPT/2 BF16 activations
    // (row stride CPT + 16 bytes) so that its global stores cover 64-byte row segments
    static constexpr int OUT_BYTES =
        EPIMODE == 0 ? EPI_WARPS * 32 * 33 * 4 : EPIMODE == 1 ? EPI_WARPS * 32 * (CPT + 16) : 0;
    // network layers: the tile's bias (and output weights) staged in shared memory once
    static constexpr int VEC_BYTES = EPIMODE ? 2 * BN * 4 : 0;
    static constexpr int SMEM = RING_BYTES + 1024 /*align*/ + 256 /*barriers*/ + OUT_BYTES + VEC_BYTES;
    static constexpr int THREADS = 32 * (EPI_WARPS + 2);    // + TMA producer warp + MMA warp
    static constexpr int TMEM_COLS = 2 * BN;                // two accumulators (ping-pong chunks)
    // K-blocks accumulated in TMEM per chunk: K = 128 for the split products (bounds the
    // tensor cores' truncation); the whole K for single BF16 products (network layers,
    // whose BF16 outputs do not need it)
    static constexpr int CHUNK = NPROD == 1 ? (1 << 20) : 128 / BK;
};

struct TcParams {
    int M, N, K;
    float *C;
    long long ldc;
    const float *Cin;
    float alpha, beta;
    double *rowsum;
    // EPIMODE == 1 (network layer): H = GELU(alpha * acc + bias[col]) stored as BF16
    const float *bias;
    __nv_bfloat16 *H;
    long long ldh;
    // EPIMODE == 2 (last hidden layer + output layer): ypart[g * M + row] =
    // sum over the columns of group g of bf16(GELU(alpha * acc + bias)) * w5[col]
    const float *w5;
    float *ypart;
    int group_m;  // M-tiles per raster group of a single product (0: 8)
    const double2 *cin_fix;  // as TcGemmArgs::cin_fix
    int ksplit;              // as TcGemmArgs::ksplit (single products; 0 or 1: none)
    long long c_slice;       // elements between the K-slices' partial outputs
    const int *band;         // as TcGemmArgs::band (single products; batched: TcProblem::band)
    int level;               // as TcGemmArgs::level
    int lolo;                // as TcGemmArgs::lolo
    int band_skip;           // as TcGemmArgs::band_skip
    int fixmode;             // as TcGemmArgs::fixmode
    __nv_bfloat16 *Shi, *Slo;  // as TcGemmArgs::Shi / Slo (single products; batched: TcProblem)
    float sscale;            // as TcGemmArgs::sscale
};

// K-blocks [kb_lo, kb_lo + nkb) that can contribute to the output tile rows [m0, m0 + tm),
// columns [n0, n0 + tn) of A.B when A and B are both zero outside the band |row - col| <= h:
// k must lie within h of some row and of some column.  The range is widened to whole
// accumulation chunks (chunk K-blocks each, counted from K = 0), so every chunk that is
// issued holds the same K-blocks as in the full product and the sums are bit-identical;
// the chunks left out hold only exact-zero products.  h < 0: the whole K range.
__device__ __forceinline__ void band_kblocks(long long h, int m0, int tm, int n0, int tn, int K, int bk, int chunk,
                                             int &kb_lo, int &nkb) {
    const int nkb_all = K / bk;
    if (h < 0 || h >= K) {
        kb_lo = 0;
        nkb = nkb_all;
        return;
    }
    const long long lo = (long long)max(m0, n0) - h;
    const long long hi = (long long)min(m0 + tm - 1, n0 + tn - 1) + h;
    if (lo > hi || hi < 0 || lo >= K) {
        kb_lo = 0;
        nkb = 0;
        return;
    }
    const int span = bk * chunk;
    const int c_lo = (int)(max(lo, 0LL) / span);
    const int c_hi = (int)(min(hi, (long long)K - 1) / span) + 1;
    kb_lo = c_lo * chunk;
    nkb = min(c_hi * chunk, nkb_all) - kb_lo;
}

// Half-bandwidth of the operands at squaring level `level` when the generator's is h0
// (E_0 = dt L has L's band; each squaring at most doubles it); -1: no band (dense).
__device__ __forceinline__ long long level_band(int h0, int level) {
    if (h0 < 0) return -1;
    if (level >= 40) return 1LL << 40;
    return (long long)h0 << level;
}

// Batched launches read per-problem tensor maps (4 per problem: Ahi, Alo, Bhi, Blo) and
// parameters from device tables and walk a work list of packed items
// (problem << 16 | m-tile << 8 | n-tile).
struct TcBatch {
    const CUtensorMap *maps;
    const TcProblem *probs;
    const uint32_t *work;
    int nwork;
};

// Persistent kernel: one CTA per SM walks the work items t = blockIdx.x + i*gridDim.x
// (single problem: its tiles in grouped raster, 8 M-tiles per group; batched: the work
// list).  The K loop of an item runs in chunks of CHUNK K-blocks; chunk g accumulates in
// TMEM accumulator g&1 starting from zero, and the epilogue warps add each finished chunk
// into FP32 register sums (round to nearest) while the MMA warp fills the other
// accumulator.  The tensor cores' truncating accumulation thus spans only 12*CHUNK MMA
// instructions, and an item's final store overlaps the next item's MMAs.
// FUSE (split products, EPIMODE 0): 0 = FP32 output (+ Cin, OPB_FIX_CIN); 1 = squaring with
// its output's parts (Shi / Slo) and OPB_FIX_SQUARE; 2 = parts only (C optional), no Cin,
// OPB_FIX_ROWSCALE.  Separate instantiations keep each epilogue's registers to its own work.
template <int BN, int STAGES, bool BATCHED, bool F16, int NPROD = 3, int EPIMODE = 0, int BK = TC_BK,
          bool PAIR = false, bool BMN = false, int FUSE = 0>
__global__ void __launch_bounds__(TcCfg<BN, STAGES, NPROD, BK, PAIR, EPIMODE>::THREADS, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
              const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo, TcParams p,
              TcBatch bt) {
    // network layers (EPIMODE >= 1) run twice the epilogue warps: their per-element GELU,
    // not the MMAs, bounds a tile
    using Cfg = TcCfg<BN, STAGES, NPROD, BK, PAIR, EPIMODE>;
    constexpr int EPI = Cfg::EPI_WARPS;
    constexpr int CPT = Cfg::CPT;
    static_assert(!BMN || (NPROD == 3 && Cfg::B_ROWS % 64 == 0), "MN-major B: split products");
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t *gbase = smem_raw + (base - raw);
    static_assert(!(Cfg::BRES && BATCHED), "resident B: single products");
    static_assert(2 * STAGES + 8 <= 32, "barrier slots");
    uint64_t *bars = reinterpret_cast<uint64_t *>(gbase + Cfg::RING_BYTES);
    const uint32_t bar0 = smem_u32(bars);
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (STAGES + s); };
    auto accf_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + a); };      // MMA -> epilogue
    auto acce_bar = [&](int a) { return bar0 + 8u * (2 * STAGES + 2 + a); };  // epilogue -> MMA
    const uint32_t drain_bar = bar0 + 8u * (2 * STAGES + 4);
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bars + 2 * STAGES + 5);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 2 * STAGES + 6);
    const uint32_t bres_bar = bar0 + 8u * (2 * STAGES + 7);        // resident B loaded
    const uint32_t bres_base = base + STAGES * Cfg::STAGE_BYTES;   // resident B, K-block kb at + kb * B_BYTES

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mtiles = p.M / Cfg::TILE_M, ntiles_n = p.N / BN;
    const int nsplit = (!BATCHED && p.ksplit > 1) ? p.ksplit : 1;  // K-slices of a single product
    const int nitems = BATCHED ? bt.nwork : mtiles * ntiles_n * nsplit;
    // pair mode: rank within the 2-CTA cluster, items walked per cluster
    const uint32_t rank = PAIR ? cluster_rank() : 0u;
    const int item0 = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const int istep = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;
    // item t -> (problem, m0, n0, K-blocks, first K-block, K-slice); a single product split
    // into nsplit K-slices has nsplit consecutive items per output tile
    auto get_item = [&](int t, int &prob, int &m0, int &n0, int &nkb, int &kb0, int &slice) {
        if constexpr (BATCHED) {
            const uint32_t w = bt.work[t];
            prob = (int)(w >> 16);
            m0 = (int)((w >> 8) & 255u) * Cfg::TILE_M;  // pair mode: 256-row items
            n0 = (int)(w & 255u) * BN;
            const TcProblem &pr = bt.probs[prob];
            const long long h = (pr.band > 0 && p.band_skip) ? level_band(pr.band, p.level) : -1;
            band_kblocks(h, m0, Cfg::TILE_M, n0, BN, pr.K, BK, Cfg::CHUNK, kb0, nkb);
            slice = 0;
        } else {
            slice = t % nsplit;
            t /= nsplit;
            const int GM = p.group_m > 0 ? p.group_m : 8;
            const int per_group = GM * ntiles_n;
            const int group = t / per_group;
            const int first_m = group * GM;
            const int gm = min(mtiles - first_m, GM);
            const int r = t - group * per_group;
            prob = 0;
            m0 = (first_m + r % gm) * Cfg::TILE_M;
            n0 = (r / gm) * BN;
            nkb = p.K / BK / nsplit;
            kb0 = slice * nkb;
            if (p.band && p.band_skip && nsplit == 1) {
                const int h0 = *p.band;
                band_kblocks(h0 > 0 ? level_band(h0, p.level) : -1, m0, Cfg::TILE_M, n0, BN, p.K, BK, Cfg::CHUNK,
                             kb0, nkb);
            }
        }
    };
    // the fourth split product lo.lo, on the launches that ask for it (p.lolo), and there
    // only while the operands are still banded (twice the band below the size), when the
    // band is known; the batched launches decide per problem
    auto item_lolo = [&](int prob) -> bool {
        if (NPROD != 3 || !p.lolo) return false;
        int h0 = -1, K = p.K;
        if constexpr (BATCHED) {
            h0 = bt.probs[prob].band;
            K = bt.probs[prob].K;
        } else if (p.band) {
            h0 = *p.band;
        }
        return h0 <= 0 || 2 * level_band(h0, p.level) < K;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(accf_bar(a), 1);
            mbar_init(acce_bar(a), PAIR ? 2 * EPI : EPI * 32);  // pair: one lane per epilogue warp of both CTAs
        }
        mbar_init(drain_bar, 1);
        if constexpr (Cfg::BRES) mbar_init(bres_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        const uint32_t slot = smem_u32(const_cast<uint32_t *>(tmem_slot));
        if constexpr (PAIR) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                         "r"(Cfg::TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                         "r"(Cfg::TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
    }
    // network layers with one column tile (N == BN, every layer of the surrogate): the bias
    // and output weights are read from shared memory in the epilogue, not from L1/L2 on the
    // dependent path of every element
    float *svec = reinterpret_cast<float *>(gbase + Cfg::RING_BYTES + 256 + Cfg::OUT_BYTES);
    const bool vec_smem = EPIMODE != 0 && p.N == BN;
    if (vec_smem) {
        for (int i = threadIdx.x; i < BN; i += blockDim.x) {
            svec[i] = p.bias[i];
            if (EPIMODE == 2) svec[BN + i] = p.w5[i];
        }
    }
    tc_fence_before();
    __syncthreads();
    if constexpr (PAIR) cluster_sync_all();  // both CTAs' barriers initialised before any cross-CTA signal
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == EPI) {
        if (lane == 0) {
            // ---------------- TMA producer
            long kbg = 0;  // K-blocks issued over the CTA's lifetime (stage ring position)
            bool ok = true;
            if constexpr (Cfg::BRES) {
                // every item's B is the whole weight matrix (N == BN, K <= 256): load it once
                if (item0 < nitems) {
                    const int nkb_all = p.K / BK;
                    mbar_expect_tx(bres_bar, (uint32_t)(nkb_all * Cfg::B_BYTES));
                    for (int kb = 0; kb < nkb_all; kb++)
                        tma_load_2d(bres_base + kb * Cfg::B_BYTES, &mBhi, bres_bar, kb * BK, 0);
                }
            }
            for (int t = item0; t < nitems && ok; t += istep) {
                int prob, m0, n0, nkb, kb0, slice;
                get_item(t, prob, m0, n0, nkb, kb0, slice);
                const int ma = m0 + (int)rank * TC_BM;          // this CTA's A rows
                const int nb = n0 + (int)rank * Cfg::B_ROWS;    // this CTA's B rows
                const CUtensorMap *mp[4] = {&mAhi, &mAlo, &mBhi, &mBlo};
                if constexpr (BATCHED) {
                    for (int i = 0; i < 4; i++) mp[i] = bt.maps + 4 * prob + i;
                }
                for (int kb = 0; kb < nkb; kb++, kbg++) {
                    const int s = (int)(kbg % STAGES);
                    if (kbg >= STAGES &&
                        !mbar_wait(empty_bar(s), (uint32_t)(((kbg / STAGES) + 1) & 1), abort_flag, TC_WAIT_NS)) {
                        ok = false;
                        break;
                    }
                    const uint32_t st = base + s * Cfg::STAGE_BYTES;
                    const int kx = (kb0 + kb) * BK;
                    if constexpr (PAIR) {
                        // both CTAs' copies complete on the leader's full barrier
                        if (rank == 0) mbar_expect_tx(full_bar(s), 2 * Cfg::STAGE_BYTES);
                        const uint32_t fb = map_to_rank(full_bar(s), 0);
                        tma_load_2d_pair(st, mp[0], fb, kx, ma);
                        tma_load_2d_pair(st + Cfg::A_BYTES, mp[1], fb, kx, ma);
                        if constexpr (BMN) {
#pragma unroll
                            for (int i = 0; i < Cfg::B_ROWS / 64; i++) {
                                tma_load_2d_pair(st + 2 * Cfg::A_BYTES + i * (BK * 128), mp[2], fb, nb + 64 * i, kx);
                                tma_load_2d_pair(st + 2 * Cfg::A_BYTES + Cfg::B_BYTES + i * (BK * 128), mp[3], fb,
                                                 nb + 64 * i, kx);
                            }
                        } else {
                            tma_load_2d_pair(st + 2 * Cfg::A_BYTES, mp[2], fb, kx, nb);
                            tma_load_2d_pair(st + 2 * Cfg::A_BYTES + Cfg::B_BYTES, mp[3], fb, kx, nb);
                        }
                    } else {
                        mbar_expect_tx(full_bar(s), Cfg::STAGE_BYTES);
                        tma_load_2d(st, mp[0], full_bar(s), kx, ma);
                        if constexpr (Cfg::BRES) {
                            // B is resident
                        } else if constexpr (NPROD == 1) {
                            tma_load_2d(st + Cfg::A_BYTES, mp[2], full_bar(s), kx, nb);
                        } else {
                            tma_load_2d(st + Cfg::A_BYTES, mp[1], full_bar(s), kx, ma);
                            if constexpr (BMN) {
#pragma unroll
                                for (int i = 0; i < Cfg::B_ROWS / 64; i++) {
                                    tma_load_2d(st + 2 * Cfg::A_BYTES + i * (BK * 128), mp[2], full_bar(s),
                                                nb + 64 * i, kx);
                                    tma_load_2d(st + 2 * Cfg::A_BYTES + Cfg::B_BYTES + i * (BK * 128), mp[3],
                                                full_bar(s), nb + 64 * i, kx);
                                }
                            } else {
                                tma_load_2d(st + 2 * Cfg::A_BYTES, mp[2], full_bar(s), kx, nb);
                                tma_load_2d(st + 2 * Cfg::A_BYTES + Cfg::B_BYTES, mp[3], full_bar(s), kx, nb);
                            }
                        }
                    }
                }
            }
            if (!ok) {
                atomicExch(&g_tc_error, 1);
                *abort_flag = 1;
                // wait (bounded) for the copies in flight; in pair mode they complete on the
                // leader's barriers, and the closing cluster barrier keeps this CTA resident
                // until the leader has drained them
                const long first = kbg > STAGES ? kbg - STAGES : 0;
                if (!PAIR || rank == 0)
                    for (long k = first; k < kbg; k++)
                        (void)mbar_wait(full_bar((int)(k % STAGES)), (uint32_t)((k / STAGES) & 1), abort_flag,
                                        100000000ull);
            }
        }
        __syncwarp();
    } else if (warp == EPI + 1) {
        if (lane == 0 && rank == 0) {
            // ---------------- MMA issuer (pair mode: the even CTA issues for both)
            const uint32_t idesc = umma_idesc_16(BN, F16, Cfg::TILE_M, BMN);
            long kbg = 0, g = 0;  // K-blocks consumed, chunks issued
            bool ok = true;
            if constexpr (Cfg::BRES) {
                if (item0 < nitems) {
                    ok = mbar_wait(bres_bar, 0u, abort_flag, TC_WAIT_NS);
                    tc_fence_after();
                }
            }
            for (int t = item0; t < nitems && ok; t += istep) {
                int prob, m0, n0, nkb, kb0, slice;
                get_item(t, prob, m0, n0, nkb, kb0, slice);
                const bool lolo = item_lolo(prob);
                const int nch = (nkb + Cfg::CHUNK - 1) / Cfg::CHUNK;
                for (int c = 0; c < nch && ok; c++, g++) {
                    const int a = (int)(g & 1);
                    if (g >= 2 && !mbar_wait(acce_bar(a), (uint32_t)(((g >> 1) + 1) & 1), abort_flag, TC_WAIT_NS)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t dacc = tmem + (uint32_t)(a * BN);
                    const int kb_end = min(nkb, (c + 1) * Cfg::CHUNK);
                    for (int kb = c * Cfg::CHUNK; kb < kb_end; kb++, kbg++) {
                        const int s = (int)(kbg % STAGES);
                        if (!mbar_wait(full_bar(s), (uint32_t)((kbg / STAGES) & 1), abort_flag, TC_WAIT_NS)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t st = base + s * Cfg::STAGE_BYTES;
                        const uint64_t dAh = umma_desc_sw<BK>(st);
                        const uint64_t dAl = umma_desc_sw<BK>(st + Cfg::A_BYTES);
                        const uint32_t sBh = Cfg::BRES ? bres_base + (uint32_t)((kb0 + kb) * Cfg::B_BYTES)
                                                       : st + Cfg::NPARTS * Cfg::A_BYTES;
                        const uint32_t sBl = st + 2 * Cfg::A_BYTES + Cfg::B_BYTES;
                        const uint64_t dBh = BMN ? umma_desc_mn<BK>(sBh) : umma_desc_sw<BK>(sBh);
                        const uint64_t dBl = BMN ? umma_desc_mn<BK>(sBl) : umma_desc_sw<BK>(sBl);
#pragma unroll
                        for (int k16 = 0; k16 < BK / 16; k16++) {
                            const uint64_t adv = (uint64_t)((k16 * 32) >> 4);  // +32 bytes along K
                            // MN-major B: +16 rows of 128 bytes along K
                            const uint64_t advb = BMN ? (uint64_t)((k16 * 16 * 128) >> 4) : adv;
                            const uint32_t acc0 = (kb > c * Cfg::CHUNK || k16 > 0) ? 1u : 0u;
                            if constexpr (PAIR) {
                                umma_bf16_pair(dacc, dAh + adv, dBh + advb, idesc, acc0);
                                umma_bf16_pair(dacc, dAh + adv, dBl + advb, idesc, 1u);
                                umma_bf16_pair(dacc, dAl + adv, dBh + advb, idesc, 1u);
                                if (lolo) umma_bf16_pair(dacc, dAl + adv, dBl + advb, idesc, 1u);
                            } else {
                                umma_bf16(dacc, dAh + adv, dBh + advb, idesc, acc0);
                                if constexpr (NPROD == 3) {
                                    umma_bf16(dacc, dAh + adv, dBl + advb, idesc, 1u);
                                    umma_bf16(dacc, dAl + adv, dBh + advb, idesc, 1u);
                                    if (lolo) umma_bf16(dacc, dAl + adv, dBl + advb, idesc, 1u);
                                }
                            }
                        }
                        if constexpr (PAIR) umma_commit_pair(empty_bar(s));
                        else umma_commit(empty_bar(s));
                    }
                    if (ok) {
                        if constexpr (PAIR) umma_commit_pair(accf_bar(a));
                        else umma_commit(accf_bar(a));
                    }
                }
            }
            if (!ok) {
                atomicExch(&g_tc_error, 2);
                *abort_flag = 1;
            }
            // arrives once every issued MMA has completed
            if constexpr (PAIR) umma_commit_pair(drain_bar);
            else umma_commit(drain_bar);
            (void)mbar_wait(drain_bar, 0, abort_flag, TC_WAIT_NS);
        }
        __syncwarp();
    } else {
        // ---------------- epilogue warps: lane quadrant q, column group h
        const int q = warp & 3, h = warp >> 2;
        const uint32_t lane_base = (uint32_t)(q * 32) << 16;
        float sum[CPT];
        long g = 0;
        bool ok = true;
        for (int t = item0; t < nitems && ok; t += istep) {
            int prob, m0, n0, nkb, kb0, slice;
            get_item(t, prob, m0, n0, nkb, kb0, slice);
            const int nch = (nkb + Cfg::CHUNK - 1) / Cfg::CHUNK;
            if constexpr (NPROD != 1) {  // single products have one chunk: its values are the sums
#pragma unroll
                for (int j = 0; j < CPT; j++) sum[j] = 0.f;
            }
            // this thread's Cin row segment is prefetched into L2 about three chunks before
            // the output needs it
            const float *pf = nullptr;
            long long pf_ld = 0;
            // a batched item's last column tile may overhang its matrix (zero B columns
            // beyond N): this thread's column group then has nothing to store
            const bool group_in = !BATCHED || n0 + h * CPT < bt.probs[prob].N;
            if constexpr (EPIMODE == 0) {
                if constexpr (BATCHED) {
                    pf = group_in ? bt.probs[prob].Cin : nullptr;
                    pf_ld = bt.probs[prob].ldc;
                } else {
                    pf = p.Cin;
                    pf_ld = p.ldc;
                }
            }
            const int pf_chunk = nch > 3 ? nch - 3 : 0;
            for (int c = 0; c < nch; c++, g++) {
                const int a = (int)(g & 1);
                if (pf && c == pf_chunk)
                    prefetch_l2(pf + (long long)(m0 + (int)rank * TC_BM + q * 32 + lane) * pf_ld + n0 + h * CPT,
                                CPT * 4);
                if (!mbar_wait(accf_bar(a), (uint32_t)((g >> 1) & 1), abort_flag, TC_WAIT_NS)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t tacc = tmem + lane_base + (uint32_t)(a * BN + h * CPT);
#pragma unroll
                for (int j = 0; j < CPT / 16; j++) {
                    uint32_t v[16];
                    tmem_ld16(tacc + (uint32_t)(16 * j), v);
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        if constexpr (NPROD == 1)
                            sum[16 * j + i] = __uint_as_float(v[i]);
                        else
                            sum[16 * j + i] = __fadd_rn(sum[16 * j + i], __uint_as_float(v[i]));
                    }
                }
                tc_fence_before();
                if constexpr (PAIR) {
                    __syncwarp();
                    if (lane == 0) mbar_arrive_remote_relaxed(map_to_rank(acce_bar(a), 0));
                } else {
                    asm volatile("mbarrier.arrive.relaxed.cta.shared::cta.b64 _, [%0];" ::"r"(acce_bar(a)) : "memory");
                }
            }
            if (!ok || *abort_flag) break;
            if (!group_in) continue;
            float *C;
            const float *Cin;
            long long ldc;
            float alpha, beta;
            double *rowsum;
            const double2 *fix;
            __nv_bfloat16 *Shi, *Slo;  // optional 16-bit parts of the stored values
            int M;
            if constexpr (BATCHED) {
                const TcProblem &pr = bt.probs[prob];
                C = pr.C; Cin = pr.Cin; ldc = pr.ldc; alpha = pr.alpha; beta = pr.beta; rowsum = pr.rowsum; M = pr.M;
                fix = pr.cin_fix; Shi = pr.Shi; Slo = pr.Slo;
            } else {
                C = p.C ? p.C + (long long)slice * p.c_slice : nullptr;  // K-slices write separate partials
                Cin = p.Cin; ldc = p.ldc; alpha = p.alpha; beta = p.beta; rowsum = p.rowsum; M = p.M;
                fix = p.cin_fix; Shi = p.Shi; Slo = p.Slo;
            }
            const int fm = fix ? (p.fixmode ? p.fixmode : OPB_FIX_CIN) : OPB_FIX_NONE;
            const int row = m0 + (int)rank * TC_BM + q * 32 + lane;
            const int col0 = n0 + h * CPT;
            if constexpr (EPIMODE == 0) {
                if (nch == 0 && C && Cin == C) {
                    // a tile that no K-block reaches (outside twice the operands' band): the
                    // product is zero there, and C, updated in place, is zero there too and
                    // keeps its values; only the row-sum partial is written
                    if (rowsum) rowsum[(long long)(col0 / CPT) * M + row] = 0.0;
                    continue;
                }
            }
            if constexpr (EPIMODE == 1) {
                // network layer: BF16 GELU(alpha * acc + bias) in two halves of CPT/2 columns.
                // Lane = row while the values are in the accumulator layout, so each lane
                // writes its row segment to the warp's staging rows (stride RS, conflict-free
                // 16-byte stores); read back, lane l stores row 8i + l/4, 16-byte chunk l%4:
                // every global store of the warp covers eight whole 64-byte row segments,
                // where stores straight from the accumulator layout touched 32 rows each
                const float4 *b4 = reinterpret_cast<const float4 *>((vec_smem ? svec - n0 : p.bias) + col0);
                constexpr int HC = CPT / 2, RS = HC * 2 + 16;
                static_assert(HC == 32, "four 16-byte chunks per staged row segment");
                uint8_t *stg = gbase + Cfg::RING_BYTES + 256 + warp * (32 * RS);
                const int rb = m0 + (int)rank * TC_BM + q * 32;
#pragma unroll
                for (int hh = 0; hh < 2; hh++) {
#pragma unroll
                    for (int j = 0; j < HC; j += 8) {
                        const int jj = hh * HC + j;
                        const float4 ba = b4[jj / 4], bb = b4[jj / 4 + 1];
                        const float bv[8] = {ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, bb.z, bb.w};
                        uint32_t pk[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            const __nv_bfloat162 h2 =
                                __floats2bfloat162_rn(gelu_as(fmaf(alpha, sum[jj + 2 * u], bv[2 * u])),
                                                      gelu_as(fmaf(alpha, sum[jj + 2 * u + 1], bv[2 * u + 1])));
                            pk[u] = *reinterpret_cast<const uint32_t *>(&h2);
                        }
                        *reinterpret_cast<uint4 *>(stg + lane * RS + j * 2) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    }
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const int r = i * 8 + (lane >> 2), c = lane & 3;
                        const uint4 v = *reinterpret_cast<const uint4 *>(stg + r * RS + c * 16);
                        *reinterpret_cast<uint4 *>(p.H + (long long)(rb + r) * p.ldh + col0 + hh * HC + c * 8) = v;
                    }
                    __syncwarp();
                }
                continue;
            }
            if constexpr (EPIMODE == 2) {
                // last hidden layer fused with the output layer: partial dot over this
                // thread's columns of the BF16-rounded activations
                const float4 *b4 = reinterpret_cast<const float4 *>((vec_smem ? svec - n0 : p.bias) + col0);
                const float4 *w4 = reinterpret_cast<const float4 *>((vec_smem ? svec + BN - n0 : p.w5) + col0);
                float acc = 0.f;
#pragma unroll
                for (int j = 0; j < CPT; j += 4) {
                    const float4 bv = b4[j / 4], wv = w4[j / 4];
                    const __nv_bfloat162 h01 = __floats2bfloat162_rn(gelu_as(fmaf(alpha, sum[j], bv.x)),
                                                                     gelu_as(fmaf(alpha, sum[j + 1], bv.y)));
                    const __nv_bfloat162 h23 = __floats2bfloat162_rn(gelu_as(fmaf(alpha, sum[j + 2], bv.z)),
                                                                     gelu_as(fmaf(alpha, sum[j + 3], bv.w)));
                    const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
                    acc = fmaf(f01.x, wv.x, acc);
                    acc = fmaf(f01.y, wv.y, acc);
                    acc = fmaf(f23.x, wv.z, acc);
                    acc = fmaf(f23.y, wv.w, acc);
                }
                p.ypart[(long long)(col0 / CPT) * p.M + row] = acc;
                continue;
            }
            // FP32 output in 32 x 32 blocks: the warp's rows (lane = row while the values are
            // in the accumulator layout) are staged in shared memory and read back so that
            // lane l handles row 4i + l/8, columns 4(l%8)..+3 of the block: every Cin load and
            // C store of the warp covers four whole 128-byte lines.  The FP64 row sum keeps
            // its order (float4 groups in column order): each group sum is parked in the
            // first two words of its group's slots (read by this lane alone) and the row's
            // lane adds them up.
            float *st = reinterpret_cast<float *>(gbase + Cfg::RING_BYTES + 256) + warp * (32 * 33);
            const int rbase = m0 + (int)rank * TC_BM + q * 32;
            const int tr = lane >> 3, tc4 = (lane & 7) * 4;
            double rs = 0.0;
#pragma unroll
            for (int j = 0; j < CPT / 32; j++) {
#pragma unroll
                for (int c = 0; c < 32; c++) st[lane * 33 + c] = sum[32 * j + c];
                // deferred squaring: the column terms s_j of this lane's four columns
                float sj[4] = {0.f, 0.f, 0.f, 0.f};
                if constexpr (FUSE == 1) {
                    if (fm == OPB_FIX_SQUARE) {
#pragma unroll
                        for (int u = 0; u < 4; u++) sj[u] = (float)fix[col0 + 32 * j + tc4 + u].x;
                    }
                }
                __syncwarp();
                // each half block's Cin loads are issued before any of its stores (with Cin = C
                // each element is read and then written by this lane alone), so that four
                // line-sized loads per warp are in flight at once
#pragma unroll
                for (int hb = 0; hb < 2; hb++) {
                    float4 cv[4];
                    if (FUSE != 2 && Cin) {
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            cv[i] = *reinterpret_cast<const float4 *>(
                                Cin + (long long)(rbase + 4 * (4 * hb + i) + tr) * ldc + col0 + 32 * j + tc4);
                    }
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const int rr = 4 * (4 * hb + i) + tr;
                        const int grow = rbase + rr, gcol = col0 + 32 * j + tc4;
                        float o[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) o[u] = alpha * st[rr * 33 + tc4 + u];
                        if constexpr (FUSE == 1) {
                            // squaring with the parts of its output: alpha acc + beta E', and with
                            // the previous level's normalisation deferred here (OPB_FIX_SQUARE):
                            // inv_i [alpha acc + (beta - s_i - s_j) E'_ij + (s_i^2 - beta s_i) [i == j]]
                            // in FP32 (s ~ 1e-5: the products with s are far below an ulp of the
                            // result's terms' rounding; inv's own rounding scales a whole row, which
                            // the next level's row sums renormalise)
                            const float c4[4] = {cv[i].x, cv[i].y, cv[i].z, cv[i].w};
                            if (fm == OPB_FIX_SQUARE) {
                                const double2 fx = fix[grow];
                                const float si = (float)fx.x, inv = (float)fx.y, bi = beta - si;
#pragma unroll
                                for (int u = 0; u < 4; u++) {
                                    float x = fmaf(bi - sj[u], c4[u], o[u]);
                                    if (grow == gcol + u) x += si * (si - beta);
                                    o[u] = x * inv;
                                }
                            } else {
#pragma unroll
                                for (int u = 0; u < 4; u++) o[u] = fmaf(beta, c4[u], o[u]);
                            }
                        } else if constexpr (FUSE == 2) {
                            // parts only, A's rows normalised here (OPB_FIX_ROWSCALE; FP32 inv:
                            // its rounding scales the whole row, renormalised by the next row sums)
                            if (fm == OPB_FIX_ROWSCALE) {
                                const float inv = (float)fix[grow].y;
#pragma unroll
                                for (int u = 0; u < 4; u++) o[u] *= inv;
                            }
                        } else if (Cin) {
                            float c4[4] = {cv[i].x, cv[i].y, cv[i].z, cv[i].w};
                            if (fm == OPB_FIX_CIN) {
                                // deferred renormalisation of Cin (the arithmetic of the
                                // E-form renormalisation kernel, so Cin reads exactly as if
                                // that kernel had stored it)
                                const double2 fx = fix[grow];
#pragma unroll
                                for (int u = 0; u < 4; u++) {
                                    double x = (double)c4[u];
                                    if (grow == gcol + u) x -= fx.x;
                                    c4[u] = (float)(x * fx.y);
                                }
                            }
#pragma unroll
                            for (int u = 0; u < 4; u++) o[u] = fmaf(beta, c4[u], o[u]);
                        }
                        if (C) *reinterpret_cast<float4 *>(C + (long long)grow * ldc + gcol) = make_float4(o[0], o[1], o[2], o[3]);
                        if constexpr (FUSE != 0) {
                            if (Shi) {
                                uint32_t hh[2], ll[2];
                                split2x2(o[0], o[1], hh[0], ll[0], p.sscale);
                                split2x2(o[2], o[3], hh[1], ll[1], p.sscale);
                                const long long so = (long long)grow * ldc + gcol;
                                *reinterpret_cast<uint2 *>(Shi + so) = make_uint2(hh[0], hh[1]);
                                *reinterpret_cast<uint2 *>(Slo + so) = make_uint2(ll[0], ll[1]);
                            }
                        }
                        const double g = (double)o[0] + (double)o[1] + (double)o[2] + (double)o[3];
                        st[rr * 33 + tc4] = __int_as_float(__double2loint(g));
                        st[rr * 33 + tc4 + 1] = __int_as_float(__double2hiint(g));
                    }
                }
                __syncwarp();
#pragma unroll
                for (int k = 0; k < 8; k++)
                    rs += __hiloint2double(__float_as_int(st[lane * 33 + 4 * k + 1]),
                                           __float_as_int(st[lane * 33 + 4 * k]));
                __syncwarp();  // before the next block overwrites the buffer
            }
            if (rowsum) rowsum[(long long)(col0 / CPT) * M + row] = rs;
        }
        if (!ok) atomicExch(&g_tc_error, 3);
    }
    tc_fence_before();
    __syncthreads();
    if constexpr (PAIR) cluster_sync_all();  // the leader's MMAs have drained before either CTA frees or exits
    if (warp == 0) {
        tc_fence_after();
        if constexpr (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS)
                         : "memory");
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS)
                         : "memory");
    }
}

// ------------------------------------------------------------------ host side

static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// rows x K bf16 row-major matrix (leading dimension ld elements), box = box_rows x bk
// (bk = 64: 128-byte swizzle; bk = 32: 64-byte swizzle).
static int make_map(CUtensorMap *m, const void *ptr, long long rows, long long K, long long ld, int box_rows,
                    int f16 = 0, int bk = TC_BK) {
    auto enc = get_encode();
    if (!enc) return OPB_E_UNSUPPORTED;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    cuuint32_t box[2] = {(cuuint32_t)bk, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, bk == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? OPB_OK : OPB_E_ARG;
}

// K x N bf16 row-major matrix (leading dimension ld elements) read as an MN-major B
// operand: box = 64 columns x bk rows, 128-byte swizzle.
static int make_map_mn(CUtensorMap *m, const void *ptr, long long K, long long N, long long ld, int f16 = 0,
                       int bk = TC_BK) {
    auto enc = get_encode();
    if (!enc) return OPB_E_UNSUPPORTED;
    cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)K};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    cuuint32_t box[2] = {64, (cuuint32_t)bk};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                     const_cast<void *>(ptr), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? OPB_OK : OPB_E_ARG;
}

// The B maps of a product: K-major (N x K, box rows = brows) or MN-major (K x N).
static int make_b_maps(CUtensorMap *hi, CUtensorMap *lo, const TcGemmArgs &a, int brows, int f16, int bk) {
    int r;
    if (a.b_kn) {
        if ((r = make_map_mn(hi, a.Bhi, a.K, a.N, a.ldb, f16, bk)) != OPB_OK) return r;
        return make_map_mn(lo, a.Blo, a.K, a.N, a.ldb, f16, bk);
    }
    if ((r = make_map(hi, a.Bhi, a.N, a.K, a.ldb, brows, f16, bk)) != OPB_OK) return r;
    return make_map(lo, a.Blo, a.N, a.K, a.ldb, brows, f16, bk);
}

static int g_tile_override = 0;  // 0 = automatic
static int g_bk256 = 64;          // K depth of a pipeline stage for 256-wide tiles (32 or 64)
static int g_pair = 1;            // 256 x 256 tiles on CTA pairs (cta_group::2) when M % 256 == 0
static int g_group_m = 0;         // M-tiles per raster group of single products (0: 8)

int tc_gemm_tile_n(int N) {
    if (g_tile_override && N % g_tile_override == 0) return g_tile_override;
    if (N % 256 == 0) return 256;
    if (N % 128 == 0) return 128;
    if (N % 64 == 0) return 64;
    return 0;
}

// Tile width for a product of M rows: the widest that still gives every SM a tile,
// else the narrowest that divides N (small-N products such as the pricing GEMM).
// A product that runs as K-slices keeps the widest tile, so that A, the large operand of a
// small-N product, is read from memory once; without K-slices narrower tiles give every SM
// a tile.
static int tile_for(int M, int N, int ksplit = 1) {
    int bn = tc_gemm_tile_n(N);
    if (g_tile_override || !bn || ksplit > 1) return bn;
    const int mt = M / TC_BM;
    while (bn > 64 && (long long)mt * (N / bn) < num_sms() && N % (bn / 2) == 0) bn /= 2;
    return bn;
}

// K-slices (at most 4, dividing K / 64) for a small-N product's widest tiles: the count
// whose items fill the SMs' waves best (items / (waves x SMs)); among equal fills, one that
// gives every SM an item, then the fewest slices.  A CTA streams A at a bounded rate
// (about 20-28 GB/s of BF16 parts through its 3-stage ring), so an idle SM is bandwidth lost:
// at d = 12288 one slice leaves 52 of 148 SMs idle (0.30 of HBM), three fill them.
int tc_gemm_split_for(int M, int N, int K) {
    const int bn = tc_gemm_tile_n(N);
    if (!bn || M % TC_BM) return 1;
    const long long tiles = (long long)(M / TC_BM) * (N / bn);
    const long long sms = num_sms();
    int best = 1;
    double best_fill = -1.0;
    bool best_all = false;
    for (int sp = 1; sp <= 4; sp++) {
        if ((K / TC_BK) % sp) continue;
        const long long items = tiles * sp;
        const long long waves = (items + sms - 1) / sms;
        const double fill = (double)items / (double)(waves * sms);
        const bool all = items >= sms;
        if (fill > best_fill + 0.02 || (fill > best_fill - 0.02 && all && !best_all)) {
            best = sp;
            best_fill = fill;
            best_all = all;
        }
    }
    return best;
}

// Row-sum partials: one per 128-column group (64 for the 64-wide tile).
int tc_gemm_nparts(int M, int N) {
    int bn = tile_for(M, N);
    if (!bn) return 0;
    return N / (bn < 128 ? bn : 128);
}

int tc_gemm_check(const TcGemmArgs &a) {
    if (a.M <= 0 || a.N <= 0 || a.K <= 0) return OPB_E_ARG;
    if (a.M % TC_BM || a.K % TC_BK || !tc_gemm_tile_n(a.N)) return OPB_E_UNSUPPORTED;
    if (!a.Ahi || !a.Alo || !a.Bhi || !a.Blo || (!a.C && !a.Shi)) return OPB_E_NULL;
    if (!a.Shi != !a.Slo) return OPB_E_NULL;
    if (a.Shi && (!aligned(a.Shi, 8) || !aligned(a.Slo, 8) || a.ksplit > 1)) return OPB_E_ARG;
    if (a.fixmode < 0 || a.fixmode > OPB_FIX_ROWSCALE || (a.fixmode && !a.cin_fix)) return OPB_E_ARG;
    // the fused epilogues: no Cin-form fix with parts, no Cin with the row scaling
    if ((a.Shi && a.fixmode == OPB_FIX_CIN) || (a.fixmode == OPB_FIX_ROWSCALE && a.Cin)) return OPB_E_ARG;
    if (a.Shi && !a.Cin && a.fixmode == OPB_FIX_NONE && a.cin_fix) return OPB_E_ARG;
    // the deferred squaring reads E' (Cin) and the column fixes of a square product
    if (a.fixmode == OPB_FIX_SQUARE && (!a.Cin || a.M != a.N)) return OPB_E_ARG;
    if (a.lda < a.K || a.ldb < (a.b_kn ? a.N : a.K) || a.ldc < a.N) return OPB_E_ARG;
    // TMA: 16-byte aligned bases and row strides; float4 epilogue: 16-byte aligned rows
    if (!aligned(a.Ahi, 16) || !aligned(a.Alo, 16) || !aligned(a.Bhi, 16) || !aligned(a.Blo, 16)) return OPB_E_ALIGN;
    if ((a.lda * 2) % 16 || (a.ldb * 2) % 16 || a.ldc % 4 || (a.C && !aligned(a.C, 16))) return OPB_E_ALIGN;
    if (a.Cin && !aligned(a.Cin, 16)) return OPB_E_ALIGN;
    if (a.cin_fix && !aligned(a.cin_fix, 16)) return OPB_E_ALIGN;
    if (a.ksplit > 1) {
        if (a.Cin || a.rowsum || a.ksplit > 64 || (a.K / TC_BK) % a.ksplit) return OPB_E_ARG;
        if (a.c_slice < (long long)a.M * a.ldc || a.c_slice % 4) return OPB_E_ARG;
    }
    // band-limited squaring: in place, square, one pass over K
    if (a.band && (a.Cin != a.C || a.M != a.N || a.N != a.K || a.ksplit > 1 || a.level < 0 || a.level > 62))
        return OPB_E_ARG;
    return OPB_OK;
}

template <int BN, int STAGES, bool BATCHED, bool F16, int NPROD = 3, int EPIMODE = 0, int BK = TC_BK,
          bool PAIR = false, bool BMN = false, int FUSE = 0>
static int set_smem_attr() {
    using Cfg = TcCfg<BN, STAGES, NPROD, BK, PAIR, EPIMODE>;
    static bool attr_set[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k_tc_gemm<BN, STAGES, BATCHED, F16, NPROD, EPIMODE, BK, PAIR, BMN, FUSE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             Cfg::SMEM);
        if (e != cudaSuccess) return (int)e;
        attr_set[dev] = true;
    }
    return 0;
}

template <int BN, int STAGES, bool F16, int BK = TC_BK, bool BMN = false, int FUSE = 0>
static int launch_tc_impl(const TcGemmArgs &a, cudaStream_t s) {
    using Cfg = TcCfg<BN, STAGES, 3, BK>;
    int e0 = set_smem_attr<BN, STAGES, false, F16, 3, 0, BK, false, BMN, FUSE>();
    if (e0) return e0;
    CUtensorMap mAh, mAl, mBh, mBl;
    int r;
    if ((r = make_map(&mAh, a.Ahi, a.M, a.K, a.lda, TC_BM, F16, BK)) != OPB_OK) return r;
    if ((r = make_map(&mAl, a.Alo, a.M, a.K, a.lda, TC_BM, F16, BK)) != OPB_OK) return r;
    if ((r = make_b_maps(&mBh, &mBl, a, BN, F16, BK)) != OPB_OK) return r;
    TcParams p{a.M, a.N, a.K, a.C, a.ldc, a.Cin, a.alpha, a.beta, a.rowsum};
    p.group_m = g_group_m;
    p.cin_fix = a.cin_fix;
    p.ksplit = a.ksplit > 1 ? a.ksplit : 1;
    p.c_slice = a.c_slice;
    p.band = a.band;
    p.level = a.level;
    p.lolo = a.lolo;
    p.band_skip = a.band_skip;
    p.fixmode = a.fixmode;
    p.Shi = a.Shi;
    p.Slo = a.Slo;
    p.sscale = a.sscale;
    const int ntiles = (a.M / TC_BM) * (a.N / BN) * p.ksplit;
    const int grid = ntiles < num_sms() ? ntiles : num_sms();
    TcBatch none{nullptr, nullptr, nullptr, 0};
    k_tc_gemm<BN, STAGES, false, F16, 3, 0, BK, false, BMN, FUSE><<<grid, Cfg::THREADS, Cfg::SMEM, s>>>(
        mAh, mAl, mBh, mBl, p, none);
    return (int)cudaGetLastError();
}

// 256 x 256 output tiles on 2-CTA clusters: each CTA loads its 128 rows of A and 128 rows
// of B, the even CTA issues cta_group::2 MMAs over both CTAs' shared memory.  The grid is
// as many clusters as can be resident at once (at most one per SM pair).
template <bool F16, bool BMN, int STAGES = 3, int BK = TC_BK, int FUSE = 0>
static int launch_tc_pair(const TcGemmArgs &a, cudaStream_t s) {
    constexpr int BN = 256;
    using Cfg = TcCfg<BN, STAGES, 3, BK, true>;
    auto kern = k_tc_gemm<BN, STAGES, false, F16, 3, 0, BK, true, BMN, FUSE>;
    int e0 = set_smem_attr<BN, STAGES, false, F16, 3, 0, BK, true, BMN, FUSE>();
    if (e0) return e0;
    CUtensorMap mAh, mAl, mBh, mBl;
    int r;
    if ((r = make_map(&mAh, a.Ahi, a.M, a.K, a.lda, TC_BM, F16, BK)) != OPB_OK) return r;
    if ((r = make_map(&mAl, a.Alo, a.M, a.K, a.lda, TC_BM, F16, BK)) != OPB_OK) return r;
    if ((r = make_b_maps(&mBh, &mBl, a, BN / 2, F16, BK)) != OPB_OK) return r;
    TcParams p{a.M, a.N, a.K, a.C, a.ldc, a.Cin, a.alpha, a.beta, a.rowsum};
    p.group_m = g_group_m;
    p.cin_fix = a.cin_fix;
    p.band = a.band;
    p.level = a.level;
    p.lolo = a.lolo;
    p.band_skip = a.band_skip;
    p.fixmode = a.fixmode;
    p.Shi = a.Shi;
    p.Slo = a.Slo;
    p.sscale = a.sscale;
    TcBatch none{nullptr, nullptr, nullptr, 0};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(Cfg::THREADS);
    cfg.dynamicSmemBytes = Cfg::SMEM;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    static int max_clusters[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return OPB_E_UNSUPPORTED;
    if (!max_clusters[dev]) {
        cfg.gridDim = dim3(2 * (num_sms() / 2));
        int n = 0;
        cudaError_t e = cudaOccupancyMaxActiveClusters(&n, kern, &cfg);
        if (e != cudaSuccess) return (int)e;
        if (n <= 0) return OPB_E_UNSUPPORTED;
        max_clusters[dev] = n;
    }
    const int ntiles = (a.M / (2 * TC_BM)) * (a.N / BN);
    const int nclusters = ntiles < max_clusters[dev] ? ntiles : max_clusters[dev];
    cfg.gridDim = dim3(2 * nclusters);
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, mAh, mAl, mBh, mBl, p, none);
    return e == cudaSuccess ? (int)cudaGetLastError() : (int)e;
}

int tc_make_maps(CUtensorMap *out4, const __nv_bfloat16 *Ahi, const __nv_bfloat16 *Alo, long long M, long long lda,
                 const __nv_bfloat16 *Bhi, const __nv_bfloat16 *Blo, long long N, long long ldb, long long K, int bn,
                 int f16, int b_kn) {
    int r;
    if ((r = make_map(&out4[0], Ahi, M, K, lda, TC_BM, f16)) != OPB_OK) return r;
    if ((r = make_map(&out4[1], Alo, M, K, lda, TC_BM, f16)) != OPB_OK) return r;
    if (b_kn) {
        if ((r = make_map_mn(&out4[2], Bhi, K, N, ldb, f16)) != OPB_OK) return r;
        return make_map_mn(&out4[3], Blo, K, N, ldb, f16);
    }
    if ((r = make_map(&out4[2], Bhi, N, K, ldb, bn, f16)) != OPB_OK) return r;
    if ((r = make_map(&out4[3], Blo, N, K, ldb, bn, f16)) != OPB_OK) return r;
    return OPB_OK;
}

template <int BN, int STAGES, bool F16, bool BMN, int FUSE>
static int launch_batched_impl(const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                               int grid, cudaStream_t s, int level, int lolo, int band_skip, int fixmode,
                               float sscale) {
    using Cfg = TcCfg<BN, STAGES>;
    int e0 = set_smem_attr<BN, STAGES, true, F16, 3, 0, TC_BK, false, BMN, FUSE>();
    if (e0) return e0;
    CUtensorMap dummy;
    std::memset(&dummy, 0, sizeof(dummy));
    TcParams p{};
    p.level = level;
    p.lolo = lolo;
    p.band_skip = band_skip;
    p.fixmode = fixmode;
    p.sscale = sscale;
    TcBatch bt{maps, probs, work, nwork};
    k_tc_gemm<BN, STAGES, true, F16, 3, 0, TC_BK, false, BMN, FUSE><<<grid, Cfg::THREADS, Cfg::SMEM, s>>>(
        dummy, dummy, dummy, dummy, p, bt);
    return (int)cudaGetLastError();
}

// Batched 256 x 256 items on 2-CTA clusters: work items (problem << 16 | m-tile << 8 |
// n-tile) in 256-row / 256-column units, maps with 128-row boxes for A and B (each CTA
// loads its own half), problems with M % 256 == 0 and N % 256 == 0.
template <bool F16, bool BMN, int FUSE>
static int launch_batched_pair_impl(const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                                    cudaStream_t s, int level, int lolo, int band_skip, int fixmode, float sscale) {
    constexpr int BN = 256, STAGES = 3;
    using Cfg = TcCfg<BN, STAGES, 3, TC_BK, true>;
    auto kern = k_tc_gemm<BN, STAGES, true, F16, 3, 0, TC_BK, true, BMN, FUSE>;
    int e0 = set_smem_attr<BN, STAGES, true, F16, 3, 0, TC_BK, true, BMN, FUSE>();
    if (e0) return e0;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(Cfg::THREADS);
    cfg.dynamicSmemBytes = Cfg::SMEM;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    static int max_clusters[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return OPB_E_UNSUPPORTED;
    if (!max_clusters[dev]) {
        cfg.gridDim = dim3(2 * (num_sms() / 2));
        int n = 0;
        cudaError_t e = cudaOccupancyMaxActiveClusters(&n, kern, &cfg);
        if (e != cudaSuccess) return (int)e;
        if (n <= 0) return OPB_E_UNSUPPORTED;
        max_clusters[dev] = n;
    }
    const int ncl = nwork < max_clusters[dev] ? nwork : max_clusters[dev];
    cfg.gridDim = dim3(2 * ncl);
    CUtensorMap dummy;
    std::memset(&dummy, 0, sizeof(dummy));
    TcParams p{};
    p.level = level;
    p.lolo = lolo;
    p.band_skip = band_skip;
    p.fixmode = fixmode;
    p.sscale = sscale;
    TcBatch bt{maps, probs, work, nwork};
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, dummy, dummy, dummy, dummy, p, bt);
    return e == cudaSuccess ? (int)cudaGetLastError() : (int)e;
}

// Batched squaring and chain products take MN-major B maps (b_kn = 1): pair and 256/128
// tiles exist only in that form; 64-wide tiles in both (pricing is K-major).
template <int FUSE>
static int batched_pair_fused(const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                              cudaStream_t s, int f16, int level, int lolo, int band_skip, int fixmode, float sscale) {
    return f16 ? launch_batched_pair_impl<true, true, FUSE>(maps, probs, work, nwork, s, level, lolo, band_skip,
                                                            fixmode, sscale)
               : launch_batched_pair_impl<false, true, FUSE>(maps, probs, work, nwork, s, level, lolo, band_skip,
                                                             fixmode, sscale);
}

int launch_tc_gemm_batched_pair(const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                                cudaStream_t s, int f16, int b_kn, int level, int lolo, int band_skip, int fixmode,
                                float sscale, int fuse) {
    if (nwork <= 0) return OPB_OK;
    if (!b_kn) return OPB_E_UNSUPPORTED;
    if (fuse == 1) return batched_pair_fused<1>(maps, probs, work, nwork, s, f16, level, lolo, band_skip, fixmode, sscale);
    if (fuse == 2) return batched_pair_fused<2>(maps, probs, work, nwork, s, f16, level, lolo, band_skip, fixmode, sscale);
    return batched_pair_fused<0>(maps, probs, work, nwork, s, f16, level, lolo, band_skip, fixmode, sscale);
}

// MN-major B (b_kn) in every tile width and epilogue form; K-major B (pricing) 64-wide only.
template <int FUSE>
static int batched_kn(int bn, const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                      int grid, cudaStream_t s, int f16, int level, int lolo, int band_skip, int fixmode,
                      float sscale) {
    switch (bn * 2 + (f16 ? 1 : 0)) {
        case 512:
            return launch_batched_impl<256, 2, false, true, FUSE>(maps, probs, work, nwork, grid, s, level, lolo,
                                                                  band_skip, fixmode, sscale);
        case 513:
            return launch_batched_impl<256, 2, true, true, FUSE>(maps, probs, work, nwork, grid, s, level, lolo,
                                                                 band_skip, fixmode, sscale);
        case 256:
            return launch_batched_impl<128, 3, false, true, FUSE>(maps, probs, work, nwork, grid, s, level, lolo,
                                                                  band_skip, fixmode, sscale);
        case 257:
            return launch_batched_impl<128, 3, true, true, FUSE>(maps, probs, work, nwork, grid, s, level, lolo,
                                                                 band_skip, fixmode, sscale);
        case 128:
            return launch_batched_impl<64, 4, false, true, FUSE>(maps, probs, work, nwork, grid, s, level, lolo,
                                                                 band_skip, fixmode, sscale);
        case 129:
            return launch_batched_impl<64, 4, true, true, FUSE>(maps, probs, work, nwork, grid, s, level, lolo,
                                                                band_skip, fixmode, sscale);
        default: return OPB_E_UNSUPPORTED;
    }
}

int launch_tc_gemm_batched(int bn, const CUtensorMap *maps, const TcProblem *probs, const uint32_t *work, int nwork,
                           int grid, cudaStream_t s, int f16, int b_kn, int level, int lolo, int band_skip, int fixmode,
                           float sscale, int fuse) {
    if (nwork <= 0) return OPB_OK;
    if (grid <= 0 || grid > nwork) grid = nwork < num_sms() ? nwork : num_sms();
    if (b_kn) {
        if (fuse == 1)
            return batched_kn<1>(bn, maps, probs, work, nwork, grid, s, f16, level, lolo, band_skip, fixmode, sscale);
        if (fuse == 2)
            return batched_kn<2>(bn, maps, probs, work, nwork, grid, s, f16, level, lolo, band_skip, fixmode, sscale);
        return batched_kn<0>(bn, maps, probs, work, nwork, grid, s, f16, level, lolo, band_skip, fixmode, sscale);
    }
    if (bn != 64 || fuse) return OPB_E_UNSUPPORTED;
    return f16 ? launch_batched_impl<64, 4, true, false, 0>(maps, probs, work, nwork, grid, s, level, lolo, band_skip,
                                                            fixmode, sscale)
               : launch_batched_impl<64, 4, false, false, 0>(maps, probs, work, nwork, grid, s, level, lolo, band_skip,
                                                             fixmode, sscale);
}

// One network layer on the tensor cores: H[M, N] = GELU(alpha * A[M, K] . W[N, K]^T + bias)
// with BF16 A, W and H (single product, FP32 accumulation); M % 128, N = 256, K % 64 and
// K <= 256 (W stays resident in shared memory).
// With w5 and ypart (N = 256): no H; instead ypart[g * M + row], g < 256 / TC_LAYER_CPT, =
// the dot of the BF16 activations of column group g with w5 (the output layer, fused).
int launch_tc_layer(int M, int N, int K, const __nv_bfloat16 *A, long long lda, const __nv_bfloat16 *W,
                    long long ldw, float alpha, const float *bias, __nv_bfloat16 *H, long long ldh, cudaStream_t s,
                    const float *w5, float *ypart) {
    constexpr int BN = 256, STAGES = 3;
    using Cfg = TcCfg<BN, STAGES, 1, TC_BK, false, 1>;
    using Cfg2 = TcCfg<BN, STAGES, 1, TC_BK, false, 2>;  // the last layer, output fused
    static_assert(Cfg::BRES && Cfg::SMEM <= 227 * 1024 && Cfg2::SMEM <= 227 * 1024, "layer kernel: resident weights");
    const bool fused = w5 != nullptr;
    // one column tile and K <= 256: the weights stay resident in shared memory
    if (M <= 0 || M % TC_BM || N != BN || K % TC_BK || K > Cfg::BRES_KB * TC_BK) return OPB_E_UNSUPPORTED;
    if (!A || !W || !bias || (fused ? !ypart : !H)) return OPB_E_NULL;
    int e0 = fused ? set_smem_attr<BN, STAGES, false, false, 1, 2>() : set_smem_attr<BN, STAGES, false, false, 1, 1>();
    if (e0) return e0;
    CUtensorMap mA, mW;
    int r;
    if ((r = make_map(&mA, A, M, K, lda, TC_BM)) != OPB_OK) return r;
    if ((r = make_map(&mW, W, N, K, ldw, BN)) != OPB_OK) return r;
    TcParams p{};
    p.M = M; p.N = N; p.K = K; p.alpha = alpha; p.bias = bias; p.H = H; p.ldh = ldh; p.w5 = w5; p.ypart = ypart;
    const int ntiles = (M / TC_BM) * (N / BN);
    const int grid = ntiles < num_sms() ? ntiles : num_sms();
    TcBatch none{nullptr, nullptr, nullptr, 0};
    if (fused)
        k_tc_gemm<BN, STAGES, false, false, 1, 2><<<grid, Cfg2::THREADS, Cfg2::SMEM, s>>>(mA, mA, mW, mW, p, none);
    else
        k_tc_gemm<BN, STAGES, false, false, 1, 1><<<grid, Cfg::THREADS, Cfg::SMEM, s>>>(mA, mA, mW, mW, p, none);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------- fused network inference
//
// The four hidden layers of one ensemble member (8 -> 256 x 4 with GELU) and the output
// layer's partial dots in one persistent kernel.  A 128-row tile's activations stay in
// shared memory between layers, written by the epilogue as BF16 in the layout the next
// layer's MMA reads (K-major, 128-byte swizzle: row r of K-block kb at kb * 16 KB + r * 128,
// its 16-byte chunk c at position c ^ (r & 7)), so HBM carries only the padded inputs and
// the output partials.  Two tiles are in flight per CTA (slots 0 and 1, each with a 64 KB
// activation buffer and a 256-column TMEM accumulator): the MMAs run the layers in the order
// (tile a, layer l), (tile b, l), (a, l + 1), (b, l + 1), ..., so the epilogue of one tile's
// layer overlaps the MMAs of the other's.  The weights stream through a two-stage ring of
// 256 x 64 K-blocks in the MMAs' order; the input tile is loaded into its slot's first
// K-block once the slot's previous tile has finished.
//
// Warp roles (576 threads): 16 epilogue warps (lane quadrant q = warp & 3, column group
// h = warp >> 2 = the K-block of the next layer's A that the warp writes), one TMA warp, one
// MMA warp.  Barriers, per slot s: xfull (input tile loaded), accf (layer's MMAs done),
// hready (epilogue done: accumulator read and, for layers 1-3, activations written and
// fenced for the async proxy), hfree (the tile's last MMA done: the slot's buffer may take
// the next input); per ring stage: wfull, wempty.  Every wait is bounded as in k_tc_gemm.
//
// Each layer is computed as launch_tc_layer computes it -- the same MMA K order into FP32
// TMEM, the same bias + GELU and BF16 rounding, the same partial dots of the output layer --
// so ypart is bit-identical to the layer-by-layer path.

constexpr int FM_EPI = 16, FM_THREADS = 32 * (FM_EPI + 2);
constexpr int FM_KB_BYTES = TC_BM * TC_BK * 2;      // one K-block of a slot's activations
constexpr int FM_HBYTES = 4 * FM_KB_BYTES;          // a slot: 128 rows x 256 BF16
constexpr int FM_WBYTES = 256 * TC_BK * 2;          // one weight K-block: 256 rows x 64 BF16
constexpr int FM_WST = 2;                           // weight ring stages
constexpr int FM_RING = 2 * FM_HBYTES + FM_WST * FM_WBYTES;
constexpr int FM_VEC = 5 * 256 * 4;                 // b1 | b2 | b3 | b4 | w5
constexpr int FM_SMEM = FM_RING + 1024 + 256 + FM_VEC;
static_assert(FM_SMEM <= 227 * 1024, "fused inference: shared memory");

struct FmParams {
    long long M;       // rows, a multiple of 128
    const float *vec;  // b1 | b2 | b3 | b4 | w5, 5 x 256 floats
    float *ypart;      // [4][M]: partial dot of column group g with w5
};

__global__ void __launch_bounds__(FM_THREADS, 1)
    k_mlp_fused(const __grid_constant__ CUtensorMap mX, const __grid_constant__ CUtensorMap mW1,
                const __grid_constant__ CUtensorMap mWH, FmParams p) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t *gbase = smem_raw + (base - raw);
    const uint32_t wbase = base + 2 * FM_HBYTES;
    uint64_t *bars = reinterpret_cast<uint64_t *>(gbase + FM_RING);
    const uint32_t bar0 = smem_u32(bars);
    auto wfull = [&](int w) { return bar0 + 8u * w; };
    auto wempty = [&](int w) { return bar0 + 8u * (2 + w); };
    auto xfull = [&](int s) { return bar0 + 8u * (4 + s); };
    auto accf = [&](int s) { return bar0 + 8u * (6 + s); };
    auto hready = [&](int s) { return bar0 + 8u * (8 + s); };
    auto hfree = [&](int s) { return bar0 + 8u * (10 + s); };
    const uint32_t drain_bar = bar0 + 8u * 12;
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bars + 13);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 14);
    float *svec = reinterpret_cast<float *>(gbase + FM_RING + 256);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (int)(p.M / TC_BM);
    const int item0 = blockIdx.x, istep = gridDim.x;
    const int nmine = item0 < ntiles ? (ntiles - item0 + istep - 1) / istep : 0;  // this CTA's tiles

    if (threadIdx.x == 0) {
        for (int i = 0; i < 12; i++) mbar_init(bar0 + 8u * i, (i == 8 || i == 9) ? FM_EPI : 1);
        mbar_init(drain_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        const uint32_t slot = smem_u32(const_cast<uint32_t *>(tmem_slot));
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    for (int i = threadIdx.x; i < 5 * 256; i += blockDim.x) svec[i] = p.vec[i];
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // The steps (tile j of this CTA, layer l) in MMA order: pairs of tiles, layer by layer,
    // the pair's two tiles alternating; tile j lives in slot j & 1 as that slot's use j >> 1.
#define FM_STEPS_BEGIN                                                     \
    for (int pp = 0; pp < nmine && ok; pp += 2)                            \
        for (int l = 0; l < 4 && ok; l++)                                  \
            for (int s = 0; s < 2 && ok; s++) {                            \
                const int j = pp + s;                                      \
                if (j >= nmine) continue;                                  \
                const int u = j >> 1;
#define FM_STEPS_END }

    if (warp == FM_EPI) {
        if (lane == 0) {
            // ---------------- TMA producer: input tiles and the weight K-blocks in MMA order
            long wk = 0;
            bool ok = true;
            FM_STEPS_BEGIN
            if (l == 0) {
                if (u >= 1 && !mbar_wait(hfree(s), (uint32_t)((u - 1) & 1), abort_flag, TC_WAIT_NS)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(xfull(s), FM_KB_BYTES);
                tma_load_2d(base + s * FM_HBYTES, &mX, xfull(s), 0, (item0 + j * istep) * TC_BM);
            }
            const int nkb = l == 0 ? 1 : 4;
            for (int kb = 0; kb < nkb; kb++, wk++) {
                const int w = (int)(wk & 1);
                if (wk >= FM_WST &&
                    !mbar_wait(wempty(w), (uint32_t)(((wk / FM_WST) + 1) & 1), abort_flag, TC_WAIT_NS)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(wfull(w), FM_WBYTES);
                if (l == 0) tma_load_2d(wbase + w * FM_WBYTES, &mW1, wfull(w), 0, 0);
                else tma_load_2d(wbase + w * FM_WBYTES, &mWH, wfull(w), kb * TC_BK, (l - 1) * 256);
            }
            FM_STEPS_END
            if (!ok) {
                atomicExch(&g_tc_error, 11);
                *abort_flag = 1;
            }
        }
        __syncwarp();
    } else if (warp == FM_EPI + 1) {
        if (lane == 0) {
            // ---------------- MMA issuer
            const uint32_t idesc = umma_idesc_16(256, false);
            long wk = 0;
            bool ok = true;
            FM_STEPS_BEGIN
            // operands of (j, l): the input tile, or layer l - 1's activations; and the
            // accumulator drained by the slot's previous epilogue (hready completion
            // 4u + l - 1 of this slot)
            if (l == 0) {
                if (u >= 1 && !mbar_wait(hready(s), 1u, abort_flag, TC_WAIT_NS)) ok = false;
                if (ok && !mbar_wait(xfull(s), (uint32_t)(u & 1), abort_flag, TC_WAIT_NS)) ok = false;
            } else if (!mbar_wait(hready(s), (uint32_t)((l - 1) & 1), abort_flag, TC_WAIT_NS)) {
                ok = false;
            }
            if (!ok) break;
            tc_fence_after();
            const uint32_t dacc = tmem + (uint32_t)(s * 256);
            const int nkb = l == 0 ? 1 : 4;
            for (int kb = 0; kb < nkb; kb++, wk++) {
                const int w = (int)(wk & 1);
                if (!mbar_wait(wfull(w), (uint32_t)((wk / FM_WST) & 1), abort_flag, TC_WAIT_NS)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint64_t dA = umma_desc_sw<TC_BK>(base + s * FM_HBYTES + kb * FM_KB_BYTES);
                const uint64_t dB = umma_desc_sw<TC_BK>(wbase + w * FM_WBYTES);
#pragma unroll
                for (int k16 = 0; k16 < TC_BK / 16; k16++) {
                    const uint64_t adv = (uint64_t)((k16 * 32) >> 4);
                    umma_bf16(dacc, dA + adv, dB + adv, idesc, (kb > 0 || k16 > 0) ? 1u : 0u);
                }
                umma_commit(wempty(w));
            }
            if (!ok) break;
            umma_commit(accf(s));
            if (l == 3) umma_commit(hfree(s));
            FM_STEPS_END
            if (!ok) {
                atomicExch(&g_tc_error, 12);
                *abort_flag = 1;
            }
            umma_commit(drain_bar);
            (void)mbar_wait(drain_bar, 0, abort_flag, TC_WAIT_NS);
        }
        __syncwarp();
    } else {
        // ---------------- epilogue warps
        const int q = warp & 3, h = warp >> 2;
        const int r = q * 32 + lane;  // row within the tile (TMEM lane)
        const uint32_t lane_base = (uint32_t)(q * 32) << 16;
        float sum[64];
        bool ok = true;
        FM_STEPS_BEGIN
        if (!mbar_wait(accf(s), (uint32_t)(l & 1), abort_flag, TC_WAIT_NS)) {
            ok = false;
            break;
        }
        tc_fence_after();
        const uint32_t tacc = tmem + lane_base + (uint32_t)(s * 256 + h * 64);
#pragma unroll
        for (int jj = 0; jj < 4; jj++) {
            uint32_t v[16];
            tmem_ld16(tacc + (uint32_t)(16 * jj), v);
#pragma unroll
            for (int i = 0; i < 16; i++) sum[16 * jj + i] = __uint_as_float(v[i]);
        }
        const float4 *b4 = reinterpret_cast<const float4 *>(svec + l * 256 + h * 64);
        if (l < 3) {
            // activations of layer l + 1: K-block h of the slot, row r, chunks swizzled
            uint8_t *hrow = gbase + s * FM_HBYTES + h * FM_KB_BYTES + r * 128;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const float4 ba = b4[2 * c], bb = b4[2 * c + 1];
                const float bv[8] = {ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, bb.z, bb.w};
                uint32_t pk[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const __nv_bfloat162 h2 = __floats2bfloat162_rn(gelu_as(fmaf(1.f, sum[8 * c + 2 * e], bv[2 * e])),
                                                                    gelu_as(fmaf(1.f, sum[8 * c + 2 * e + 1], bv[2 * e + 1])));
                    pk[e] = *reinterpret_cast<const uint32_t *>(&h2);
                }
                *reinterpret_cast<uint4 *>(hrow + ((c ^ (r & 7)) << 4)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
            // the MMAs read these through the async proxy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        } else {
            // output layer: partial dot of the BF16-rounded activations with w5
            const float4 *w4 = reinterpret_cast<const float4 *>(svec + 4 * 256 + h * 64);
            float acc = 0.f;
#pragma unroll
            for (int c = 0; c < 64; c += 4) {
                const float4 bv = b4[c / 4], wv = w4[c / 4];
                const __nv_bfloat162 h01 = __floats2bfloat162_rn(gelu_as(fmaf(1.f, sum[c], bv.x)),
                                                                 gelu_as(fmaf(1.f, sum[c + 1], bv.y)));
                const __nv_bfloat162 h23 = __floats2bfloat162_rn(gelu_as(fmaf(1.f, sum[c + 2], bv.z)),
                                                                 gelu_as(fmaf(1.f, sum[c + 3], bv.w)));
                const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
                acc = fmaf(f01.x, wv.x, acc);
                acc = fmaf(f01.y, wv.y, acc);
                acc = fmaf(f23.x, wv.z, acc);
                acc = fmaf(f23.y, wv.w, acc);
            }
            p.ypart[(long long)h * p.M + (long long)(item0 + j * istep) * TC_BM + r] = acc;
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(hready(s)) : "memory");
        FM_STEPS_END
        if (!ok) atomicExch(&g_tc_error, 13);
    }
#undef FM_STEPS_BEGIN
#undef FM_STEPS_END
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// One ensemble member's inference: Xp [M x 64] padded BF16 inputs, W1 [256 x 64], WH three
// [256 x 256] matrices back to back (BF16, K-major), vec = b1 | b2 | b3 | b4 | w5 (FP32);
// ypart [4][M] receives the output layer's partial dots (as launch_tc_layer's fused last
// layer writes them).  M % 128 == 0.
int launch_mlp_fused(long long M, const __nv_bfloat16 *Xp, const __nv_bfloat16 *W1, const __nv_bfloat16 *WH,
                     const float *vec, float *ypart, cudaStream_t s) {
    if (M <= 0 || M % TC_BM || M / TC_BM > 0x7fffffffLL) return OPB_E_UNSUPPORTED;
    if (!Xp || !W1 || !WH || !vec || !ypart) return OPB_E_NULL;
    static bool attr_set[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, FM_SMEM);
        if (e != cudaSuccess) return (int)e;
        attr_set[dev] = true;
    }
    CUtensorMap mX, mW1, mWH;
    int r;
    if ((r = make_map(&mX, Xp, M, 64, 64, TC_BM)) != OPB_OK) return r;
    if ((r = make_map(&mW1, W1, 256, 64, 64, 256)) != OPB_OK) return r;
    if ((r = make_map(&mWH, WH, 3 * 256, 256, 256, 256)) != OPB_OK) return r;
    FmParams p{M, vec, ypart};
    const long long ntiles = M / TC_BM;
    const int grid = ntiles < num_sms() ? (int)ntiles : num_sms();
    k_mlp_fused<<<grid, FM_THREADS, FM_SMEM, s>>>(mX, mW1, mWH, p);
    return (int)cudaGetLastError();
}

// The epilogue form of a product (the FUSE template parameter of k_tc_gemm).
static int fuse_of(const TcGemmArgs &a) {
    if (a.fixmode == OPB_FIX_SQUARE || (a.Shi && a.Cin)) return 1;
    if (a.fixmode == OPB_FIX_ROWSCALE || a.Shi) return 2;
    return 0;
}

// Products with B given K x N row-major (MN-major operand; BK = 64 only): the squaring and
// chain products, in any of the three epilogue forms.
template <int FUSE>
static int launch_tc_kn(const TcGemmArgs &a, cudaStream_t s, bool pair) {
    switch (tile_for(a.M, a.N, a.ksplit) * 2 + (a.f16 ? 1 : 0)) {
        case 512:
            if (pair)
                return g_bk256 == 32 ? launch_tc_pair<false, true, 6, 32, FUSE>(a, s)
                                     : launch_tc_pair<false, true, 3, TC_BK, FUSE>(a, s);
            return launch_tc_impl<256, 2, false, 64, true, FUSE>(a, s);
        case 513:
            if (pair)
                return g_bk256 == 32 ? launch_tc_pair<true, true, 6, 32, FUSE>(a, s)
                                     : launch_tc_pair<true, true, 3, TC_BK, FUSE>(a, s);
            return launch_tc_impl<256, 2, true, 64, true, FUSE>(a, s);
        case 256: return launch_tc_impl<128, 3, false, 64, true, FUSE>(a, s);
        case 257: return launch_tc_impl<128, 3, true, 64, true, FUSE>(a, s);
        case 128: return launch_tc_impl<64, 4, false, 64, true, FUSE>(a, s);
        case 129: return launch_tc_impl<64, 4, true, 64, true, FUSE>(a, s);
        default: return OPB_E_UNSUPPORTED;
    }
}

int launch_tc_gemm(const TcGemmArgs &a, cudaStream_t s) {
    int c = tc_gemm_check(a);
    if (c != OPB_OK) return c;
    // K-sliced products (pricing, induction) stay on one CTA per tile: on CTA pairs, which
    // share the B tile and so hold four stages of A instead of three, they ran 6% slower
    const bool pair = g_pair && a.M % (2 * TC_BM) == 0 && a.ksplit <= 1;
    const int fuse = fuse_of(a);
    if (a.b_kn) {
        if (fuse == 1) return launch_tc_kn<1>(a, s, pair);
        if (fuse == 2) return launch_tc_kn<2>(a, s, pair);
        return launch_tc_kn<0>(a, s, pair);
    }
    if (fuse) return OPB_E_UNSUPPORTED;  // fused epilogues: MN-major B only
    switch (tile_for(a.M, a.N, a.ksplit) * 2 + (a.f16 ? 1 : 0)) {
        case 512:
            if (pair) return launch_tc_pair<false, false>(a, s);
            return g_bk256 == 32 ? launch_tc_impl<256, 4, false, 32>(a, s) : launch_tc_impl<256, 2, false>(a, s);
        case 513:
            if (pair) return launch_tc_pair<true, false>(a, s);
            return g_bk256 == 32 ? launch_tc_impl<256, 4, true, 32>(a, s) : launch_tc_impl<256, 2, true>(a, s);
        case 256: return launch_tc_impl<128, 3, false>(a, s);
        case 257: return launch_tc_impl<128, 3, true>(a, s);
        case 128: return launch_tc_impl<64, 4, false>(a, s);
        case 129: return launch_tc_impl<64, 4, true>(a, s);
        default: return OPB_E_UNSUPPORTED;
    }
}

}  // namespace opb

using namespace opb;

// Split-BF16 GEMM with typed pointers (row-major, K-major operands; see top of file).
OPB_API int opb_gemm_bf16x3(int M, int N, int K, const __nv_bfloat16 *Ahi, const __nv_bfloat16 *Alo, long long lda,
                            const __nv_bfloat16 *Bhi, const __nv_bfloat16 *Blo, long long ldb, float alpha,
                            const float *Cin, float beta, float *C, long long ldc, double *rowsum) {
    TcGemmArgs a{};
    a.M = M; a.N = N; a.K = K; a.Ahi = Ahi; a.Alo = Alo; a.Bhi = Bhi; a.Blo = Blo; a.lda = lda; a.ldb = ldb;
    a.C = C; a.ldc = ldc; a.Cin = Cin; a.alpha = alpha; a.beta = beta; a.rowsum = rowsum;
    return set_status(launch_tc_gemm(a, stream()));
}

// The same product with B given K x N row-major (ldb >= N), read as an MN-major operand:
// the form the lattice solve uses (a squaring's B is E's own row-major parts).  Results are
// identical to opb_gemm_bf16x3 on the transposed B.
OPB_API int opb_gemm_bf16x3_kn(int M, int N, int K, const __nv_bfloat16 *Ahi, const __nv_bfloat16 *Alo,
                               long long lda, const __nv_bfloat16 *Bhi, const __nv_bfloat16 *Blo, long long ldb,
                               float alpha, const float *Cin, float beta, float *C, long long ldc, double *rowsum) {
    TcGemmArgs a{};
    a.M = M; a.N = N; a.K = K; a.Ahi = Ahi; a.Alo = Alo; a.Bhi = Bhi; a.Blo = Blo; a.lda = lda; a.ldb = ldb;
    a.C = C; a.ldc = ldc; a.Cin = Cin; a.alpha = alpha; a.beta = beta; a.rowsum = rowsum; a.b_kn = 1;
    return set_status(launch_tc_gemm(a, stream()));
}

// The same product with FP16 parts (e.g. of a power-of-two-scaled split; undo the scales
// through alpha).
OPB_API int opb_gemm_f16x3(int M, int N, int K, const uint16_t *Ahi, const uint16_t *Alo, long long lda,
                           const uint16_t *Bhi, const uint16_t *Blo, long long ldb, float alpha, const float *Cin,
                           float beta, float *C, long long ldc, double *rowsum) {
    TcGemmArgs a{};
    a.M = M; a.N = N; a.K = K;
    a.Ahi = reinterpret_cast<const __nv_bfloat16 *>(Ahi); a.Alo = reinterpret_cast<const __nv_bfloat16 *>(Alo);
    a.Bhi = reinterpret_cast<const __nv_bfloat16 *>(Bhi); a.Blo = reinterpret_cast<const __nv_bfloat16 *>(Blo);
    a.lda = lda; a.ldb = ldb; a.C = C; a.ldc = ldc; a.Cin = Cin; a.alpha = alpha; a.beta = beta; a.rowsum = rowsum;
    a.f16 = 1;
    return set_status(launch_tc_gemm(a, stream()));
}

// The FP16-part product with B given K x N row-major (as opb_gemm_bf16x3_kn).
OPB_API int opb_gemm_f16x3_kn(int M, int N, int K, const uint16_t *Ahi, const uint16_t *Alo, long long lda,
                              const uint16_t *Bhi, const uint16_t *Blo, long long ldb, float alpha, const float *Cin,
                              float beta, float *C, long long ldc, double *rowsum) {
    TcGemmArgs a{};
    a.M = M; a.N = N; a.K = K;
    a.Ahi = reinterpret_cast<const __nv_bfloat16 *>(Ahi); a.Alo = reinterpret_cast<const __nv_bfloat16 *>(Alo);
    a.Bhi = reinterpret_cast<const __nv_bfloat16 *>(Bhi); a.Blo = reinterpret_cast<const __nv_bfloat16 *>(Blo);
    a.lda = lda; a.ldb = ldb; a.C = C; a.ldc = ldc; a.Cin = Cin; a.alpha = alpha; a.beta = beta; a.rowsum = rowsum;
    a.f16 = 1;
    a.b_kn = 1;
    return set_status(launch_tc_gemm(a, stream()));
}

OPB_API int opb_gemm_bf16x3_nparts(int M, int N) { return tc_gemm_nparts(M, N); }

// The product of a skinny B (N <= 128 columns: payoffs, option values) as ksplit K-slices:
// slice s (of K / ksplit) writes its FP32 partial product to C + s * c_slice (c_slice >=
// M * ldc), for the caller to sum.  B is N x K row-major (K-major).  ksplit = 0 picks the
// slice count that brings the tiles to about one per SM (at most 4), as the lattice solve's
// pricing products do; the count used is returned through ksplit_used (optional).
OPB_API int opb_gemm_bf16x3_ksliced(int M, int N, int K, const __nv_bfloat16 *Ahi, const __nv_bfloat16 *Alo,
                                    long long lda, const __nv_bfloat16 *Bhi, const __nv_bfloat16 *Blo, long long ldb,
                                    float *C, long long ldc, int ksplit, long long c_slice, int *ksplit_used) {
    OPB_REQUIRE(ksplit >= 0 && ksplit <= 64 && N > 0 && N <= 128, OPB_E_ARG);
    TcGemmArgs a{};
    a.M = M; a.N = N; a.K = K; a.Ahi = Ahi; a.Alo = Alo; a.Bhi = Bhi; a.Blo = Blo; a.lda = lda; a.ldb = ldb;
    a.C = C; a.ldc = ldc; a.alpha = 1.f; a.beta = 0.f;
    a.ksplit = ksplit > 0 ? ksplit : tc_gemm_split_for(M, N, K);
    a.c_slice = c_slice;
    if (ksplit_used) *ksplit_used = a.ksplit;
    return set_status(launch_tc_gemm(a, stream()));
}

// Tuning knob: force the output tile width (64, 128 or 256) of single products; 0 = automatic.
OPB_API int opb_set_tile_n(int bn) {
    OPB_REQUIRE(bn == 0 || bn == 64 || bn == 128 || bn == 256, OPB_E_ARG);
    g_tile_override = bn;
    return set_status(OPB_OK);
}

// Tuning knob: K depth of a pipeline stage of 256-wide tiles: 64 (the default: 2 stages of
// 96 KB for one CTA, 3 of 64 KB per CTA of a pair) or 32 (4 stages of 48 KB, 6 of 32 KB for
// a pair with B given K x N; A in 64-byte swizzle).  Results are identical; at d = 6144
// the 64-deep stages are faster for both kernels.
OPB_API int opb_set_stage_k(int bk) {
    OPB_REQUIRE(bk == 32 || bk == 64, OPB_E_ARG);
    g_bk256 = bk;
    return set_status(OPB_OK);
}

// Tuning knob: 256 x 256 tiles on CTA pairs (cta_group::2) for products with M % 256 == 0
// and 256-wide tiles: 1 = on (default), 0 = off (one CTA per 128 x 256 tile).
OPB_API int opb_set_cta_pair(int on) {
    OPB_REQUIRE(on == 0 || on == 1, OPB_E_ARG);
    g_pair = on;
    return set_status(OPB_OK);
}

// Tuning knob: M-tiles per raster group of single products (operand-strip reuse in L2);
// 0 = 8.  Results are identical.
OPB_API int opb_set_group_m(int gm) {
    OPB_REQUIRE(gm >= 0 && gm <= 64, OPB_E_ARG);
    g_group_m = gm;
    return set_status(OPB_OK);
}

// Reads and clears the tensor-core kernels' device error word (0 = no bounded wait expired)
// after the calling thread's library stream has drained (it may be a non-blocking stream,
// which the symbol copies below would not wait for).
OPB_API int opb_tc_error(void) {
    int v = 0, z = 0;
    OPB_TRY(cudaStreamSynchronize(stream()));
    OPB_TRY(cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)));
    OPB_TRY(cudaMemcpyToSymbol(g_tc_error, &z, sizeof(int)));
    set_status(OPB_OK);
    return v;
}
