// Cumulative normalised transition rows and the per-row bracket ("guide") table.
//
// C[y, z] = min(1, (sum_{w<=z} P[y, w]) / (sum_w P[y, w])) with a sequential FP32 running
// sum in z order, one FP32 division per entry and the clamp at 1 -- the arithmetic of
// oplib/opcuda/sck.cu:43-84, so the rows are bit-identical to a sequential CPU loop.
// Negative entries (FP32 rounding residue of a squared kernel) are taken as 0 so the
// rows are non-decreasing and every correct inverse-CDF search returns the same state.
//
// The guide table follows the bracket table the reference builds on the host
// (oplib/opmodel/models/CModel Host Double.cs:434-455): for bucket b of nb (a power of
// two) it stores lb = first z with C[z] > b/nb and ub = first z with C[z] >= (b+1)/nb
// (d-1 for the last bucket or if none), packed lb | ub << 16.  A uniform u with
// floor(u*nb) = b has its answer "smallest z with u < C[z], capped at d-1" in [lb, ub].
#include "common.cuh"
#include "lattice.h"

namespace opb {

// Row-major rows (row y contiguous).  One warp handles 32 rows (lane = row while summing)
// in two passes over the row block: the row totals, then the running sums again in the
// same order, divided and clamped.  Each pass walks 32-column tiles staged through shared
// memory (coalesced loads and stores), with the next tile's loads in flight while the
// current one is summed; the outputs are written once.
__global__ void k_sck_rm(int d, int nrows, const float *__restrict__ P, float *__restrict__ C) {
    __shared__ float t[32][33];
    const int lane = threadIdx.x;
    const int r0 = blockIdx.x * 32;
    float nxt[32];
    auto load = [&](int c0) {
#pragma unroll
        for (int i = 0; i < 32; i++) {
            const int r = r0 + i, c = c0 + lane;
            nxt[i] = (r < nrows && c < d) ? P[(long long)r * d + c] : 0.f;
        }
    };
    float total = 0.f;
    for (int pass = 0; pass < 2; pass++) {
        float acc = 0.f;
        load(0);
        for (int c0 = 0; c0 < d; c0 += 32) {
#pragma unroll
            for (int i = 0; i < 32; i++) t[i][lane] = nxt[i];
            __syncwarp();
            if (c0 + 32 < d) load(c0 + 32);
            const int cmax = min(32, d - c0);
            if (cmax == 32) {
                // whole tile: the row's 32 values into registers, the dependent additions,
                // then the (independent) divisions
                float pv[32];
#pragma unroll
                for (int j = 0; j < 32; j++) pv[j] = t[lane][j];
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    const float p = pv[j] > 0.f ? pv[j] : 0.f;
                    acc = (c0 + j == 0) ? p : __fadd_rn(acc, p);
                    pv[j] = acc;
                }
                if (pass == 1) {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        const float v = __fdiv_rn(pv[j], total);
                        t[lane][j] = v < 1.0f ? v : 1.0f;
                    }
                }
            } else {
                for (int j = 0; j < cmax; j++) {
                    float p = t[lane][j];
                    p = p > 0.f ? p : 0.f;
                    acc = (c0 + j == 0) ? p : __fadd_rn(acc, p);
                    if (pass == 1) {
                        const float v = __fdiv_rn(acc, total);
                        t[lane][j] = v < 1.0f ? v : 1.0f;
                    }
                }
            }
            __syncwarp();
            if (pass == 1) {
#pragma unroll
                for (int i = 0; i < 32; i++) {
                    const int r = r0 + i, c = c0 + lane;
                    if (r < nrows && c < d) C[(long long)r * d + c] = t[i][lane];
                }
            }
            __syncwarp();
        }
        total = acc;
    }
}

// Column-major rows as in the reference: element (y1, y2) at m*d*d + y1 + d*y2, thread
// per (m, y1) -- consecutive threads touch consecutive addresses.
__global__ void k_sck_cm(int d, int nm, const float *__restrict__ P, float *__restrict__ C) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nm * d) return;
    long long m = t / d;
    int y1 = (int)(t - m * d);
    const float *p = P + m * d * (long long)d + y1;
    float *c = C + m * d * (long long)d + y1;
    float acc = 0.f;
    for (int z = 0; z < d; z++) {
        float v = p[(long long)z * d];
        v = v > 0.f ? v : 0.f;
        acc = (z == 0) ? v : __fadd_rn(acc, v);
        c[(long long)z * d] = acc;
    }
    for (int z = 0; z < d; z++) {
        float v = __fdiv_rn(c[(long long)z * d], acc);
        c[(long long)z * d] = v < 1.0f ? v : 1.0f;
    }
}

// One warp per row; lanes scan the row for each bucket boundary.
__global__ void k_guide(int d, int nrows, int nb, const float *__restrict__ C, uint32_t *__restrict__ guide) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nrows) return;
    const float *row = C + (long long)warp * d;
    const float inv = 1.0f / (float)nb;  // exact: nb is a power of two
    for (int b = lane; b < nb; b += 32) {
        float lo_t = (float)b * inv, hi_t = (float)(b + 1) * inv;
        // first z with C[z] > lo_t (binary search on the non-decreasing row)
        int lo = 0, hi = d;  // answer in [lo, hi], d = none
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (row[mid] > lo_t) hi = mid; else lo = mid + 1;
        }
        int lb = lo < d ? lo : d - 1;
        int ub;
        if (b == nb - 1) {
            ub = d - 1;
        } else {
            lo = 0; hi = d;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (row[mid] >= hi_t) hi = mid; else lo = mid + 1;
            }
            ub = lo < d ? lo : d - 1;
        }
        if (ub < lb) ub = lb;
        guide[(long long)warp * nb + b] = (uint32_t)lb | ((uint32_t)ub << 16);
    }
}

int launch_sck_rm(int d, int nrows, const float *P, float *C, cudaStream_t s) {
    k_sck_rm<<<(nrows + 31) / 32, 32, 0, s>>>(d, nrows, P, C);
    return (int)cudaGetLastError();
}

int launch_guide(int d, int nrows, int nb, const float *C, uint32_t *guide, cudaStream_t s) {
    long long threads = (long long)nrows * 32;
    k_guide<<<(int)((threads + 255) / 256), 256, 0, s>>>(d, nrows, nb, C, guide);
    return (int)cudaGetLastError();
}

}  // namespace opb

// Reference entry point: nm column-major d x d kernels -> cumulative rows
// (oplib/opcuda/sck.cu:88-93).
OPB_API int opcuda_sck(int d, int nm, uint64_t tpker_yy_m, uint64_t ctpker_yy_m) {
    OPB_REQUIRE(d >= 0 && nm >= 0, OPB_E_ARG);
    if (d == 0 || nm == 0) return opb::set_status(OPB_OK);
    OPB_REQUIRE(tpker_yy_m != 0 && ctpker_yy_m != 0, OPB_E_NULL);
    long long n = (long long)nm * d;
    opb::k_sck_cm<<<(int)((n + 127) / 128), 128, 0, opb::stream()>>>(
        d, nm, reinterpret_cast<const float *>(tpker_yy_m), reinterpret_cast<float *>(ctpker_yy_m));
    return opb::launch_check();
}

// Row-major (source-major) cumulative rows for nrows rows of length d.
OPB_API int opb_sck_rm(int d, int nrows, const float *P, float *C) {
    OPB_REQUIRE(d > 0 && nrows >= 0, OPB_E_ARG);
    if (nrows == 0) return opb::set_status(OPB_OK);
    OPB_REQUIRE(P && C, OPB_E_NULL);
    return opb::set_status(opb::launch_sck_rm(d, nrows, P, C, opb::stream()));
}

OPB_API int opb_guide_table(int d, int nrows, int nb, const float *C, uint32_t *guide) {
    OPB_REQUIRE(d > 0 && d <= 65535 && nrows >= 0, OPB_E_ARG);
    OPB_REQUIRE(nb >= 1 && nb <= 4096 && (nb & (nb - 1)) == 0, OPB_E_ARG);
    if (nrows == 0) return opb::set_status(OPB_OK);
    OPB_REQUIRE(C && guide, OPB_E_NULL);
    return opb::set_status(opb::launch_guide(d, nrows, nb, C, guide, opb::stream()));
}
