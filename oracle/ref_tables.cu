// Test harness around the reference's kernels that take device tables of 32-bit device
// pointers: global_ssqmm (oplib/opcuda/ssqmm.cu:119-179), global_sgemm4
// (oplib/opcuda/sgemm4.cu:84-154) and global_sgemv4 (oplib/opcuda/sgemv4.cu:88-180).
// TEST INFRASTRUCTURE ONLY, built by oracle/Makefile into oracle/_ref/libref_opcuda.so.
//
// The three reference files each define the same device helpers (rank1_update, ...), so each
// is included in a translation unit of its own: oracle/Makefile compiles this file three
// times, with REF_FILE = 1 (ssqmm.cu), 2 (sgemm4.cu) and 3 (sgemv4.cu).  The kernels read
// 32-bit pointers, so every table, record and matrix they touch must lie below 4 GB of
// device address space: the tests place them in memory from ref_low_alloc (ref_lowmem.cu),
// and the entry points here refuse any table address at or above 2^32.
#include <cstdint>

#include <cuda_runtime.h>

// (inside an unnamed namespace: their device helpers also get host definitions, whose names
// would otherwise collide between the objects, and with sgemv3.cu's in ref_opcuda.cu)
namespace {
#if REF_FILE == 1
#include "ssqmm.cu"
#elif REF_FILE == 2
#include "sgemm4.cu"
#else
#include "sgemv4.cu"
#endif
}  // namespace

#define REF_API extern "C" __attribute__((visibility("default")))

static int ref_done() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    return (int)cudaDeviceSynchronize();
}

static bool low(unsigned long long p) { return p != 0 && p < (1ull << 32); }

#if REF_FILE == 1
// ni column-major d x d products C_i = A_i . B_i from three device tables of 32-bit pointers,
// launched as opcuda_ssqmm launches them (ssqmm.cu:174-179); d % 64 == 0.
REF_API int ref_ssqmm(int d, int ni, unsigned long long A_i, unsigned long long B_i, unsigned long long C_i) {
    if (d <= 0 || d % 64 || ni < 1 || !low(A_i) || !low(B_i) || !low(C_i)) return -1;
    const int nb = (d + 63) / 64;
    dim3 grid(ni * nb, (d + 15) / 16), threads(16, 4);
    global_ssqmm<<<grid, threads>>>(nb, d, ni, (unsigned)A_i, (unsigned)B_i, (unsigned)C_i);
    return ref_done();
}
#elif REF_FILE == 2
// One block per task: argptr_bid is a device array of nblocks 32-bit pointers to 9-word
// task records {i, bx, by, m, n, k, A, B, C} (sgemm4.cu:84-102, launch 148-154).
REF_API int ref_sgemm4(int nblocks, unsigned long long argptr_bid) {
    if (nblocks < 1 || !low(argptr_bid)) return -1;
    global_sgemm4<<<dim3(nblocks, 1), dim3(16, 4)>>>((unsigned int *)argptr_bid);
    return ref_done();
}
#else
// One block per task: 10-word records {i, bx, by, d, nz, ncol, A, Z, col0, col1}
// (sgemv4.cu:90-107, launch 174-180).
REF_API int ref_sgemv4(int nblocks, unsigned long long argptr_bid) {
    if (nblocks < 1 || !low(argptr_bid)) return -1;
    global_sgemv4<<<dim3(nblocks, 1), dim3(16, 4)>>>((unsigned int *)argptr_bid);
    return ref_done();
}
#endif
