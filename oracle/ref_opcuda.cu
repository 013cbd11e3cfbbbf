// Test harness around the reference's own CUDA kernels.  TEST INFRASTRUCTURE ONLY: nothing
// in oplib_b200 links or loads it; only tests/ use it, as the checker of the drop-in entry
// points that replace these kernels.
//
// oracle/Makefile compiles this file with the reference's own flags (-DLINUX, nvcc defaults,
// so FMA contraction on as in oplib/opcuda/Makefile_osc_64:1-2) and with the reference's
// kernel directory (oplib/opcuda) on the include path, into oracle/_ref/libref_opcuda.so.
// The reference's sources are included unchanged; nothing of them is copied here.
//
// Why a harness: the reference's exported wrappers take 32-bit `unsigned` device handles
// (oplib/opcuda/util.cu:182-221), which truncate 64-bit addresses.  The __global__ kernels
// themselves take typed pointers, so this file launches them directly, with the launch
// shapes of the reference's own wrappers, and 64-bit pointers.  Only kernels that stay in
// bounds on the sizes the tests use are wrapped:
//   global_sck       (sck.cu:43-84, launch sck.cu:88-93)            any d, nm
//   global_sek/sekd/sekd_lambda (sek.cu:40-103, launches 106-137)     any d
//   global_sdot2     (sdot2.cu:48-68, launch sdot2.cu:72-83)         any m, n
//   global_sgemv3    (sgemv3.cu:92-159, launch sgemv3.cu:163-176)     d % 64 == 0, column
//                    lists padded to a multiple of 16 entries
//   global_sgsvg     (sgsvg.cu:40-209, launch sgsvg.cu:215-234)      nx*nr % 32 == 0, output
//                    zeroed by the caller
//   global_ssetall/ssetone (sset.cu:41-75)                           any n
// Wrapped in ref_tables.cu instead: global_ssqmm and global_sgemm4/sgemv4, whose device
// tables hold 32-bit pointers (run on memory below 4 GB, ref_lowmem.cu).  Not wrapped:
// global_sglvg (a __syncthreads inside a divergent branch) and the Monte Carlo kernels (their
// MT607 parameter file is not shipped).
//
// Every entry synchronises the device and returns the CUDA error code (0 = success).

#include <cstdint>

#include <cuda_runtime.h>

#include "sck.cu"
#include "sek.cu"
#include "sdot2.cu"
#include "sgemv3.cu"
#include "sgsvg.cu"
#include "sset.cu"

#define REF_API extern "C" __attribute__((visibility("default")))

static int ref_done() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    return (int)cudaDeviceSynchronize();
}

REF_API int ref_sck(int d, int nm, float *tpk, float *ctpk) {
    global_sck<<<32, 128>>>(d, nm, tpk, ctpk);
    return ref_done();
}

static dim3 sek_grid(int d) {
    int n = (d + 15) / 16;
    return dim3(n, n);
}

REF_API int ref_sek(int d, const float *gen, float dt, float *tpk) {
    global_sek<<<sek_grid(d), dim3(16, 16)>>>(d, gen, dt, tpk);
    return ref_done();
}

REF_API int ref_sekd(int d, const float *gen, float dt, float *tpk, float *r) {
    global_sekd<<<sek_grid(d), dim3(16, 16)>>>(d, gen, dt, tpk, r);
    return ref_done();
}

REF_API int ref_sekd_lambda(int d, const float *gen, float dt, float *tpk, float *r, float *lambda) {
    global_sekd_lambda<<<sek_grid(d), dim3(16, 16)>>>(d, gen, dt, tpk, r, lambda);
    return ref_done();
}

REF_API int ref_sdot2(float *a, float *b, float *c, int m, int n) {
    global_sdot2<<<GRIDDIM, BLOCKDIM>>>(a, b, c, m, n);
    return ref_done();
}

REF_API int ref_sgemv3(int d, int nz, int ncol, float *A, float *B, const int *col0, const int *col1) {
    if (d % 64 != 0) return -1;  // the kernel reads rows up to the next multiple of 64
    dim3 grid((d + 63) / 64, (ncol + 15) / 16), threads(16, 4);
    global_sgemv3<<<grid, threads>>>(d, nz, ncol, A, B, col0, col1);
    return ref_done();
}

// pars as in sgsvg.cu:221-230: xval[d], then SDrift, SVol, VolDrift, VolVol, Jumpsz_minus,
// Jumpsz_plus, each ni*d
REF_API int ref_sgsvg(float *gen, int ni, int nx, int nr, float *invm, float *pars) {
    int d = nx * nr;
    if (d % 32 != 0) return -1;
    global_sgsvg<<<ni * d / 32, 32>>>(gen, ni, nx, nr, invm, pars, pars + d, pars + d + ni * d,
                                      pars + d + 2 * ni * d, pars + d + 3 * ni * d, pars + d + 4 * ni * d,
                                      pars + d + 5 * ni * d);
    return ref_done();
}

REF_API int ref_ssetall(float *x, int n, float c, int incx) {
    global_ssetall<<<32, 128>>>(x, n, c, incx);
    return ref_done();
}

REF_API int ref_ssetone(float *x, int n, float c, int i) {
    global_ssetone<<<1, 128>>>(x, n, c, i);
    return ref_done();
}
