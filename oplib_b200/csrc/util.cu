// Runtime support surface of the opcuda C-ABI: status, devices, memory, copies, fills
// and timers.  Replaces oplib/opcuda/util.cu, scopy2.cu (scopy1) and sset.cu with
// 64-bit device handles (the reference truncates device pointers to 32 bits,
// oplib/opcuda/util.cu:209-213, which cannot work on a 64-bit host).
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>

#include "common.cuh"

namespace opb {

static thread_local int t_status = 0;
static thread_local cudaStream_t t_stream = nullptr;

int set_status(int s) {
    t_status = s;
    return s;
}
int set_cuda(cudaError_t e) { return set_status(static_cast<int>(e)); }
cudaStream_t stream() { return t_stream; }

int num_sms() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

int launch_check() {
    cudaError_t e = cudaGetLastError();
    return set_cuda(e);
}

}  // namespace opb

using opb::set_cuda;
using opb::set_status;

// ------------------------------------------------------------------ status / streams

OPB_API int opcuda_get_status(void) { return opb::t_status; }

OPB_API int opb_set_stream(uint64_t stream) {
    opb::t_stream = reinterpret_cast<cudaStream_t>(stream);
    return set_status(OPB_OK);
}

OPB_API uint64_t opb_get_stream(void) { return reinterpret_cast<uint64_t>(opb::t_stream); }

OPB_API const char *opb_version(void) { return "opcuda-b200 1.0 (sm_100a)"; }

OPB_API const char *opb_status_string(int status) {
    switch (status) {
        case OPB_OK: return "ok";
        case OPB_E_ARG: return "invalid size or count";
        case OPB_E_NULL: return "null pointer";
        case OPB_E_ALIGN: return "misaligned pointer or size";
        case OPB_E_UNSUPPORTED: return "unsupported configuration";
        case OPB_E_NOMEM: return "out of memory";
        case OPB_E_TIMEOUT: return "bounded device wait expired";
        case OPB_E_STATE: return "call out of order";
        default: break;
    }
    if (status > 0) return cudaGetErrorString(static_cast<cudaError_t>(status));
    return "unknown status";
}

// ------------------------------------------------------------------ context / devices

// The reference initialises legacy cuBLAS here (oplib/opcuda/util.cu:123-126).  This
// library needs no cuBLAS context; the call creates the CUDA context on the current
// device so that later timings do not include context creation.
OPB_API int opcuda_cublas_init(void) {
    OPB_TRY(cudaFree(nullptr));
    (void)opb::num_sms();
    return set_status(OPB_OK);
}

OPB_API int opcuda_shutdown(void) {
    OPB_TRY(cudaDeviceSynchronize());
    return set_status(OPB_OK);
}

OPB_API int opcuda_thread_synchronize(void) {
    OPB_TRY(cudaDeviceSynchronize());
    return set_status(OPB_OK);
}

OPB_API int opcuda_set_device(int dev) {
    OPB_TRY(cudaSetDevice(dev));
    return set_status(OPB_OK);
}

OPB_API int opcuda_get_device(void) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    set_cuda(e);
    return e == cudaSuccess ? dev : -1;
}

OPB_API int opcuda_device_get_count(void) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    set_cuda(e);
    return e == cudaSuccess ? n : 0;
}

OPB_API int opcuda_device_count(void) { return opcuda_device_get_count(); }

OPB_API int opcuda_device_get_name(char *name, int len, int dev) {
    OPB_REQUIRE(name != nullptr, OPB_E_NULL);
    OPB_REQUIRE(len > 0, OPB_E_ARG);
    cudaDeviceProp p;
    OPB_TRY(cudaGetDeviceProperties(&p, dev));
    std::strncpy(name, p.name, static_cast<size_t>(len) - 1);
    name[len - 1] = '\0';
    return set_status(OPB_OK);
}

OPB_API int opcuda_device_total_memory(uint64_t *bytes, int dev) {
    OPB_REQUIRE(bytes != nullptr, OPB_E_NULL);
    cudaDeviceProp p;
    OPB_TRY(cudaGetDeviceProperties(&p, dev));
    *bytes = static_cast<uint64_t>(p.totalGlobalMem);
    return set_status(OPB_OK);
}

OPB_API int opcuda_multi_processor_count(int dev) {
    int n = 0;
    cudaError_t e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    set_cuda(e);
    return e == cudaSuccess ? n : 0;
}

OPB_API int opcuda_max_threads_per_block(int dev) {
    int n = 0;
    cudaError_t e = cudaDeviceGetAttribute(&n, cudaDevAttrMaxThreadsPerBlock, dev);
    set_cuda(e);
    return e == cudaSuccess ? n : 0;
}

// ------------------------------------------------------------------ memory

// Test hook: when positive, the n-th next device allocation fails with OPB_E_NOMEM
// (injected allocation failure for host-side fault tests; no device is touched).
static std::atomic<int> g_fail_alloc_countdown{0};

OPB_API int opb_test_fail_next_alloc(int n) {
    g_fail_alloc_countdown.store(n);
    return set_status(OPB_OK);
}

OPB_API uint64_t opcuda_mem_alloc(uint64_t sz) {
    int c = g_fail_alloc_countdown.load();
    if (c > 0) {
        if (g_fail_alloc_countdown.fetch_sub(1) == 1) {
            set_status(OPB_E_NOMEM);
            return 0;
        }
    }
    if (sz == 0) {
        set_status(OPB_E_ARG);
        return 0;
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, static_cast<size_t>(sz));
    set_cuda(e);
    return e == cudaSuccess ? reinterpret_cast<uint64_t>(p) : 0;
}

OPB_API int opcuda_mem_free_device(uint64_t ptr) {
    if (ptr == 0) return set_status(OPB_OK);
    OPB_TRY(cudaDeviceSynchronize());  // the reference synchronises before freeing
    OPB_TRY(cudaFree(reinterpret_cast<void *>(ptr)));
    return set_status(OPB_OK);
}

OPB_API uint64_t opcuda_mem_alloc_host(uint64_t sz) {
    if (sz == 0) {
        set_status(OPB_E_ARG);
        return 0;
    }
    void *p = nullptr;
    cudaError_t e = cudaMallocHost(&p, static_cast<size_t>(sz));
    set_cuda(e);
    return e == cudaSuccess ? reinterpret_cast<uint64_t>(p) : 0;
}

OPB_API int opcuda_mem_free_host(uint64_t hptr) {
    if (hptr == 0) return set_status(OPB_OK);
    OPB_TRY(cudaFreeHost(reinterpret_cast<void *>(hptr)));
    return set_status(OPB_OK);
}

// The reference's copies are blocking (cudaMemcpy, oplib/opcuda/util.cu:182-201); these
// keep that contract but order the copy on the library stream.
static int copy_blocking(uint64_t dst, uint64_t src, uint64_t sz, cudaMemcpyKind kind) {
    if (sz == 0) return set_status(OPB_OK);
    OPB_REQUIRE(dst != 0 && src != 0, OPB_E_NULL);
    cudaStream_t s = opb::stream();
    OPB_TRY(cudaMemcpyAsync(reinterpret_cast<void *>(dst), reinterpret_cast<const void *>(src),
                            static_cast<size_t>(sz), kind, s));
    OPB_TRY(cudaStreamSynchronize(s));
    return set_status(OPB_OK);
}

OPB_API int opcuda_memcpy_h2d(uint64_t dptr, uint64_t hptr, uint64_t sz) {
    return copy_blocking(dptr, hptr, sz, cudaMemcpyHostToDevice);
}
OPB_API int opcuda_memcpy_d2h(uint64_t dptr, uint64_t hptr, uint64_t sz) {
    return copy_blocking(hptr, dptr, sz, cudaMemcpyDeviceToHost);
}
OPB_API int opcuda_memcpy_d2d(uint64_t dptr2, uint64_t dptr1, uint64_t sz) {
    return copy_blocking(dptr2, dptr1, sz, cudaMemcpyDeviceToDevice);
}

// ------------------------------------------------------------------ timers (wall clock)

static std::chrono::steady_clock::time_point g_t0, g_t1;

OPB_API void opcuda_create_timer(void) { g_t0 = g_t1 = std::chrono::steady_clock::now(); }
OPB_API void opcuda_reset_timer(void) { g_t0 = g_t1 = std::chrono::steady_clock::now(); }
OPB_API void opcuda_stop_timer(void) { g_t1 = std::chrono::steady_clock::now(); }
OPB_API double opcuda_get_timer_value(void) {
    return std::chrono::duration<double>(g_t1 - g_t0).count();
}

// ------------------------------------------------------------------ copies and fills

__global__ void k_scopy(long n, const float *__restrict__ x, int incx, float *__restrict__ y, int incy) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long step = (long)gridDim.x * blockDim.x;
    for (; i < n; i += step) y[i * incy] = x[i * incx];
}

__global__ void k_sset(long n, float *__restrict__ x, int incx, float c) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long step = (long)gridDim.x * blockDim.x;
    for (; i < n; i += step) x[i * incx] = c;
}

static int grid_for(long n) {
    long b = (n + 255) / 256;
    long cap = 8L * opb::num_sms();
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return static_cast<int>(b);
}

OPB_API int opcuda_scopy(int n, uint64_t x, int incx, uint64_t y, int incy) {
    OPB_REQUIRE(n >= 0, OPB_E_ARG);
    if (n == 0) return set_status(OPB_OK);
    OPB_REQUIRE(x != 0 && y != 0, OPB_E_NULL);
    OPB_REQUIRE(incx > 0 && incy > 0, OPB_E_ARG);
    k_scopy<<<grid_for(n), 256, 0, opb::stream()>>>(n, reinterpret_cast<const float *>(x), incx,
                                                     reinterpret_cast<float *>(y), incy);
    return opb::launch_check();
}

// Contiguous float copy (oplib/opcuda/scopy2.cu:137-143 stages it through shared memory;
// a device-to-device async copy is the B200 equivalent).
OPB_API int opcuda_scopy1(uint64_t destination, uint64_t source, uint64_t n) {
    if (n == 0) return set_status(OPB_OK);
    OPB_REQUIRE(destination != 0 && source != 0, OPB_E_NULL);
    OPB_TRY(cudaMemcpyAsync(reinterpret_cast<void *>(destination), reinterpret_cast<const void *>(source),
                            static_cast<size_t>(n) * sizeof(float), cudaMemcpyDeviceToDevice, opb::stream()));
    return set_status(OPB_OK);
}

OPB_API int opcuda_ssetall(uint64_t x, int n, float c, int incx) {
    OPB_REQUIRE(n >= 0, OPB_E_ARG);
    if (n == 0) return set_status(OPB_OK);
    OPB_REQUIRE(x != 0, OPB_E_NULL);
    OPB_REQUIRE(incx > 0, OPB_E_ARG);
    k_sset<<<grid_for(n), 256, 0, opb::stream()>>>(n, reinterpret_cast<float *>(x), incx, c);
    return opb::launch_check();
}

OPB_API int opcuda_ssetone(uint64_t x, int n, float c, int i) {
    OPB_REQUIRE(x != 0, OPB_E_NULL);
    OPB_REQUIRE(i >= 0 && i < n, OPB_E_ARG);
    OPB_TRY(cudaMemcpyAsync(reinterpret_cast<float *>(x) + i, &c, sizeof(float), cudaMemcpyHostToDevice,
                            opb::stream()));
    OPB_TRY(cudaStreamSynchronize(opb::stream()));
    return set_status(OPB_OK);
}
