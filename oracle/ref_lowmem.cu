// Device memory below 4 GB of address space, for the reference kernels that read 32-bit
// device pointers (oracle/ref_tables.cu).  TEST INFRASTRUCTURE ONLY.
//
// The reference passes device addresses as 32-bit `unsigned` (oplib/opcuda/util.cu:182-221),
// which was safe on the 32-bit hosts it was written for.  Here a virtual address range is
// reserved with a requested start below 2^32 (cuMemAddressReserve, the driver API's virtual
// memory management) and backed by device memory; a range the driver places at or above
// 2^32 is released and the next start tried.  ref_low_alloc fails cleanly (no memory is
// handed out) when no such range is available, and the tests then skip.
#include <cstdint>

#include <cuda.h>
#include <cuda_runtime.h>

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {
// driver entry points resolved through the runtime, so the library does not link libcuda
using PfnGran = CUresult (*)(size_t *, const CUmemAllocationProp *, CUmemAllocationGranularity_flags);
using PfnReserve = CUresult (*)(CUdeviceptr *, size_t, size_t, CUdeviceptr, unsigned long long);
using PfnAddrFree = CUresult (*)(CUdeviceptr, size_t);
using PfnCreate = CUresult (*)(CUmemGenericAllocationHandle *, size_t, const CUmemAllocationProp *,
                               unsigned long long);
using PfnRelease = CUresult (*)(CUmemGenericAllocationHandle);
using PfnMap = CUresult (*)(CUdeviceptr, size_t, size_t, CUmemGenericAllocationHandle, unsigned long long);
using PfnUnmap = CUresult (*)(CUdeviceptr, size_t);
using PfnAccess = CUresult (*)(CUdeviceptr, size_t, const CUmemAccessDesc *, size_t);
struct Drv {
    PfnGran gran = nullptr;
    PfnReserve reserve = nullptr;
    PfnAddrFree addr_free = nullptr;
    PfnCreate create = nullptr;
    PfnRelease release = nullptr;
    PfnMap map = nullptr;
    PfnUnmap unmap = nullptr;
    PfnAccess access = nullptr;
};
template <class F>
bool entry(const char *name, F &f) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return false;
    f = reinterpret_cast<F>(p);
    return true;
}
bool drv(Drv &d) {
    return entry("cuMemGetAllocationGranularity", d.gran) && entry("cuMemAddressReserve", d.reserve) &&
           entry("cuMemAddressFree", d.addr_free) && entry("cuMemCreate", d.create) &&
           entry("cuMemRelease", d.release) && entry("cuMemMap", d.map) && entry("cuMemUnmap", d.unmap) &&
           entry("cuMemSetAccess", d.access);
}
Drv g_drv;

struct LowBlock {
    CUdeviceptr p;
    size_t size;
    CUmemGenericAllocationHandle h;
};
LowBlock g_blocks[16];
int g_nblocks = 0;
}  // namespace

REF_API int ref_low_alloc(unsigned long long bytes, unsigned long long *out) {
    if (!out || bytes == 0 || g_nblocks >= 16) return -1;
    *out = 0;
    if (cudaFree(0) != cudaSuccess) return -2;  // the runtime's primary context is current
    if (!g_drv.gran && !drv(g_drv)) return -2;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -2;
    CUmemAllocationProp prop = {};
    prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
    prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
    prop.location.id = dev;
    size_t gran = 0;
    if (g_drv.gran(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_MINIMUM) != CUDA_SUCCESS || !gran)
        return -3;
    const size_t size = (bytes + gran - 1) / gran * gran;
    CUdeviceptr p = 0;
    for (unsigned long long start = 0x40000000ull; start + size <= (1ull << 32); start += 0x10000000ull) {
        CUdeviceptr q = 0;
        if (g_drv.reserve(&q, size, gran, (CUdeviceptr)start, 0) != CUDA_SUCCESS) continue;
        if (q != 0 && (unsigned long long)q + size <= (1ull << 32)) {
            p = q;
            break;
        }
        g_drv.addr_free(q, size);
    }
    if (!p) return -4;
    CUmemGenericAllocationHandle h;
    if (g_drv.create(&h, size, &prop, 0) != CUDA_SUCCESS) {
        g_drv.addr_free(p, size);
        return -5;
    }
    if (g_drv.map(p, size, 0, h, 0) != CUDA_SUCCESS) {
        g_drv.release(h);
        g_drv.addr_free(p, size);
        return -6;
    }
    CUmemAccessDesc acc = {};
    acc.location = prop.location;
    acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
    if (g_drv.access(p, size, &acc, 1) != CUDA_SUCCESS) {
        g_drv.unmap(p, size);
        g_drv.release(h);
        g_drv.addr_free(p, size);
        return -7;
    }
    g_blocks[g_nblocks++] = LowBlock{p, size, h};
    *out = (unsigned long long)p;
    return 0;
}

REF_API int ref_low_free_all(void) {
    cudaDeviceSynchronize();
    for (int i = 0; i < g_nblocks; i++) {
        g_drv.unmap(g_blocks[i].p, g_blocks[i].size);
        g_drv.release(g_blocks[i].h);
        g_drv.addr_free(g_blocks[i].p, g_blocks[i].size);
    }
    g_nblocks = 0;
    return 0;
}

// plain copies, so that the tests can fill and read low memory without another library
REF_API int ref_memcpy_h2d(unsigned long long dst, const void *src, unsigned long long bytes) {
    return (int)cudaMemcpy(reinterpret_cast<void *>(dst), src, bytes, cudaMemcpyHostToDevice);
}
REF_API int ref_memcpy_d2h(void *dst, unsigned long long src, unsigned long long bytes) {
    return (int)cudaMemcpy(dst, reinterpret_cast<const void *>(src), bytes, cudaMemcpyDeviceToHost);
}
