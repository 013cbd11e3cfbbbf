// Shared definitions for the opcuda-b200 library (sm_100a).
//
// Error model: every exported entry point returns an int status -- 0 on success, a
// negative OPB_E* code for an argument error detected on the host, or a positive
// cudaError_t.  The last status is also kept per host thread and can be read through
// opcuda_get_status(), which is how the reference's callers read it
// (oplib/opcuda/util.cu:59,204-207; oplib/opmodel/types/CArray.cs:577-578).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#define OPB_API extern "C" __attribute__((visibility("default")))

enum {
    OPB_OK = 0,
    OPB_E_ARG = -1,       // bad size / count
    OPB_E_NULL = -2,      // null pointer where one is required
    OPB_E_ALIGN = -3,     // pointer or size misaligned for the kernel's vector access
    OPB_E_UNSUPPORTED = -4,
    OPB_E_NOMEM = -5,
    OPB_E_TIMEOUT = -6,   // a bounded device wait ran out
    OPB_E_STATE = -7,     // call out of order (missing init, plan not built, ...)
};

namespace opb {

int set_status(int s);            // records and returns s
int set_cuda(cudaError_t e);      // records and returns (int)e
cudaStream_t stream();            // the calling thread's current library stream
int num_sms();                    // SM count of the current device (cached per device)
int launch_check();               // cudaGetLastError -> status

inline bool aligned(const void *p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

// Profiler range over one library call (NVTX; a no-op unless a profiler is attached), so
// that a capture can select a call's kernels by name.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace opb

#define OPB_NVTX(name) opb::NvtxRange opb_nvtx_range_(name)

#define OPB_TRY(expr)                                  \
    do {                                               \
        cudaError_t _e = (expr);                       \
        if (_e != cudaSuccess) return opb::set_cuda(_e); \
    } while (0)

#define OPB_REQUIRE(cond, code)                        \
    do {                                               \
        if (!(cond)) return opb::set_status(code);     \
    } while (0)
