// The static device scratch of s2dwc_plan_analysis_noalloc.
//
// The array is a file-scope __device__ object, so it is part of this file's
// module: the CUDA driver reserves it on a device when it loads the module
// there (with the default lazy module loading, at the first lookup below),
// and nothing in the library ever allocates or frees it.  Its contents start
// at zero, but the entry point that uses it writes every element before it
// reads it, so no call depends on what an earlier call left behind.
#include <cuda_runtime.h>

#include <mutex>

#include "s2dw_internal.h"

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[S2DWC_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_ptr[kMaxDevices] = {};

}  // namespace

namespace s2dw {

int noalloc_scratch(int device, void **ptr)
{
    if (device < 0 || device >= kMaxDevices)
        return set_error(S2DWC_ERROR_ARG_INVALID, "noalloc scratch: device %d out of range", device);
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_ptr[device]) {
        // `device` is current (the caller holds a device guard)
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(S2DWC_ERROR_CUDA, "cudaGetSymbolAddress of the static scratch on device %d failed: %s",
                             device, cudaGetErrorString(e));
        g_ptr[device] = p;
    }
    *ptr = g_ptr[device];
    return S2DWC_OK;
}

void noalloc_forget()
{
    std::lock_guard<std::mutex> g(g_mu);
    for (auto &q : g_ptr) q = nullptr;
}

}  // namespace s2dw
