// noalloc.cu -- ndlgpu_gaussian_blur_noalloc: gaussian_blur with its scratch
// in a fixed device array, for callers that cannot allocate device memory
// (see include/ndlgpu.h).  No counterpart in the reference.
#include <mutex>
#include <string>

#include "internal.h"

namespace ndlgpu {
namespace {

constexpr size_t kScratchBytes = NDLGPU_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// The scratch.  In host code this name is only a stand-in for the device
// array (passing it to a kernel would hand over a host address); the device
// address comes from cudaGetSymbolAddress, per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of the scratch on the current device; looked up once per
// device, with that device current.
ndlgpu_status scratch_address(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(NDLGPU_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(NDLGPU_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return set_error(NDLGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_addr[dev] = ptr;
    }
    *out = g_addr[dev];
    return NDLGPU_OK;
}

}  // namespace
}  // namespace ndlgpu

extern "C" ndlgpu_status ndlgpu_gaussian_blur_noalloc(const ndlgpu_view* src, const ndlgpu_view* dst, double sigma,
                                                      int border, void* stream)
{
    using namespace ndlgpu;
    size_t need = 0;
    ndlgpu_status st = ndlgpu_gaussian_blur_workspace_size(src, dst, sigma, border, &need);
    if (st != NDLGPU_OK) return st;
    if (need > kScratchBytes)
        return set_error(NDLGPU_ERR_WORKSPACE,
                         "this blur needs " + std::to_string(need) + " bytes of scratch; the allocation-free entry "
                         "point has a fixed " + std::to_string(kScratchBytes) + " bytes");
    // the array goes along even when the query reports no scratch: a route
    // that needs some then finds it there (or fails with
    // NDLGPU_ERR_WORKSPACE), and never falls back to allocating
    void* ws = nullptr;
    if ((st = scratch_address(&ws)) != NDLGPU_OK) return st;
    return ndlgpu_gaussian_blur(src, dst, sigma, border, ws, kScratchBytes, stream);
}
