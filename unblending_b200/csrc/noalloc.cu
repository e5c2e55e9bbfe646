// Fixed device scratch for unblending_unmix_device_noalloc.
//
// The first-pass solve needs scratch beyond its inputs and outputs: the
// work-queue heads, the miss counters and two lists of pixels that missed
// the feasibility tolerance (for the FP64 re-solve). The allocation-free entry
// point takes that scratch from this file-scope array instead of cudaMalloc.
// The array exists once per device that loads this module and lives until
// the process exits.
#include <mutex>

#include "solver_dispatch.hpp"

namespace unb {

// 256 bytes of queue heads and counters, then two int32 pixel lists of up to
// kNoAllocMaxPixels entries each.
constexpr size_t kNoAllocMaxPixels = size_t(2048) * 2048;
constexpr size_t kNoAllocScratchBytes = 256 + 2 * sizeof(int32_t) * kNoAllocMaxPixels;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

size_t noalloc_max_pixels() { return kNoAllocMaxPixels; }

// Device address of the scratch array on the current device. In host code the
// array's name is only a host-side stand-in, so the address is resolved with
// cudaGetSymbolAddress, once per device (with that device current), on the
// first call, and cached.
cudaError_t noalloc_scratch(void** ptr, size_t* bytes, size_t* max_pixels) {
    static std::mutex mutex;
    static void* cache[256] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mutex);
    if (!cache[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        cache[dev] = p;
    }
    *ptr = cache[dev];
    *bytes = kNoAllocScratchBytes;
    *max_pixels = kNoAllocMaxPixels;
    return cudaSuccess;
}

}  // namespace unb
