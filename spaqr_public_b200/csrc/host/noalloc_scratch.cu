// Fixed device workspace for spq_gmres_dev_noalloc.
//
// Some callers may not allocate device memory once they are running (a
// serving process that reserves all of its memory up front, or code between
// allocation-free checkpoints of a real-time loop). For them the GMRES
// workspace (the Householder basis H, five work vectors, reduction partials and
// scalars) lives in this file-scope array instead of cudaMalloc'd buffers.
// The array exists on every GPU that loads the library, for the life of the
// process, so it is kept to 32 MiB.
#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>

namespace spq {

constexpr size_t kNoAllocScratchDoubles = size_t(4) << 20;  // 4 Mi doubles = 32 MiB per device

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of the workspace on the CURRENT device. In host code the
// array's name is only a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress, once per device (the first call on each device), with
// that device current; later calls return the cached address.
cudaError_t noalloc_scratch(double** ptr, size_t* elems) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static double* cache[256] = {};
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!cache[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        cache[dev] = static_cast<double*>(p);
    }
    *ptr = cache[dev];
    *elems = kNoAllocScratchDoubles;
    return cudaSuccess;
}

}  // namespace spq
