// Device memory of the library's handles: stream-ordered allocations from one memory
// pool per device that keeps freed blocks for reuse (release threshold = unlimited), so
// that factorizations done one after another (a Newton loop that builds a new handle per
// step, a batch of models) do not pay cudaMalloc / cudaFree for their multi-GB arenas
// every time. rfg_release_cached_memory() hands the cached blocks back to the driver.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"

namespace rfg {

namespace {

std::mutex g_mu;
std::vector<cudaMemPool_t> g_pools;  // per device ordinal, created on first use

cudaMemPool_t pool_for_current_device() {
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_mu);
    if ((int)g_pools.size() <= dev) g_pools.resize(dev + 1, nullptr);
    if (!g_pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        RFG_CUDA(cudaMemPoolCreate(&p, &props));
        uint64_t keep = UINT64_MAX;
        RFG_CUDA(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
        g_pools[dev] = p;
    }
    return g_pools[dev];
}

}  // namespace

void* dev_alloc(size_t bytes, cudaStream_t st) {
    void* p = nullptr;
    if (bytes == 0) bytes = 256;
    RFG_CUDA(cudaMallocFromPoolAsync(&p, bytes, pool_for_current_device(), st));
    return p;
}

void dev_free(void* p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
}

void release_cached_memory() {
    std::lock_guard<std::mutex> lock(g_mu);
    for (cudaMemPool_t p : g_pools)
        if (p) cudaMemPoolTrimTo(p, 0);
}

}  // namespace rfg
