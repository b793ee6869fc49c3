// Device memory of the library's handles: stream-ordered allocations from one memory
// pool per device that keeps freed blocks for reuse (release threshold = unlimited), so
// that factorizations done one after another (a Newton loop that builds a new handle per
// step, a batch of models) do not pay cudaMalloc / cudaFree for their multi-GB arenas
// every time. rfg_release_cached_memory() hands the cached blocks back to the driver.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "par.h"

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

// Large host -> device copies from pageable memory: the driver stages such copies through
// its own pinned buffers with one thread. Here all host threads copy chunk i into one of two
// reusable pinned staging buffers while the DMA of chunk i-1 from the other runs, so the
// copy runs at the link's rate instead of one core's memcpy rate. On return the source may
// be reused (as after a pageable cudaMemcpyAsync); the last DMA may still be in flight from
// the staging buffer, which the next upload waits for.
namespace {
constexpr size_t STAGE_BYTES = (size_t)32 << 20;
std::mutex g_stage_mu;
void* g_stage[2] = {nullptr, nullptr};
cudaEvent_t g_stage_ev[2] = {nullptr, nullptr};
}  // namespace

void host_upload(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes < ((size_t)8 << 20)) {
        if (bytes) RFG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        return;
    }
    std::lock_guard<std::mutex> lock(g_stage_mu);
    for (int b = 0; b < 2; b++)
        if (!g_stage[b]) {
            RFG_CUDA(cudaHostAlloc(&g_stage[b], STAGE_BYTES, cudaHostAllocPortable));
            RFG_CUDA(cudaEventCreateWithFlags(&g_stage_ev[b], cudaEventDisableTiming));
        }
    const char* s = static_cast<const char*>(src);
    char* d = static_cast<char*>(dst);
    int b = 0;
    for (size_t off = 0; off < bytes; off += STAGE_BYTES, b ^= 1) {
        const size_t len = std::min(STAGE_BYTES, bytes - off);
        RFG_CUDA(cudaEventSynchronize(g_stage_ev[b]));  // the previous DMA out of this buffer
        char* stage = static_cast<char*>(g_stage[b]);
        parallel_chunks((int64_t)len, (int64_t)1 << 20,
                        [&](int64_t a, int64_t e) { std::memcpy(stage + a, s + off + a, (size_t)(e - a)); });
        RFG_CUDA(cudaMemcpyAsync(d + off, stage, len, cudaMemcpyHostToDevice, st));
        RFG_CUDA(cudaEventRecord(g_stage_ev[b], st));
    }
}

void release_cached_memory() {
    std::lock_guard<std::mutex> lock(g_mu);
    for (cudaMemPool_t p : g_pools)
        if (p) cudaMemPoolTrimTo(p, 0);
}

}  // namespace rfg
