// Process-wide cache of large host blocks (the NoInitAlloc allocator of symbolic.h sends
// every block of HOST_BLOCK_MIN bytes and more here).
//
// One factorization call builds several hundred MB of host scratch (the node graph and its
// transpose, the front patterns, the plan's maps), and freshly mapped pages are faulted in
// one 4 KB page at a time, partly under the kernel's address-space lock when threads fault
// together. Freed blocks are kept (up to CACHE_MAX bytes, largest evicted first) and handed
// to the next request they fit within a factor of two, so a model analysed again reuses
// pages that are already mapped. (No transparent huge pages are asked for: on a host whose
// memory is fragmented a huge-page fault may compact memory first and stall the caller.)

#include "symbolic.h"

#include <sys/types.h>
#include <unistd.h>

#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <new>
#include <unordered_map>

namespace rfg {

namespace {

constexpr size_t PAGE = 4096;
constexpr size_t CACHE_MAX = (size_t)4 << 30;

struct HostBlocks {
    std::mutex mu;
    std::unordered_map<void*, size_t> live;  // block → capacity in bytes
    std::multimap<size_t, void*> cached;     // capacity → block
    size_t cached_bytes = 0;
};

// never destroyed: vectors freed during static destruction still find it. A forked child
// starts a cache of its own (the parent's lock may have been held by another thread at the
// fork); blocks it inherited are then not found on release and simply stay allocated.
HostBlocks& blocks() {
    static std::atomic<HostBlocks*> b{nullptr};
    static std::atomic<pid_t> owner{0};
    const pid_t me = ::getpid();
    if (owner.load(std::memory_order_acquire) == me) return *b.load(std::memory_order_acquire);  // b is set before owner
    static std::mutex init_mu;
    std::lock_guard<std::mutex> lock(init_mu);
    HostBlocks* cur = b.load(std::memory_order_acquire);
    if (!cur || owner.load(std::memory_order_acquire) != me) {
        cur = new HostBlocks();
        b.store(cur, std::memory_order_release);
        owner.store(me, std::memory_order_release);
    }
    return *cur;
}

}  // namespace

void* host_block_alloc(size_t bytes) {
    HostBlocks& B = blocks();
    const size_t cap = (bytes + PAGE - 1) / PAGE * PAGE;
    {
        std::lock_guard<std::mutex> lock(B.mu);
        auto it = B.cached.lower_bound(cap);
        if (it != B.cached.end() && it->first / 2 <= cap) {
            void* p = it->second;
            B.live[p] = it->first;
            B.cached_bytes -= it->first;
            B.cached.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    if (posix_memalign(&p, 64, cap) != 0) throw std::bad_alloc();
    std::lock_guard<std::mutex> lock(B.mu);
    B.live[p] = cap;
    return p;
}

void host_block_free(void* p) {
    if (!p) return;
    HostBlocks& B = blocks();
    std::lock_guard<std::mutex> lock(B.mu);
    auto it = B.live.find(p);
    if (it == B.live.end()) return;  // not a block of this cache: nothing to do
    const size_t cap = it->second;
    B.live.erase(it);
    B.cached.emplace(cap, p);
    B.cached_bytes += cap;
    while (B.cached_bytes > CACHE_MAX && !B.cached.empty()) {
        auto last = std::prev(B.cached.end());
        B.cached_bytes -= last->first;
        std::free(last->second);
        B.cached.erase(last);
    }
}

void host_release_cached() {
    HostBlocks& B = blocks();
    std::lock_guard<std::mutex> lock(B.mu);
    for (auto& e : B.cached) std::free(e.second);
    B.cached.clear();
    B.cached_bytes = 0;
}

}  // namespace rfg
