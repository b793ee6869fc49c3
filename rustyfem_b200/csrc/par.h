// Host fork-join helper: fn(first, last) over [0, n) in chunks, on all hardware threads
// (the analogue of the reference's src/par.rs for the host-side stages).
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <vector>

namespace rfg {

template <class F>
void parallel_chunks(int64_t n, int64_t chunk, F fn) {
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    if (n <= chunk || nt == 1) {
        if (n > 0) fn(0, n);
        return;
    }
    std::atomic<int64_t> next{0};
    auto work = [&] {
        for (;;) {
            int64_t a = next.fetch_add(chunk);
            if (a >= n) return;
            fn(a, std::min(n, a + chunk));
        }
    };
    std::vector<std::thread> th;
    for (unsigned i = 1; i < nt; i++) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

// Wall-clock laps of a host stage, printed to stderr when RFG_HOST_TIMING is set.
struct HostTimer {
    const char* what;
    bool on;
    std::chrono::steady_clock::time_point last;
    explicit HostTimer(const char* w) : what(w), on(enabled()), last(std::chrono::steady_clock::now()) {}
    void lap(const char* name) {
        if (!on) return;
        auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[rfg-host] %s: %s %.1f ms\n", what, name,
                     std::chrono::duration<double, std::milli>(now - last).count());
        last = now;
    }
    static bool enabled() {
        static const bool e = std::getenv("RFG_HOST_TIMING") != nullptr;
        return e;
    }
};

}  // namespace rfg
