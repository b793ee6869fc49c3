// Host fork-join helper: fn(first, last) over [0, n) in chunks, on all hardware threads
// (the analogue of the reference's src/par.rs for the host-side stages).
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <vector>

#include <sys/types.h>
#include <unistd.h>

namespace rfg {

// Persistent workers for parallel_chunks: threads are created once per process (and again
// after a fork), so a call costs a wake-up instead of thread creation, and per-thread
// scratch (thread_local tables) survives from one call to the next.
class HostPool {
   public:
    static HostPool& get() {
        static std::mutex m;
        static HostPool* p = nullptr;
        std::lock_guard<std::mutex> lock(m);
        if (!p || p->pid_ != ::getpid()) p = new HostPool();  // the old one (other process) is left alone
        return *p;
    }
    unsigned workers() const { return (unsigned)th_.size(); }
    // runs f on every worker and on the caller; false (nothing run) when the pool is busy or
    // the caller is itself running a pool job (a nested call)
    template <class F>
    bool try_run(F& f) {
        if (in_job()) return false;
        std::unique_lock<std::mutex> run(run_mu_, std::try_to_lock);
        if (!run.owns_lock()) return false;
        {
            std::lock_guard<std::mutex> lock(mu_);
            job_ = [&f] { f(); };
            active_ = (int)th_.size();
            gen_++;
        }
        cv_.notify_all();
        in_job() = true;
        f();
        in_job() = false;
        std::unique_lock<std::mutex> lock(mu_);
        done_.wait(lock, [&] { return active_ == 0; });
        job_ = nullptr;
        return true;
    }

   private:
    static bool& in_job() {
        static thread_local bool b = false;
        return b;
    }
    HostPool() : pid_(::getpid()) {
        unsigned nt = std::max(1u, std::thread::hardware_concurrency());
        for (unsigned i = 1; i < nt; i++) th_.emplace_back([this] { loop(); });
        for (auto& t : th_) t.detach();
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            std::function<void()> f;
            {
                std::unique_lock<std::mutex> lock(mu_);
                cv_.wait(lock, [&] { return gen_ != seen; });
                seen = gen_;
                f = job_;
            }
            in_job() = true;
            if (f) f();
            in_job() = false;
            std::lock_guard<std::mutex> lock(mu_);
            if (--active_ == 0) done_.notify_one();
        }
    }
    pid_t pid_;
    std::vector<std::thread> th_;
    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_;
    std::function<void()> job_;
    uint64_t gen_ = 0;
    int active_ = 0;
};

// fn over [0, n) in chunks on the pool's workers and the caller when the pool is free,
// else on the calling thread alone: for callers that may run beside other users of the
// pool and would rather wait than start threads of their own.
template <class F>
void pool_chunks_or_serial(int64_t n, int64_t chunk, F fn) {
    if (n <= chunk) {
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
    if (!HostPool::get().try_run(work)) work();
}

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
    if (HostPool::get().try_run(work)) return;
    // the pool is busy (a nested call, or another host thread): threads of our own
    std::vector<std::thread> th;
    for (unsigned i = 1; i < nt; i++) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

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
