// Stress test of sp3mm::HostPool (sp3mm4amg_b200/csrc/host_pool.h), built
// and run by tests/test_host_native.py: many short runs back to back, so that
// workers wake late for runs that already finished.  Every index of every
// run must be processed exactly once, and no chunk may still be running
// when run() returns.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <thread>
#include <vector>

#include "host_pool.h"

int main(int argc, char** argv) {
    const int runs = argc > 1 ? std::atoi(argv[1]) : 100000;
    const int workers = argc > 2 ? std::atoi(argv[2]) : 7;
    // Kept for the life of the process, as the library keeps its pool.
    sp3mm::HostPool& pool = *new sp3mm::HostPool(workers);
    std::mt19937 rng(12345);
    std::vector<std::atomic<int>> hits(4096);
    std::atomic<int> in_flight{0};
    std::atomic<long long> bad{0};
    for (int r = 0; r < runs; ++r) {
        const int chunks = 2 + static_cast<int>(rng() % 15);
        const long long chunk = 1 + rng() % 64;
        const long long n = chunks * chunk - static_cast<long long>(rng() % chunk);
        for (long long i = 0; i < n; ++i) hits[i].store(0, std::memory_order_relaxed);
        const bool yield = (r & 7) == 0;
        const sp3mm::HostPool::Fn fn = [&](long long lo, long long hi) {
            in_flight.fetch_add(1);
            for (long long i = lo; i < hi; ++i) hits[i].fetch_add(1, std::memory_order_relaxed);
            if (yield) std::this_thread::yield();
            in_flight.fetch_sub(1);
        };
        {
            std::lock_guard<std::mutex> lk(pool.use);
            pool.run(fn, n, chunk, static_cast<int>((n + chunk - 1) / chunk));
        }
        if (in_flight.load() != 0) ++bad;
        for (long long i = 0; i < n; ++i)
            if (hits[i].load(std::memory_order_relaxed) != 1) ++bad;
        if (bad) {
            std::printf("run %d: %lld bad\n", r, bad.load());
            return 1;
        }
    }
    std::printf("ok %d runs\n", runs);
    return 0;
}
