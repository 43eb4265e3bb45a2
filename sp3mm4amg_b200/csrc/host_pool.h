// host_pool.h -- persistent host worker threads for the transfer loops
// (narrowing, widening, copies into caller arrays): creating threads per
// call cost more than the work of a call.
//
// One caller at a time runs work on a pool (it holds `use`); the caller
// takes chunks too and returns when every chunk is done.  Each run has a
// generation, and the chunk counter carries it in its high half: a worker
// claims a chunk only while the counter still names the run it woke for,
// so a worker that wakes late can neither run a chunk of the next run with
// the previous run's bounds nor count its chunk toward the wrong run.
// Plain host C++ (no CUDA), so the pool is tested on its own.
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <thread>

namespace sp3mm {

class HostPool {
public:
    using Fn = std::function<void(long long, long long)>;

    // n worker threads (detached: a pool lives as long as the process).
    explicit HostPool(int n) : nthreads_(n) {
        for (int k = 0; k < n; ++k) std::thread([this] { work(); }).detach();
    }
    // Never destroyed: its workers wait on its condition variable for good
    // (create pools with new and keep them).
    ~HostPool() = delete;
    HostPool(const HostPool&) = delete;
    HostPool& operator=(const HostPool&) = delete;
    int size() const { return nthreads_; }
    std::mutex use;

    // Run fn over `chunks` pieces [i*chunk, min(n, (i+1)*chunk)); the caller
    // (holding `use`) takes pieces too and returns when all are done.
    void run(const Fn& fn, long long n, long long chunk, int chunks) {
        Job j{&fn, n, chunk, chunks, 0};
        {
            std::lock_guard<std::mutex> lk(m_);
            j.gen = ++gen_;
            job_ = j;
            finished_ = 0;
            next_.store(static_cast<uint64_t>(j.gen) << 32);
        }
        cv_.notify_all();
        pull(j);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return finished_ == chunks; });
        job_.fn = nullptr;
    }

private:
    struct Job {
        const Fn* fn;
        long long n, chunk;
        int chunks;
        uint32_t gen;
    };

    // Claim and run chunks of run j.gen until none is left or another run
    // has started; count the chunks done toward run j.gen (which cannot
    // complete before they are counted, so `finished_` is still its count).
    void pull(const Job& j) {
        int done = 0;
        uint64_t v = next_.load();
        for (;;) {
            if (static_cast<uint32_t>(v >> 32) != j.gen) break;
            const int i = static_cast<int>(v & 0xffffffffu);
            if (i >= j.chunks) break;
            if (!next_.compare_exchange_weak(v, v + 1)) continue;   // v reloaded
            const long long lo = i * j.chunk;
            (*j.fn)(lo, std::min(j.n, lo + j.chunk));
            ++done;
            v = next_.load();
        }
        if (done) {
            std::lock_guard<std::mutex> lk(m_);
            finished_ += done;
            if (finished_ == j.chunks) done_.notify_all();
        }
    }

    void work() {
        uint32_t seen = 0;
        for (;;) {
            Job j{};
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (!job_.fn) continue;
                j = job_;
            }
            pull(j);
        }
    }

    const int nthreads_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    Job job_{nullptr, 0, 1, 0, 0};   // guarded by m_
    int finished_ = 0;               // guarded by m_
    uint32_t gen_ = 0;               // guarded by m_
    std::atomic<uint64_t> next_{0};  // (generation << 32) | next chunk
};

}  // namespace sp3mm
