// buffer_cache.h -- a process-wide cache of host buffers whose allocation
// is slow (page-locked staging: cudaHostAlloc costs about 0.4 ms per MB).
// A context gives its buffer back when it is destroyed or grows; the next
// context that needs one takes the smallest cached buffer that is large
// enough.  At most `max_held` bytes stay cached; a buffer given beyond that
// is released at once.  Allocation and release are passed in, so the
// policy is plain host C++ and is tested on its own.
#pragma once

#include <cstddef>
#include <map>
#include <mutex>

namespace sp3mm {

template <class Alloc, class Release>
class BufferCache {
public:
    BufferCache(Alloc alloc, Release release, size_t max_held)
        : alloc_(alloc), release_(release), max_held_(max_held) {}

    // A cached buffer of at least `bytes`, else a new one of `bytes`
    // (nullptr when allocation fails); *got = its size.
    void* take(size_t bytes, size_t* got) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = free_.lower_bound(bytes);
            if (it != free_.end()) {
                void* p = it->second;
                *got = it->first;
                held_ -= it->first;
                free_.erase(it);
                return p;
            }
        }
        void* p = alloc_(bytes);
        *got = p ? bytes : 0;
        return p;
    }

    // Hand back a buffer of `bytes` that nothing uses any more.
    void give(void* p, size_t bytes) {
        if (!p) return;
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (held_ + bytes <= max_held_) {
                free_.emplace(bytes, p);
                held_ += bytes;
                return;
            }
        }
        release_(p);
    }

    // Release every cached buffer.
    void drain() {
        std::multimap<size_t, void*> all;
        {
            std::lock_guard<std::mutex> lk(mu_);
            all.swap(free_);
            held_ = 0;
        }
        for (auto& kv : all) release_(kv.second);
    }

    size_t held() {
        std::lock_guard<std::mutex> lk(mu_);
        return held_;
    }

private:
    Alloc alloc_;
    Release release_;
    const size_t max_held_;
    std::mutex mu_;
    std::multimap<size_t, void*> free_;   // size -> buffer, guarded by mu_
    size_t held_ = 0;                     // guarded by mu_
};

}  // namespace sp3mm
