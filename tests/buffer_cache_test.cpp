// Test of sp3mm::BufferCache (sp3mm4amg_b200/csrc/buffer_cache.h), built and
// run by tests/test_host_native.py with a fake allocator that records every
// buffer's state: the policy (smallest large-enough buffer, the cap on
// cached bytes, drain), then 8 threads taking and giving buffers, where no
// buffer may be handed to two holders and nothing may leak.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <random>
#include <set>
#include <thread>
#include <vector>

#include "buffer_cache.h"

namespace {

std::mutex g_mu;
std::set<void*> g_live;   // allocated, not released
std::atomic<long long> g_allocs{0}, g_releases{0};

struct FakeAlloc {
    void* operator()(size_t bytes) const {
        void* p = std::malloc(bytes ? bytes : 1);
        std::lock_guard<std::mutex> lk(g_mu);
        g_live.insert(p);
        ++g_allocs;
        return p;
    }
};
struct FakeRelease {
    void operator()(void* p) const {
        {
            std::lock_guard<std::mutex> lk(g_mu);
            if (!g_live.erase(p)) std::abort();   // released twice or never allocated
        }
        ++g_releases;
        std::free(p);
    }
};

#define CHECK(c)                                              \
    do {                                                      \
        if (!(c)) {                                           \
            std::printf("check failed line %d: %s\n", __LINE__, #c); \
            return 1;                                         \
        }                                                     \
    } while (0)

}  // namespace

int main() {
    using Cache = sp3mm::BufferCache<FakeAlloc, FakeRelease>;
    {
        Cache c(FakeAlloc{}, FakeRelease{}, 3 << 20);
        size_t got = 0;
        void* a = c.take(1 << 20, &got);
        CHECK(a && got == (1u << 20) && g_allocs == 1);
        void* b = c.take(2 << 20, &got);
        CHECK(b && got == (2u << 20) && g_allocs == 2);
        c.give(a, 1 << 20);
        c.give(b, 2 << 20);
        CHECK(c.held() == (3u << 20));
        void* x = c.take(1536 << 10, &got);   // smallest buffer >= 1.5 MB
        CHECK(x == b && got == (2u << 20) && g_allocs == 2);
        void* y = c.take(512 << 10, &got);    // the 1 MB one
        CHECK(y == a && got == (1u << 20) && c.held() == 0);
        void* z = c.take(4 << 20, &got);      // nothing large enough: allocate
        CHECK(z && got == (4u << 20) && g_allocs == 3);
        c.give(z, 4 << 20);                   // over the 3 MB cap: released
        CHECK(g_releases == 1 && c.held() == 0);
        c.give(x, 2 << 20);
        c.give(y, 1 << 20);
        CHECK(c.held() == (3u << 20));
        c.drain();
        CHECK(c.held() == 0 && g_releases == 3 && g_live.empty());
    }
    {
        Cache c(FakeAlloc{}, FakeRelease{}, 64 << 20);
        std::mutex own_mu;
        std::set<void*> owned;   // buffers currently held by some thread
        std::atomic<int> bad{0};
        std::vector<std::thread> th;
        for (int t = 0; t < 8; ++t) {
            th.emplace_back([&, t] {
                std::mt19937 rng(100 + t);
                for (int i = 0; i < 20000; ++i) {
                    const size_t bytes = size_t(1) << (10 + rng() % 12);
                    size_t got = 0;
                    void* p = c.take(bytes, &got);
                    if (!p || got < bytes) ++bad;
                    {
                        std::lock_guard<std::mutex> lk(own_mu);
                        if (!owned.insert(p).second) ++bad;   // two holders
                    }
                    if (rng() % 4 == 0) std::this_thread::yield();
                    {
                        std::lock_guard<std::mutex> lk(own_mu);
                        owned.erase(p);
                    }
                    c.give(p, got);
                }
            });
        }
        for (auto& x : th) x.join();
        CHECK(bad == 0);
        CHECK(c.held() <= (64u << 20));
        c.drain();
        CHECK(g_live.empty() && g_allocs == g_releases);
    }
    std::printf("ok\n");
    return 0;
}
