// Host test of the per-context caching allocator (gp::Device in
// horkxg_b200/csrc/gp_common.cuh), built and run by tests/test_host.py with
// no GPU: its driver calls are replaced by a fake device that hands out host
// memory within a byte budget and refuses requests beyond it.  Prints one
// line per failed check and exits non-zero if any failed.
#include <cstdio>
#include <cstdlib>
#include <map>

#include "../horkxg_b200/csrc/gp_common.cuh"

namespace {

size_t g_budget = 0, g_used = 0;
int g_mallocs = 0, g_frees = 0;
std::map<void*, size_t> g_blocks;

cudaError_t fake_malloc(void** p, size_t bytes) {
    if (g_used + bytes > g_budget) return cudaErrorMemoryAllocation;
    *p = std::malloc(bytes);
    g_blocks[*p] = bytes;
    g_used += bytes;
    ++g_mallocs;
    return cudaSuccess;
}

cudaError_t fake_free(void* p) {
    auto it = g_blocks.find(p);
    if (it == g_blocks.end()) return cudaErrorInvalidValue;
    g_used -= it->second;
    g_blocks.erase(it);
    std::free(p);
    ++g_frees;
    return cudaSuccess;
}

void fake_device(gp::Device& d, size_t budget) {
    d.malloc_fn = fake_malloc;
    d.free_fn = fake_free;
    g_budget = budget;
}

int failures = 0;
#define CHECK(c)                                                        \
    do {                                                                \
        if (!(c)) {                                                     \
            std::printf("FAIL line %d: %s\n", __LINE__, #c);            \
            ++failures;                                                 \
        }                                                               \
    } while (0)

constexpr size_t KiB = size_t{1} << 10, MiB = size_t{1} << 20;

}  // namespace

int main() {
    using gp::Device;

    // size classes: 256-byte steps up to 4 KiB, then 1/16 of the power of two
    CHECK(Device::size_class(1) == 256);
    CHECK(Device::size_class(4096) == 4096);
    CHECK(Device::size_class(4097) == 4608);
    CHECK(Device::size_class(MiB) == MiB);
    CHECK(Device::size_class(MiB + 1) == MiB + 128 * KiB);

    {
        Device d;
        fake_device(d, 64 * MiB);
        void* a = d.alloc(MiB);                    // class 1 MiB, from the driver
        CHECK(a && g_mallocs == 1 && d.driver_allocs == 1);
        d.release(a);
        CHECK(d.cached_bytes == MiB && d.live_bytes == 0);

        // class 960 KiB: the cached 1 MiB block is within 25% and serves it
        void* b = d.alloc(900 * KiB);
        CHECK(b == a && g_mallocs == 1 && d.live_bytes == MiB);
        d.release(b);                              // back into its own class
        CHECK(d.free_blocks[MiB].size() == 1);

        // class 640 KiB: the 1 MiB block is more than 25% larger, so the driver
        void* c = d.alloc(600 * KiB);
        CHECK(c != a && g_mallocs == 2 && d.free_blocks[MiB].size() == 1);
        d.release(c);

        // under pressure only the exact class is reused
        d.pressure = true;
        void* e = d.alloc(900 * KiB);
        CHECK(e != a && g_mallocs == 3 && d.free_blocks[MiB].size() == 1);
        void* f = d.alloc(MiB);                    // exact class: the cached block
        CHECK(f == a && g_mallocs == 3);
        d.release(e);
        d.release(f);
        CHECK(d.live_bytes == 0 && d.alloc_calls == 5);
        d.release_cached();
        CHECK(d.cached_bytes == 0 && g_used == 0);
    }

    {
        // out of device memory: the smallest cached block that is large
        // enough is freed and the request retried, and the context switches
        // to exact classes
        g_mallocs = g_frees = 0;
        Device d;
        fake_device(d, 3 * MiB);
        void* x = d.alloc(2 * MiB);
        d.release(x);                              // 2 MiB cached, 1 MiB of budget left
        CHECK(!d.pressure);
        void* y = d.alloc(1536 * KiB);             // 2 MiB is > 1.25x: driver, refused, evict, retry
        CHECK(y != nullptr && d.pressure && d.cache_frees == 1 && g_frees == 1 && d.cached_bytes == 0);
        CHECK(g_used == 1536 * KiB && d.live_bytes == 1536 * KiB);

        // a request the device cannot hold even with the cache empty fails
        // with GP_ENOMEM and leaves the context usable
        bool enomem = false;
        try {
            d.alloc(8 * MiB);
        } catch (const gp::Error& err) {
            enomem = err.status == GP_ENOMEM;
        }
        CHECK(enomem);
        d.release(y);
        void* z = d.alloc(1536 * KiB);             // exact class, cached
        CHECK(z == y && g_mallocs == 2);
        d.release(z);
        d.release_cached();
        CHECK(g_used == 0);
    }

    if (failures == 0) std::printf("allocator policy: all checks passed\n");
    return failures == 0 ? 0 : 1;
}
