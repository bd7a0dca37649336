// Common infrastructure of the B200 partitioner: graph type widths, status
// codes and exceptions, the per-context stream-ordered allocator and small
// device helpers shared by every stage.
#pragma once

#include <cuda_runtime.h>

#include <chrono>

#include <cstdint>
#include <cstring>
#include <cstdio>
#include <iterator>
#include <map>
#include <unordered_map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/gpart_b200.h"

namespace gp {

using u64 = std::uint64_t;
using u32 = std::uint32_t;
using i64 = std::int64_t;
using i32 = std::int32_t;

// The reference's two graph widths (include/graph_types.hpp:7-17):
// "standard" = int32 offsets + uint32 weights, "big" = int64 offsets +
// uint64 weights.  Vertex ids are int32 in both.
struct Std { using O = i32; using W = u32; static constexpr const char* name = "standard"; };
struct Big { using O = i64; using W = u64; static constexpr const char* name = "big"; };

// Errors carry the C-ABI status.  The classes mirror the reference's
// exception classes: invalid_argument -> GP_EINVAL, runtime_error ->
// GP_ERUNTIME, overflow_error -> GP_EOVERFLOW.
struct Error : std::runtime_error {
    gp_status status;
    Error(gp_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};
[[noreturn]] inline void fail(gp_status s, const std::string& what) { throw Error(s, what); }

struct Device;

#define GP_CUDA(call)                                                              \
    do {                                                                           \
        const cudaError_t e__ = (call);                                            \
        if (e__ != cudaSuccess)                                                    \
            ::gp::fail(e__ == cudaErrorMemoryAllocation ? GP_ENOMEM : GP_ECUDA,    \
                       std::string("CUDA failure at ") + __FILE__ + ":" +          \
                           std::to_string(__LINE__) + " " + #call + ": " +         \
                           cudaGetErrorString(e__));                               \
    } while (0)

#define GP_LAUNCH() GP_CUDA(cudaGetLastError())

// Device error word bits (set by kernels, read at host sync points).
enum DeviceError : u32 {
    kErrNone = 0,
    kErrTimeout = 1u << 0,        // a bounded wait gave up
    kErrCapacity = 1u << 1,       // SCLP cluster above its cap
    kErrSplit = 1u << 2,          // spectral split cannot satisfy capacity
    kErrBalance = 1u << 3,        // initial partition above capacity
    kErrCutUnderflow = 1u << 4,   // incremental cut underflow
    kErrOddCut = 1u << 5,         // directed cut odd (asymmetric input)
    kErrTableFull = 1u << 6,      // hash table overflow (sizing bug)
    kErrBadInput = 1u << 7,       // input validation failure
};

// ---------------------------------------------------------------------------
// Device memory: a caching allocator per context.  Blocks are cudaMalloc'd in
// size classes (<= 12.5% rounding) and kept on free lists when released.
// All of a context's work runs on its one stream, so a released block can be
// handed to the next allocation immediately: later work on the stream is
// ordered after every earlier use.  Repeated partitions of similar graphs
// therefore allocate nothing from the driver.
// ---------------------------------------------------------------------------
struct Device {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sms = 148;
    // Contexts expected to run at once on the device (a server's slots): the
    // grid-stride kernels of this context take at most 1/share of the
    // device's block slots, so kernels of the other contexts fit beside them.
    int share = 1;
    // Small coarsest graphs take the one-block diffusion (same values as the
    // cooperative kernel); off only to compare the two.
    bool small_diffusion = true;
    // SCLP affinity of hubs with on-chip tables where they fit (same
    // results as the global tables); off only to compare the two.
    bool hub_chip = true;
    // The default mode's rebalance loop as a CUDA graph with a device-side
    // loop condition: 0 never (host loop, same kernels; the default), 1 once
    // a level's host loop has run a few iterations, 2 always.
    int graph_loops = 0;
    size_t total_bytes = 0;     // device memory, read once when the context is created
    int grid_limit(int per_sm) const { return std::max(sms / 2, sms * per_sm / std::max(1, share)); }
    u32* err = nullptr;         // device error word
    void* pinned = nullptr;     // small pinned host staging area
    static constexpr size_t kPinnedBytes = 1 << 16;

    // The driver calls behind the cache.  A host test replaces them with a
    // fake device (a byte budget) to exercise the reuse policy and the
    // out-of-memory path without a GPU.
    cudaError_t (*malloc_fn)(void**, size_t) = [](void** p, size_t bytes) { return cudaMalloc(p, bytes); };
    cudaError_t (*free_fn)(void*) = [](void* p) { return cudaFree(p); };
    cudaError_t driver_alloc(void** p, size_t bytes) { return malloc_fn(p, bytes); }
    void driver_free(void* p) { free_fn(p); }

    std::map<size_t, std::vector<void*>> free_blocks;
    std::unordered_map<void*, size_t> live;
    size_t cached_bytes = 0, live_bytes = 0, peak_bytes = 0;
    u64 alloc_calls = 0, driver_allocs = 0, cache_frees = 0;
    double alloc_ms = 0.0;   // host time spent inside the allocator

    static size_t size_class(size_t bytes) {
        if (bytes <= 4096) return (bytes + 255) & ~size_t{255};
        int b = 0;
        for (size_t x = bytes; x; x >>= 1) ++b;
        const size_t q = size_t{1} << (b - 4);
        return (bytes + q - 1) / q * q;
    }
    void release_cached() {
        if (cached_bytes == 0) return;
        cudaStreamSynchronize(stream);
        for (auto& kv : free_blocks)
            for (void* p : kv.second) driver_free(p);
        free_blocks.clear();
        cached_bytes = 0;
    }
    // Makes room for a `bytes` allocation that the driver refused: frees the
    // smallest cached block at least that large, or, without one, cached
    // blocks largest first until `bytes` are returned.  The rest of the cache
    // stays for the blocks that will be asked for again (a full flush made
    // every partition of the largest graphs re-allocate most of its blocks).
    void release_cached(size_t bytes) {
        if (cached_bytes == 0) return;
        cudaStreamSynchronize(stream);
        for (auto fit = free_blocks.lower_bound(bytes); fit != free_blocks.end(); ++fit) {
            if (fit->second.empty()) continue;
            driver_free(fit->second.back());
            fit->second.pop_back();
            cached_bytes -= fit->first;
            ++cache_frees;
            if (fit->second.empty()) free_blocks.erase(fit);
            return;
        }
        size_t freed = 0;
        while (freed < bytes && !free_blocks.empty()) {
            auto it = std::prev(free_blocks.end());
            while (!it->second.empty() && freed < bytes) {
                driver_free(it->second.back());
                it->second.pop_back();
                freed += it->first;
                cached_bytes -= it->first;
                ++cache_frees;
            }
            if (it->second.empty()) free_blocks.erase(it);
        }
    }
    // The cached list a request of class c is served from: its own class,
    // else the smallest larger class within kReuseSlack (a block at most 25%
    // larger than asked for).  Hierarchies of the same graph at another seed,
    // or of a graph of similar size, differ by a few percent per buffer;
    // exact classes alone sent those buffers to the driver, at several
    // milliseconds per cudaMalloc.  Near the device's capacity (`pressure`:
    // set once the driver has refused an allocation, or up front for a graph
    // whose projected footprint exceeds half the device) only exact classes
    // are reused, so that no live block carries an unused tail there and the
    // cache keeps the classes the graph asks for (RMAT-26: reusing larger
    // blocks without bound ran out of memory, and a cache shaped by the slack
    // before the first refusal thrashed afterwards).
    static constexpr size_t kReuseSlack = 4;   // c + c / 4
    bool pressure = false;
    std::map<size_t, std::vector<void*>>::iterator cached_for(size_t c) {
        auto it = free_blocks.find(c);
        if (it != free_blocks.end() && !it->second.empty()) return it;
        if (pressure) return free_blocks.end();
        for (it = free_blocks.upper_bound(c); it != free_blocks.end() && it->first <= c + c / kReuseSlack; ++it)
            if (!it->second.empty()) return it;
        return free_blocks.end();
    }
    void* alloc(size_t bytes) {
        if (bytes == 0) return nullptr;
        const auto t0 = std::chrono::steady_clock::now();
        size_t c = size_class(bytes);
        void* p = nullptr;
        auto it = cached_for(c);
        if (it != free_blocks.end()) {
            c = it->first;   // the block keeps its own class (release files it there)
            p = it->second.back();
            it->second.pop_back();
            cached_bytes -= c;
        } else {
            cudaError_t e = driver_alloc(&p, c);
            if (e != cudaSuccess) {   // release part of the cache, then all of it
                cudaGetLastError();
                pressure = true;
                release_cached(c);
                e = driver_alloc(&p, c);
            }
            if (e != cudaSuccess) {
                cudaGetLastError();
                release_cached();
                e = driver_alloc(&p, c);
            }
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw_oom(c);
            }
            ++driver_allocs;
        }
        live[p] = c;
        live_bytes += c;
        peak_bytes = std::max(peak_bytes, live_bytes);
        ++alloc_calls;
        alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return p;
    }
    void release(void* p) {
        if (!p) return;
        auto it = live.find(p);
        if (it == live.end()) return;
        free_blocks[it->second].push_back(p);
        cached_bytes += it->second;
        live_bytes -= it->second;
        live.erase(it);
    }
    [[noreturn]] static void throw_oom(size_t bytes);
    u64 syncs = 0;     // host waits on the stream (round trips)
    // Blocking waits put the host thread to sleep until the stream's work is
    // done instead of spinning on a core (for processes with many contexts).
    cudaEvent_t sync_event = nullptr;
    bool blocking_sync = false;
    void sync() {
        ++syncs;
        if (blocking_sync) {
            GP_CUDA(cudaEventRecord(sync_event, stream));
            GP_CUDA(cudaEventSynchronize(sync_event));
        } else {
            GP_CUDA(cudaStreamSynchronize(stream));
        }
    }
    // Read a device error word; throws on any set bit.
    void check_errors();

    // Launch accounting and optional per-kernel CUDA-event timing.
    u64 launches = 0;
    bool prof = false;
    struct ProfEntry {
        u64 launches = 0;
        double ms = 0.0;
        double bytes = 0.0;     // algorithmic bytes recorded by the call sites
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    };
    std::map<std::string, ProfEntry> prof_table;
    std::vector<cudaEvent_t> event_pool;
    cudaEvent_t event() {
        if (!event_pool.empty()) { auto e = event_pool.back(); event_pool.pop_back(); return e; }
        cudaEvent_t e;
        GP_CUDA(cudaEventCreate(&e));
        return e;
    }
    void prof_bytes(const char* name, double bytes) { if (prof) prof_table[name].bytes += bytes; }
    // Resolve pending event pairs (synchronises the stream).
    void prof_resolve() {
        sync();
        for (auto& kv : prof_table) {
            for (auto& pr : kv.second.pending) {
                float ms = 0.f;
                GP_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
                kv.second.ms += ms;
                event_pool.push_back(pr.first);
                event_pool.push_back(pr.second);
            }
            kv.second.pending.clear();
        }
    }
};

// Every kernel launch of the library goes through this helper: it counts
// launches and, when profiling is on, brackets the launch with CUDA events on
// the context stream.
template <typename... KArgs, typename... Args>
void launch(Device& d, const char* name, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, Args&&... args) {
    static_assert(sizeof...(KArgs) == sizeof...(Args), "kernel argument count");
    cudaEvent_t a = nullptr;
    if (d.prof) {
        a = d.event();
        GP_CUDA(cudaEventRecord(a, d.stream));
    }
    k<<<grid, block, smem, d.stream>>>(static_cast<KArgs>(args)...);
    GP_CUDA(cudaGetLastError());
    ++d.launches;
    if (d.prof) {
        cudaEvent_t b = d.event();
        GP_CUDA(cudaEventRecord(b, d.stream));
        auto& e = d.prof_table[name];
        e.pending.push_back({a, b});
        ++e.launches;
    }
}

inline void Device::throw_oom(size_t bytes) {
    fail(GP_ENOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
}

template <typename T>
class Buf {
public:
    Buf() = default;
    Buf(Device& d, size_t count) : dev_(&d), count_(count) {
        ptr_ = static_cast<T*>(d.alloc(count * sizeof(T)));
    }
    ~Buf() { reset(); }
    Buf(Buf&& o) noexcept : dev_(o.dev_), ptr_(o.ptr_), count_(o.count_) { o.ptr_ = nullptr; o.count_ = 0; }
    Buf& operator=(Buf&& o) noexcept {
        if (this != &o) { reset(); dev_ = o.dev_; ptr_ = o.ptr_; count_ = o.count_; o.ptr_ = nullptr; o.count_ = 0; }
        return *this;
    }
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    void reset() { if (ptr_ && dev_) dev_->release(ptr_); ptr_ = nullptr; count_ = 0; dev_ = nullptr; }
    // Non-owning view of caller memory (never freed by this Buf).
    void borrow(T* p, size_t count) { reset(); ptr_ = p; count_ = count; }
    // Grow without preserving contents.
    void ensure(Device& d, size_t count) {
        if (count <= count_ && ptr_) return;
        reset();
        dev_ = &d;
        count_ = count;
        ptr_ = static_cast<T*>(d.alloc(count * sizeof(T)));
    }
    T* get() const { return ptr_; }
    size_t size() const { return count_; }
    void zero(Device& d) { if (count_) GP_CUDA(cudaMemsetAsync(ptr_, 0, count_ * sizeof(T), d.stream)); }
    void fill_bytes(Device& d, int byte) { if (count_) GP_CUDA(cudaMemsetAsync(ptr_, byte, count_ * sizeof(T), d.stream)); }
    void swap(Buf& o) { std::swap(dev_, o.dev_); std::swap(ptr_, o.ptr_); std::swap(count_, o.count_); }

private:
    Device* dev_ = nullptr;
    T* ptr_ = nullptr;
    size_t count_ = 0;
};

template <typename T>
void to_host(Device& d, T* host, const T* dev, size_t count) {
    if (count) GP_CUDA(cudaMemcpyAsync(host, dev, count * sizeof(T), cudaMemcpyDeviceToHost, d.stream));
}
template <typename T>
void to_device(Device& d, T* dev, const T* host, size_t count) {
    if (count) GP_CUDA(cudaMemcpyAsync(dev, host, count * sizeof(T), cudaMemcpyHostToDevice, d.stream));
}
// Synchronously fetch a few scalars through the pinned staging area.
template <typename T>
void fetch(Device& d, T* host, const T* dev, size_t count) {
    static_assert(std::is_trivially_copyable_v<T>);
    if (!count) return;
    const size_t bytes = count * sizeof(T);
    if (bytes > Device::kPinnedBytes) { to_host(d, host, dev, count); d.sync(); return; }
    GP_CUDA(cudaMemcpyAsync(d.pinned, dev, bytes, cudaMemcpyDeviceToHost, d.stream));
    d.sync();
    std::memcpy(host, d.pinned, bytes);
}

inline int blocks_for(i64 items, int per_block) {
    const i64 b = (items + per_block - 1) / per_block;
    return static_cast<int>(b < 1 ? 1 : b);
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
// The reference's 32-bit mixer (src/coarsen.cu:112-118, refine.cu:38-44,
// initial_partition_gpu.cu:36-39).
__host__ __device__ __forceinline__ u32 mix32(u32 x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    return x ^ (x >> 16);
}

template <typename W>
__device__ __forceinline__ W weight_at(const W* w, i64 i) { return w ? w[i] : W(1); }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ void atomic_add_w(u32* p, u32 v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_w(u64* p, u64 v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}
__device__ __forceinline__ u64 atomic_add_u64(u64* p, u64 v) {
    return atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}
__device__ __forceinline__ u64 atomic_max_u64(u64* p, u64 v) {
    return atomicMax(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}
__device__ __forceinline__ u64 atomic_cas_u64(u64* p, u64 c, u64 v) {
    return atomicCAS(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(c),
                     static_cast<unsigned long long>(v));
}

__device__ __forceinline__ void set_error(u32* err, u32 bit) { atomicOr(err, bit); }

}  // namespace gp
