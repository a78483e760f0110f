// Every device and pinned host allocation of the library goes through dev_malloc / dev_free /
// pinned_malloc / pinned_free:
//  * so that the handling of a failed allocation can be tested on the host, without exhausting or
//    faulting a GPU: while the environment variable PG_TEST_FAIL_DEVICE_ALLOC is set to a non-empty
//    value other than "0", dev_malloc returns cudaErrorMemoryAllocation without allocating (the
//    variable is read on every call, so a test can set and clear it around one operation);
//  * so that the trace can say how many allocations and frees a phase made and how long they took
//    (alloc_stats(); a one-shot process pays for every buffer it grows, and cudaFree waits for the
//    device).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace pg {

struct AllocStats {
    std::atomic<uint64_t> allocs{0}, alloc_bytes{0}, alloc_ns{0};
    std::atomic<uint64_t> frees{0}, free_ns{0};
    std::atomic<uint64_t> pinned{0}, pinned_bytes{0}, pinned_ns{0};
};

inline AllocStats& alloc_stats() {
    static AllocStats s;
    return s;
}

inline uint64_t alloc_clock_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

inline bool device_alloc_failure_injected() {
    const char* e = std::getenv("PG_TEST_FAIL_DEVICE_ALLOC");
    return e && e[0] && !(e[0] == '0' && e[1] == 0);
}

// Deferred frees. cudaFree waits until the whole device is idle, and while it waits it holds the
// runtime's lock, so that a buffer freed on one host thread (a workspace growing on the helper
// stream) drains the queue of the other (the splitting's launches). Inside a DeferFrees scope
// (the pi pipeline's calls), dev_free therefore only records the buffer; the recorded buffers are
// freed by the first dev_malloc or dev_free made after the last scope has closed (or when an
// allocation fails for want of memory, or the recorded bytes pass a quarter of the device's
// memory), i.e. with the semantics of cudaFree, one call later.
struct FreeList {
    std::mutex mu;
    std::unordered_map<void*, size_t> sizes;  // live allocations made by dev_malloc
    std::vector<void*> pending;
    size_t pending_bytes = 0;
    size_t pending_cap = 0;                   // 0: not queried yet
    std::atomic<int> scopes{0};
};

inline FreeList& free_list() {
    static FreeList f;
    return f;
}

inline cudaError_t timed_cuda_free(void* p) {
    const uint64_t t0 = alloc_clock_ns();
    const cudaError_t e = cudaFree(p);
    AllocStats& s = alloc_stats();
    s.frees += 1;
    s.free_ns += alloc_clock_ns() - t0;
    return e;
}

// Frees every recorded buffer (caller holds f.mu).
inline void flush_pending_locked(FreeList& f) {
    for (void* q : f.pending) timed_cuda_free(q);
    f.pending.clear();
    f.pending_bytes = 0;
}

struct DeferFrees {
    DeferFrees() { free_list().scopes.fetch_add(1); }
    ~DeferFrees() { free_list().scopes.fetch_sub(1); }
    DeferFrees(const DeferFrees&) = delete;
    DeferFrees& operator=(const DeferFrees&) = delete;
};

template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
    if (device_alloc_failure_injected()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    FreeList& f = free_list();
    std::lock_guard<std::mutex> lk(f.mu);
    if (!f.pending.empty() && f.scopes.load() == 0) flush_pending_locked(f);
    const uint64_t t0 = alloc_clock_ns();
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e == cudaErrorMemoryAllocation && !f.pending.empty()) {  // the recorded buffers first
        cudaGetLastError();
        flush_pending_locked(f);
        e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    }
    AllocStats& s = alloc_stats();
    s.allocs += 1;
    s.alloc_bytes += bytes;
    s.alloc_ns += alloc_clock_ns() - t0;
    if (e == cudaSuccess) f.sizes[static_cast<void*>(*p)] = bytes;
    return e;
}

inline cudaError_t dev_free(void* p) {
    FreeList& f = free_list();
    std::lock_guard<std::mutex> lk(f.mu);
    if (!p) {
        if (!f.pending.empty() && f.scopes.load() == 0) flush_pending_locked(f);
        return cudaSuccess;
    }
    size_t bytes = 0;
    auto it = f.sizes.find(p);
    if (it != f.sizes.end()) {
        bytes = it->second;
        f.sizes.erase(it);
    }
    if (f.scopes.load() > 0 && bytes) {  // a buffer of dev_malloc's, inside a scope
        if (!f.pending_cap) {
            size_t fr = 0, tot = 0;
            f.pending_cap = (cudaMemGetInfo(&fr, &tot) == cudaSuccess && tot) ? tot / 4 : ((size_t)8 << 30);
        }
        if (f.pending_bytes + bytes <= f.pending_cap) {
            f.pending.push_back(p);
            f.pending_bytes += bytes;
            return cudaSuccess;
        }
    }
    if (!f.pending.empty() && f.scopes.load() == 0) flush_pending_locked(f);
    return timed_cuda_free(p);
}

template <class T>
inline cudaError_t pinned_malloc(T** p, size_t bytes) {
    const uint64_t t0 = alloc_clock_ns();
    const cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(p), bytes);
    AllocStats& s = alloc_stats();
    s.pinned += 1;
    s.pinned_bytes += bytes;
    s.pinned_ns += alloc_clock_ns() - t0;
    return e;
}

inline cudaError_t pinned_free(void* p) { return cudaFreeHost(p); }

}  // namespace pg
