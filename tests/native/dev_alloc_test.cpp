// Host test of the library's allocation layer (pi-compute_b200/csrc/dev_alloc.h) against a fake
// CUDA runtime: cudaMalloc / cudaFree / cudaMemGetInfo are defined below and record what the layer
// asks of them, so the deferred-free rules are checked without a GPU:
//  * outside a DeferFrees scope a free is immediate;
//  * inside one it is only recorded, and the recorded buffers are freed by the first allocation or
//    free made after the last scope closed;
//  * recorded bytes stay under a quarter of the device's memory (a free past that is immediate);
//  * an allocation that fails for want of memory frees the recorded buffers and tries again;
//  * PG_TEST_FAIL_DEVICE_ALLOC makes every allocation fail without calling cudaMalloc.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <set>

#include "dev_alloc.h"

namespace {
std::set<void*> g_live;           // buffers the fake device holds
size_t g_live_bytes = 0, g_capacity = 0;
int g_mallocs = 0, g_frees = 0;
std::set<std::pair<void*, size_t>> g_sizes;
size_t g_total = (size_t)16 << 30;  // the fake device's memory (cudaMemGetInfo)

size_t size_of(void* p) {
    for (auto& s : g_sizes)
        if (s.first == p) return s.second;
    return 0;
}
}  // namespace

extern "C" {
cudaError_t cudaMalloc(void** p, size_t bytes) {
    ++g_mallocs;
    if (g_capacity && g_live_bytes + bytes > g_capacity) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    static uintptr_t next = 0x10000;  // fresh addresses, never reused; the bytes are not touched
    *p = reinterpret_cast<void*>(next);
    next += 0x1000;
    g_live.insert(*p);
    g_sizes.insert({*p, bytes});
    g_live_bytes += bytes;
    return cudaSuccess;
}
cudaError_t cudaFree(void* p) {
    ++g_frees;
    if (!g_live.count(p)) return cudaErrorInvalidValue;
    g_live.erase(p);
    const size_t b = size_of(p);
    g_sizes.erase({p, b});
    g_live_bytes -= b;
    return cudaSuccess;
}
cudaError_t cudaMemGetInfo(size_t* fr, size_t* tot) {
    *tot = g_total;
    *fr = g_total - g_live_bytes;
    return cudaSuccess;
}
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
cudaError_t cudaMallocHost(void** p, size_t bytes) {
    *p = std::malloc(bytes ? bytes : 1);
    return cudaSuccess;
}
cudaError_t cudaFreeHost(void* p) {
    std::free(p);
    return cudaSuccess;
}
}

#define CHECK(c)                                                        \
    do {                                                                \
        if (!(c)) {                                                     \
            std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #c); \
            return 1;                                                   \
        }                                                               \
    } while (0)

int main() {
    using namespace pg;
    const size_t MB = (size_t)1 << 20;
    void* a = nullptr;
    void* b = nullptr;
    void* c = nullptr;
    // outside a scope: immediate
    CHECK(dev_malloc(&a, 10 * MB) == cudaSuccess && g_live.count(a));
    CHECK(dev_free(a) == cudaSuccess && !g_live.count(a) && g_frees == 1);
    // inside a scope: recorded, not freed
    {
        DeferFrees d;
        CHECK(dev_malloc(&a, 10 * MB) == cudaSuccess);
        CHECK(dev_malloc(&b, 20 * MB) == cudaSuccess);
        CHECK(dev_free(a) == cudaSuccess && g_live.count(a) && g_frees == 1);
        {
            DeferFrees inner;  // nested scopes
            CHECK(dev_free(b) == cudaSuccess && g_live.count(b));
        }
        CHECK(dev_malloc(&c, MB) == cudaSuccess && g_live.count(a) && g_live.count(b));  // still in a scope
        CHECK(free_list().pending.size() == 2 && free_list().pending_bytes == 30 * MB);
    }
    // the first allocation after the last scope frees the recorded buffers
    void* e = nullptr;
    CHECK(dev_malloc(&e, MB) == cudaSuccess && !g_live.count(a) && !g_live.count(b));
    CHECK(free_list().pending.empty() && free_list().pending_bytes == 0);
    CHECK(dev_free(c) == cudaSuccess && dev_free(e) == cudaSuccess && g_live.empty());
    // the cap: a quarter of the device's memory (4 GB of the fake 16 GB)
    {
        DeferFrees d;
        void* big[3];
        for (auto& p : big) CHECK(dev_malloc(&p, (size_t)1536 * MB) == cudaSuccess);
        CHECK(dev_free(big[0]) == cudaSuccess && dev_free(big[1]) == cudaSuccess);  // 3 GB recorded
        CHECK(g_live.count(big[0]) && g_live.count(big[1]));
        CHECK(dev_free(big[2]) == cudaSuccess && !g_live.count(big[2]));  // would pass 4 GB: immediate
        CHECK(free_list().pending_bytes == (size_t)3072 * MB);
    }
    CHECK(dev_free(nullptr) == cudaSuccess && free_list().pending.empty() && g_live.empty());  // flushed
    // an allocation failing for want of memory frees the recorded buffers and retries
    g_capacity = 100 * MB;
    {
        DeferFrees d;
        CHECK(dev_malloc(&a, 60 * MB) == cudaSuccess);
        CHECK(dev_free(a) == cudaSuccess && g_live.count(a));
        CHECK(dev_malloc(&b, 60 * MB) == cudaSuccess && !g_live.count(a) && g_live.count(b));
        CHECK(free_list().pending.empty());
        CHECK(dev_malloc(&c, 60 * MB) == cudaErrorMemoryAllocation);  // nothing left to free
        CHECK(dev_free(b) == cudaSuccess);
    }
    CHECK(dev_malloc(&a, MB) == cudaSuccess && dev_free(a) == cudaSuccess && g_live.empty());
    g_capacity = 0;
    // injected failures never reach cudaMalloc
    setenv("PG_TEST_FAIL_DEVICE_ALLOC", "1", 1);
    const int m0 = g_mallocs;
    CHECK(dev_malloc(&a, MB) == cudaErrorMemoryAllocation && a == nullptr && g_mallocs == m0);
    setenv("PG_TEST_FAIL_DEVICE_ALLOC", "0", 1);
    CHECK(dev_malloc(&a, MB) == cudaSuccess && dev_free(a) == cudaSuccess);
    // the counters saw every dev_malloc that reached cudaMalloc (the retry after freeing the
    // recorded buffers counts with its call: one retry above)
    CHECK(alloc_stats().allocs.load() == (uint64_t)g_mallocs - 1);
    std::puts("ok");
    return 0;
}
