// Every device allocation of the library goes through dev_malloc, so that the handling of a
// failed allocation can be tested on the host, without exhausting or faulting a GPU: while the
// environment variable PG_TEST_FAIL_DEVICE_ALLOC is set to a non-empty value other than "0",
// dev_malloc returns cudaErrorMemoryAllocation without allocating (the variable is read on every
// call, so a test can set and clear it around one operation).
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>

namespace pg {

inline bool device_alloc_failure_injected() {
    const char* e = std::getenv("PG_TEST_FAIL_DEVICE_ALLOC");
    return e && e[0] && !(e[0] == '0' && e[1] == 0);
}

template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
    if (device_alloc_failure_injected()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

}  // namespace pg
