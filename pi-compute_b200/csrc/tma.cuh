// Tensor-memory-accelerator (TMA) tile loads for the pass kernels: an mbarrier in shared memory and
// cp.async.bulk.tensor loads of a tile from a CUtensorMap built on the host for the launch (this
// GPU's own memory only, no cluster multicast). The tensor map uses the 128-byte swizzle: in every
// 1024-byte group of the destination, the 16-byte chunk c of 128-byte line l lands at chunk c ^ l
// (tma_swz below), so a tile arrives in a layout other than the passes' own (swz); the first
// radix round reads it and writes the passes' layout back.
#pragma once
#include <cuda.h>
#include <cstdint>

namespace pg {

// Word index of tile element x in the layout the 128-byte swizzle gives (chunks of 4 words
// permuted within each 32-word line by the line's low three bits). Linear over GF(2).
__device__ __forceinline__ uint32_t tma_swz(uint32_t x) { return x ^ (((x >> 5) & 7u) << 2); }

// tma_swz(x0 | (q << qb)) for x0 whose bits [qb, qb + log2 R) are zero, as a base plus a constant
// (see swz_elem): the bits >= 5 of the two parts do not overlap, so XOR is addition there.
__device__ __forceinline__ uint32_t tma_elem(uint32_t b0, uint32_t q, int qb) {
    const uint32_t k = tma_swz(q << qb);
    return (b0 ^ (k & 31u)) + (k & ~31u);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialised barrier visible to the asynchronous proxy (the TMA unit).
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6}], [%2];\n" ::"r"(smem_addr(dst)),
        "l"(map), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6, %7}], [%2];\n" ::"r"(smem_addr(dst)),
        "l"(map), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
}

// Polls of the tile barrier before a pass gives up (each poll is a hardware-bounded try_wait);
// giving up sets bit 4 of the launch's error word and leaves the tile as it is.
constexpr uint32_t kTmaSpinLimit = 1u << 22;
constexpr uint32_t kErrTmaWait = 4u;

}  // namespace pg
