// Plain parameter/table types shared by the kernels and the host-side engine.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "modarith.cuh"

namespace pg {

__host__ __device__ inline int __builtin_clz_portable(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __clz(x);
#else
    return __builtin_clz(x);
#endif
}

constexpr int kStageLog = 14;  // stage twiddles come from w_{2^14}: sub-transforms up to 2^13 points
constexpr int kFsLog = 13;     // four-step twiddles: w_{2^26}^e = lo[e & 8191] * hi[e >> 13]

// Exponent of w_{2^14} stored at stage-table entry i = h + x (h = 2^k <= i < 2h): w_{2h}^x.
__host__ __device__ inline uint32_t stage_exponent(uint32_t i) {
    if (i == 0) return 0;
    int k = 31 - __builtin_clz_portable(i);
    return (i - (1u << k)) << (kStageLog - 1 - k);
}

struct TwiddleTables {
    // (w, w') Shoup pairs, [dir][prime]; dir 0 = forward (w), 1 = inverse (w^-1).
    const uint2* stage[2][kNumPrimes];  // entry h + x = w_{2h}^x (h = 2^k, x < h), 2^13 entries
    const uint2* fs_lo[2][kNumPrimes];  // w_{2^26}^j,           j < 2^13
    const uint2* fs_hi[2][kNumPrimes];  // w_{2^26}^(2^13 * i),  i < 2^13
};

enum class Layout : int { Strided = 0, Contig = 1 };
enum class Source : int { Residues = 0, Limbs = 1 };
enum class Fuse : int { None = 0, MulInverse = 1, SqrInverse = 2 };

struct PassParams {
    uint32_t* data;          // residue array of this operand: prime j at data + j*L
    const uint32_t* other;   // Fuse::MulInverse: fully transformed other operand (same layout)
    uint32_t* out;           // where the tile is written (== data for in-place passes)
    const uint32_t* words;   // Source::Limbs: operand as 32-bit words (little-endian)
    uint64_t ncoef;          // Source::Limbs: number of valid 32-bit coefficients
    uint64_t L;              // transform length (elements per prime)
    int logS;                // log2 of the element stride of this pass (0 for Contig)
    int logNp;               // log2 of the block size N' = N * S (four-step twiddle)
    uint32_t nrows;          // Contig: number of valid rows (blocks of N) in the array
};

struct CrtConsts {
    // Shoup pairs (value, companion) for the Garner steps.
    uint32_t c00, c00p;   // f0                       mod p0
    uint32_t c11, c11p;   // f1 * p0^-1               mod p1
    uint32_t k01, k01p;   // p0^-1                    mod p1
    uint32_t c22, c22p;   // f2 * p0^-1 * p1^-1       mod p2
    uint32_t k02, k02p;   // p0^-1 * p1^-1            mod p2
    uint32_t k12, k12p;   // p1^-1                    mod p2
    uint64_t p01;         // p0 * p1
};

struct CrtParams {
    const uint32_t* res;     // residues: prime j at res + j*L, natural order
    uint64_t L;
    uint64_t nwords;         // output words (2 * output limbs)
    uint32_t* out;           // output words
    uint32_t* status;        // one word per CTA, zeroed before launch
    uint32_t* ticket;        // zeroed before launch
    uint32_t* error;         // set non-zero on a look-back timeout or a final carry
    CrtConsts k;
};

constexpr int kCrtThreads = 256;
constexpr int kCrtWords = 16;  // words per thread

}  // namespace pg
