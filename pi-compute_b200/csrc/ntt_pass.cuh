// Shared-memory-staged NTT passes (sm_100a).
//
// A transform of length L = 2^logL over Z/p is split into passes. Pass j does
// length-N_j sub-transforms on elements at stride S_j = N_{j+1} * ... * N_last
// (the four-step / six-step decomposition): the block of N' = N_j * S_j points
// at offset blk*N', column t in [0, S_j), holds x[t + S_j*m], m in [0, N_j).
//
//   forward (decimation in frequency, natural order in):
//     Y = DFT_N(x[t + S m]); Y[k] *= w_{N'}^{t k}; store Y[k] at t + S*bitrev_N(k)
//   inverse (decimation in time, exact reverse of the forward pass):
//     read Z at t + S*pos; Z *= w_{N'}^{-t bitrev(pos)}; y = IDFT_N(Z) (natural order out)
//
// The forward transform therefore leaves a fixed permutation of the DFT in
// memory; the inverse undoes it, and the pointwise product in between does not
// care about the order (convolution theorem). No bit-reversal pass exists.
//
// A CTA holds a tile of E = 2^LOGE residues of one prime in shared memory:
//   STRIDED tile: C = E/N adjacent columns t0..t0+C-1 of one block (rows of C
//                 contiguous words in HBM, coalesced 16-byte vector accesses);
//   CONTIG tile:  C = E/N consecutive blocks of length N (S = 1), contiguous.
// Inside the tile each sub-transform runs as radix-16 (then 8/4/2) rounds:
// a thread loads R elements of one group into registers, does log2(R) radix-2
// stages there, and writes them back; rounds are separated by __syncthreads.
#pragma once
#include <cstdint>

#include "modarith.cuh"
#include "series.cuh"
#include "tma.cuh"
#include "types.cuh"

namespace pg {

#ifndef PG_STRIDED_MINB
#define PG_STRIDED_MINB 4
#endif
// CTAs per SM each pass kernel's register budget is sized for (4: <= 64 registers). At 4 the
// strided passes spill a few words to L1 and still run faster than at 3 (80 registers): more
// warps hide the global-load latency they are bound by.
#ifndef PG_FUSED_MINB
#define PG_FUSED_MINB 4
#endif
template <Layout LAY, Fuse FUSE, int LOGE>
constexpr int pass_min_blocks() {
    return LOGE > 13 ? 2 : (LAY == Layout::Strided ? PG_STRIDED_MINB : (FUSE == Fuse::None ? 4 : PG_FUSED_MINB));
}

__device__ __forceinline__ uint32_t bitrev_n(uint32_t x, int logn) {
    return logn == 0 ? 0u : (__brev(x) >> (32 - logn));
}

// Four-step twiddles of a strided tile. Element (row m, tile column c) of the tile whose
// first column is t0 is multiplied by w_{N'}^{(t0 + c) k}, k = bitrev(m), written as
//   A[m] * B[m][c],  A[m] = w_{N'}^{t0 k} (per tile, kept in shared memory),
//                    B[m][c] = w_{N'}^{c k} (the tile-shape table of (N', N), row-major).
// The four consecutive columns c..c+3 of one row are two 16-byte loads, consecutive across the
// lanes of a warp. Each factor is a (w, w') Shoup pair, so an element costs two Shoup products;
// the first may stay lazy because Shoup accepts any 32-bit input.
__device__ __forceinline__ void fourstep_twiddle4(uint4& x, uint32_t c, uint32_t m, int logc, uint2 A,
                                                  const uint2* B, uint32_t p) {
    const uint4* b = reinterpret_cast<const uint4*>(B + ((size_t)m << logc) + c);
    const uint4 b01 = __ldg(b), b23 = __ldg(b + 1);
    x.x = mul_shoup(mul_shoup_lazy(x.x, b01.x, b01.y, p), A.x, A.y, p);
    x.y = mul_shoup(mul_shoup_lazy(x.y, b01.z, b01.w, p), A.x, A.y, p);
    x.z = mul_shoup(mul_shoup_lazy(x.z, b23.x, b23.y, p), A.x, A.y, p);
    x.w = mul_shoup(mul_shoup_lazy(x.w, b23.z, b23.w, p), A.x, A.y, p);
}

// One decimation-in-frequency round of radix R = 2^LR on v[0..R), the group's
// elements sitting at sub-transform positions t' + s*q within a block of R*s.
// Stage k (half size h = (R/2 >> k) * s) pairs q with q + 2^(LR-1-k) and uses
// twiddle w_{2h}^(t' + s*(q mod 2^(LR-1-k))).
// When logs == 0 the group offset t' is 0 and every twiddle exponent is a compile-time
// constant after unrolling; exponent 0 (twiddle 1) then skips its multiply.
template <int LR>
__device__ __forceinline__ void dif_round(uint32_t (&v)[1 << LR], uint32_t tp, int logs, const uint2* stw,
                                          uint32_t p) {
#pragma unroll
    for (int k = 0; k < LR; ++k) {
        const int half = 1 << (LR - 1 - k);     // pair distance in q
        const int logh = logs + (LR - 1 - k);   // log2 of stage half size h
#pragma unroll
        for (int q = 0; q < (1 << LR); ++q) {
            if (q & half) continue;
            uint32_t a = v[q], b = v[q + half];
            v[q] = add_mod(a, b, p);
            if (logs == 0 && (q & (half - 1)) == 0) {
                v[q + half] = sub_mod(a, b, p);
            } else {
                uint32_t x = tp + ((uint32_t)(q & (half - 1)) << logs);
                // stride 1: w_{2h}^x = w_{2^LR}^(x 2^k), all from the round's top entries, so equal
                // twiddles of different stages share one load
                const uint32_t idx = logs == 0 ? (1u << (LR - 1)) + (x << k) : (1u << logh) + x;
                uint2 w = __ldg(stw + idx);
                v[q + half] = mul_shoup(a - b + p, w.x, w.y, p);
            }
        }
    }
}

// Decimation-in-time round (inverse): stage k has half size h = 2^k * s, pairs
// q with q + 2^k, twiddle w_{2h}^-(t' + s*(q mod 2^k)).
template <int LR>
__device__ __forceinline__ void dit_round(uint32_t (&v)[1 << LR], uint32_t tp, int logs, const uint2* stw,
                                          uint32_t p) {
#pragma unroll
    for (int k = 0; k < LR; ++k) {
        const int half = 1 << k;
        const int logh = logs + k;
#pragma unroll
        for (int q = 0; q < (1 << LR); ++q) {
            if (q & half) continue;
            uint32_t a = v[q];
            uint32_t b = v[q + half];
            if (!(logs == 0 && (q & (half - 1)) == 0)) {
                uint32_t x = tp + ((uint32_t)(q & (half - 1)) << logs);
                // stride 1: stage k's w_{2^(k+1)}^x = w_{2^LR}^(x 2^(LR-1-k)) from the top entries
                const uint32_t idx = logs == 0 ? (1u << (LR - 1)) + (x << (LR - 1 - k)) : (1u << logh) + x;
                uint2 w = __ldg(stw + idx);
                b = mul_shoup(b, w.x, w.y, p);
            }
            v[q] = add_mod(a, b, p);
            v[q + half] = sub_mod(a, b, p);
        }
    }
}

// Shared-memory address of linear tile index x: the eight 16-byte chunks of each 128-byte
// line are permuted by f = ((x >> 5) ^ (x >> 7) ^ (x >> 8 << 2)) & 7 (bits 5-9 of x select the
// permutation, bits 2-4 are permuted, bits 0-1 stay: 16-byte vectors stay whole). The access
// patterns of a warp:
//   global<->shared copies, 16-byte vectors of consecutive chunks: one line per 8 lanes;
//   stride-1 rounds of contiguous tiles, 16-byte vectors at a 64-byte lane stride;
//   stride-16 rounds of contiguous tiles, 16 lanes on consecutive words and the other 16 lanes
//     256 words further;
//   stride-1 rounds of strided tiles with C = 4 or 8 columns: 32 / C row groups, 16 C words apart;
//   every other round: 32 consecutive words.
// Every pattern above touches each bank once per 128 bytes moved, for every tile shape the passes
// use except the radix-2 remainder round of a 64-point contiguous transform (2 ways).
__device__ __forceinline__ uint32_t swz(uint32_t x) {
    return x ^ ((((x >> 5) ^ (x >> 7) ^ ((x >> 8) << 2)) & 7u) << 2);
}

// 16-byte asynchronous copy global -> shared (no register staging, so every copy of a thread is in
// flight at once); both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(uint32_t* smem, const uint32_t* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// swz is linear over GF(2) (shifts, XOR and a constant mask), so for index bits that do not
// overlap, swz(x0 | y) = swz(x0) ^ swz(y). A round's group of R elements sits at
// x0 | (q << qb) for q < R, with x0's bits [qb, qb + log2 R) zero: one swizzle per group and a
// compile-time constant per element (the rounds are unrolled, so qb and q are constants).
// The constant splits into bits 0-4 (XORed into the group's base: at most 8 distinct bases per
// group, since only bits 2-4 can be set) and bits >= 5, which are zero in b0 (they are x0's bits,
// zero in [qb, qb + log2 R)) and so add: a register base plus an immediate offset per element.
__device__ __forceinline__ uint32_t swz_elem(uint32_t b0, uint32_t q, int qb) {
    const uint32_t k = swz(q << qb);
    return (b0 ^ (k & 31u)) + (k & ~31u);
}

// Run the radix rounds of one sub-transform direction over the whole tile.
// Stages are processed from half size N/2 down to 1 (DIF) or 1 up to N/2 (DIT).
// Rounds [RR0, RR1) of the schedule run (in the direction's order); the default is all of them.
// TIN: the tile arrived by TMA (layout tma_swz); the first round run reads that layout and writes
// the passes' own. Every warp's groups of that round cover whole 128-byte lines that no other warp
// (or other group of the same warp) touches, so the warp only has to finish its reads before it
// writes (__syncwarp).
template <Layout LAY, int LOGN, int LOGE, int NTHREADS, bool INV, int RR0 = 0, int RR1 = 64, bool TIN = false>
__device__ __forceinline__ void tile_transform(uint32_t* sm, const uint2* stw, uint32_t p) {
    constexpr int LOGC = LOGE - LOGN;
    // Radix schedule: the remainder (LOGN % 4 stages) is the top round (largest stride), then
    // radix-16 rounds at strides 2^(4k), down to the round at stride 1. Every radix-16 round
    // therefore has stride 1, 16 or >= 256, the strides the swizzle makes conflict-free.
    constexpr int NFULL = LOGN / 4;
    constexpr int REM = LOGN % 4;
    constexpr int NROUND = NFULL + (REM ? 1 : 0);
#pragma unroll
    for (int rr = 0; rr < NROUND; ++rr) {
        if (rr < RR0 || rr >= RR1) continue;
        const bool tin = TIN && rr == RR0;
        // DIF: the first rounds take the highest stages. DIT: reversed order.
        const int r = INV ? (NROUND - 1 - rr) : rr;
        const bool is_rem = (REM != 0) && (r == 0);
        const int LRr = is_rem ? REM : 4;
        // round r (r >= 1 when REM != 0) covers log-half-sizes [logs, logs + 4)
        const int logs = is_rem ? (LOGN - REM) : (LOGN - REM - 4 * (r - (REM ? 1 : 0) + 1));
        // groups: E / R
        if (LRr == 4) {
            constexpr int R = 16;
            constexpr int NG = (1 << LOGE) / R;
            static_assert(NG % NTHREADS == 0, "whole groups per thread");
#pragma unroll 1
            for (int it = 0; it < NG / NTHREADS; ++it) {
                const int g = threadIdx.x + it * NTHREADS;
                uint32_t c, tp, blk;
                const uint32_t s = 1u << logs;
                if constexpr (LAY == Layout::Strided) {
                    c = g & ((1u << LOGC) - 1);
                    uint32_t rest = g >> LOGC;
                    tp = rest & (s - 1);
                    blk = rest >> logs;
                } else {
                    tp = g & (s - 1);
                    uint32_t rest = g >> logs;
                    blk = rest & ((1u << (LOGN - logs - 4)) - 1);
                    c = rest >> (LOGN - logs - 4);
                }
                // m0's bits [logs, logs + 4) are zero (tp < s), so element q is at x0 | (q << qb)
                const uint32_t m0 = (blk << (logs + 4)) | tp;
                const uint32_t x0 = (LAY == Layout::Strided) ? ((m0 << LOGC) | c) : ((c << LOGN) | m0);
                const int qb = (LAY == Layout::Strided) ? logs + LOGC : logs;
                const uint32_t b0 = swz(x0);
                uint32_t v[R];
                // A contiguous tile's stride-1 round reads 16 consecutive words: 4 vectors.
                const bool vec = (LAY == Layout::Contig) && logs == 0;
                if (tin) {
                    const uint32_t bt = tma_swz(x0);
                    if (vec) {
#pragma unroll
                        for (int q4 = 0; q4 < R / 4; ++q4) {
                            const uint4 t = *reinterpret_cast<const uint4*>(sm + tma_elem(bt, 4 * q4, 0));
                            v[4 * q4] = t.x;
                            v[4 * q4 + 1] = t.y;
                            v[4 * q4 + 2] = t.z;
                            v[4 * q4 + 3] = t.w;
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < R; ++q) v[q] = sm[tma_elem(bt, q, qb)];
                    }
                } else if (vec) {
#pragma unroll
                    for (int q4 = 0; q4 < R / 4; ++q4) {
                        const uint4 t = *reinterpret_cast<const uint4*>(sm + swz_elem(b0, 4 * q4, 0));
                        v[4 * q4] = t.x;
                        v[4 * q4 + 1] = t.y;
                        v[4 * q4 + 2] = t.z;
                        v[4 * q4 + 3] = t.w;
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < R; ++q) v[q] = sm[swz_elem(b0, q, qb)];
                }
                if (INV)
                    dit_round<4>(v, tp, logs, stw, p);
                else
                    dif_round<4>(v, tp, logs, stw, p);
                if (tin) __syncwarp();
                if (vec) {
#pragma unroll
                    for (int q4 = 0; q4 < R / 4; ++q4)
                        *reinterpret_cast<uint4*>(sm + swz_elem(b0, 4 * q4, 0)) =
                            make_uint4(v[4 * q4], v[4 * q4 + 1], v[4 * q4 + 2], v[4 * q4 + 3]);
                } else {
#pragma unroll
                    for (int q = 0; q < R; ++q) sm[swz_elem(b0, q, qb)] = v[q];
                }
            }
        } else {
            // remainder round: the top LRX stages, stride s = 2^(LOGN - LRX), one block
            constexpr int LRX = (REM == 0) ? 1 : REM;
            constexpr int R = 1 << LRX;
            constexpr int NG = (1 << LOGE) / R;
            static_assert(NG % NTHREADS == 0, "whole groups per thread");
            constexpr int LOGSR = LOGN - LRX;
#pragma unroll 2
            for (int it = 0; it < NG / NTHREADS; ++it) {
                const int g = threadIdx.x + it * NTHREADS;
                uint32_t c, tp;
                if constexpr (LAY == Layout::Strided) {
                    c = g & ((1u << LOGC) - 1);
                    tp = g >> LOGC;
                } else {
                    tp = g & ((1u << LOGSR) - 1);
                    c = g >> LOGSR;
                }
                // tp < 2^LOGSR: element q is at x0 | (q << qb)
                const uint32_t x0 = (LAY == Layout::Strided) ? ((tp << LOGC) | c) : ((c << LOGN) | tp);
                constexpr int qb = (LAY == Layout::Strided) ? LOGSR + LOGC : LOGSR;
                const uint32_t b0 = swz(x0);
                uint32_t v[R];
                if (tin) {
                    const uint32_t bt = tma_swz(x0);
#pragma unroll
                    for (int q = 0; q < R; ++q) v[q] = sm[tma_elem(bt, q, qb)];
                } else {
#pragma unroll
                    for (int q = 0; q < R; ++q) v[q] = sm[swz_elem(b0, q, qb)];
                }
                if (INV)
                    dit_round<LRX>(v, tp, LOGSR, stw, p);
                else
                    dif_round<LRX>(v, tp, LOGSR, stw, p);
                if (tin) __syncwarp();
#pragma unroll
                for (int q = 0; q < R; ++q) sm[swz_elem(b0, q, qb)] = v[q];
            }
        }
        __syncthreads();
    }
}

// Global index of tile element (m, c) within its job's array. For Strided tiles `tile` is the
// tile index inside the job; for Contig tiles `row` is the row index inside the job.
template <Layout LAY, int LOGN, int LOGE>
__device__ __forceinline__ uint64_t gidx(uint64_t tile, uint32_t m, uint32_t c, int logS) {
    constexpr int LOGC = LOGE - LOGN;
    if constexpr (LAY == Layout::Strided) {
        // tiles per block = S / C
        const int logTpb = logS - LOGC;
        uint64_t blk = tile >> logTpb;
        uint64_t t0 = (tile & ((1ull << logTpb) - 1)) << LOGC;
        return (blk << (LOGN + logS)) + t0 + c + ((uint64_t)m << logS);
    } else {
        return (tile << LOGN) + m;  // here `tile` is the row inside the job
    }
}

// Column index t (within the block) of tile element column c, for the four-step twiddle.
template <Layout LAY, int LOGN, int LOGE>
__device__ __forceinline__ uint32_t tcol(uint64_t tile, uint32_t c, int logS) {
    constexpr int LOGC = LOGE - LOGN;
    const int logTpb = logS - LOGC;
    return (uint32_t)(((tile & ((1ull << logTpb) - 1)) << LOGC) + c);
}

// Residue words from the launch's data (or out) pointer to job `job`'s arrays.
__device__ __forceinline__ uint64_t job_offset(const PassParams& P, uint64_t job) {
    if (P.comb3) {
        const uint64_t m = job / 3;
        return (6 * m + comb_out_slot((int)(job - 3 * m))) * P.comb_slot;
    }
    return job * P.job_stride;
}

// Source limbs of job `job` (first forward pass); ncoef counts the source's coefficients (two
// per limb for 32-bit ones, one for 64-bit ones).
template <Source SRC>
__device__ __forceinline__ void job_source(const PassParams& P, uint64_t job, const uint32_t*& words,
                                           uint64_t& ncoef) {
    if (P.merge == 2) {
        words = P.src[job].words;
        ncoef = P.src[job].ncoef;
    } else if (P.merge == 1) {
        const uint64_t m = job / 6;
        const int o = (int)(job - 6 * m);
        const uint64_t child = 2 * m + merge_slot_child(o);
        const int which = merge_slot_value(o);
        words = reinterpret_cast<const uint32_t*>(P.ms.X[which] + child * P.ms.cap[which]);
        ncoef = (SRC == Source::Limbs64 ? 1ull : 2ull) * P.ms.len[3 * child + which];
    } else {
        words = P.words + job * P.words_stride;
        ncoef = P.ncoef;
    }
}

// What a contiguous tile's load needs of each of its rows, looked up once per row rather than per
// 16-byte chunk: the source limbs (first forward pass) or, for the splitting's combining pass, the
// sign of R's second product (ncoef = 1 for +, 0 for -).
struct RowSrc {
    const uint32_t* words;
    uint64_t ncoef;
};

// The pass kernel. grid = tiles over all jobs x primes (1-D, tile-major). Tile contents move with 16-byte
// vector accesses along the contiguous dimension. Job j's residues are the array at
// data + j * job_stride (prime i at + i * L).
//
// TMA: the tile (residues, uniform job layout) is loaded by the TMA unit from `tmap` (built by the
// launcher: contiguous tiles as [job][prime][line][32 words], strided ones as
// [job * NP + prime][block][row][column chunk][32 words]) into the 128-byte-swizzled layout, and the
// first radix round (or, for an inverse strided tile, the four-step twiddle loop) rewrites it in the
// passes' own layout. Without TMA the tile is copied by cp.async (tmap unused).
template <Layout LAY, int LOGN, int LOGE, int NTHREADS, bool INV, Source SRC, Fuse FUSE, int NP = kNumPrimes,
          bool TMA = false>
__global__ void __launch_bounds__(NTHREADS, pass_min_blocks<LAY, FUSE, LOGE>())
    ntt_pass_kernel(PassParams P, TwiddleTables T, const __grid_constant__ CUtensorMap tmap) {
    extern __shared__ __align__(1024) uint32_t sm[];
    static_assert(!TMA || (SRC == Source::Residues && FUSE != Fuse::Combine), "TMA tiles hold residues");
    static_assert(!TMA || LAY == Layout::Contig || LOGE - LOGN >= 5, "TMA strided tiles: rows of >= 32 words");
    constexpr int LOGC = LOGE - LOGN;
    constexpr uint32_t E = 1u << LOGE;
    static_assert(E % (4 * NTHREADS) == 0, "tile copies: whole 16-byte chunks per thread");
    // 1-D grid, the NP primes of a tile adjacent: CTAs that read the same operand limbs (first pass)
    // run together, so the limbs come from L2 for all but the first prime
    const uint32_t tile = blockIdx.x / NP;
    const int j = (int)(blockIdx.x - tile * NP);  // prime index
    const uint32_t p = prime_of(NP, j);
    const int dir = INV ? 1 : 0;
    const uint32_t pinv = inv_mod_2_32(p);
    const uint64_t prime_off = (uint64_t)j * P.L;

    // Strided: one job per tile. Contig: row c of the tile is global row R = tile*C + c.
    uint64_t sjob = 0, stile = 0;
    if constexpr (LAY == Layout::Strided) {
        const int logTpj = P.logL - LOGE;
        sjob = (uint64_t)tile >> logTpj;
        stile = (uint64_t)tile & ((1ull << logTpj) - 1);
    }
    const uint64_t total_rows = (uint64_t)P.njobs << (P.logL - LOGN);
    const int logRows = P.logL - LOGN;

    // Contiguous tiles: the per-row sources, after the tile in shared memory.
    static_assert(FUSE != Fuse::Combine || LAY == Layout::Contig, "the combining pass is contiguous");
    constexpr bool kRowSrc = LAY == Layout::Contig && (SRC != Source::Residues || FUSE == Fuse::Combine);
    RowSrc* rsrc = reinterpret_cast<RowSrc*>(sm + E);
    if constexpr (kRowSrc) {
        for (uint32_t c = threadIdx.x; c < (1u << LOGC); c += NTHREADS) {
            const uint64_t R = ((uint64_t)tile << LOGC) + c;
            RowSrc r{nullptr, 0};
            if (R < total_rows) {
                const uint64_t job = R >> logRows;
                if constexpr (SRC != Source::Residues) job_source<SRC>(P, job, r.words, r.ncoef);
                if constexpr (FUSE == Fuse::Combine) {
                    const uint64_t mrg = job / 3;
                    if (job - 3 * mrg == 1) {  // R^
                        uint64_t a, b;
                        node_range(P.comb_a0, P.comb_b0, P.comb_depth, mrg, a, b);
                        r.ncoef = merge_r_sign(a, b) > 0 ? 1 : 0;
                    }
                }
            }
            rsrc[c] = r;
        }
        __syncthreads();
    }

    // Strided tiles: four-step row factors A[m] = w_{N'}^{t0 bitrev(m)} of this tile's first
    // column t0, after the tile in shared memory; B is the row power table of N'.
    uint2* smA = reinterpret_cast<uint2*>(sm + E);
    const uint2* rowB = nullptr;
    if constexpr (LAY == Layout::Strided) {
        rowB = P.rowB + ((size_t)j << LOGE);  // one table per prime, an entry per tile element
        const uint32_t t0 = tcol<LAY, LOGN, LOGE>(stile, 0, P.logS);
        const int sh = root_log_of(NP) - P.logNp;
        const uint2* lo = T.fs_lo[dir][j];
        const uint2* hi = T.fs_hi[dir][j];
        const uint64_t R = recip64_of(NP, j);
        for (uint32_t i = threadIdx.x; i < (1u << LOGN); i += NTHREADS) {
            const uint32_t E0 = (t0 * bitrev_n(i, LOGN)) << sh;  // t0 * k < N', exponent of w_{2^root_log}
            const uint2 a = __ldg(lo + (E0 & ((1u << kFsLog) - 1)));
            const uint2 b = __ldg(hi + (E0 >> kFsLog));
            const uint32_t w = mul_shoup(a.x, b.x, b.y, p);
            smA[i] = make_uint2(w, shoup_companion_dev(w, p, R));
        }
        if constexpr (INV) __syncthreads();  // used by the load loop below
    }

    // Strided tiles: this thread's chunk `it` is row m_0 + it * (4 NTHREADS / C), column c_0, so its
    // element index moves by a fixed step per chunk.
    static_assert(LAY != Layout::Strided || (4 * NTHREADS) % (1u << LOGC) == 0, "chunk rows advance evenly");
    uint64_t sg0 = 0, sgstep = 0;
    if constexpr (LAY == Layout::Strided) {
        const uint32_t e0 = threadIdx.x * 4;
        sg0 = gidx<LAY, LOGN, LOGE>(stile, e0 >> LOGC, e0 & ((1u << LOGC) - 1), P.logS);
        sgstep = (uint64_t)((4 * NTHREADS) >> LOGC) << P.logS;
    }

    // A strided tile belongs to one job: its source words are looked up once, not per element.
    const uint32_t* swords = nullptr;
    uint64_t sncoef = 0;
    if constexpr (SRC != Source::Residues && LAY == Layout::Strided) job_source<SRC>(P, sjob, swords, sncoef);
    // 64-bit coefficients: x = hi 2^32 + lo = hi * (2^32 mod p) + lo (mod p)
    uint32_t one_p64 = 0, r32 = 0, r32p = 0;
    if constexpr (SRC == Source::Limbs64) {
        one_p64 = (uint32_t)(0x100000000ull / p);
        r32 = 0u - one_p64 * p;  // 2^32 - p floor(2^32 / p) < p
        r32p = shoup_companion_dev(r32, p, recip64_of(NP, j));
    }

    // ---- load (4 consecutive elements along the contiguous dimension per thread step)
    if constexpr (TMA) {
        // the barrier sits after the tile and its row data (pass_smem's 16 extra bytes)
        uint64_t* bar = reinterpret_cast<uint64_t*>(
            reinterpret_cast<char*>(sm) + ((size_t)4 << LOGE) +
            (LAY == Layout::Strided ? ((size_t)8 << LOGN) : ((size_t)16 << (LOGE - LOGN))));
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(bar, 4u << LOGE);
            if constexpr (LAY == Layout::Contig) {
                const uint64_t first = (uint64_t)tile << LOGE;  // over all jobs' arrays
                const int job = (int)(first >> P.logL);
                if (P.logL >= LOGE) {
                    // boxes of 256 lines (32 KB)
                    const int line = (int)((first & (P.L - 1)) >> 5);
#pragma unroll
                    for (int k = 0; k < ((1 << LOGE) >> 13); ++k)
                        tma_load_4d(sm + (k << 13), &tmap, bar, 0, line + 256 * k, j, job);
                } else {
                    tma_load_4d(sm, &tmap, bar, 0, 0, j, job);  // one box of E / L whole arrays
                }
            } else {
                const int logTpb = P.logS - LOGC;
                const int blk = (int)(stile >> logTpb);
                const int cc0 = (int)((stile & ((1ull << logTpb) - 1)) << LOGC) >> 5;
                const int jp = (int)(sjob * NP + (uint64_t)j);
                constexpr int kRows = LOGN > 8 ? 256 : (1 << LOGN);
#pragma unroll
                for (int k = 0; k < (1 << LOGN) / kRows; ++k)
                    tma_load_5d(sm + ((k * kRows) << LOGC), &tmap, bar, 0, cc0, k * kRows, blk, jp);
            }
        }
        uint32_t polls = 0;
        while (!mbar_try_wait(bar, 0)) {
            if (++polls >= kTmaSpinLimit) {
                if (P.error) atomicOr(P.error, kErrTmaWait);
                break;
            }
        }
        if constexpr (INV && LAY == Layout::Strided) {
            // inverse four-step twiddle, reading the TMA layout and writing the passes' own: each
            // step's chunks fill whole lines of this warp (8 lanes a line)
#pragma unroll
            for (uint32_t it = 0; it < E / (4 * NTHREADS); ++it) {
                const uint32_t e4 = threadIdx.x * 4 + it * (NTHREADS * 4);
                const uint32_t m = e4 >> LOGC, c = e4 & ((1u << LOGC) - 1);
                uint4 x = *reinterpret_cast<uint4*>(sm + tma_swz(e4));
                fourstep_twiddle4(x, c, m, LOGC, smA[m], rowB, p);
                __syncwarp();
                *reinterpret_cast<uint4*>(sm + swz(e4)) = x;
            }
        }
    } else {
#pragma unroll(LAY == Layout::Strided ? E / (4 * NTHREADS) : 1)
    for (uint32_t it = 0; it < E / (4 * NTHREADS); ++it) {
        const uint32_t e4 = threadIdx.x * 4 + it * (NTHREADS * 4);
        uint32_t m, c;
        uint64_t job, g;
        if constexpr (LAY == Layout::Strided) {
            m = e4 >> LOGC;
            c = e4 & ((1u << LOGC) - 1);
            job = sjob;
            g = sg0 + it * sgstep;
        } else {
            c = e4 >> LOGN;
            m = e4 & ((1u << LOGN) - 1);
            const uint64_t R = ((uint64_t)tile << LOGC) + c;
            if (R >= total_rows) {
                *reinterpret_cast<uint4*>(sm + swz(e4)) = make_uint4(0, 0, 0, 0);
                continue;
            }
            job = R >> logRows;
            g = gidx<LAY, LOGN, LOGE>(R & ((1ull << logRows) - 1), m, c, 0);
        }
        if constexpr (SRC == Source::Residues && FUSE != Fuse::Combine) {
            // residues: an asynchronous copy straight into shared memory (the inverse strided
            // twiddle, if any, is applied below once the copies have landed)
            cp_async16(sm + swz(e4), P.data + job_offset(P, job) + prime_off + g);
        } else if constexpr (SRC == Source::Limbs64) {
            // four 64-bit coefficients (32 bytes of limbs) reduced modulo p in registers; past the
            // operand's end (ncoef limbs), zeros
            const uint32_t* words = swords;
            uint64_t ncoef = sncoef;
            if constexpr (LAY == Layout::Contig) {
                words = rsrc[c].words;
                ncoef = rsrc[c].ncoef;
            }
            uint32_t w[8];
            if (g + 4 <= ncoef) {
                const uint4 v0 = __ldg(reinterpret_cast<const uint4*>(words + 2 * g));
                const uint4 v1 = __ldg(reinterpret_cast<const uint4*>(words + 2 * g + 4));
                w[0] = v0.x; w[1] = v0.y; w[2] = v0.z; w[3] = v0.w;
                w[4] = v1.x; w[5] = v1.y; w[6] = v1.z; w[7] = v1.w;
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const bool in = g + u < ncoef;
                    w[2 * u] = in ? __ldg(words + 2 * (g + u)) : 0u;
                    w[2 * u + 1] = in ? __ldg(words + 2 * (g + u) + 1) : 0u;
                }
            }
            uint32_t r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                r[u] = add_mod(reduce_u32(w[2 * u], p, one_p64), mul_shoup(w[2 * u + 1], r32, r32p, p), p);
            *reinterpret_cast<uint4*>(sm + swz(e4)) = make_uint4(r[0], r[1], r[2], r[3]);
        } else if constexpr (SRC == Source::Limbs) {
            // operand words: whole 16-byte groups copied asynchronously, the ragged end (and the
            // zero padding) written directly; reduced modulo p below once landed
            const uint32_t* words = swords;
            uint64_t ncoef = sncoef;
            if constexpr (LAY == Layout::Contig) {
                words = rsrc[c].words;
                ncoef = rsrc[c].ncoef;
            }
            if (g + 4 <= ncoef) {
                cp_async16(sm + swz(e4), words + g);
            } else {
                uint32_t w[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) w[u] = (g + u < ncoef) ? __ldg(words + g + u) : 0u;
                *reinterpret_cast<uint4*>(sm + swz(e4)) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        } else {
            uint4 x;
            if constexpr (FUSE == Fuse::Combine) {
                // the merge's products in the transform domain (Montgomery: the 2^-32 is in the CRT scale)
                const uint64_t mrg = job / 3;
                const int ck = (int)(job - 3 * mrg);
                const uint32_t* slot0 = P.data + 6 * mrg * P.comb_slot + prime_off + g;
                auto at = [&](int o) { return *reinterpret_cast<const uint4*>(slot0 + (uint64_t)o * P.comb_slot); };
                if (ck == 1) {  // R^ = Qr Rl +- Pl Rr
                    const int sgn = rsrc[c].ncoef ? 1 : -1;
                    const uint4 pl = at(0), rl = at(2), qr = at(3), rr = at(4);
                    uint32_t u, v;
#define PG_RCOMB(f)                                         \
    u = mul_mont(qr.f, rl.f, p, pinv);                      \
    v = mul_mont(pl.f, rr.f, p, pinv);                      \
    x.f = sgn > 0 ? add_mod(u, v, p) : sub_mod(u, v, p);
                    PG_RCOMB(x) PG_RCOMB(y) PG_RCOMB(z) PG_RCOMB(w)
#undef PG_RCOMB
                } else {
                    const uint4 l = ck == 0 ? at(1) : at(0), r = ck == 0 ? at(3) : at(5);  // Ql Qr or Pl Pr
                    x = make_uint4(mul_mont(l.x, r.x, p, pinv), mul_mont(l.y, r.y, p, pinv), mul_mont(l.z, r.z, p, pinv),
                                   mul_mont(l.w, r.w, p, pinv));
                }
            }
            *reinterpret_cast<uint4*>(sm + swz(e4)) = x;
        }
    }
    if constexpr (SRC == Source::Limbs) {
        cp_async_wait_all();  // this thread's copies; each word of its elements reduced modulo p
        const uint32_t one_p = (uint32_t)(0x100000000ull / p);
#pragma unroll(LAY == Layout::Strided ? E / (4 * NTHREADS) : 1)
        for (uint32_t it = 0; it < E / (4 * NTHREADS); ++it) {
        const uint32_t e4 = threadIdx.x * 4 + it * (NTHREADS * 4);
            uint4 w = *reinterpret_cast<uint4*>(sm + swz(e4));
            w = make_uint4(reduce_u32(w.x, p, one_p), reduce_u32(w.y, p, one_p), reduce_u32(w.z, p, one_p),
                           reduce_u32(w.w, p, one_p));
            *reinterpret_cast<uint4*>(sm + swz(e4)) = w;
        }
    }
    if constexpr (SRC == Source::Residues && FUSE != Fuse::Combine) {
        cp_async_wait_all();  // this thread's copies (the barrier below publishes them to the block)
        if constexpr (INV && LAY == Layout::Strided) {
            // inverse four-step twiddle before the sub-transform: w_{N'}^-(t * bitrev(m)), on the
            // same elements this thread copied
#pragma unroll
            for (uint32_t it = 0; it < E / (4 * NTHREADS); ++it) {
        const uint32_t e4 = threadIdx.x * 4 + it * (NTHREADS * 4);
                const uint32_t m = e4 >> LOGC, c = e4 & ((1u << LOGC) - 1);
                uint4 x = *reinterpret_cast<uint4*>(sm + swz(e4));
                fourstep_twiddle4(x, c, m, LOGC, smA[m], rowB, p);
                *reinterpret_cast<uint4*>(sm + swz(e4)) = x;
            }
        }
    }
    }  // cp.async load
    __syncthreads();
    // the first round reads a TMA tile's layout (an inverse strided tile was rewritten above)
    constexpr bool kTin = TMA && !(INV && LAY == Layout::Strided);

    if constexpr (FUSE == Fuse::None || FUSE == Fuse::Combine) {
        tile_transform<LAY, LOGN, LOGE, NTHREADS, INV, 0, 64, kTin>(sm, T.stage[dir][j], p);
    } else {
        // Forward rounds but the last; then, per 16-word group, the last forward round (stride 1),
        // the pointwise product and the first inverse round (stride 1, the same 16 words) in
        // registers; then the remaining inverse rounds.
        static_assert(LAY == Layout::Contig && !INV, "pointwise fusion happens in the last forward pass");
        constexpr int NROUND = LOGN / 4 + ((LOGN % 4) ? 1 : 0);
        const uint2* stw_f = T.stage[0][j];
        const uint2* stw_i = T.stage[1][j];
        tile_transform<LAY, LOGN, LOGE, NTHREADS, false, 0, NROUND - 1, kTin>(sm, stw_f, p);
        constexpr int NG = (1 << LOGE) / 16;
#pragma unroll 1
        for (uint32_t it = 0; it < NG / NTHREADS; ++it) {
            const uint32_t g = threadIdx.x + it * NTHREADS;
            const uint32_t blk = g & ((1u << (LOGN - 4)) - 1);
            const uint32_t c = g >> (LOGN - 4);
            const uint32_t m0 = blk * 16;
            const uint32_t b0 = swz((c << LOGN) | m0);  // vector q4 at swz_elem(b0, 4 q4, 0)
            const uint64_t R = ((uint64_t)tile << LOGC) + c;
            const bool live = R < total_rows;
            uint4 o[4];
            if constexpr (FUSE == Fuse::MulInverse) {
                // the other operand's 16 words, issued before the butterflies so the load overlaps
                // them (rows past the end hold zeros: skip them)
                const uint64_t job = R >> logRows;
                const uint4* src = reinterpret_cast<const uint4*>(
                    P.other + job * P.other_stride + prime_off + ((R & ((1ull << logRows) - 1)) << LOGN) + m0);
#pragma unroll
                for (int q4 = 0; q4 < 4; ++q4) o[q4] = live ? __ldg(src + q4) : make_uint4(0, 0, 0, 0);
            }
            uint32_t v[16];
#pragma unroll
            for (int q4 = 0; q4 < 4; ++q4) {
                const uint4 t = *reinterpret_cast<const uint4*>(sm + swz_elem(b0, 4 * q4, 0));
                v[4 * q4] = t.x;
                v[4 * q4 + 1] = t.y;
                v[4 * q4 + 2] = t.z;
                v[4 * q4 + 3] = t.w;
            }
            dif_round<4>(v, 0, 0, stw_f, p);
            if constexpr (FUSE == Fuse::MulInverse) {
#pragma unroll
                for (int q4 = 0; q4 < 4; ++q4) {
                    const uint4 b = o[q4];
                    v[4 * q4] = mul_mont(v[4 * q4], b.x, p, pinv);
                    v[4 * q4 + 1] = mul_mont(v[4 * q4 + 1], b.y, p, pinv);
                    v[4 * q4 + 2] = mul_mont(v[4 * q4 + 2], b.z, p, pinv);
                    v[4 * q4 + 3] = mul_mont(v[4 * q4 + 3], b.w, p, pinv);
                }
            } else {
#pragma unroll
                for (int q = 0; q < 16; ++q) v[q] = mul_mont(v[q], v[q], p, pinv);
            }
            dit_round<4>(v, 0, 0, stw_i, p);
#pragma unroll
            for (int q4 = 0; q4 < 4; ++q4)
                *reinterpret_cast<uint4*>(sm + swz_elem(b0, 4 * q4, 0)) =
                    make_uint4(v[4 * q4], v[4 * q4 + 1], v[4 * q4 + 2], v[4 * q4 + 3]);
        }
        __syncthreads();
        tile_transform<LAY, LOGN, LOGE, NTHREADS, true, 1, 64>(sm, stw_i, p);
    }

    // ---- store
#pragma unroll(LAY == Layout::Strided ? E / (4 * NTHREADS) : 1)
    for (uint32_t it = 0; it < E / (4 * NTHREADS); ++it) {
        const uint32_t e4 = threadIdx.x * 4 + it * (NTHREADS * 4);
        uint32_t m, c;
        uint64_t job, g;
        if constexpr (LAY == Layout::Strided) {
            m = e4 >> LOGC;
            c = e4 & ((1u << LOGC) - 1);
            job = sjob;
            g = sg0 + it * sgstep;
        } else {
            c = e4 >> LOGN;
            m = e4 & ((1u << LOGN) - 1);
            const uint64_t R = ((uint64_t)tile << LOGC) + c;
            if (R >= total_rows) continue;
            job = R >> logRows;
            g = gidx<LAY, LOGN, LOGE>(R & ((1ull << logRows) - 1), m, c, 0);
        }
        uint4 x = *reinterpret_cast<uint4*>(sm + swz(e4));
        if constexpr (!INV && LAY == Layout::Strided) {
            fourstep_twiddle4(x, c, m, LOGC, smA[m], rowB, p);
        }
        *reinterpret_cast<uint4*>(P.out + job_offset(P, job) + prime_off + g) = x;
    }
}


}  // namespace pg
