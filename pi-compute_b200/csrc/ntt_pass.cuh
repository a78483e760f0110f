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
#include "types.cuh"

namespace pg {

__device__ __forceinline__ uint32_t bitrev_n(uint32_t x, int logn) {
    return logn == 0 ? 0u : (__brev(x) >> (32 - logn));
}

// Four-step twiddles for four consecutive columns t..t+3 of one row (output index k):
// x.x *= w, x.y *= w*s, x.z *= w*s^2, x.w *= w*s^3 with w = w_{N'}^{t k}, s = w_{N'}^k.
// Only w and s come from the tables (s is the same for a whole row, so its loads broadcast
// across the warp); the other three twiddles follow by Montgomery products in registers.
// r32 = 2^32 mod p with Shoup companion r32p (conversion into Montgomery form).
__device__ __forceinline__ void fourstep_twiddle4(uint4& x, uint64_t t, uint64_t k, int logNp, const uint2* lo,
                                                  const uint2* hi, uint32_t p, uint32_t pinv, uint32_t r32,
                                                  uint32_t r32p) {
    const uint32_t mask26 = (1u << kMaxLogL) - 1, mask13 = (1u << kFsLog) - 1;
    const uint32_t E0 = (uint32_t)(((t * k) << (kMaxLogL - logNp)) & mask26);
    const uint32_t Es = (uint32_t)((k << (kMaxLogL - logNp)) & mask26);
    const uint2 a = __ldg(lo + (E0 & mask13));
    const uint2 b = __ldg(hi + (E0 >> kFsLog));
    const uint2 c = __ldg(lo + (Es & mask13));
    const uint2 d = __ldg(hi + (Es >> kFsLog));
    const uint32_t w = mul_shoup(a.x, b.x, b.y, p);
    const uint32_t st = mul_shoup(c.x, d.x, d.y, p);
    uint32_t wm = mul_shoup(w, r32, r32p, p);   // w * 2^32  (Montgomery form)
    const uint32_t sm = mul_shoup(st, r32, r32p, p);
    x.x = mul_mont(x.x, wm, p, pinv);
    wm = mul_mont(wm, sm, p, pinv);
    x.y = mul_mont(x.y, wm, p, pinv);
    wm = mul_mont(wm, sm, p, pinv);
    x.z = mul_mont(x.z, wm, p, pinv);
    wm = mul_mont(wm, sm, p, pinv);
    x.w = mul_mont(x.w, wm, p, pinv);
}

// One decimation-in-frequency round of radix R = 2^LR on v[0..R), the group's
// elements sitting at sub-transform positions t' + s*q within a block of R*s.
// Stage k (half size h = (R/2 >> k) * s) pairs q with q + 2^(LR-1-k) and uses
// twiddle w_{2h}^(t' + s*(q mod 2^(LR-1-k))).
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
            uint32_t x = tp + ((uint32_t)(q & (half - 1)) << logs);
            uint2 w = __ldg(stw + ((1u << logh) + x));
            v[q] = add_mod(a, b, p);
            v[q + half] = mul_shoup(a - b + p, w.x, w.y, p);
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
            uint32_t x = tp + ((uint32_t)(q & (half - 1)) << logs);
            uint2 w = __ldg(stw + ((1u << logh) + x));
            uint32_t a = v[q];
            uint32_t b = mul_shoup(v[q + half], w.x, w.y, p);
            v[q] = add_mod(a, b, p);
            v[q + half] = sub_mod(a, b, p);
        }
    }
}

// Shared-memory address of linear tile index x: 16-byte chunks are permuted inside each
// 128-byte line by bits of the line index (x >> 5) and (x >> 8), so the strided access
// patterns of the radix rounds (strides of 16 and 256 words across lanes) and the 16-byte
// vector accesses of the global<->shared copies all fall on distinct banks.
__device__ __forceinline__ uint32_t swz(uint32_t x) { return x ^ ((((x >> 5) ^ (x >> 8)) & 7u) << 2); }

// Shared-memory address of tile element (m, c).
template <Layout LAY, int LOGN, int LOGE>
__device__ __forceinline__ uint32_t sidx(uint32_t m, uint32_t c) {
    if constexpr (LAY == Layout::Strided) {
        return swz((m << (LOGE - LOGN)) + c);
    } else {
        return swz((c << LOGN) + m);
    }
}

// Run the radix rounds of one sub-transform direction over the whole tile.
// Stages are processed from half size N/2 down to 1 (DIF) or 1 up to N/2 (DIT).
template <Layout LAY, int LOGN, int LOGE, int NTHREADS, bool INV>
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
            for (int g = threadIdx.x; g < NG; g += NTHREADS) {
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
                uint32_t m0 = blk * (R << logs) + tp;
                uint32_t v[R];
#pragma unroll
                for (int q = 0; q < R; ++q) v[q] = sm[sidx<LAY, LOGN, LOGE>(m0 + (q << logs), c)];
                if (INV)
                    dit_round<4>(v, tp, logs, stw, p);
                else
                    dif_round<4>(v, tp, logs, stw, p);
#pragma unroll
                for (int q = 0; q < R; ++q) sm[sidx<LAY, LOGN, LOGE>(m0 + (q << logs), c)] = v[q];
            }
        } else {
            // remainder round: the top LRX stages, stride s = 2^(LOGN - LRX), one block
            constexpr int LRX = (REM == 0) ? 1 : REM;
            constexpr int R = 1 << LRX;
            constexpr int NG = (1 << LOGE) / R;
            constexpr int LOGSR = LOGN - LRX;
            for (int g = threadIdx.x; g < NG; g += NTHREADS) {
                uint32_t c, tp;
                if constexpr (LAY == Layout::Strided) {
                    c = g & ((1u << LOGC) - 1);
                    tp = g >> LOGC;
                } else {
                    tp = g & ((1u << LOGSR) - 1);
                    c = g >> LOGSR;
                }
                uint32_t v[R];
#pragma unroll
                for (int q = 0; q < R; ++q) v[q] = sm[sidx<LAY, LOGN, LOGE>(tp + ((uint32_t)q << LOGSR), c)];
                if (INV)
                    dit_round<LRX>(v, tp, LOGSR, stw, p);
                else
                    dif_round<LRX>(v, tp, LOGSR, stw, p);
#pragma unroll
                for (int q = 0; q < R; ++q) sm[sidx<LAY, LOGN, LOGE>(tp + ((uint32_t)q << LOGSR), c)] = v[q];
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

// Source limbs of job `job` (first forward pass).
__device__ __forceinline__ void job_source(const PassParams& P, uint64_t job, const uint32_t*& words,
                                           uint64_t& ncoef) {
    if (P.merge) {
        const uint64_t m = job / 6, o = job % 6;
        const uint64_t child = 2 * m + (o >= 3 ? 1 : 0);
        const int which = (int)(o % 3);
        words = reinterpret_cast<const uint32_t*>(P.ms.X[which] + child * P.ms.cap[which]);
        ncoef = 2ull * P.ms.len[3 * child + which];
    } else {
        words = P.words;
        ncoef = P.ncoef;
    }
}

// The pass kernel. grid = (tiles over all jobs, primes). Tile contents move with 16-byte
// vector accesses along the contiguous dimension. Job j's residues are the array at
// data + j * job_stride (prime i at + i * L).
template <Layout LAY, int LOGN, int LOGE, int NTHREADS, bool INV, Source SRC, Fuse FUSE>
__global__ void __launch_bounds__(NTHREADS) ntt_pass_kernel(PassParams P, TwiddleTables T) {
    extern __shared__ uint32_t sm[];
    constexpr int LOGC = LOGE - LOGN;
    constexpr uint32_t E = 1u << LOGE;
    const int j = blockIdx.y;
    const uint32_t p = kPrime(j);
    const int dir = INV ? 1 : 0;
    const uint32_t pinv = inv_mod_2_32(p);
    const uint32_t r32 = (uint32_t)(0x100000000ull % p);
    const uint32_t r32p = (uint32_t)(((uint64_t)r32 << 32) / p);
    const uint64_t prime_off = (uint64_t)j * P.L;

    // Strided: one job per tile. Contig: row c of the tile is global row R = tile*C + c.
    uint64_t sjob = 0, stile = 0;
    if constexpr (LAY == Layout::Strided) {
        const int logTpj = P.logL - LOGE;
        sjob = (uint64_t)blockIdx.x >> logTpj;
        stile = (uint64_t)blockIdx.x & ((1ull << logTpj) - 1);
    }
    const uint64_t total_rows = (uint64_t)P.njobs << (P.logL - LOGN);
    const int logRows = P.logL - LOGN;

    // ---- load (4 consecutive elements along the contiguous dimension per thread step)
    for (uint32_t e4 = threadIdx.x * 4; e4 < E; e4 += NTHREADS * 4) {
        uint32_t m, c;
        uint64_t job, g;
        if constexpr (LAY == Layout::Strided) {
            m = e4 >> LOGC;
            c = e4 & ((1u << LOGC) - 1);
            job = sjob;
            g = gidx<LAY, LOGN, LOGE>(stile, m, c, P.logS);
        } else {
            c = e4 >> LOGN;
            m = e4 & ((1u << LOGN) - 1);
            const uint64_t R = ((uint64_t)blockIdx.x << LOGC) + c;
            if (R >= total_rows) {
                *reinterpret_cast<uint4*>(sm + swz(e4)) = make_uint4(0, 0, 0, 0);
                continue;
            }
            job = R >> logRows;
            g = gidx<LAY, LOGN, LOGE>(R & ((1ull << logRows) - 1), m, c, 0);
        }
        uint4 x;
        if constexpr (SRC == Source::Limbs) {
            const uint32_t* words;
            uint64_t ncoef;
            job_source(P, job, words, ncoef);
            const uint32_t one_p = (uint32_t)(0x100000000ull / p);
            uint32_t w[4];
            if (g + 4 <= ncoef) {
                uint4 raw = __ldg(reinterpret_cast<const uint4*>(words + g));
                w[0] = raw.x; w[1] = raw.y; w[2] = raw.z; w[3] = raw.w;
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) w[u] = (g + u < ncoef) ? __ldg(words + g + u) : 0u;
            }
            x = make_uint4(reduce_u32(w[0], p, one_p), reduce_u32(w[1], p, one_p), reduce_u32(w[2], p, one_p),
                           reduce_u32(w[3], p, one_p));
        } else {
            x = *reinterpret_cast<const uint4*>(P.data + job * P.job_stride + prime_off + g);
        }
        if constexpr (INV && LAY == Layout::Strided) {
            // inverse four-step twiddle before the sub-transform: w_{N'}^-(t * bitrev(m))
            uint32_t t = tcol<LAY, LOGN, LOGE>(stile, c, P.logS);
            uint64_t k = bitrev_n(m, LOGN);
            fourstep_twiddle4(x, t, k, P.logNp, T.fs_lo[1][j], T.fs_hi[1][j], p, pinv, r32, r32p);
        }
        *reinterpret_cast<uint4*>(sm + swz(e4)) = x;
    }
    __syncthreads();

    tile_transform<LAY, LOGN, LOGE, NTHREADS, INV>(sm, T.stage[dir][j], p);

    if constexpr (FUSE != Fuse::None) {
        static_assert(LAY == Layout::Contig && !INV, "pointwise fusion happens in the last forward pass");
        for (uint32_t e4 = threadIdx.x * 4; e4 < E; e4 += NTHREADS * 4) {
            uint32_t c = e4 >> LOGN, m = e4 & ((1u << LOGN) - 1);
            const uint64_t R = ((uint64_t)blockIdx.x << LOGC) + c;
            if (R >= total_rows) continue;
            const uint64_t job = R >> logRows;
            uint64_t g = gidx<LAY, LOGN, LOGE>(R & ((1ull << logRows) - 1), m, c, 0);
            uint4 a = *reinterpret_cast<uint4*>(sm + swz(e4));
            uint4 b;
            if constexpr (FUSE == Fuse::MulInverse) {
                b = *reinterpret_cast<const uint4*>(P.other + job * P.job_stride + prime_off + g);
            } else {
                b = a;
            }
            a.x = mul_mont(a.x, b.x, p, pinv);
            a.y = mul_mont(a.y, b.y, p, pinv);
            a.z = mul_mont(a.z, b.z, p, pinv);
            a.w = mul_mont(a.w, b.w, p, pinv);
            *reinterpret_cast<uint4*>(sm + swz(e4)) = a;
        }
        __syncthreads();
        tile_transform<LAY, LOGN, LOGE, NTHREADS, true>(sm, T.stage[1][j], p);
    }

    // ---- store
    for (uint32_t e4 = threadIdx.x * 4; e4 < E; e4 += NTHREADS * 4) {
        uint32_t m, c;
        uint64_t job, g;
        if constexpr (LAY == Layout::Strided) {
            m = e4 >> LOGC;
            c = e4 & ((1u << LOGC) - 1);
            job = sjob;
            g = gidx<LAY, LOGN, LOGE>(stile, m, c, P.logS);
        } else {
            c = e4 >> LOGN;
            m = e4 & ((1u << LOGN) - 1);
            const uint64_t R = ((uint64_t)blockIdx.x << LOGC) + c;
            if (R >= total_rows) continue;
            job = R >> logRows;
            g = gidx<LAY, LOGN, LOGE>(R & ((1ull << logRows) - 1), m, c, 0);
        }
        uint4 x = *reinterpret_cast<uint4*>(sm + swz(e4));
        if constexpr (!INV && LAY == Layout::Strided) {
            uint32_t t = tcol<LAY, LOGN, LOGE>(stile, c, P.logS);
            uint64_t k = bitrev_n(m, LOGN);
            fourstep_twiddle4(x, t, k, P.logNp, T.fs_lo[0][j], T.fs_hi[0][j], p, pinv, r32, r32p);
        }
        *reinterpret_cast<uint4*>(P.out + job * P.job_stride + prime_off + g) = x;
    }
}

}  // namespace pg
