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

constexpr int kStageLog = 14;  // stage twiddles come from w_{2^14}: sub-transforms up to 2^14 points
constexpr int kStageEnt = 1 << 14;  // entries per stage table (entry h + x for h <= 2^13)
constexpr int kFsLog = 13;     // four-step twiddles: w_{2^26}^e = lo[e & 8191] * hi[e >> 13]

// Exponent of w_{2^14} stored at stage-table entry i = h + x (h = 2^k <= i < 2h): w_{2h}^x.
__host__ __device__ inline uint32_t stage_exponent(uint32_t i) {
    if (i == 0) return 0;
    int k = 31 - __builtin_clz_portable(i);
    return (i - (1u << k)) << (kStageLog - 1 - k);
}

constexpr int kRowLogMin = 14;  // row tables exist for four-step blocks of 2^14 .. 2^26 points
constexpr int kRowNMin = 5, kRowNMax = 10;  // and strided sub-transforms of 2^5 .. 2^10 points (2^13 tiles)
constexpr int kRowNBigMin = 11, kRowNBigMax = 12;  // or of 2^11 .. 2^12 points (2^14 tiles)
constexpr int kRowTables = (kMaxLogL - kRowLogMin + 1) * (kRowNMax - kRowNMin + 1);  // per (dir, prime)
constexpr int kRowTablesBig = (kMaxLogL - kRowLogMin + 1) * (kRowNBigMax - kRowNBigMin + 1);

struct TwiddleTables {
    // (w, w') Shoup pairs, [dir][prime]; dir 0 = forward (w), 1 = inverse (w^-1). The tables of one
    // configuration: nprimes primes (3, or 5 for the wide one) with roots w_{2^root_log} (26 or 25).
    int nprimes;
    int root_log;
    const uint2* stage[2][kMaxPrimes];  // entry h + x = w_{2h}^x (h = 2^k, x < h), kStageEnt entries
    const uint2* fs_lo[2][kMaxPrimes];  // w_{2^root_log}^j,           j < 2^13
    const uint2* fs_hi[2][kMaxPrimes];  // w_{2^root_log}^(2^13 * i),  i < 2^13
    // Four-step factors of strided tiles: for a block of N' = 2^n points split into sub-transforms
    // of N = 2^l points (tile of C = 2^(13 - l) columns), table
    // (((n - kRowLogMin) * 6 + l - kRowNMin) * 2 + dir) * nprimes + prime holds
    // w_{N'}^(c * bitrev_l(m)) at entry m * C + c (row-major, so a tile row reads consecutively).
    const uint2* row;
    // The same for sub-transforms of 2^11 and 2^12 points in tiles of 2^14 (C = 2^(14 - l) columns,
    // 2^14 entries): table (((n - kRowLogMin) * 2 + l - kRowNBigMin) * 2 + dir) * nprimes + prime.
    const uint2* row_big;
    // 0: the layouts above for every (n, l); 1: only (14, 7) then (15, 7) (the fixed-size tables
    // of pg_mul_noalloc), [n][dir][prime].
    int row_layout;
    // Transforms of 3 * 2^m points (the wide configuration; null otherwise): W a root of order
    // 3 * 2^25, t3_lo[dir][prime][j] = W^(+-j) and t3_hi[dir][prime][i] = W^(+-2^13 i) (2^13 entries
    // each); the radix-3 butterfly's constants as Shoup pairs: t3_c[dir] = (w3 - w3^2) / 2 with
    // w3 = W^(+-2^25), and t3_h = 1/2.
    const uint2* t3_lo[2][kMaxPrimes];
    const uint2* t3_hi[2][kMaxPrimes];
    uint2 t3_c[2][kMaxPrimes];
    uint2 t3_h[kMaxPrimes];
};

// Prime-0 four-step factor table of a strided pass (prime j at + j * 2^(tile log)), or null.
inline const uint2* row_table(const TwiddleTables& T, int logNp, int logN, int dir) {
    if (T.row_layout == 1) {
        if (logN != 7 || logNp < 14 || logNp > 15) return nullptr;
        return T.row + ((size_t)((logNp - 14) * 2 + dir) * kNumPrimes) * (1u << kFsLog);
    }
    if (logNp < kRowLogMin || logNp > T.root_log) return nullptr;
    if (logN >= kRowNBigMin && logN <= kRowNBigMax) {
        if (!T.row_big) return nullptr;
        const int t = ((logNp - kRowLogMin) * (kRowNBigMax - kRowNBigMin + 1) + (logN - kRowNBigMin)) * 2 + dir;
        return T.row_big + ((size_t)t * T.nprimes) * (1u << 14);
    }
    if (logN < kRowNMin || logN > kRowNMax) return nullptr;
    const int t = ((logNp - kRowLogMin) * (kRowNMax - kRowNMin + 1) + (logN - kRowNMin)) * 2 + dir;
    return T.row + ((size_t)t * T.nprimes) * (1u << kFsLog);
}

enum class Layout : int { Strided = 0, Contig = 1 };
// Residues: a previous pass's output. Limbs: operand limbs as 32-bit coefficients (two per limb).
// Limbs64: operand limbs as 64-bit coefficients (the wide configuration), one per element.
enum class Source : int { Residues = 0, Limbs = 1, Limbs64 = 2 };
// Combine (inverse contiguous pass of a binary-splitting level only): the tile is formed on load
// from the merge's forward-transformed operands, P^ = Pl Pr, Q^ = Ql Qr or R^ = Qr Rl +- Pl Rr.
enum class Fuse : int { None = 0, MulInverse = 1, SqrInverse = 2, Combine = 3 };

// Table-driven batch (merge == 2): operand j of a pass launch comes from src[j], CRT job j
// writes dst[j].
struct SrcEntry {
    const uint32_t* words;  // operand as 32-bit words (device)
    uint64_t ncoef;         // valid words
};
struct DstEntry {
    uint32_t* out;          // output words (device)
    uint64_t nwords;        // words written
    uint32_t centred;       // 1: coefficients are signed (lift to (-P/2, P/2])
    uint32_t pad;
};

// One depth of the binary-splitting tree in device memory: node i's P, Q, R magnitudes at
// X[k] + i * cap[k] (k = 0, 1, 2), lengths in limbs at len[3 i + k].
struct LevelView {
    uint64_t* X[3];    // P, Q, R slot arrays
    uint32_t cap[3];   // limbs per slot
    uint32_t* len;     // len[3 i + k]
};

// Child level of a merge batch: node i's P/Q/R limbs at X[k] + i * cap[k] (k = 0, 1, 2),
// lengths (limbs) at len[3 * i + k].
struct MergeSrc {
    const uint64_t* X[3];
    uint32_t cap[3];
    const uint32_t* len;
};

// A merge's six operand slots in a transform batch, in the order Pl Ql Rl Qr Rr Pr, and its three
// outputs in the order Q^ = Ql Qr, R^ = Qr Rl +- Pl Rr, P^ = Pl Pr: the P's last, so that a batch
// whose last merge needs no P (the rightmost node of every depth when the root's P is not wanted)
// just ends one slot and one output early.
// Slot o holds the value (0 P, 1 Q, 2 R) of the left (child 0) or right (child 1) child:
__host__ __device__ constexpr int merge_slot_child(int o) { return o >= 3 ? 1 : 0; }
__host__ __device__ constexpr int merge_slot_value(int o) { return o < 3 ? o : (o == 3 ? 1 : (o == 4 ? 2 : 0)); }
// Output k holds the value (0 P, 1 Q, 2 R):
__host__ __device__ constexpr int merge_out_value(int k) { return k == 0 ? 1 : (k == 1 ? 2 : 0); }
// Output k is written over the operand slot that only it reads: Q^ over Ql, R^ over Rr, P^ over Pr.
__host__ __device__ constexpr int comb_out_slot(int k) { return k == 0 ? 1 : (k == 1 ? 4 : 5); }

struct PassParams {
    uint32_t* data;          // residues of job 0: prime i at data + i*L; job j at data + j*job_stride
    const uint32_t* other;   // Fuse::MulInverse: fully transformed other operand (same layout)
    uint64_t other_stride;   // residue words between jobs' `other` arrays (0: one operand shared by all)
    uint64_t words_stride;   // Source::Limbs, merge == 0: 32-bit words between jobs' operands
    uint32_t* out;           // where tiles are written (== data for in-place passes)
    const uint32_t* words;   // Source::Limbs, single job: operand as 32-bit words (little-endian)
    uint64_t ncoef;          // Source::Limbs, single job: number of valid 32-bit coefficients
    uint64_t L;              // transform length (elements per prime)
    uint64_t job_stride;     // residue words between consecutive jobs (>= 3*L)
    uint32_t njobs;          // number of transforms in this launch
    int logL;
    int logS;                // log2 of the element stride of this pass (0 for Contig)
    int logNp;               // log2 of the block size N' = N * S (four-step twiddle)
    int merge;               // Source::Limbs per job: 0 words + job*words_stride, 1 from `ms`
                             // (job = 6*merge + operand), 2 from src[job]
    MergeSrc ms;
    const SrcEntry* src;
    const uint2* rowB;       // strided passes: four-step factor table of prime 0 (set by launch_pass)
    // comb3 = 1 (the splitting's Fuse::Combine pass and the inverse passes after it): job j of the
    // launch is output k = j % 3 (0 Q^, 1 R^, 2 P^) of merge m = j / 3. Merge m's operands o (Pl Ql
    // Rl Qr Rr Pr) are at data + (6 m + o) * comb_slot, and output k is written over operand slot
    // comb_out_slot(k), which no other output of the merge reads, so all three outputs of every
    // merge run in one launch.
    int comb3;
    uint64_t comb_slot;
    uint64_t comb_a0, comb_b0;  // the splitting's range and this level's depth (R's sign per merge)
    int comb_depth;
    uint32_t* error;         // optional: bounded waits that give up OR a flag into it (TMA tile loads)
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
    // centred lift: Garner digits of floor(P/2) and P = p0*p1*p2 as (P_hi << 64) + P_lo
    uint32_t h0, h1, h2;
    uint64_t P_lo, P_hi;
};

struct CrtParams {
    const uint32_t* res;     // single product: residues, prime j at res + j*L, natural order
    uint64_t L;
    uint64_t nwords;         // single product: output words (2 * output limbs)
    uint32_t* out;           // single product: output words
    uint32_t* status;        // blocks_per_job words per job, zeroed before launch
    uint32_t* ticket;        // one per job, zeroed before launch
    uint32_t* error;         // set non-zero on a look-back timeout or a final carry
    uint64_t blocks_per_job; // grid = jobs * blocks_per_job
    CrtConsts k;
    // plain batch (merge == 0): job i's residues at res + i * res_stride, its words at
    // out + i * out_stride, its length (if dlen) at dlen[i]; every job has `nwords` words.
    uint64_t out_stride;
    // merge batch: job = 3 * merge + k, output k (0 Q^, 1 R^, 2 P^) of value v = merge_out_value(k);
    // its residues at res + (6m + comb_out_slot(k)) * res_stride; the words go to dst[v] + m * dcap[v]
    // (limbs), the length to dlen[3m + v]; node ranges of the level come from [a0, b0) and depth.
    int merge;
    uint64_t res_stride;
    uint64_t* dst[3];
    uint32_t dcap[3];
    uint32_t* dlen;
    uint64_t a0, b0;
    int depth;
    // table batch (merge == 2): job i's residues at res + i * res_stride, output per dtab[i]
    const DstEntry* dtab;
    // Look-back wait limit in polls (0: kSpinLimit) and a test hook: when withhold1 = b + 1, the
    // block with ticket b never publishes its status, so its successor's wait runs out (0: none).
    // launch_crt fills both from the environment (PG_TEST_CRT_SPIN_LIMIT, PG_TEST_CRT_WITHHOLD).
    uint32_t spin_limit;
    uint32_t withhold1;
    // 1: a carry out of a job's top word is dropped instead of reported (a wrapped product, whose
    // words past the transform length are not wanted).
    int top_ok;
};

constexpr int kCrtThreads = 256;
constexpr int kCrtWords = 16;  // words per thread

}  // namespace pg
