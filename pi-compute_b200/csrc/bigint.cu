// Device big-integer kernels (bigint.cuh) and the DevArith host wrapper (devnum.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "bigint.cuh"
#include "dev_alloc.h"
#include "devnum.h"

namespace pg {
namespace {

// ------------------------------------------------------------------ carry-chain sums
template <AddForm F>
__device__ __forceinline__ void add_fetch(const AddArgs& A, uint64_t job, uint64_t i, uint64_t& u, uint64_t& v) {
    const uint64_t* x = A.x + job * A.sx;
    if constexpr (F == AddForm::Plain) {
        const uint64_t xi = i < A.nx ? x[i] : 0;
        const uint64_t yi = (A.y && i < A.ny) ? A.y[job * A.sy + i] : 0;
        u = xi ^ A.mx;
        v = yi ^ A.my;
    } else {
        const uint64_t xi = i < A.nx ? x[i] : 0;
        const uint64_t xp = (i >= 1 && i - 1 < A.nx) ? x[i - 1] : 0;
        u = xi * A.c;
        v = __umul64hi(xp, A.c);
    }
}

// (g, p) of a range: bit 0 = carry out with carry-in 0, bit 1 = a carry-in passes through.
__device__ __forceinline__ uint32_t gp_compose(uint32_t hi, uint32_t lo) {
    const uint32_t g = (hi & 1u) | ((hi >> 1) & lo & 1u);
    const uint32_t p = (hi >> 1) & (lo >> 1) & 1u;
    return g | (p << 1);
}
__device__ __forceinline__ uint32_t gp_apply(uint32_t gp, uint32_t cin) { return (gp & 1u) | ((gp >> 1) & cin); }

// Inclusive warp scan of (g, p) pairs, lane order = limb order.
__device__ __forceinline__ uint32_t gp_warp_scan(uint32_t gp, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t lo = __shfl_up_sync(0xffffffffu, gp, off);
        if (lane >= off) gp = gp_compose(gp, lo);
    }
    return gp;
}

// *p = v (a single word written by the device, so the host does not wait to reuse a pinned word)
__global__ void set_word_kernel(uint64_t* p, uint64_t v) { *p = v; }

// *out = (*in == 0): the enable flag of a negation that runs only after a borrow
__global__ void not_flag_kernel(const uint32_t* in, uint32_t* out) { *out = (*in & 1u) ? 0u : 1u; }

// Short numbers: one warp per job, K = ceil(n / 32) <= 8 limbs per lane.
template <AddForm F>
__global__ void add_warp_kernel(AddArgs A) {
    const uint64_t job = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (job >= A.njobs) return;
    if (A.enable && !A.enable[job]) return;
    const uint32_t K = (uint32_t)((A.n + 31) / 32);
    const uint64_t base = (uint64_t)lane * K;
    uint64_t s[kBigLimbs];
    uint32_t gen = 0, gp = 2;  // empty range: passes carries
#pragma unroll
    for (int k = 0; k < kBigLimbs; ++k) {
        s[k] = 0;
        if ((uint32_t)k < K && base + k < A.n) {
            uint64_t u, v;
            add_fetch<F>(A, job, base + k, u, v);
            s[k] = u + v;
            const uint32_t gk = s[k] < u ? 1u : 0u;
            gen |= gk << k;
            gp = gp_compose(gk | ((s[k] == ~0ull ? 1u : 0u) << 1), gp);
        }
    }
    const uint32_t incl = gp_warp_scan(gp, lane);
    const uint32_t prev = __shfl_up_sync(0xffffffffu, incl, 1);
    uint32_t carry = lane == 0 ? A.cin : gp_apply(prev, A.cin);
    uint64_t* z = A.z + job * A.sz;
#pragma unroll
    for (int k = 0; k < kBigLimbs; ++k) {
        if ((uint32_t)k < K && base + k < A.n) {
            const uint64_t r = s[k] + carry;
            carry = ((gen >> k) & 1u) | (r < s[k] ? 1u : 0u);
            z[base + k] = r;
        }
    }
    if (lane == 31 && A.carry_out) A.carry_out[job] = carry;
}

// Long numbers, phase 1: (g, p) of each 2048-limb segment.
template <AddForm F>
__global__ void __launch_bounds__(kBigThreads) add_seg_kernel(AddArgs A, uint64_t nseg) {
    __shared__ uint32_t s_w[kBigThreads / 32];
    const uint64_t job = blockIdx.x / nseg, seg = blockIdx.x % nseg;
    if (A.enable && !A.enable[job]) return;
    const uint64_t base = seg * kBigSeg + (uint64_t)threadIdx.x * kBigLimbs;
    uint32_t gp = 2;
#pragma unroll
    for (int k = 0; k < kBigLimbs; ++k) {
        if (base + k < A.n) {
            uint64_t u, v;
            add_fetch<F>(A, job, base + k, u, v);
            const uint64_t s = u + v;
            gp = gp_compose((s < u ? 1u : 0u) | ((s == ~0ull ? 1u : 0u) << 1), gp);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = gp_warp_scan(gp, lane);
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 2;
        for (int w = 0; w < kBigThreads / 32; ++w) t = gp_compose(s_w[w], t);
        A.seg[blockIdx.x] = t;
    }
}

// Phase 2: carry into every segment of a job (bit 2 of its word) and the job's carry out.
// One block per job scans the job's segment words 256 at a time.
__global__ void __launch_bounds__(kBigThreads) add_scan_kernel(AddArgs A, uint64_t nseg) {
    __shared__ uint32_t s_w[kBigThreads / 32];
    const uint64_t job = blockIdx.x;
    if (A.enable && !A.enable[job]) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t carry = A.cin;  // carry into the current chunk of segments
    uint32_t* w = A.seg + job * nseg;
    for (uint64_t base = 0; base < nseg; base += kBigThreads) {
        const uint64_t s = base + threadIdx.x;
        const uint32_t gp = s < nseg ? w[s] : 2u;
        const uint32_t incl = gp_warp_scan(gp, lane);
        if (lane == 31) s_w[warp] = incl;
        __syncthreads();
        uint32_t cw = carry;
        for (int k = 0; k < warp; ++k) cw = gp_apply(s_w[k], cw);
        const uint32_t prev = __shfl_up_sync(0xffffffffu, incl, 1);
        const uint32_t cin = lane == 0 ? cw : gp_apply(prev, cw);
        if (s < nseg) w[s] = gp | (cin << 2);
        uint32_t tot = carry;
        for (int k = 0; k < kBigThreads / 32; ++k) tot = gp_apply(s_w[k], tot);
        __syncthreads();  // s_w is rewritten by the next chunk
        carry = tot;
    }
    if (threadIdx.x == 0 && A.carry_out) A.carry_out[job] = carry;
}

// Phase 3: the sums with each segment's carry in.
template <AddForm F>
__global__ void __launch_bounds__(kBigThreads) add_final_kernel(AddArgs A, uint64_t nseg) {
    __shared__ uint32_t s_w[kBigThreads / 32];
    const uint64_t job = blockIdx.x / nseg, seg = blockIdx.x % nseg;
    if (A.enable && !A.enable[job]) return;
    const uint64_t base = seg * kBigSeg + (uint64_t)threadIdx.x * kBigLimbs;
    uint64_t s[kBigLimbs];
    uint32_t gen = 0, gp = 2;
#pragma unroll
    for (int k = 0; k < kBigLimbs; ++k) {
        s[k] = 0;
        if (base + k < A.n) {
            uint64_t u, v;
            add_fetch<F>(A, job, base + k, u, v);
            s[k] = u + v;
            const uint32_t gk = s[k] < u ? 1u : 0u;
            gen |= gk << k;
            gp = gp_compose(gk | ((s[k] == ~0ull ? 1u : 0u) << 1), gp);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = gp_warp_scan(gp, lane);
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    const uint32_t segcin = (A.seg[blockIdx.x] >> 2) & 1u;
    // carry into this warp: segment carry-in through the earlier warps
    uint32_t cw = segcin;
    for (int w = 0; w < warp; ++w) cw = gp_apply(s_w[w], cw);
    const uint32_t prev = __shfl_up_sync(0xffffffffu, incl, 1);
    uint32_t carry = lane == 0 ? cw : gp_apply(prev, cw);
    uint64_t* z = A.z + job * A.sz;
#pragma unroll
    for (int k = 0; k < kBigLimbs; ++k) {
        if (base + k < A.n) {
            const uint64_t r = s[k] + carry;
            carry = ((gen >> k) & 1u) | (r < s[k] ? 1u : 0u);
            z[base + k] = r;
        }
    }
}

// Plain sums of long numbers in one launch (njobs x nseg blocks): block b sums segment
// s = b % nseg of job b / nseg, publishes the segment's (g, p), looks back over the job's earlier
// segments, 32 at a time across a warp, until one has published its carry out (composing the
// aggregates passed over), publishes its own carry out and writes its limbs. Status word: bits 0-1 (g, p), bit 2 the
// carry out, bit 3 (g, p) valid, bit 4 carry out valid, bits 8-31 the call's epoch (words of
// earlier calls never pass for this one's, so the array needs no reset between calls). Blocks
// start in index order, so a wait is on a block already running; past kAddSpinLimit polls the
// block records kErrAddWait and goes on with carry 0 (the result is then wrong and flagged).
__global__ void __launch_bounds__(kBigThreads) add_onepass_kernel(AddArgs A, uint64_t nseg, uint32_t epoch) {
    __shared__ uint32_t s_w[kBigThreads / 32];
    __shared__ uint32_t s_cin;
    const uint64_t job = blockIdx.x / nseg, seg = blockIdx.x % nseg;
    if (A.enable && !A.enable[job]) return;
    const uint64_t base = seg * kBigSeg + (uint64_t)threadIdx.x * kBigLimbs;
    uint64_t s[kBigLimbs];
    uint32_t gen = 0, gp = 2;
#pragma unroll
    for (int k = 0; k < kBigLimbs; ++k) {
        s[k] = 0;
        if (base + k < A.n) {
            uint64_t u, v;
            add_fetch<AddForm::Plain>(A, job, base + k, u, v);
            s[k] = u + v;
            const uint32_t gk = s[k] < u ? 1u : 0u;
            gen |= gk << k;
            gp = gp_compose(gk | ((s[k] == ~0ull ? 1u : 0u) << 1), gp);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = gp_warp_scan(gp, lane);
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        // the segment's aggregate, published first: later segments may pass over this one
        uint32_t agg = 2;
        for (int w = 0; w < kBigThreads / 32; ++w) agg = gp_compose(s_w[w], agg);
        volatile uint32_t* stw = A.seg + (blockIdx.x - seg);  // the job's status words
        const uint32_t tag = epoch << 8;
        const bool withheld = A.withhold1 && seg + 1 == A.withhold1;
        const uint32_t limit = A.spin_limit ? A.spin_limit : kAddSpinLimit;
        if (lane == 0 && seg > 0 && !withheld) stw[seg] = tag | 8u | agg;
        // look back 32 segments at a time: lane l reads segment j - l (j the window's nearest);
        // once every word of the window is valid, the nearest lane holding a carry out ends the
        // walk, and the window's function is the composition of the aggregates nearer than it
        // (lane order = from the nearest segment down). Segment -1 stands for the carry in.
        uint32_t cin = A.cin;
        if (seg > 0) {
            uint32_t acc = 2;  // (g, p) of the segments passed over so far (identity)
            long long j = (long long)seg - 1;
            uint32_t polls = 0;
            bool timed_out = false;
            for (;;) {
                const long long idx = j - lane;
                uint32_t w = idx < 0 ? (tag | 16u | (A.cin << 2)) : stw[idx];
                bool valid = (w >> 8) == epoch && (w & 24u);
                while (!__all_sync(0xffffffffu, valid)) {
                    if (++polls > limit) {
                        timed_out = true;
                        break;
                    }
                    if (!valid) {
                        w = stw[idx];
                        valid = (w >> 8) == epoch && (w & 24u);
                    }
                }
                if (timed_out) break;
                const unsigned inc = __ballot_sync(0xffffffffu, (w & 16u) != 0);
                const int first = inc ? __ffs(inc) - 1 : 32;  // nearest segment with a carry out
                // lane function: the aggregate before `first`, the carry out at `first` (a constant:
                // g = carry, p = 0), identity beyond
                uint32_t x = lane < first ? (w & 3u) : (lane == first ? ((w >> 2) & 1u) : 2u);
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const uint32_t y = __shfl_down_sync(0xffffffffu, x, off);
                    if (lane + off < 32) x = gp_compose(x, y);
                }
                x = __shfl_sync(0xffffffffu, x, 0);
                acc = gp_compose(acc, x);
                if (inc) {
                    cin = acc & 1u;  // p = 0 past a carry out: g is the carry
                    break;
                }
                j -= 32;
            }
            if (timed_out) {
                if (lane == 0 && A.err) atomicOr(A.err, kErrAddWait);
                cin = 0;
            }
        }
        if (lane == 0) {
            const uint32_t cout = gp_apply(agg, cin);
            if (!withheld) stw[seg] = tag | 16u | 8u | (cout << 2) | agg;
            if (seg == nseg - 1 && A.carry_out) A.carry_out[job] = cout;
            s_cin = cin;
        }
    }
    __syncthreads();
    uint32_t cw = s_cin;
    for (int w = 0; w < warp; ++w) cw = gp_apply(s_w[w], cw);
    const uint32_t prev = __shfl_up_sync(0xffffffffu, incl, 1);
    uint32_t carry = lane == 0 ? cw : gp_apply(prev, cw);
    uint64_t* z = A.z + job * A.sz;
#pragma unroll
    for (int k = 0; k < kBigLimbs; ++k) {
        if (base + k < A.n) {
            const uint64_t r = s[k] + carry;
            carry = ((gen >> k) & 1u) | (r < s[k] ? 1u : 0u);
            z[base + k] = r;
        }
    }
}

// ------------------------------------------------------------------ shifts, compares, lengths
// z_j[0..n) = floor(x_j / 2^s) (x_j has nx limbs, z != x).
__global__ void shr_kernel(const uint64_t* x, uint64_t sx, uint64_t nx, uint64_t* z, uint64_t sz, uint64_t n,
                           uint64_t s, uint64_t njobs) {
    const uint64_t w = s >> 6;
    const uint32_t b = (uint32_t)(s & 63);
    const uint64_t total = n * njobs;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t job = t / n, i = t - job * n;
        const uint64_t* xj = x + job * sx;
        const uint64_t lo = (i + w < nx) ? xj[i + w] : 0;
        const uint64_t hi = (i + w + 1 < nx) ? xj[i + w + 1] : 0;
        z[job * sz + i] = b ? ((lo >> b) | (hi << (64 - b))) : lo;
    }
}

// z[0..n) = x * 2^s (single job, z != x).
__global__ void shl_kernel(const uint64_t* x, uint64_t nx, uint64_t* z, uint64_t n, uint64_t s) {
    const uint64_t w = s >> 6;
    const uint32_t b = (uint32_t)(s & 63);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t lo = (i >= w + 1 && i - w - 1 < nx) ? x[i - w - 1] : 0;
        const uint64_t hi = (i >= w && i - w < nx) ? x[i - w] : 0;
        z[i] = b ? ((hi << b) | (lo >> (64 - b))) : hi;
    }
}

// z[0..n) = x[0..n) masked to its low s bits (s <= 64 n).
__global__ void lowbits_kernel(const uint64_t* x, uint64_t nx, uint64_t* z, uint64_t n, uint64_t s) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t v = i < nx ? x[i] : 0;
        if (64 * (i + 1) > s) v = (64 * i >= s) ? 0 : (v & ((1ull << (s - 64 * i)) - 1));
        z[i] = v;
    }
}

// Block-wide maximum (unsigned), result valid in thread 0.
__device__ __forceinline__ unsigned long long block_max(unsigned long long v) {
    __shared__ unsigned long long s_m[32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, off));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_m[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = max(v, s_m[w]);
    return v;
}

// flag |= 1 if any of the low s bits of x is set (one atomic per block).
__global__ void sticky_kernel(const uint64_t* x, uint64_t nx, uint64_t s, uint32_t* flag) {
    const uint64_t w = s >> 6;
    const uint32_t b = (uint32_t)(s & 63);
    unsigned long long hit = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= w && i < nx;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = x[i];
        if ((i < w) ? (v != 0) : (b && (v & ((1ull << b) - 1)) != 0)) hit = 1;
    }
    hit = block_max(hit);
    if (threadIdx.x == 0 && hit) atomicOr(flag, 1u);
}

// *top = 1 + index of the highest non-zero limb of x (0 if x == 0); *top zeroed before.
__global__ void top_kernel(const uint64_t* x, uint64_t n, unsigned long long* top) {
    unsigned long long m = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (x[i] != 0) m = i + 1;
    m = block_max(m);
    if (threadIdx.x == 0 && m) atomicMax(top, m);
}

// *diff = 1 + highest index where x and y differ (0: equal); *diff zeroed before.
__global__ void diff_kernel(const uint64_t* x, const uint64_t* y, uint64_t n, unsigned long long* diff) {
    unsigned long long m = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (x[i] != y[i]) m = i + 1;
    m = block_max(m);
    if (threadIdx.x == 0 && m) atomicMax(diff, m);
}

// ge[j] = x_j >= y_j over n limbs, one warp per job (no atomics).
__global__ void ge_warp_kernel(const uint64_t* x, uint64_t sx, const uint64_t* y, uint64_t sy, uint64_t n,
                               uint64_t njobs, uint32_t* ge) {
    const uint64_t job = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (job >= njobs) return;
    const uint64_t* xj = x + job * sx;
    const uint64_t* yj = y + job * sy;
    unsigned long long m = 0;
    for (uint64_t i = lane; i < n; i += 32)
        if (xj[i] != yj[i]) m = i + 1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (lane == 0) ge[job] = (m == 0) ? 1u : (xj[m - 1] > yj[m - 1] ? 1u : 0u);
}

// Long numbers, many blocks per job: diff[j] = 1 + highest differing index (grid (blocks, jobs),
// one atomic per block), then ge_from_diff_kernel decides.
__global__ void diff_jobs_kernel(const uint64_t* x, uint64_t sx, const uint64_t* y, uint64_t sy, uint64_t n,
                                 unsigned long long* diff) {
    const uint64_t job = blockIdx.y;
    const uint64_t* xj = x + job * sx;
    const uint64_t* yj = y + job * sy;
    unsigned long long m = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (xj[i] != yj[i]) m = i + 1;
    m = block_max(m);
    if (threadIdx.x == 0 && m) atomicMax(diff + job, m);
}

__global__ void ge_from_diff_kernel(const uint64_t* x, uint64_t sx, const uint64_t* y, uint64_t sy, uint64_t njobs,
                                    const unsigned long long* diff, uint32_t* ge) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = diff[j];
        ge[j] = (k == 0) ? 1u : (x[j * sx + k - 1] > y[j * sy + k - 1] ? 1u : 0u);
    }
}

// The same with one block per job (long numbers).
__global__ void __launch_bounds__(256) ge_block_kernel(const uint64_t* x, uint64_t sx, const uint64_t* y, uint64_t sy,
                                                       uint64_t n, uint32_t* ge) {
    const uint64_t job = blockIdx.x;
    const uint64_t* xj = x + job * sx;
    const uint64_t* yj = y + job * sy;
    unsigned long long m = 0;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x)
        if (xj[i] != yj[i]) m = i + 1;
    m = block_max(m);
    if (threadIdx.x == 0) ge[job] = (m == 0) ? 1u : (xj[m - 1] > yj[m - 1] ? 1u : 0u);
}

// Decimal digits of job j (< 10^digits) written most significant first to out[j * digits ...];
// only characters at global positions [skip, total) are stored, shifted down by skip. *bad is
// set when a job does not fit its digits or a digit below `skip` is not zero.
// (u1 2^64 + u0) / d for the normalised divisor d = 10^19 (d >= 2^63) and u1 < d, with the
// precomputed v = floor((2^128 - 1) / d) - 2^64: the division by an invariant integer of Moller and
// Granlund ("Improved division by invariant integers", IEEE Trans. Computers 60(2), 2011, Alg. 4):
// one 64x64 -> 128 product and at most two corrections instead of a 128-bit division.
__device__ __forceinline__ uint64_t div_ten19(uint64_t u1, uint64_t u0, uint64_t& rem) {
    constexpr uint64_t d = 10000000000000000000ull;
    constexpr uint64_t v = 0xd83c94fb6d2ac34aull;
    uint64_t q0 = v * u1;
    uint64_t q1 = __umul64hi(v, u1);
    const uint64_t s = q0 + u0;
    q1 += u1 + 1 + (s < q0 ? 1 : 0);
    q0 = s;
    uint64_t r = u0 - q1 * d;
    if (r > q0) {
        --q1;
        r += d;
    }
    if (r >= d) {
        ++q1;
        r -= d;
    }
    rem = r;
    return q1;
}

constexpr int kLeafMaxLimbs = 64;

__global__ void leaves_kernel(const uint64_t* x, uint64_t sx, uint64_t nl, uint64_t njobs, uint64_t digits, char* out,
                              uint64_t skip, uint64_t total, uint32_t* bad) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t v[kLeafMaxLimbs];
        const uint64_t* xj = x + j * sx;
        for (uint64_t i = 0; i < nl; ++i) v[i] = xj[i];
        uint64_t top = nl;
        while (top > 0 && v[top - 1] == 0) --top;
        int64_t pos = (int64_t)(j * digits + digits);  // one past the last digit of this job
        uint64_t left = digits;
        while (left > 0) {
            // remainder of v / 10^19, v <- quotient
            uint64_t r = 0;
            for (int64_t i = (int64_t)top - 1; i >= 0; --i) v[i] = div_ten19(r, v[i], r);
            while (top > 0 && v[top - 1] == 0) --top;
            uint64_t g = r;
            const uint64_t nd = left < 19 ? left : 19;
            for (uint64_t d = 0; d < nd; ++d) {
                --pos;
                const char ch = (char)('0' + (g % 10));
                g /= 10;
                if ((uint64_t)pos >= skip && (uint64_t)pos < total)
                    out[pos - skip] = ch;
                else if (ch != '0')
                    atomicOr(bad, 1u);
            }
            left -= nd;
        }
        if (top != 0) atomicOr(bad, 1u);
    }
}

unsigned grid_for(uint64_t work, unsigned per = 256) {
    const uint64_t b = (work + per - 1) / per;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 32));
}

}  // namespace

// ------------------------------------------------------------------ DevArith
void DevPool::trim() {
    for (auto& p : all_) dev_free(p.first);
    all_.clear();
    for (void* a : arenas_) dev_free(a);
    arenas_.clear();
    carved_.clear();
    arena_next_ = nullptr;
    arena_left_ = 0;
    free_.clear();
    if (scratch_) dev_free(scratch_);
    if (flags_) dev_free(flags_);
    if (seg_) dev_free(seg_);
    if (host_word_) pinned_free(host_word_);
    scratch_ = nullptr;
    flags_ = nullptr;
    seg_ = nullptr;
    host_word_ = nullptr;
    scratch_cap_ = flags_cap_ = seg_cap_ = 0;
}

bool DevPool::reserve_arena(size_t bytes) {
    if (arena_left_ >= bytes) return true;
    void* a = nullptr;
    if (pg::dev_malloc(&a, bytes) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    arenas_.push_back(a);
    arena_next_ = static_cast<char*>(a);
    arena_left_ = bytes;
    return true;
}

uint64_t* DevPool::carve(size_t bytes) {
    const size_t step = (bytes + 511) & ~(size_t)511;
    if (!arena_next_ || step > arena_left_) return nullptr;
    uint64_t* p = reinterpret_cast<uint64_t*>(arena_next_);
    arena_next_ += step;
    arena_left_ -= step;
    carved_.push_back({p, bytes / 8});
    return p;
}

size_t DevPool::held_bytes() const {
    size_t b = 0;
    for (const auto& x : all_) b += x.second * 8;
    for (const auto& x : carved_) b += x.second * 8;
    return b;
}

DevArith::DevArith(const DeviceTables& T, Workspace& W, cudaStream_t st, uint64_t* launches, DevPool& pool)
    : T_(T), W_(W), st_(st), launches_(launches), P_(pool), pool_(pool.free_), all_(pool.all_),
      scratch_(pool.scratch_), scratch_cap_(pool.scratch_cap_), flags_(pool.flags_), flags_cap_(pool.flags_cap_),
      seg_(pool.seg_), seg_cap_(pool.seg_cap_), host_word_(pool.host_word_) {
    if (!host_word_ && pinned_malloc(&host_word_, 64) != cudaSuccess) throw DevError(4, "pinned word");
}

DevArith::~DevArith() { cudaStreamSynchronize(st_); }

static void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw DevError(e == cudaErrorMemoryAllocation ? 1 : 4, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

void DevArith::reserve(DevNum& x, size_t limbs) {
    limbs = std::max<size_t>(limbs, 2);
    if (x.d && x.cap >= limbs) return;
    release(x);
    size_t cap = 2;
    while (cap < limbs) cap <<= 1;  // size classes: powers of two
    auto it = pool_.find(cap);
    if (it != pool_.end()) {
        x.d = it->second;
        pool_.erase(it);
    } else if (!(x.d = P_.carve(cap * 8))) {
        check(pg::dev_malloc((void**)&x.d, cap * 8), "DevArith allocation");
        all_.push_back({x.d, cap});
    }
    x.cap = cap;
}

void DevArith::release(DevNum& x) {
    if (x.d) pool_.insert({x.cap, x.d});
    x.d = nullptr;
    x.cap = x.n = 0;
    x.sign = 0;
    x.slack = 0;
}

uint64_t* DevArith::scratch(size_t limbs) {
    if (limbs > scratch_cap_) {
        if (scratch_) {
            cudaStreamSynchronize(st_);
            dev_free(scratch_);
        }
        const size_t cap = std::max(limbs, scratch_cap_ * 3 / 2);
        scratch_ = nullptr;
        scratch_cap_ = 0;
        check(pg::dev_malloc((void**)&scratch_, cap * 8), "DevArith scratch");
        scratch_cap_ = cap;
    }
    return scratch_;
}

uint32_t* DevArith::flags(size_t n) {
    if (n > flags_cap_) {
        if (flags_) {
            cudaStreamSynchronize(st_);
            dev_free(flags_);
        }
        const size_t cap = std::max<size_t>({n, 1024, flags_cap_ + flags_cap_ / 2});
        flags_ = nullptr;
        flags_cap_ = 0;
        check(pg::dev_malloc((void**)&flags_, cap * 8), "DevArith flags");
        flags_cap_ = cap;
    }
    return flags_;
}

void DevArith::sync() {
    check(cudaStreamSynchronize(st_), "DevArith");
}

// Plain long sums in one launch (add_onepass_kernel) unless PG_ADD_ONEPASS=0 (three launches, no
// wait between blocks).
static bool add_onepass() {
    static const bool on = [] {
        const char* e = std::getenv("PG_ADD_ONEPASS");
        return !(e && e[0] == '0' && e[1] == 0);
    }();
    return on;
}

void DevArith::run_add(const AddArgs& a0, int form) {
    AddArgs a = a0;
    if (a.n == 0) return;
    if (a.n <= kBigWarpMax) {
        const uint64_t threads = a.njobs * 32;
        const unsigned blocks = (unsigned)((threads + 255) / 256);
        if (form == 0)
            add_warp_kernel<AddForm::Plain><<<blocks, 256, 0, st_>>>(a);
        else
            add_warp_kernel<AddForm::MulSmall><<<blocks, 256, 0, st_>>>(a);
        check(cudaGetLastError(), "add");
        ++*launches_;
        return;
    }
    const uint64_t nseg = (a.n + kBigSeg - 1) / kBigSeg;
    if (a.njobs * nseg > seg_cap_) {
        if (seg_) {
            cudaStreamSynchronize(st_);
            dev_free(seg_);
        }
        const size_t cap = std::max<size_t>({a.njobs * nseg, 4096, seg_cap_ + seg_cap_ / 2});
        seg_ = nullptr;
        seg_cap_ = 0;
        check(pg::dev_malloc((void**)&seg_, cap * 4), "DevArith segments");
        // no stale epoch may match a later call's (one-pass status words)
        check(cudaMemsetAsync(seg_, 0, cap * 4, st_), "DevArith segments");
        seg_cap_ = cap;
    }
    a.seg = seg_;
    const unsigned blocks = (unsigned)(a.njobs * nseg);
    if (form == 0 && add_onepass()) {
        if (!W_.sync) check(W_.ensure_sync(1), "error word");
        a.err = W_.sync;
        // test hooks, read on every call so that a test can set and clear them around one
        // operation: PG_TEST_ADD_SPIN_LIMIT=n ends each wait after n polls, PG_TEST_ADD_WITHHOLD=s
        // keeps segment s from publishing its status, so that the later segments' waits run out
        // (kErrAddWait; no GPU fault). Unset: the built-in limit, no hook.
        if (const char* e = std::getenv("PG_TEST_ADD_SPIN_LIMIT")) a.spin_limit = (uint32_t)std::strtoul(e, nullptr, 10);
        if (const char* e = std::getenv("PG_TEST_ADD_WITHHOLD")) a.withhold1 = (uint32_t)std::strtoul(e, nullptr, 10) + 1;
        if (++P_.add_epoch_ > 0xffffffu) {  // the epoch field wraps: clear the words, start again
            check(cudaMemsetAsync(seg_, 0, seg_cap_ * 4, st_), "DevArith segments");
            P_.add_epoch_ = 1;
        }
        add_onepass_kernel<<<blocks, kBigThreads, 0, st_>>>(a, nseg, P_.add_epoch_);
        check(cudaGetLastError(), "add");
        ++*launches_;
        return;
    }
    if (form == 0)
        add_seg_kernel<AddForm::Plain><<<blocks, kBigThreads, 0, st_>>>(a, nseg);
    else
        add_seg_kernel<AddForm::MulSmall><<<blocks, kBigThreads, 0, st_>>>(a, nseg);
    add_scan_kernel<<<(unsigned)a.njobs, kBigThreads, 0, st_>>>(a, nseg);
    if (form == 0)
        add_final_kernel<AddForm::Plain><<<blocks, kBigThreads, 0, st_>>>(a, nseg);
    else
        add_final_kernel<AddForm::MulSmall><<<blocks, kBigThreads, 0, st_>>>(a, nseg);
    check(cudaGetLastError(), "add");
    *launches_ += 3;
}

void DevArith::normalize(DevNum& x) {
    if (x.n == 0) {
        x.sign = 0;
        return;
    }
    unsigned long long* top = reinterpret_cast<unsigned long long*>(flags(2));
    check(cudaMemsetAsync(top, 0, 8, st_), "normalize");
    top_kernel<<<grid_for(x.n), 256, 0, st_>>>(x.d, x.n, top);
    ++*launches_;
    check(cudaMemcpyAsync(host_word_, top, 8, cudaMemcpyDeviceToHost, st_), "normalize");
    sync();
    x.n = (size_t)host_word_[0];
    if (x.n == 0) x.sign = 0;
    x.slack = 0;
}

void DevArith::set_ui(DevNum& x, uint64_t v) {
    reserve(x, 2);
    set_word_kernel<<<1, 1, 0, st_>>>(x.d, v);  // a launch, not a copy from a reused pinned word
    check(cudaGetLastError(), "set_ui");
    ++*launches_;
    x.n = v ? 1 : 0;
    x.sign = v ? 1 : 0;
    x.slack = 0;
}

void DevArith::set_pow2(DevNum& x, size_t e) {
    const size_t n = e / 64 + 1;
    reserve(x, n);
    if (n > 1) check(cudaMemsetAsync(x.d, 0, (n - 1) * 8, st_), "set_pow2");
    set_word_kernel<<<1, 1, 0, st_>>>(x.d + n - 1, 1ull << (e % 64));
    check(cudaGetLastError(), "set_pow2");
    ++*launches_;
    x.n = n;
    x.sign = 1;
    x.slack = 0;
}

void DevArith::copy(DevNum& z, const DevNum& x) {
    if (&z == &x) return;
    reserve(z, x.n);
    if (x.n) check(cudaMemcpyAsync(z.d, x.d, x.n * 8, cudaMemcpyDeviceToDevice, st_), "copy");
    z.n = x.n;
    z.sign = x.sign;
    z.slack = x.slack;
}

void DevArith::upload(DevNum& x, const uint64_t* host, size_t n, int sign) {
    while (n && host[n - 1] == 0) --n;
    reserve(x, n);
    if (n) check(cudaMemcpyAsync(x.d, host, n * 8, cudaMemcpyHostToDevice, st_), "upload");
    sync();
    x.n = n;
    x.slack = 0;
    x.sign = n ? (sign < 0 ? -1 : 1) : 0;
}

void DevArith::download(const DevNum& x, uint64_t* host) {
    exact(const_cast<DevNum&>(x));  // the value is unchanged; only its recorded length
    if (x.n) check(cudaMemcpyAsync(host, x.d, x.n * 8, cudaMemcpyDeviceToHost, st_), "download");
    sync();
}

size_t DevArith::bits(const DevNum& x) {
    exact(const_cast<DevNum&>(x));
    if (x.n == 0) return 0;
    check(cudaMemcpyAsync(host_word_, x.d + x.n - 1, 8, cudaMemcpyDeviceToHost, st_), "bits");
    sync();
    const uint64_t top = host_word_[0];
    return 64 * (x.n - 1) + (64 - (size_t)__builtin_clzll(top));
}

int DevArith::cmp_abs(const DevNum& x, const DevNum& y) {
    exact(const_cast<DevNum&>(x));
    exact(const_cast<DevNum&>(y));
    if (x.n != y.n) return x.n < y.n ? -1 : 1;
    if (x.n == 0) return 0;
    unsigned long long* diff = reinterpret_cast<unsigned long long*>(flags(2));
    check(cudaMemsetAsync(diff, 0, 8, st_), "cmp");
    diff_kernel<<<grid_for(x.n), 256, 0, st_>>>(x.d, y.d, x.n, diff);
    ++*launches_;
    check(cudaMemcpyAsync(host_word_, diff, 8, cudaMemcpyDeviceToHost, st_), "cmp");
    sync();
    const uint64_t k = host_word_[0];
    if (k == 0) return 0;
    check(cudaMemcpyAsync(host_word_ + 1, x.d + k - 1, 8, cudaMemcpyDeviceToHost, st_), "cmp");
    check(cudaMemcpyAsync(host_word_ + 2, y.d + k - 1, 8, cudaMemcpyDeviceToHost, st_), "cmp");
    sync();
    return host_word_[1] > host_word_[2] ? 1 : -1;
}

int DevArith::cmp(const DevNum& x, const DevNum& y) {
    exact(const_cast<DevNum&>(x));  // a zero value gets sign 0
    exact(const_cast<DevNum&>(y));
    if (x.sign != y.sign) return x.sign < y.sign ? -1 : 1;
    const int c = cmp_abs(x, y);
    return x.sign >= 0 ? c : -c;
}

// |z| = |x| + |y| with sign `sign`.
void DevArith::add_mag(DevNum& z, const DevNum& x, const DevNum& y, int sign) {
    const size_t n = std::max(x.n, y.n) + 1;
    DevNum t;
    const bool alias = (&z == &x) || (&z == &y);
    DevNum& out = alias ? t : z;
    reserve(out, n);
    AddArgs a{};
    a.x = x.d;
    a.nx = x.n;
    a.y = y.d;
    a.ny = y.n;
    a.z = out.d;
    a.n = n;
    a.njobs = 1;
    run_add(a, 0);
    out.n = n;
    out.sign = sign;
    out.slack = std::max(x.slack, y.slack) + 1;
    if (alias) {
        std::swap(z, t);
        release(t);
    }
}

// z = |x| - |y|, signed: sign_if_pos when |x| >= |y|, else -sign_if_pos.
void DevArith::sub_mag(DevNum& z, const DevNum& x, const DevNum& y, int sign_if_pos) {
    const size_t n = std::max(x.n, y.n);
    DevNum t;
    const bool alias = (&z == &x) || (&z == &y);
    DevNum& out = alias ? t : z;
    reserve(out, n);
    // f[0]: carry out of x - y (0 <=> |x| < |y|), f[1]: 1 - f[0], f[2..3]: exact length
    uint32_t* f = flags(4);
    unsigned long long* top = reinterpret_cast<unsigned long long*>(f + 2);
    check(cudaMemsetAsync(f, 0, 16, st_), "sub");
    AddArgs a{};
    a.x = x.d;
    a.nx = x.n;
    a.y = y.d;
    a.ny = y.n;
    a.my = ~0ull;
    a.cin = 1;
    a.z = out.d;
    a.n = n;
    a.njobs = 1;
    a.carry_out = f;
    run_add(a, 0);
    not_flag_kernel<<<1, 1, 0, st_>>>(f, f + 1);
    ++*launches_;
    AddArgs b{};  // on a borrow, two's complement in place: magnitude = ~out + 1
    b.x = out.d;
    b.nx = n;
    b.mx = ~0ull;
    b.cin = 1;
    b.z = out.d;
    b.n = n;
    b.enable = f + 1;
    b.njobs = 1;
    run_add(b, 0);
    top_kernel<<<grid_for(n), 256, 0, st_>>>(out.d, n, top);
    ++*launches_;
    // the borrow and the exact length come back together: the one host wait of a subtraction
    check(cudaMemcpyAsync(host_word_, f, 16, cudaMemcpyDeviceToHost, st_), "sub");
    sync();
    const bool borrow = (host_word_[0] & 1u) == 0;
    out.n = (size_t)host_word_[1];
    out.sign = out.n ? (borrow ? -sign_if_pos : sign_if_pos) : 0;
    out.slack = 0;
    if (alias) {
        std::swap(z, t);
        release(t);
    }
}

void DevArith::add(DevNum& z, const DevNum& x, const DevNum& y) {
    if (y.sign == 0) return copy(z, x);
    if (x.sign == 0) return copy(z, y);
    if (x.sign == y.sign) return add_mag(z, x, y, x.sign);
    sub_mag(z, x, y, x.sign);
}

void DevArith::sub(DevNum& z, const DevNum& x, const DevNum& y) {
    if (y.sign == 0) return copy(z, x);
    if (x.sign == 0) {
        copy(z, y);
        z.sign = -z.sign;
        return;
    }
    if (x.sign != y.sign) return add_mag(z, x, y, x.sign);
    sub_mag(z, x, y, x.sign);
}

void DevArith::add_si(DevNum& z, const DevNum& x, int64_t v) {
    DevNum c;
    set_ui(c, (uint64_t)(v < 0 ? -v : v));
    c.sign = v < 0 ? -1 : (v > 0 ? 1 : 0);
    add(z, x, c);
    release(c);
}

void DevArith::mul(DevNum& z, const DevNum& x, const DevNum& y) {
    if (x.sign == 0 || y.sign == 0) {
        reserve(z, 1);
        z.n = 0;
        z.sign = 0;
        return;
    }
    // upper-bound lengths compound through chains of products (a squaring doubles the slack):
    // operands more than a few limbs over their exact length are measured first
    if (x.slack > 4) exact(const_cast<DevNum&>(x));
    if (y.slack > 4) exact(const_cast<DevNum&>(y));
    DevNum t;
    reserve(t, x.n + y.n);
    mul_limbs(x.d, x.n, y.d, y.n, t.d);
    t.n = x.n + y.n;
    t.sign = x.sign * y.sign;
    t.slack = x.slack + y.slack + 1;
    std::swap(z, t);
    release(t);
}

void DevArith::sqr(DevNum& z, const DevNum& x) { mul(z, x, x); }

void DevArith::mul_limbs(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out) {
    const bool square = (a == b && na == nb);
    // the transform's first pass reads operand limbs with 16-byte vector loads
    if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(out)) & 15)
        throw DevError(3, "product: operands must be 16-byte aligned");
    if (product_logL(na, nb) <= split_logL()) {
        check(enqueue_product(T_, W_, a, na, square ? nullptr : b, nb, out, st_, launches_), square ? "square" : "product");
        return;
    }
    // Blocks of at most 2^(l-2) limbs, so that a block product (< 2^(l-1) limbs) fits one
    // transform of 2^l points; k_a x k_b block products, each added into out at its offset.
    // Block sizes are even: every block (and every offset in out) starts on a 16-byte boundary,
    // which the transform's vector loads of the operand limbs need.
    const size_t cap = (size_t)1 << (split_logL() - 2);
    const size_t ka = (na + cap - 1) / cap, kb = (nb + cap - 1) / cap;
    const size_t Ba = ((na + ka - 1) / ka + 1) & ~(size_t)1, Bb = ((nb + kb - 1) / kb + 1) & ~(size_t)1;
    const size_t total = na + nb;
    check(cudaMemsetAsync(out, 0, total * 8, st_), "block product");
    DevNum t;
    reserve(t, Ba + Bb);
    for (size_t i = 0; i < ka && i * Ba < na; ++i) {
        const size_t la = std::min(Ba, na - i * Ba);
        for (size_t j = (square ? i : 0); j < kb && j * Bb < nb; ++j) {
            const size_t lb = std::min(Bb, nb - j * Bb);
            const uint64_t* bj = (square && i == j) ? nullptr : b + j * Bb;
            check(enqueue_product(T_, W_, a + i * Ba, la, bj, lb, t.d, st_, launches_), "block product");
            // out[off ..) += t (twice for an off-diagonal block of a square)
            const size_t off = i * Ba + j * Bb;
            for (int rep = 0; rep < ((square && i != j) ? 2 : 1); ++rep) {
                AddArgs g{};
                g.x = out + off;
                g.nx = total - off;
                g.y = t.d;
                g.ny = la + lb;
                g.z = out + off;
                g.n = total - off;
                g.njobs = 1;
                run_add(g, 0);
            }
        }
    }
    release(t);
}

void DevArith::fold(DevNum& z, const DevNum& x, int logL) {
    const size_t half = (size_t)1 << (logL - 1);  // limbs of 2^(32 L)
    if (x.n <= half) return copy(z, x);
    if (x.n > half + 2) throw DevError(3, "fold: value too long");
    const int sign = x.sign;
    DevNum lo, hi;  // views of x (never released); lo may have zero top limbs, which add() allows
    lo.d = x.d;
    lo.n = half;
    lo.sign = 1;
    lo.slack = half;
    hi.d = x.d + half;
    hi.n = x.n - half;
    hi.sign = 1;
    hi.slack = hi.n;
    DevNum t;
    add(t, lo, hi);  // < 2^(32 L) + 2^128
    exact(t);
    if (t.n > half) {  // 2^(32 L) = M + 1: drop it and add one
        tdiv_r_2exp(t, t, 64 * half);
        add_si(t, t, 1);
    }
    if (t.n) t.sign = sign;
    std::swap(z, t);
    release(t);
}

void DevArith::mul_wrap(DevNum& z, const DevNum& x, const DevNum& y, int logL) {
    const size_t half = (size_t)1 << (logL - 1);
    if (x.sign == 0 || y.sign == 0) {
        reserve(z, 1);
        z.n = 0;
        z.sign = 0;
        return;
    }
    if (2 * x.n > 2 * half || 2 * y.n > 2 * half) throw DevError(3, "mul_wrap: operand longer than the transform");
    DevNum t;
    reserve(t, half + 1);
    const bool sq = (&x == &y || x.d == y.d);
    check(enqueue_product_wrap(T_, W_, x.d, x.n, sq ? nullptr : y.d, y.n, logL, t.d, st_, launches_), "wrapped product");
    t.n = half + 1;  // an upper bound: fold() adds the top limb in whether or not it is zero
    t.sign = 1;
    t.slack = half + 1;
    fold(z, t, logL);
    release(t);
    if (z.n) z.sign = x.sign * y.sign;
}

void DevArith::mul_ui(DevNum& z, const DevNum& x, uint64_t c) {
    if (x.sign == 0 || c == 0) {
        reserve(z, 1);
        z.n = 0;
        z.sign = 0;
        return;
    }
    DevNum t;
    reserve(t, x.n + 1);
    AddArgs a{};
    a.x = x.d;
    a.nx = x.n;
    a.c = c;
    a.z = t.d;
    a.n = x.n + 1;
    a.njobs = 1;
    run_add(a, 1);
    t.n = x.n + 1;
    t.sign = x.sign;
    t.slack = x.slack + 1;
    std::swap(z, t);
    release(t);
}

void DevArith::shl(DevNum& z, const DevNum& x, size_t s) {
    if (x.sign == 0) return copy(z, x);
    DevNum t;
    const size_t n = x.n + s / 64 + 1;
    reserve(t, n);
    shl_kernel<<<grid_for(n), 256, 0, st_>>>(x.d, x.n, t.d, n, s);
    check(cudaGetLastError(), "shl");
    ++*launches_;
    t.n = n;
    t.sign = x.sign;
    t.slack = x.slack + 1;
    std::swap(z, t);
    release(t);
}

void DevArith::tdiv_q_2exp(DevNum& z, const DevNum& x, size_t s) {
    if (x.sign == 0 || s >= 64 * x.n) {
        reserve(z, 1);
        z.n = 0;
        z.sign = 0;
        return;
    }
    DevNum t;
    const size_t n = x.n - s / 64;
    reserve(t, n);
    shr_kernel<<<grid_for(n), 256, 0, st_>>>(x.d, 0, x.n, t.d, 0, n, s, 1);
    check(cudaGetLastError(), "shr");
    ++*launches_;
    t.n = n;
    t.sign = x.sign;
    t.slack = x.slack + 1;
    std::swap(z, t);
    release(t);
}

void DevArith::fdiv_q_2exp(DevNum& z, const DevNum& x, size_t s) {
    if (x.sign >= 0 || x.n == 0) return tdiv_q_2exp(z, x, s);
    // floor of a negative quotient: -(trunc(|x| / 2^s) + (any low bit set)); the +1 is applied on
    // the device under the sticky flag, so the host does not wait for it
    const size_t q = s / 64;
    const size_t n = x.n > q ? x.n - q : 0;
    DevNum t;
    reserve(t, n + 1);
    uint32_t* f = flags(1);
    check(cudaMemsetAsync(f, 0, 4, st_), "fdiv");
    sticky_kernel<<<grid_for(std::min<uint64_t>(x.n, q + 1)), 256, 0, st_>>>(x.d, x.n, s, f);
    ++*launches_;
    if (n) {
        shr_kernel<<<grid_for(n), 256, 0, st_>>>(x.d, 0, x.n, t.d, 0, n, s, 1);
        ++*launches_;
    }
    check(cudaMemsetAsync(t.d + n, 0, 8, st_), "fdiv");
    AddArgs a{};
    a.x = t.d;
    a.nx = n + 1;
    a.cin = 1;
    a.z = t.d;
    a.n = n + 1;
    a.enable = f;  // in place, only when a dropped bit was set
    a.njobs = 1;
    run_add(a, 0);
    t.n = n + 1;
    t.sign = -1;
    t.slack = x.slack + 2;
    std::swap(z, t);
    release(t);
}

void DevArith::tdiv_r_2exp(DevNum& z, const DevNum& x, size_t s) {
    DevNum t;
    const size_t n = std::min<size_t>(x.n, (s + 63) / 64);
    reserve(t, std::max<size_t>(n, 1));
    if (n) {
        lowbits_kernel<<<grid_for(n), 256, 0, st_>>>(x.d, x.n, t.d, n, s);
        check(cudaGetLastError(), "lowbits");
        ++*launches_;
    }
    t.n = n;
    t.sign = x.sign;
    t.slack = n;  // the low bits may have zero limbs on top: length unknown
    std::swap(z, t);
    release(t);
}

// ------------------------------------------------------------------ batched forms
void DevArith::batch_add(const uint64_t* x, uint64_t sx, uint64_t nx, const uint64_t* y, uint64_t sy, uint64_t ny,
                         uint64_t* z, uint64_t sz, uint64_t n, bool subtract, uint32_t cin, const uint32_t* enable,
                         uint64_t njobs) {
    AddArgs a{};
    a.x = x;
    a.sx = sx;
    a.nx = nx;
    a.y = y;
    a.sy = sy;
    a.ny = ny;
    a.z = z;
    a.sz = sz;
    a.n = n;
    a.my = subtract ? ~0ull : 0;
    a.cin = subtract ? 1u : cin;
    a.enable = enable;
    a.njobs = njobs;
    run_add(a, 0);
}

void DevArith::batch_shr(const uint64_t* x, uint64_t sx, uint64_t nx, uint64_t* z, uint64_t sz, uint64_t n, uint64_t s,
                         uint64_t njobs) {
    shr_kernel<<<grid_for(n * njobs), 256, 0, st_>>>(x, sx, nx, z, sz, n, s, njobs);
    check(cudaGetLastError(), "batch shr");
    ++*launches_;
}

void DevArith::batch_ge(const uint64_t* x, uint64_t sx, const uint64_t* y, uint64_t sy, uint64_t n, uint32_t* ge,
                        uint64_t njobs) {
    if (n <= 1024) {
        ge_warp_kernel<<<(unsigned)((njobs * 32 + 255) / 256), 256, 0, st_>>>(x, sx, y, sy, n, njobs, ge);
        ++*launches_;
    } else if (n <= 16384 || njobs >= 1024) {
        ge_block_kernel<<<(unsigned)njobs, 256, 0, st_>>>(x, sx, y, sy, n, ge);
        ++*launches_;
    } else {
        // few long jobs: spread each over many blocks
        unsigned long long* diff = reinterpret_cast<unsigned long long*>(scratch(njobs));
        check(cudaMemsetAsync(diff, 0, njobs * 8, st_), "batch ge");
        const unsigned per = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(n / 8192, 148ull * 8 / njobs + 1));
        dim3 grid(per, (unsigned)njobs);
        diff_jobs_kernel<<<grid, 256, 0, st_>>>(x, sx, y, sy, n, diff);
        ge_from_diff_kernel<<<grid_for(njobs), 256, 0, st_>>>(x, sx, y, sy, njobs, diff, ge);
        *launches_ += 2;
    }
    check(cudaGetLastError(), "batch ge");
}

bool DevArith::leaves(const uint64_t* x, uint64_t sx, uint64_t nlimbs, uint64_t njobs, uint64_t digits, char* out,
                      uint64_t skip, uint64_t total) {
    if (nlimbs > (uint64_t)kLeafMaxLimbs) throw DevError(3, "leaves: chunk longer than 64 limbs");
    uint32_t* bad = flags(1);
    check(cudaMemsetAsync(bad, 0, 4, st_), "leaves");
    leaves_kernel<<<grid_for(njobs, 128), 128, 0, st_>>>(x, sx, nlimbs, njobs, digits, out, skip, total, bad);
    check(cudaGetLastError(), "leaves");
    ++*launches_;
    check(cudaMemcpyAsync(host_word_, bad, 4, cudaMemcpyDeviceToHost, st_), "leaves");
    sync();
    return (host_word_[0] & 1u) == 0;
}

}  // namespace pg
