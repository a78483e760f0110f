// Exact CRT recombination of the three inverse-transformed residue arrays and
// the carry-propagation scan that turns the convolution into product limbs.
//
// Coefficient i of the (w = 32) convolution is x_i, rebuilt by Garner's method with all
// constants precomputed (the scale L^-1 * 2^32 for the unnormalised inverse transform and
// the Montgomery pointwise product are folded into them). For a plain product x_i lies in
// [0, p0*p1*p2) and is < 2^91. For a signed combination (the binary-splitting R = Qr*Rl -
// Pl*Rr done in the transform domain) coefficients may be negative: the CRT value is lifted
// to (-p0p1p2/2, p0p1p2/2] and held as a 96-bit two's-complement number.
//
// Output 32-bit word j receives W_j = x_j[0] + x_{j-1}[1] + x_{j-2}[2] (x[2] signed), so
// W_j lies in (-2^31, 2^33 + 2^31) and every carry between words is in {-1, 0, 1, 2}.
//
// The scan: each thread owns 16 consecutive words; its carry behaviour is the transfer
// function f: {-1,0,1,2} -> {-1,0,1,2} (carry in -> carry out), stored as 4 two-bit
// entries of (carry + 1). Functions compose associatively, so a warp scan, a block scan
// and a decoupled look-back across blocks (single pass, CTA order fixed by an atomic
// ticket so every predecessor is resident; one warp inspects 32 predecessors per step)
// give each thread its exact carry in. Every spin in the look-back has an iteration limit
// (kSpinLimit polls, or CrtParams::spin_limit); running out sets an error word the host checks,
// and the kernel finishes without hanging.
//
// One launch can recombine many products (the three outputs of every merge of a
// binary-splitting level); each has its own ticket and status words.
#pragma once
#include <cstdint>

#include "modarith.cuh"
#include "series.cuh"
#include "types.cuh"

namespace pg {

constexpr uint32_t kSpinLimit = 1u << 22;

struct X3 {
    uint32_t w0, w1, w2;
};

__device__ __forceinline__ X3 crt3(uint32_t r0, uint32_t r1, uint32_t r2, const CrtConsts& k, bool centred) {
    const uint32_t p0 = kPrime(0), p1 = kPrime(1), p2 = kPrime(2);
    uint32_t x0 = mul_shoup(r0, k.c00, k.c00p, p0);
    uint32_t y1 = sub_mod(mul_shoup(r1, k.c11, k.c11p, p1), mul_shoup(x0, k.k01, k.k01p, p1), p1);
    uint32_t t1 = mul_shoup(r2, k.c22, k.c22p, p2);
    uint32_t t2 = mul_shoup(x0, k.k02, k.k02p, p2);
    uint32_t t3 = mul_shoup(y1, k.k12, k.k12p, p2);
    uint32_t y2 = sub_mod(sub_mod(t1, t2, p2), t3, p2);
    uint64_t lo = (uint64_t)x0 + (uint64_t)p0 * y1;  // < 2^63
    uint64_t plo = k.p01 * (uint64_t)y2;
    uint64_t phi = __umul64hi(k.p01, (uint64_t)y2);
    uint64_t s = lo + plo;
    phi += (s < lo);
    if (centred) {
        // x > P/2  <=>  Garner digits (y2, y1, x0) > those of floor(P/2), compared lexicographically
        const bool neg = (y2 > k.h2) || (y2 == k.h2 && (y1 > k.h1 || (y1 == k.h1 && x0 > k.h0)));
        if (neg) {  // x - P as a 96-bit two's-complement number
            const uint64_t b0 = s - k.P_lo;
            phi = phi - k.P_hi - (s < k.P_lo ? 1 : 0);
            s = b0;
        }
    }
    X3 r;
    r.w0 = (uint32_t)s;
    r.w1 = (uint32_t)(s >> 32);
    r.w2 = (uint32_t)phi;
    return r;
}

// f packed as (f(-1)+1) | (f(0)+1) << 2 | (f(1)+1) << 4 | (f(2)+1) << 6, indexed by u = carry + 1.
__device__ __forceinline__ uint32_t fapply(uint32_t f, uint32_t u) { return (f >> (2 * u)) & 3u; }
__device__ __forceinline__ uint32_t fcompose(uint32_t g, uint32_t f) {  // g o f (apply f first)
    return fapply(g, fapply(f, 0)) | (fapply(g, fapply(f, 1)) << 2) | (fapply(g, fapply(f, 2)) << 4) |
           (fapply(g, fapply(f, 3)) << 6);
}
constexpr uint32_t kFIdentity = 0u | (1u << 2) | (2u << 4) | (3u << 6);
__device__ __forceinline__ uint32_t fconst(uint32_t u) { return u | (u << 2) | (u << 4) | (u << 6); }

enum : uint32_t { kStNone = 0, kStAgg = 1, kStIncl = 2 };

// Job description resolved per block: where the residues are, where the words go.
struct CrtJob {
    const uint32_t* res;
    uint32_t* out;
    uint64_t nwords;
    uint32_t* len;     // if non-null: receives the product's length in limbs (atomicMax)
    bool centred;
};

__device__ __forceinline__ CrtJob crt_job(const CrtParams& P, uint64_t job) {
    CrtJob J;
    if (P.merge == 2) {
        const DstEntry d = P.dtab[job];
        J.res = P.res + job * P.res_stride;
        J.out = d.out;
        J.nwords = d.nwords;
        J.len = nullptr;
        J.centred = d.centred != 0;
        return J;
    }
    if (!P.merge) {
        J.res = P.res + job * P.res_stride;
        J.out = P.out + job * P.out_stride;
        J.nwords = P.nwords;
        J.len = P.dlen ? P.dlen + job : nullptr;
        J.centred = false;
        return J;
    }
    const uint64_t m = job / 3;
    const int k = (int)(job - 3 * m);  // output: 0 Q^, 1 R^, 2 P^
    const int which = merge_out_value(k);
    J.res = P.res + (6 * m + comb_out_slot(k)) * P.res_stride;
    J.out = reinterpret_cast<uint32_t*>(P.dst[which] + m * P.dcap[which]);
    J.nwords = 2ull * P.dcap[which];
    J.len = P.dlen + 3 * m + which;
    J.centred = false;
    if (which == 2) {
        uint64_t a, b;
        node_range(P.a0, P.b0, P.depth, m, a, b);
        J.centred = merge_r_sign(a, b) < 0;
    }
    return J;
}

// Carry resolution of one block: each thread holds the signed sums W[0..NW) of NW consecutive output
// words (thread order = word order; the block is number `bid` of its job, j0 = this thread's first
// word); the carries between words lie in {-1, 0, 1, 2}. Per-thread carry transfer functions are
// composed by a warp scan, a block scan and the decoupled look-back across blocks; o receives the
// exact words and top the index of this thread's highest non-zero word below nwords (-1: none).
template <int NW, int NT = kCrtThreads>
__device__ __forceinline__ void carry_resolve(const int64_t (&W)[NW], uint32_t (&o)[NW], int& top, uint32_t bid,
                                              uint64_t j0, uint64_t nwords, volatile uint32_t* st, const CrtParams& P,
                                              uint32_t (&s_wagg)[NT / 32], uint32_t& s_carry_in) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t f;
    {
        int64_t acc = 0;
        bool ones_hi = true, zero_hi = true;
        uint32_t low0 = 0;
#pragma unroll
        for (int u = 0; u < NW; ++u) {
            acc += W[u];
            uint32_t o = (uint32_t)acc;
            if (u == 0) {
                low0 = o;
            } else {
                ones_hi &= (o == 0xffffffffu);
                zero_hi &= (o == 0u);
            }
            acc >>= 32;  // arithmetic: floor division by 2^32
        }
        const int c0 = (int)acc;
        const int fm1 = c0 - ((zero_hi && low0 == 0u) ? 1 : 0);
        const int f1 = c0 + ((ones_hi && low0 == 0xffffffffu) ? 1 : 0);
        const int f2 = c0 + ((ones_hi && low0 >= 0xfffffffeu) ? 1 : 0);
        f = (uint32_t)(fm1 + 1) | ((uint32_t)(c0 + 1) << 2) | ((uint32_t)(f1 + 1) << 4) | ((uint32_t)(f2 + 1) << 6);
    }

    // Warp inclusive scan of transfer functions (lane order = word order).
    uint32_t incl = f;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = fcompose(incl, o);
    }
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = kFIdentity;
    if (lane == 31) s_wagg[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        // Exclusive prefix over the block's warps, block aggregate in lane NWARP - 1.
        constexpr int NWARP = NT / 32;
        uint32_t wf = (lane < NWARP) ? s_wagg[lane] : kFIdentity;
        uint32_t wincl = wf;
#pragma unroll
        for (int off = 1; off < NWARP; off <<= 1) {
            uint32_t o = __shfl_up_sync(0xffffffffu, wincl, off);
            if (lane >= off) wincl = fcompose(wincl, o);
        }
        uint32_t wexcl = __shfl_up_sync(0xffffffffu, wincl, 1);
        if (lane == 0) wexcl = kFIdentity;
        const uint32_t blk = __shfl_sync(0xffffffffu, wincl, NWARP - 1);
        __syncwarp();
        if (lane < NWARP) s_wagg[lane] = wexcl;

        // Decoupled look-back, one window of 32 predecessors per step (lane l reads block
        // base - l). The window's functions compose into one; the nearest block that already
        // knows its carry out ends the walk. Carries are stored as u = carry + 1.
        uint32_t u_in = 1;
        const bool publish = bid + 1 != P.withhold1;  // false only under the test hook
        const uint32_t spin_limit = P.spin_limit ? P.spin_limit : kSpinLimit;
        if (bid == 0) {
            if (lane == 0 && publish) st[0] = kStIncl | (fapply(blk, 1) << 8);
        } else {
            if (lane == 0 && publish) {
                __threadfence();
                st[bid] = kStAgg | (blk << 8);
            }
            uint32_t look = kFIdentity;
            int64_t base = (int64_t)bid - 1;
            uint32_t spins = 0;
            while (true) {
                const int64_t jb = base - lane;
                const uint32_t v = (jb >= 0) ? st[jb] : (uint32_t)(kStIncl | (1u << 8));  // before block 0: carry 0
                const uint32_t sv = v & 0xffu;
                const unsigned incl_mask = __ballot_sync(0xffffffffu, sv == kStIncl);
                const unsigned none_mask = __ballot_sync(0xffffffffu, sv == kStNone);
                const int first = incl_mask ? (__ffs(incl_mask) - 1) : 32;
                const unsigned upto = (first >= 31) ? 0xffffffffu : ((2u << first) - 1u);
                if (none_mask & upto) {
                    if (++spins > spin_limit) {
                        if (lane == 0) atomicExch(P.error, 1u);
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                __threadfence();
                const uint32_t pay = (v >> 8) & 0xffu;
                uint32_t g = (lane < first) ? pay : (lane == first ? fconst(pay) : kFIdentity);
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    uint32_t o = __shfl_down_sync(0xffffffffu, g, off);
                    if (lane + off < 32) g = fcompose(g, o);
                }
                g = __shfl_sync(0xffffffffu, g, 0);
                look = fcompose(look, g);
                if (first < 32) {
                    u_in = fapply(look, 1);
                    break;
                }
                base -= 32;
            }
            if (lane == 0 && publish) {
                __threadfence();
                st[bid] = kStIncl | (fapply(blk, u_in) << 8);
            }
        }
        if (lane == 0) {
            s_carry_in = u_in;
            if ((uint64_t)(bid + 1) * NT * NW >= nwords && fapply(blk, u_in) != 1 && !P.top_ok)
                atomicExch(P.error, 2u);  // carry out of the top word: the result does not fit
        }
    }
    __syncthreads();
    const int c = (int)fapply(excl, fapply(s_wagg[warp], s_carry_in)) - 1;

    // Final words.
    top = -1;
    {
        int64_t acc = c;
#pragma unroll
        for (int u = 0; u < NW; ++u) {
            acc += W[u];
            o[u] = (uint32_t)acc;
            if (o[u] != 0 && j0 + u < nwords) top = u;
            acc >>= 32;
        }
    }
}

// Carry transfer function of NW consecutive signed word sums: f packed as above, entry u = carry-in
// + 1 -> carry-out + 1 (carries in {-1, 0, 1, 2}).
template <int NW>
__device__ __forceinline__ uint32_t words_transfer(const int64_t (&W)[NW]) {
    int64_t acc = 0;
    bool ones_hi = true, zero_hi = true;
    uint32_t low0 = 0;
#pragma unroll
    for (int u = 0; u < NW; ++u) {
        acc += W[u];
        const uint32_t o = (uint32_t)acc;
        if (u == 0) {
            low0 = o;
        } else {
            ones_hi &= (o == 0xffffffffu);
            zero_hi &= (o == 0u);
        }
        acc >>= 32;
    }
    const int c0 = (int)acc;
    const int fm1 = c0 - ((zero_hi && low0 == 0u) ? 1 : 0);
    const int f1 = c0 + ((ones_hi && low0 == 0xffffffffu) ? 1 : 0);
    const int f2 = c0 + ((ones_hi && low0 >= 0xfffffffeu) ? 1 : 0);
    return (uint32_t)(fm1 + 1) | ((uint32_t)(c0 + 1) << 2) | ((uint32_t)(f1 + 1) << 4) | ((uint32_t)(f2 + 1) << 6);
}

// Carry resolution inside one block only, with carry-in 0 at the block's first word: o receives
// the words, the return value (valid in every thread) is the block's transfer function. The
// blocks' carries are then joined by crt_fix_kernel (a scan over the block functions and a
// correction of each block's first words), so no block waits for another.
template <int NW, int NT>
__device__ __forceinline__ uint32_t carry_local(const int64_t (&W)[NW], uint32_t (&o)[NW], uint32_t (&s_wagg)[NT / 32],
                                                uint32_t& s_blk) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NWARP = NT / 32;
    const uint32_t f = words_transfer<NW>(W);
    uint32_t incl = f;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = fcompose(incl, x);
    }
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = kFIdentity;
    if (lane == 31) s_wagg[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t wincl = (lane < NWARP) ? s_wagg[lane] : kFIdentity;
#pragma unroll
        for (int off = 1; off < NWARP; off <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, wincl, off);
            if (lane >= off) wincl = fcompose(wincl, x);
        }
        uint32_t wexcl = __shfl_up_sync(0xffffffffu, wincl, 1);
        if (lane == 0) wexcl = kFIdentity;
        const uint32_t blk = __shfl_sync(0xffffffffu, wincl, NWARP - 1);
        __syncwarp();
        if (lane < NWARP) s_wagg[lane] = wexcl;
        if (lane == 0) s_blk = blk;
    }
    __syncthreads();
    int64_t acc = (int)fapply(excl, fapply(s_wagg[warp], 1u)) - 1;
#pragma unroll
    for (int u = 0; u < NW; ++u) {
        acc += W[u];
        o[u] = (uint32_t)acc;
        acc >>= 32;
    }
    return s_blk;
}

__global__ void __launch_bounds__(kCrtThreads, 4) crt_carry_kernel(CrtParams P) {
    __shared__ uint32_t s_tail[kCrtThreads / 32][3];
    __shared__ uint32_t s_wagg[kCrtThreads / 32];
    __shared__ uint32_t s_bid;
    __shared__ uint32_t s_carry_in;

    const uint64_t job = blockIdx.x / P.blocks_per_job;
    const CrtJob J = crt_job(P, job);
    const uint64_t nblocks = (J.nwords + kCrtThreads * kCrtWords - 1) / (kCrtThreads * kCrtWords);
    if (blockIdx.x % P.blocks_per_job >= nblocks) return;  // this job needs fewer blocks
    uint32_t* ticket = P.ticket + job;
    volatile uint32_t* st = P.status + job * P.blocks_per_job;

    if (threadIdx.x == 0) s_bid = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t bid = s_bid;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t j0 = ((uint64_t)bid * kCrtThreads + threadIdx.x) * kCrtWords;

    const uint32_t* r0 = J.res;
    const uint32_t* r1 = J.res + P.L;
    const uint32_t* r2 = J.res + 2 * P.L;
    const bool cen = J.centred;

    uint32_t a0[kCrtWords], a1[kCrtWords], a2[kCrtWords];
    if (j0 + kCrtWords <= P.L) {
#pragma unroll
        for (int u = 0; u < kCrtWords; u += 4) {
            uint4 v0 = *reinterpret_cast<const uint4*>(r0 + j0 + u);
            uint4 v1 = *reinterpret_cast<const uint4*>(r1 + j0 + u);
            uint4 v2 = *reinterpret_cast<const uint4*>(r2 + j0 + u);
            X3 x;
            x = crt3(v0.x, v1.x, v2.x, P.k, cen); a0[u] = x.w0; a1[u] = x.w1; a2[u] = x.w2;
            x = crt3(v0.y, v1.y, v2.y, P.k, cen); a0[u + 1] = x.w0; a1[u + 1] = x.w1; a2[u + 1] = x.w2;
            x = crt3(v0.z, v1.z, v2.z, P.k, cen); a0[u + 2] = x.w0; a1[u + 2] = x.w1; a2[u + 2] = x.w2;
            x = crt3(v0.w, v1.w, v2.w, P.k, cen); a0[u + 3] = x.w0; a1[u + 3] = x.w1; a2[u + 3] = x.w2;
        }
    } else {
#pragma unroll
        for (int u = 0; u < kCrtWords; ++u) {
            uint64_t i = j0 + u;
            if (i < P.L) {
                X3 x = crt3(r0[i], r1[i], r2[i], P.k, cen);
                a0[u] = x.w0; a1[u] = x.w1; a2[u] = x.w2;
            } else {
                a0[u] = a1[u] = a2[u] = 0;
            }
        }
    }

    // Words 1 and 2 of the two coefficients just below j0 (from the previous thread).
    uint32_t pw1 = __shfl_up_sync(0xffffffffu, a1[kCrtWords - 1], 1);
    uint32_t pw2a = __shfl_up_sync(0xffffffffu, a2[kCrtWords - 1], 1);
    uint32_t pw2b = __shfl_up_sync(0xffffffffu, a2[kCrtWords - 2], 1);
    if (lane == 31) {
        s_tail[warp][0] = a1[kCrtWords - 1];
        s_tail[warp][1] = a2[kCrtWords - 1];
        s_tail[warp][2] = a2[kCrtWords - 2];
    }
    __syncthreads();
    if (lane == 0) {
        if (warp > 0) {
            pw1 = s_tail[warp - 1][0];
            pw2a = s_tail[warp - 1][1];
            pw2b = s_tail[warp - 1][2];
        } else if (j0 >= 2) {
            // first thread of the CTA: rebuild the two coefficients below its range
            X3 xm1 = {0, 0, 0}, xm2 = {0, 0, 0};
            if (j0 - 1 < P.L) xm1 = crt3(r0[j0 - 1], r1[j0 - 1], r2[j0 - 1], P.k, cen);
            if (j0 - 2 < P.L) xm2 = crt3(r0[j0 - 2], r1[j0 - 2], r2[j0 - 2], P.k, cen);
            pw1 = xm1.w1; pw2a = xm1.w2; pw2b = xm2.w2;
        } else {
            pw1 = pw2a = pw2b = 0;
        }
    }

    // Raw word sums (signed) and the carry-in-0 pass.
    int64_t W[kCrtWords];
#pragma unroll
    for (int u = 0; u < kCrtWords; ++u) {
        int64_t w = (int64_t)a0[u];
        w += (int64_t)((u >= 1) ? a1[u - 1] : pw1);
        w += (int64_t)(int32_t)((u >= 2) ? a2[u - 2] : (u == 1 ? pw2a : pw2b));
        W[u] = w;
    }
    uint32_t o[kCrtWords];
    int top = -1;
    carry_resolve<kCrtWords>(W, o, top, bid, j0, J.nwords, st, P, s_wagg, s_carry_in);
    if (j0 + kCrtWords <= J.nwords) {
#pragma unroll
        for (int u = 0; u < kCrtWords; u += 4)
            *reinterpret_cast<uint4*>(J.out + j0 + u) = make_uint4(o[u], o[u + 1], o[u + 2], o[u + 3]);
    } else {
#pragma unroll
        for (int u = 0; u < kCrtWords; ++u)
            if (j0 + u < J.nwords) J.out[j0 + u] = o[u];
    }
    if (J.len) {
        // length in limbs = (index of the highest non-zero word) / 2 + 1
        uint32_t lim = top >= 0 ? (uint32_t)((j0 + top) / 2 + 1) : 0u;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lim = max(lim, __shfl_xor_sync(0xffffffffu, lim, off));
        if (lane == 0 && lim) atomicMax(J.len, lim);
    }
}

// ---- The wide configuration: 64-bit coefficients over five primes (modarith.cuh).
// Coefficient i is rebuilt by Garner's method as x = y0 + y1 q0 + y2 q0 q1 + y3 q0 q1 q2 +
// y4 q0 q1 q2 q3 (y_k < q_k), with y_k = r_k c_k - sum_{m<k} y_m k_mk (mod q_k): fifteen Shoup
// products, the inverse transform's 1/L and the pointwise product's 2^-32 folded into c_k. x < 2^154
// sits in five 32-bit words at bit 64 i, so output word 2i receives x_i[0] + x_{i-1}[2] + x_{i-2}[4]
// and word 2i+1 receives x_i[1] + x_{i-1}[3]: at most three words, carries in {0, 1, 2}, resolved by
// the same scan as above.
struct CrtWideConsts {
    uint32_t c[kWidePrimes], cp[kWidePrimes];            // c_k and Shoup companions (mod q_k)
    uint32_t k[kWidePrimes][kWidePrimes], kp[kWidePrimes][kWidePrimes];  // k_mk = P_m / P_k mod q_k, m < k
    uint32_t Pw[kWidePrimes][kWidePrimes - 1];           // words of P_m = q0 ... q_{m-1}
    uint32_t h[kWidePrimes];                             // Garner digits of floor(P_5 / 2)
    uint32_t Pi[kWidePrimes];                            // words of P_5 = q0 ... q4
};

struct X5 {
    uint32_t w[5];
};

// Coefficient x from its five residues; centred: x - P_5 when x > P_5 / 2 (a signed combination of
// products), as a 160-bit two's-complement number (the top word then reads as a negative int32).
__device__ __forceinline__ X5 crt5(const uint32_t (&r)[kWidePrimes], const CrtWideConsts& K, bool centred) {
    uint32_t y[kWidePrimes];
#pragma unroll
    for (int kk = 0; kk < kWidePrimes; ++kk) {
        const uint32_t q = prime_of(kWidePrimes, kk);
        uint32_t acc = mul_shoup(r[kk], K.c[kk], K.cp[kk], q);
#pragma unroll
        for (int m = 0; m < kk; ++m) acc = sub_mod(acc, mul_shoup(y[m], K.k[m][kk], K.kp[m][kk], q), q);
        y[kk] = acc;
    }
    uint64_t col[5] = {y[0], 0, 0, 0, 0};
#pragma unroll
    for (int m = 1; m < kWidePrimes; ++m)
#pragma unroll
        for (int w = 0; w < m; ++w) {
            const uint64_t pr = (uint64_t)y[m] * K.Pw[m][w];
            col[w] += (uint32_t)pr;
            col[w + 1] += pr >> 32;
        }
    X5 x;
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        col[w + 1] += col[w] >> 32;
        x.w[w] = (uint32_t)col[w];
    }
    x.w[4] = (uint32_t)col[4];
    if (centred) {
        // x > P/2 <=> its Garner digits (y4 .. y0) exceed those of floor(P/2), lexicographically
        int cmp = 0;
#pragma unroll
        for (int kk = kWidePrimes - 1; kk >= 0; --kk)
            if (cmp == 0) cmp = y[kk] > K.h[kk] ? 1 : (y[kk] < K.h[kk] ? -1 : 0);
        if (cmp > 0) {
            int64_t br = 0;
#pragma unroll
            for (int w = 0; w < 5; ++w) {
                const int64_t t = (int64_t)x.w[w] - K.Pi[w] + br;
                x.w[w] = (uint32_t)t;
                br = t >> 32;
            }
        }
    }
    return x;
}

constexpr int kWideCoefs = 4;                  // coefficients per thread
constexpr int kWideWords = 2 * kWideCoefs;     // output words per thread

// Products in the wide configuration, any batch form of CrtParams (crt_job): blocks_per_job blocks
// of kWideThreads * kWideWords words per job (grid = jobs * blocks_per_job). Each block computes its
// words with carry-in 0 and stores its carry transfer function in status[block];
// crt_scan_kernel / crt_scan_warp_kernel and crt_apply_kernel then join the blocks of each job.
//
// status[block] = f | (t << 8): f the block's carry transfer function (8 bits), t - 1 the index
// within the block of its highest non-zero word with carry-in 0 (t = 0: none), which bounds where a
// job's final length can lie (crt_len_kernel).
constexpr int kWideThreads = 512;
__global__ void __launch_bounds__(kWideThreads, 2) crt_wide_kernel(CrtParams P, CrtWideConsts K) {
    __shared__ uint32_t s_tail[kWideThreads / 32][4];
    __shared__ uint32_t s_wagg[kWideThreads / 32];
    __shared__ uint32_t s_blk;
    __shared__ uint32_t s_top;
    if (threadIdx.x == 0) s_top = 0;
    const uint64_t bid = blockIdx.x;
    const uint64_t job = bid / P.blocks_per_job;
    const uint64_t blk = bid - job * P.blocks_per_job;
    const CrtJob J = crt_job(P, job);
    const bool cen = J.centred;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t i0 = (blk * kWideThreads + threadIdx.x) * kWideCoefs;  // first coefficient
    const uint64_t j0 = 2 * i0;                                           // first word
    auto coef = [&](uint64_t i) {
        X5 x = {{0, 0, 0, 0, 0}};
        if (i < P.L) {
            uint32_t r[kWidePrimes];
#pragma unroll
            for (int kk = 0; kk < kWidePrimes; ++kk) r[kk] = J.res[(uint64_t)kk * P.L + i];
            x = crt5(r, K, cen);
        }
        return x;
    };
    X5 x[kWideCoefs];
    if (i0 + kWideCoefs <= P.L) {
        uint4 v[kWidePrimes];
#pragma unroll
        for (int kk = 0; kk < kWidePrimes; ++kk) v[kk] = *reinterpret_cast<const uint4*>(J.res + (uint64_t)kk * P.L + i0);
#pragma unroll
        for (int u = 0; u < kWideCoefs; ++u) {
            uint32_t r[kWidePrimes];
#pragma unroll
            for (int kk = 0; kk < kWidePrimes; ++kk) r[kk] = u == 0 ? v[kk].x : u == 1 ? v[kk].y : u == 2 ? v[kk].z : v[kk].w;
            x[u] = crt5(r, K, cen);
        }
    } else {
#pragma unroll
        for (int u = 0; u < kWideCoefs; ++u) x[u] = coef(i0 + u);
    }
    // Words 2..4 of the coefficient just below i0 and word 4 of the one below that.
    uint32_t b2 = __shfl_up_sync(0xffffffffu, x[kWideCoefs - 1].w[2], 1);
    uint32_t b3 = __shfl_up_sync(0xffffffffu, x[kWideCoefs - 1].w[3], 1);
    uint32_t b4 = __shfl_up_sync(0xffffffffu, x[kWideCoefs - 1].w[4], 1);
    uint32_t bb4 = __shfl_up_sync(0xffffffffu, x[kWideCoefs - 2].w[4], 1);
    if (lane == 31) {
        s_tail[warp][0] = x[kWideCoefs - 1].w[2];
        s_tail[warp][1] = x[kWideCoefs - 1].w[3];
        s_tail[warp][2] = x[kWideCoefs - 1].w[4];
        s_tail[warp][3] = x[kWideCoefs - 2].w[4];
    }
    __syncthreads();
    if (lane == 0) {
        if (warp > 0) {
            b2 = s_tail[warp - 1][0];
            b3 = s_tail[warp - 1][1];
            b4 = s_tail[warp - 1][2];
            bb4 = s_tail[warp - 1][3];
        } else if (i0 >= 1) {
            // first thread of the block: rebuild the two coefficients below its range
            const X5 m1 = coef(i0 - 1);
            const X5 m2 = i0 >= 2 ? coef(i0 - 2) : X5{{0, 0, 0, 0, 0}};
            b2 = m1.w[2];
            b3 = m1.w[3];
            b4 = m1.w[4];
            bb4 = m2.w[4];
        } else {
            b2 = b3 = b4 = bb4 = 0;
        }
    }
    int64_t W[kWideWords];
#pragma unroll
    for (int u = 0; u < kWideCoefs; ++u) {
        // word 2 (i0 + u): x_i[0] + x_{i-1}[2] + x_{i-2}[4]; word 2 (i0 + u) + 1: x_i[1] + x_{i-1}[3]
        // (the top word x[4] is signed: below 2^26 for a plain coefficient, negative for a lifted one)
        const uint32_t p2 = u >= 1 ? x[u - 1].w[2] : b2;
        const uint32_t p3 = u >= 1 ? x[u - 1].w[3] : b3;
        const uint32_t p4 = u >= 2 ? x[u - 2].w[4] : (u == 1 ? b4 : bb4);
        W[2 * u] = (int64_t)x[u].w[0] + p2 + (int32_t)p4;
        W[2 * u + 1] = (int64_t)x[u].w[1] + p3;
    }
    uint32_t o[kWideWords];
    const uint32_t fb = carry_local<kWideWords, kWideThreads>(W, o, s_wagg, s_blk);
    uint32_t t = 0;  // 1 + index within the block of this thread's highest non-zero word
#pragma unroll
    for (int u = 0; u < kWideWords; ++u)
        if (o[u] != 0 && j0 + u < J.nwords) t = threadIdx.x * kWideWords + u + 1;
    t = __reduce_max_sync(0xffffffffu, t);
    if (lane == 0 && t) atomicMax(&s_top, t);
    __syncthreads();
    if (threadIdx.x == 0) P.status[bid] = fb | (s_top << 8);
    if (j0 + kWideWords <= J.nwords) {
#pragma unroll
        for (int u = 0; u < kWideWords; u += 4)
            *reinterpret_cast<uint4*>(J.out + j0 + u) = make_uint4(o[u], o[u + 1], o[u + 2], o[u + 3]);
    } else {
#pragma unroll
        for (int u = 0; u < kWideWords; ++u)
            if (j0 + u < J.nwords) J.out[j0 + u] = o[u];
    }
}

// Joins the blocks of crt_wide_kernel per job in two launches.
// crt_scan_kernel (one block of kFixThreads threads per job) / crt_scan_warp_kernel (one warp per
// job, for at most 64 blocks a job): scan the job's block transfer functions (fblk + job * bpj, in
// word order) and overwrite each with its block's carry-in + 1. A carry out of the job's top word
// sets *error = 2 (the result does not fit) unless top_ok (a wrapped product, whose top is dropped).
// crt_apply_kernel: one warp per block adds its carry-in to the block's words, 128 words per step
// (a warp scan of the words' carry transfer functions), and stops as soon as the carry does or at
// the block's end, past which the next block's carry-in accounts for it. A carry that runs through
// a long stretch of all-ones (or, borrowing, all-zero) words therefore costs one step per 128 words
// on one warp, not a serial walk word by word.
constexpr int kFixThreads = 1024;
constexpr uint64_t kFixMaxBlocks = 16384;  // shared-memory staging of one job: 64 KB
constexpr uint64_t kScanWarpMax = 64;      // blocks per job up to which a warp scans a job
__global__ void __launch_bounds__(kFixThreads) crt_scan_kernel(uint32_t* fblk, uint64_t nb, uint32_t* error,
                                                             int top_ok) {
    extern __shared__ uint32_t s_f[];
    __shared__ uint32_t s_w[kFixThreads / 32];
    fblk += (uint64_t)blockIdx.x * nb;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t i = threadIdx.x; i < nb; i += kFixThreads) s_f[i] = fblk[i] & 0xffu;
    __syncthreads();
    const uint64_t per = (nb + kFixThreads - 1) / kFixThreads;  // consecutive blocks per thread
    const uint64_t b0 = (uint64_t)threadIdx.x * per;
    uint32_t tf = kFIdentity;  // this thread's blocks composed
    for (uint64_t i = 0; i < per; ++i)
        if (b0 + i < nb) tf = fcompose(s_f[b0 + i], tf);
    uint32_t incl = tf;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = fcompose(incl, x);
    }
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = kFIdentity;
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t wi = s_w[lane];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi = fcompose(wi, x);
        }
        uint32_t we = __shfl_up_sync(0xffffffffu, wi, 1);
        if (lane == 0) we = kFIdentity;
        __syncwarp();
        s_w[lane] = we;
    }
    __syncthreads();
    uint32_t u = fapply(excl, fapply(s_w[warp], 1u));  // carry-in + 1 of this thread's first block
    for (uint64_t i = 0; i < per && b0 + i < nb; ++i) {
        fblk[b0 + i] = (fblk[b0 + i] & ~0xffu) | u;
        u = fapply(s_f[b0 + i], u);
    }
    if (!top_ok && b0 < nb && b0 + per >= nb && u != 1) atomicExch(error, 2u);  // the last block's carry out
}

__global__ void __launch_bounds__(256) crt_scan_warp_kernel(uint32_t* fblk, uint64_t nb, uint64_t njobs,
                                                          uint32_t* error, int top_ok) {
    const uint64_t job = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (job >= njobs) return;
    fblk += job * nb;
    const uint64_t per = (nb + 31) / 32;  // at most 2
    const uint64_t b0 = (uint64_t)lane * per;
    uint32_t f[2] = {kFIdentity, kFIdentity}, hi[2] = {0, 0};
    uint32_t tf = kFIdentity;
#pragma unroll
    for (int i = 0; i < 2; ++i)
        if (i < (int)per && b0 + i < nb) {
            const uint32_t st = fblk[b0 + i];
            f[i] = st & 0xffu;
            hi[i] = st & ~0xffu;
            tf = fcompose(f[i], tf);
        }
    uint32_t incl = tf;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = fcompose(incl, x);
    }
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = kFIdentity;
    uint32_t u = fapply(excl, 1u);
#pragma unroll
    for (int i = 0; i < 2; ++i)
        if (i < (int)per && b0 + i < nb) {
            fblk[b0 + i] = hi[i] | u;
            u = fapply(f[i], u);
        }
    if (!top_ok && b0 < nb && b0 + per >= nb && u != 1) atomicExch(error, 2u);
}

constexpr int kApplyWarps = 8;
__global__ void __launch_bounds__(32 * kApplyWarps) crt_apply_kernel(CrtParams P, uint64_t nblocks,
                                                                  uint64_t block_words) {
    const int lane = threadIdx.x & 31;
    const uint64_t wb = (uint64_t)blockIdx.x * kApplyWarps + (threadIdx.x >> 5);  // block over all jobs
    if (wb >= nblocks) return;
    uint32_t u = P.status[wb] & 0xffu;  // carry + 1 entering the block's first word
    if (u == 1) return;
    const uint64_t job = wb / P.blocks_per_job;
    const uint64_t b = wb - job * P.blocks_per_job;
    const CrtJob J = crt_job(P, job);
    uint32_t* out = J.out;
    const uint64_t end = min((b + 1) * block_words, J.nwords);
    for (uint64_t j0 = b * block_words; j0 < end && u != 1; j0 += 128) {
        const uint64_t j = j0 + 4 * (uint64_t)lane;
        int64_t W[4];
        const bool whole = j + 4 <= end;
        if (whole) {
            const uint4 v = *reinterpret_cast<const uint4*>(out + j);
            W[0] = v.x; W[1] = v.y; W[2] = v.z; W[3] = v.w;
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) W[q] = j + q < end ? out[j + q] : 0;
        }
        // words past the end transfer carries unchanged: identity
        const uint32_t f = j < end ? words_transfer<4>(W) : kFIdentity;
        uint32_t incl = f;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl = fcompose(incl, x);
        }
        uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) excl = kFIdentity;
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t my = fapply(excl, u);  // carry + 1 entering this lane's first word
        if (my != 1 && j < end) {
            int64_t acc = (int)my - 1;
            uint32_t o[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                acc += W[q];
                o[q] = (uint32_t)acc;
                acc >>= 32;
            }
            if (whole) {
                *reinterpret_cast<uint4*>(out + j) = make_uint4(o[0], o[1], o[2], o[3]);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (j + q < end) out[j + q] = o[q];
            }
        }
        u = fapply(total, u);
    }
}

// Lengths in limbs of the jobs' final words (jobs with a length slot), one warp per job. The job's
// highest non-zero word lies in its highest block b with a non-zero word at carry-in 0 or a non-zero
// carry-in: a carry-in adds at most one word above the block's own top (the words above it are zero,
// so a carry stops there), and a block whose final words were all zero would pass a carry to the
// block above. So the warp finds b from the status words (scanning down 32 blocks a step), then
// scans b's final words down from just above its own top.
__global__ void __launch_bounds__(256) crt_len_kernel(CrtParams P, uint64_t njobs, uint64_t block_words) {
    const uint64_t job = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (job >= njobs) return;
    const CrtJob J = crt_job(P, job);
    if (!J.len) return;
    const uint32_t* st = P.status + job * P.blocks_per_job;
    const uint64_t nb = min(P.blocks_per_job, (J.nwords + block_words - 1) / block_words);
    uint64_t b = ~0ull;
    uint32_t sb = 0;
    for (uint64_t top = nb; top > 0; top = top > 32 ? top - 32 : 0) {
        const uint64_t i = top - 1 - lane;
        const uint32_t v = top > (uint64_t)lane ? st[i] : 0x1u;  // carry-in 0, no words
        const uint32_t m = __ballot_sync(0xffffffffu, (v >> 8) != 0 || (v & 0xffu) != 1);
        if (m) {
            const int l = __ffs(m) - 1;
            b = top - 1 - (uint64_t)l;
            sb = __shfl_sync(0xffffffffu, v, l);
            break;
        }
    }
    uint32_t len = 0;
    if (b != ~0ull) {
        const uint64_t start = b * block_words;
        const uint64_t end = min(min(start + (uint64_t)(sb >> 8) + 1, (b + 1) * block_words), J.nwords);
        for (uint64_t top = end; top > start; top = top - start > 32 ? top - 32 : start) {
            const uint64_t i = top - 1 - lane;
            const bool nz = top - start > (uint64_t)lane && J.out[i] != 0;
            const uint32_t m = __ballot_sync(0xffffffffu, nz);
            if (m) {
                len = (uint32_t)((top - 1 - (uint64_t)(__ffs(m) - 1)) / 2 + 1);
                break;
            }
        }
    }
    if (lane == 0) *J.len = len;
}

// Short jobs (at most 32 * kCrtWords output words): one warp per job, no look-back. The same
// arithmetic as crt_carry_kernel: Garner lift, word sums, per-lane carry transfer functions, a
// warp scan; the job's final carry must be zero.
constexpr uint64_t kCrtWarpWords = 32 * kCrtWords;

__global__ void __launch_bounds__(256) crt_warp_kernel(CrtParams P, uint64_t njobs) {
    const uint64_t job = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (job >= njobs) return;
    const CrtJob J = crt_job(P, job);
    const uint64_t j0 = (uint64_t)lane * kCrtWords;
    const uint32_t* r0 = J.res;
    const uint32_t* r1 = J.res + P.L;
    const uint32_t* r2 = J.res + 2 * P.L;
    const bool cen = J.centred;
    uint32_t a0[kCrtWords], a1[kCrtWords], a2[kCrtWords];
#pragma unroll
    for (int u = 0; u < kCrtWords; ++u) {
        const uint64_t i = j0 + u;
        if (i < P.L) {
            const X3 x = crt3(r0[i], r1[i], r2[i], P.k, cen);
            a0[u] = x.w0;
            a1[u] = x.w1;
            a2[u] = x.w2;
        } else {
            a0[u] = a1[u] = a2[u] = 0;
        }
    }
    uint32_t pw1 = __shfl_up_sync(0xffffffffu, a1[kCrtWords - 1], 1);
    uint32_t pw2a = __shfl_up_sync(0xffffffffu, a2[kCrtWords - 1], 1);
    uint32_t pw2b = __shfl_up_sync(0xffffffffu, a2[kCrtWords - 2], 1);
    if (lane == 0) pw1 = pw2a = pw2b = 0;
    int64_t W[kCrtWords];
#pragma unroll
    for (int u = 0; u < kCrtWords; ++u) {
        int64_t w = (int64_t)a0[u];
        w += (int64_t)((u >= 1) ? a1[u - 1] : pw1);
        w += (int64_t)(int32_t)((u >= 2) ? a2[u - 2] : (u == 1 ? pw2a : pw2b));
        W[u] = w;
    }
    uint32_t f;
    {
        int64_t acc = 0;
        bool ones_hi = true, zero_hi = true;
        uint32_t low0 = 0;
#pragma unroll
        for (int u = 0; u < kCrtWords; ++u) {
            acc += W[u];
            const uint32_t o = (uint32_t)acc;
            if (u == 0) {
                low0 = o;
            } else {
                ones_hi &= (o == 0xffffffffu);
                zero_hi &= (o == 0u);
            }
            acc >>= 32;
        }
        const int c0 = (int)acc;
        const int fm1 = c0 - ((zero_hi && low0 == 0u) ? 1 : 0);
        const int f1 = c0 + ((ones_hi && low0 == 0xffffffffu) ? 1 : 0);
        const int f2 = c0 + ((ones_hi && low0 >= 0xfffffffeu) ? 1 : 0);
        f = (uint32_t)(fm1 + 1) | ((uint32_t)(c0 + 1) << 2) | ((uint32_t)(f1 + 1) << 4) | ((uint32_t)(f2 + 1) << 6);
    }
    uint32_t incl = f;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = fcompose(incl, o);
    }
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = kFIdentity;
    const int c = (int)fapply(excl, 1u) - 1;  // carry into this lane's words (job carry-in 0)
    uint32_t o[kCrtWords];
    int top = -1;
    bool spill = false;  // a non-zero word past the job's end
    {
        int64_t acc = c;
#pragma unroll
        for (int u = 0; u < kCrtWords; ++u) {
            acc += W[u];
            o[u] = (uint32_t)acc;
            if (o[u] != 0) {
                if (j0 + u < J.nwords)
                    top = u;
                else
                    spill = true;
            }
            acc >>= 32;
        }
    }
    if (j0 + kCrtWords <= J.nwords) {
#pragma unroll
        for (int u = 0; u < kCrtWords; u += 4)
            *reinterpret_cast<uint4*>(J.out + j0 + u) = make_uint4(o[u], o[u + 1], o[u + 2], o[u + 3]);
    } else {
#pragma unroll
        for (int u = 0; u < kCrtWords; ++u)
            if (j0 + u < J.nwords) J.out[j0 + u] = o[u];
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const bool bad = !P.top_ok && (__any_sync(0xffffffffu, spill) || fapply(total, 1u) != 1u);
    if (lane == 0 && bad) atomicExch(P.error, 2u);  // the result does not fit its words
    if (J.len) {
        uint32_t lim = top >= 0 ? (uint32_t)((j0 + top) / 2 + 1) : 0u;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lim = max(lim, __shfl_xor_sync(0xffffffffu, lim, off));
        if (lane == 0 && lim) atomicMax(J.len, lim);
    }
}

}  // namespace pg
