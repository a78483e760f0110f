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
    const int which = (int)(job % 3);
    J.res = P.res + (6 * m + comb_out_slot(which)) * P.res_stride;
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
    uint32_t f;
    {
        int64_t acc = 0;
        bool ones_hi = true, zero_hi = true;
        uint32_t low0 = 0;
#pragma unroll
        for (int u = 0; u < kCrtWords; ++u) {
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
        // Exclusive prefix over the block's warps (lanes 0..7), block aggregate in lane 7.
        constexpr int NW = kCrtThreads / 32;
        uint32_t wf = (lane < NW) ? s_wagg[lane] : kFIdentity;
        uint32_t wincl = wf;
#pragma unroll
        for (int off = 1; off < NW; off <<= 1) {
            uint32_t o = __shfl_up_sync(0xffffffffu, wincl, off);
            if (lane >= off) wincl = fcompose(wincl, o);
        }
        uint32_t wexcl = __shfl_up_sync(0xffffffffu, wincl, 1);
        if (lane == 0) wexcl = kFIdentity;
        const uint32_t blk = __shfl_sync(0xffffffffu, wincl, NW - 1);
        __syncwarp();
        if (lane < NW) s_wagg[lane] = wexcl;

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
            if ((uint64_t)(bid + 1) * kCrtThreads * kCrtWords >= J.nwords && fapply(blk, u_in) != 1)
                atomicExch(P.error, 2u);  // carry out of the top word: the result does not fit
        }
    }
    __syncthreads();
    const int c = (int)fapply(excl, fapply(s_wagg[warp], s_carry_in)) - 1;

    // Final words.
    uint32_t o[kCrtWords];
    int top = -1;
    {
        int64_t acc = c;
#pragma unroll
        for (int u = 0; u < kCrtWords; ++u) {
            acc += W[u];
            o[u] = (uint32_t)acc;
            if (o[u] != 0 && j0 + u < J.nwords) top = u;
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
    if (J.len) {
        // length in limbs = (index of the highest non-zero word) / 2 + 1
        uint32_t lim = top >= 0 ? (uint32_t)((j0 + top) / 2 + 1) : 0u;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lim = max(lim, __shfl_xor_sync(0xffffffffu, lim, off));
        if (lane == 0 && lim) atomicMax(J.len, lim);
    }
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
    const bool bad = __any_sync(0xffffffffu, spill) || fapply(total, 1u) != 1u;
    if (lane == 0 && bad) atomicExch(P.error, 2u);  // the result does not fit its words
    if (J.len) {
        uint32_t lim = top >= 0 ? (uint32_t)((j0 + top) / 2 + 1) : 0u;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lim = max(lim, __shfl_xor_sync(0xffffffffu, lim, off));
        if (lane == 0 && lim) atomicMax(J.len, lim);
    }
}

}  // namespace pg
