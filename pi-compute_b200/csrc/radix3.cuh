// Transforms of 3 * 2^m points in the wide configuration (five primes, each with 3 * 2^25 | q - 1):
// one radix-3 step across the three thirds of the operand, then the 2^m-point passes on the three
// rows as three jobs (the four-step split L = 3 x 2^m):
//   forward: y_r[i] = W_L^(i r) * sum_{j<3} x[i + M j] w3^(j r)   (r = 0, 1, 2; M = 2^m; L = 3M),
//            the rows y_r then transformed by the 2^m-point forward passes;
//   inverse: the 2^m-point inverse passes, then z_r[i] = W_L^(-i r) y_r[i] and
//            x[i + M j] = sum_r z_r[i] w3^(-j r) (the 1/L is folded into the CRT constants).
// W_L = W^(2^(25 - m)) for W of order 3 * 2^25, its powers as products of two table entries
// (t3_lo, t3_hi); the radix-3 butterfly uses w3 + w3^2 = -1: with s = x1 + x2, d = x1 - x2,
// y1 = x0 - s/2 + c d and y2 = x0 - s/2 - c d, c = (w3 - w3^2) / 2 (two Shoup products).
#pragma once
#include <cstdint>

#include "modarith.cuh"
#include "types.cuh"

namespace pg {

constexpr int kR3Threads = 256;  // 4 points per thread

__device__ __forceinline__ uint32_t r3_twiddle(uint32_t y, uint32_t e, const uint2* lo, const uint2* hi, uint32_t p) {
    const uint2 a = __ldg(lo + (e & ((1u << kFsLog) - 1)));
    const uint2 b = __ldg(hi + (e >> kFsLog));
    return mul_shoup(mul_shoup(y, a.x, a.y, p), b.x, b.y, p);
}

// Forward step from the operand's 64-bit limbs (ncoef of them; zeros beyond): rows r at
// out + r * job_stride + prime * M. Grid: (M / (4 kR3Threads)) * NP blocks, a tile's primes adjacent.
template <int NP>
__global__ void __launch_bounds__(kR3Threads) radix3_fwd_kernel(const uint32_t* words, uint64_t ncoef, uint32_t* out,
                                                             uint64_t M, int logM, uint64_t job_stride, TwiddleTables T) {
    const uint32_t chunk = blockIdx.x / NP;
    const int k = (int)(blockIdx.x - chunk * NP);
    const uint64_t i0 = ((uint64_t)chunk * kR3Threads + threadIdx.x) * 4;
    if (i0 >= M) return;
    const uint32_t p = prime_of(NP, k);
    const uint32_t one_p = (uint32_t)(0x100000000ull / p);
    const uint32_t r32 = 0u - one_p * p;  // 2^32 mod p
    const uint32_t r32p = shoup_companion_dev(r32, p, recip64_of(NP, k));
    uint32_t x[3][4];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const uint64_t n0 = i0 + (uint64_t)j * M;
        uint32_t w[8];
        if (n0 + 4 <= ncoef) {
            const uint4 v0 = __ldg(reinterpret_cast<const uint4*>(words + 2 * n0));
            const uint4 v1 = __ldg(reinterpret_cast<const uint4*>(words + 2 * n0 + 4));
            w[0] = v0.x; w[1] = v0.y; w[2] = v0.z; w[3] = v0.w;
            w[4] = v1.x; w[5] = v1.y; w[6] = v1.z; w[7] = v1.w;
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool in = n0 + u < ncoef;
                w[2 * u] = in ? __ldg(words + 2 * (n0 + u)) : 0u;
                w[2 * u + 1] = in ? __ldg(words + 2 * (n0 + u) + 1) : 0u;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            x[j][u] = add_mod(reduce_u32(w[2 * u], p, one_p), mul_shoup(w[2 * u + 1], r32, r32p, p), p);
    }
    const uint2 h = T.t3_h[k], c = T.t3_c[0][k];
    const uint2* lo = T.t3_lo[0][k];
    const uint2* hi = T.t3_hi[0][k];
    const int sh = kWideMaxLogL - logM;
    uint32_t y[3][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const uint32_t s = add_mod(x[1][u], x[2][u], p), d = sub_mod(x[1][u], x[2][u], p);
        y[0][u] = add_mod(x[0][u], s, p);
        const uint32_t half_s = mul_shoup(s, h.x, h.y, p);
        const uint32_t a = sub_mod(x[0][u], half_s, p);
        const uint32_t v = mul_shoup(d, c.x, c.y, p);
        const uint32_t e1 = (uint32_t)(i0 + u) << sh;  // W_L^(i) = W^(i 2^(25-m)), < 2^25
        y[1][u] = r3_twiddle(add_mod(a, v, p), e1, lo, hi, p);
        y[2][u] = r3_twiddle(sub_mod(a, v, p), e1 << 1, lo, hi, p);
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
        *reinterpret_cast<uint4*>(out + (uint64_t)r * job_stride + (uint64_t)k * M + i0) =
            make_uint4(y[r][0], y[r][1], y[r][2], y[r][3]);
}

// Inverse step: rows r at in + r * job_stride + prime * M (natural order, after the 2^m-point inverse
// passes) -> coefficients at out + prime * 3M + i + M j.
template <int NP>
__global__ void __launch_bounds__(kR3Threads) radix3_inv_kernel(const uint32_t* in, uint32_t* out, uint64_t M,
                                                             int logM, uint64_t job_stride, TwiddleTables T) {
    const uint32_t chunk = blockIdx.x / NP;
    const int k = (int)(blockIdx.x - chunk * NP);
    const uint64_t i0 = ((uint64_t)chunk * kR3Threads + threadIdx.x) * 4;
    if (i0 >= M) return;
    const uint32_t p = prime_of(NP, k);
    const uint2 h = T.t3_h[k], c = T.t3_c[1][k];
    const uint2* lo = T.t3_lo[1][k];
    const uint2* hi = T.t3_hi[1][k];
    const int sh = kWideMaxLogL - logM;
    uint4 z[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        z[r] = *reinterpret_cast<const uint4*>(in + (uint64_t)r * job_stride + (uint64_t)k * M + i0);
    uint32_t x[3][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const uint32_t e1 = (uint32_t)(i0 + u) << sh;
        const uint32_t z0 = u == 0 ? z[0].x : u == 1 ? z[0].y : u == 2 ? z[0].z : z[0].w;
        const uint32_t z1 = r3_twiddle(u == 0 ? z[1].x : u == 1 ? z[1].y : u == 2 ? z[1].z : z[1].w, e1, lo, hi, p);
        const uint32_t z2 =
            r3_twiddle(u == 0 ? z[2].x : u == 1 ? z[2].y : u == 2 ? z[2].z : z[2].w, e1 << 1, lo, hi, p);
        const uint32_t s = add_mod(z1, z2, p), d = sub_mod(z1, z2, p);
        x[0][u] = add_mod(z0, s, p);
        const uint32_t a = sub_mod(z0, mul_shoup(s, h.x, h.y, p), p);
        const uint32_t v = mul_shoup(d, c.x, c.y, p);
        x[1][u] = add_mod(a, v, p);
        x[2][u] = sub_mod(a, v, p);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j)
        *reinterpret_cast<uint4*>(out + (uint64_t)k * 3 * M + (uint64_t)j * M + i0) =
            make_uint4(x[j][0], x[j][1], x[j][2], x[j][3]);
}

}  // namespace pg
