// Modular arithmetic on the 32-bit integer pipes for the three NTT primes.
//
// Primes (all < 2^31, so a + b of two residues never overflows 32 bits):
//   p0 = 2013265921 = 15 * 2^27 + 1   generator 31
//   p1 = 1811939329 = 27 * 2^26 + 1   generator 13
//   p2 =  469762049 =  7 * 2^26 + 1   generator 3
// Every prime has a primitive 2^26-th root of unity, so transforms up to
// L = 2^26 points exist for all three. p0*p1*p2 ~ 2^90.47.
//
// Exactness bound (checked per product on the host, see plan.h): with w-bit
// coefficients, the largest cyclic-convolution coefficient of an na x nb
// product is min(ca, cb) * (2^w - 1)^2 (ca, cb = coefficient counts), and a
// sum of `terms` such products stays below terms * that. It must be < p0*p1*p2
// for the CRT to recover it; with w = 32 and L <= 2^26 that always holds for
// terms <= 2.
//
// Two multiplication forms are used:
//   * Shoup: x * w mod p for a constant w with companion w' = floor(w * 2^32 / p).
//     q = mulhi(x, w'); r = x*w - q*p lies in [0, 2p) for any 32-bit x.
//     Used for every twiddle and every CRT constant (3 IMAD + 2 ALU).
//   * Montgomery (R = 2^32): a * b * 2^-32 mod p for two variables. Used once
//     per element for the pointwise product; the stray 2^-32 is folded into
//     the CRT scale constants.
#pragma once
#include <cstdint>

namespace pg {

constexpr int kNumPrimes = 3;
constexpr int kMaxLogL = 26;

struct PrimeConst {
    uint32_t p;
    uint32_t pinv;   // p^-1 mod 2^32 (Montgomery)
};

__host__ __device__ constexpr uint32_t kPrime(int j) {
    return j == 0 ? 2013265921u : (j == 1 ? 1811939329u : 469762049u);
}
__host__ __device__ constexpr uint32_t kGenerator(int j) {
    return j == 0 ? 31u : (j == 1 ? 13u : 3u);
}

// p^-1 mod 2^32 by Newton iteration (x <- x * (2 - p*x)), exact after 5 steps from x = p.
__host__ __device__ constexpr uint32_t inv_mod_2_32(uint32_t p) {
    uint32_t x = p;
    x *= 2u - p * x;
    x *= 2u - p * x;
    x *= 2u - p * x;
    x *= 2u - p * x;
    x *= 2u - p * x;
    return x;
}

__device__ __forceinline__ uint32_t reduce_once(uint32_t x, uint32_t p) {
    // x in [0, 2p) -> [0, p). Unsigned min: if x < p then x - p wraps above x.
    return min(x, x - p);
}

__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
    return reduce_once(a + b, p);
}

__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
    return reduce_once(a - b + p, p);
}

// x * w mod p, result in [0, p); x any 32-bit value, w < p with companion wp.
__device__ __forceinline__ uint32_t mul_shoup(uint32_t x, uint32_t w, uint32_t wp, uint32_t p) {
    uint32_t q = __umulhi(x, wp);
    uint32_t r = x * w - q * p;
    return reduce_once(r, p);
}

// x * w mod p, result in [0, 2p) (lazy).
__device__ __forceinline__ uint32_t mul_shoup_lazy(uint32_t x, uint32_t w, uint32_t wp, uint32_t p) {
    uint32_t q = __umulhi(x, wp);
    return x * w - q * p;
}

// floor((2^64 - 1) / p), used to form Shoup companions on the device without a division.
__host__ __device__ constexpr uint64_t kRecip64(int j) { return ~0ull / kPrime(j); }

// Shoup companion floor(w * 2^32 / p) of w < p. With R = floor(2^64 / p) = 2^64/p - d
// (0 <= d < 1), floor(w * R / 2^32) undershoots floor(w * 2^32 / p) by at most one because
// w * d / 2^32 < 1/2; the remainder w * 2^32 - q * p (in [0, 2p), exact modulo 2^32)
// says which.
__device__ __forceinline__ uint32_t shoup_companion_dev(uint32_t w, uint32_t p, uint64_t R) {
    const uint32_t q = w * (uint32_t)(R >> 32) + __umulhi(w, (uint32_t)R);
    const uint32_t r = 0u - q * p;
    return r >= p ? q + 1 : q;
}

// a * b * 2^-32 mod p for a, b < p; result in [0, p).
__device__ __forceinline__ uint32_t mul_mont(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    uint32_t lo = a * b;
    uint32_t hi = __umulhi(a, b);
    uint32_t m = lo * pinv;
    uint32_t t = __umulhi(m, p);
    uint32_t r = hi - t;   // in (-p, p); m*p has the same low word as a*b
    return min(r, r + p);
}

// x mod p for any 32-bit x (reduces with a Shoup multiply by one).
__device__ __forceinline__ uint32_t reduce_u32(uint32_t x, uint32_t p, uint32_t one_p) {
    uint32_t q = __umulhi(x, one_p);
    return reduce_once(x - q * p, p);
}

}  // namespace pg
