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

// The wide configuration: 64-bit coefficients (one per limb, no repacking) over five primes,
//   q0 = 2113929217 = 63 * 2^25 + 1   generator 5
//   q1 = 2013265921 = 15 * 2^27 + 1   generator 31
//   q2 = 1811939329 = 27 * 2^26 + 1   generator 13
//   q3 = 1711276033 = 51 * 2^25 + 1   generator 29
//   q4 = 1107296257 = 33 * 2^25 + 1   generator 10
// all < 2^31, each with a primitive 2^25-th root of unity; q0 q1 q2 q3 q4 ~ 2^153.36. A product of
// na x nb limbs has na + nb - 1 coefficients (half as many as with 32-bit coefficients) and its
// largest coefficient min(na, nb) (2^64 - 1)^2 stays below the modulus for min(na, nb) < 2^25.35,
// i.e. for every product of up to 2^25 limbs. Five transforms of L points against three of 2L:
// 5/6 of the residue work per product bit.
constexpr int kWidePrimes = 5;
constexpr int kWideMaxLogL = 25;
constexpr int kMaxPrimes = 5;

// Primes and generators of a configuration with NP primes (3: 32-bit coefficients, 5: wide).
__host__ __device__ constexpr uint32_t prime_of(int np, int j) {
    return np == 5 ? (j == 0 ? 2113929217u : j == 1 ? 2013265921u : j == 2 ? 1811939329u : j == 3 ? 1711276033u
                                                                                                   : 1107296257u)
                   : (j == 0 ? 2013265921u : (j == 1 ? 1811939329u : 469762049u));
}
__host__ __device__ constexpr uint32_t generator_of(int np, int j) {
    return np == 5 ? (j == 0 ? 5u : j == 1 ? 31u : j == 2 ? 13u : j == 3 ? 29u : 10u) : (j == 0 ? 31u : (j == 1 ? 13u : 3u));
}
// log2 of the longest transform (the 2-power order of the common roots of unity).
__host__ __device__ constexpr int root_log_of(int np) { return np == 5 ? kWideMaxLogL : kMaxLogL; }

struct PrimeConst {
    uint32_t p;
    uint32_t pinv;   // p^-1 mod 2^32 (Montgomery)
};

__host__ __device__ constexpr uint32_t kPrime(int j) { return prime_of(3, j); }
__host__ __device__ constexpr uint32_t kGenerator(int j) { return generator_of(3, j); }

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
__host__ __device__ constexpr uint64_t recip64_of(int np, int j) { return ~0ull / prime_of(np, j); }

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
