// Integer Newton iterations on Multiplier products: reciprocal, scaled square root, the pi
// final formula and divide-and-conquer binary-to-decimal conversion.
//
// Replace, for the pi pipeline, the reference's GMP floating-point finish and its radix
// conversion:
//   NewtonDivider::sqrt_to_precision / divide (src/arithmetic/newton_divider.cpp:13-39):
//     mpf_sqrt / mpf_div at digits*3.3219281+64 bits;
//   PiEngine::compute final step (src/engine/pi_engine.cpp:437-491): pi = 426880 Q sqrt(10005) / R,
//     times 10^digits, truncated by mpz_set_f;
//   BaseConverter::parallel_to_decimal (src/io/base_converter.cpp:48-147, 201-246): a power tree
//     10^(2^k) and mpz_tdiv_qr splits down to mpz_get_str leaves.
// Here every large product goes through a pi::Multiplier (the B200 for large operands), precision
// doubles from one Newton step to the next with each step's products sized to it, and there is
// no floating-point arithmetic: every quotient, root and digit is corrected to its exact integer
// value, so the digits equal the reference's.
#pragma once

#include <cstddef>
#include <string>

#include "multiplier.h"

namespace pi {

// Z = floor(2^(2k) / R), k = bit length of R (R > 0). Exact.
void recip_floor(mpz_t Z, const mpz_t R, Multiplier& mul);

// S = floor(sqrt(a) * 2^s). Exact.
void sqrt_scaled(mpz_t S, unsigned long a, size_t s, Multiplier& mul);

// pi_int = floor(426880 * Q * sqrt(10005) * 10^digits / R) (Chudnovsky with Q = Q(0,N),
// R = R(0,N) of binary splitting). Exact: the result is accepted only when the computed
// fraction is provably away from an integer, otherwise precision grows and it retries.
void final_formula_newton(mpz_t pi_int, const mpz_t Q, const mpz_t R, size_t digits, Multiplier& mul);

// Decimal digits of x >= 0, left-padded with '0' to exactly `ndigits` characters (x < 10^ndigits).
// Divide-and-conquer over 10^(2^j) with exact quotients from verified reciprocals; subtrees
// below `leaf_digits` run on `threads` host threads with mpz_get_str.
std::string to_decimal(const mpz_t x, size_t ndigits, Multiplier& mul, unsigned threads = 0,
                       size_t leaf_digits = 200000);

}  // namespace pi
