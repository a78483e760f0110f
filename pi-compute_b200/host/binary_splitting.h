// Chudnovsky binary splitting over a pi::Multiplier (per-call form).
//
// Same series, same leaves and the same tree shape as the reference's BinarySplitting
// (src/engine/binary_splitting.h:22-102, .cpp:100-102, 137-159, 161-293, 295-348): the range
// [a, b) splits at m = a + (b - a) / 2 down to single terms, so every P/Q/R and every digit
// matches the reference exactly. Each merge issues its four products through the Multiplier,
// one call at a time or from up to four host threads (the reference's tier-2 merge); that is
// the per-call drop-in form. The level-batched device form lives in device_bs.h.
#pragma once

#include <cstddef>

#include "multiplier.h"

namespace pi {

struct BSResult {
    mpz_t P, Q, R;
    BSResult();
    ~BSResult();
    BSResult(const BSResult&) = delete;
    BSResult& operator=(const BSResult&) = delete;
    BSResult(BSResult&& o) noexcept;
    BSResult& operator=(BSResult&& o) noexcept;
};

class BinarySplitting {
public:
    // num_threads: host threads issuing products concurrently (1 = sequential).
    explicit BinarySplitting(Multiplier& multiplier, unsigned int num_threads = 1);

    BSResult compute(unsigned long a, unsigned long b);

    // ceil(digits / 14.1816474627) + 1 (binary_splitting.cpp:100-102).
    static unsigned long terms_needed(size_t digits);
    // Leaf values for term a (binary_splitting.cpp:137-159).
    static void leaf(unsigned long a, mpz_t P, mpz_t Q, mpz_t R);

private:
    BSResult rec(unsigned long a, unsigned long b, int depth);
    BSResult merge(BSResult& l, BSResult& r, bool concurrent);
    Multiplier& mult_;
    unsigned int threads_;
};

}  // namespace pi
