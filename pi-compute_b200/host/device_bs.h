// DeviceBinarySplitting: the level-batched, device-resident binary splitting (pg_bs in
// include/pi_b200.h) with mpz_t results, for the pi engine's batched mode. Computes the
// same P, Q, R as BinarySplitting (binary_splitting.h) and the reference's
// BinarySplitting::compute (src/engine/binary_splitting.cpp:605-644).
#pragma once

#include "gmp.h"
#include "pi_b200.h"

namespace pi {

class DeviceBinarySplitting {
public:
    explicit DeviceBinarySplitting(int device = 0);
    // Use an existing context (not destroyed here).
    explicit DeviceBinarySplitting(pg_ctx* shared);
    ~DeviceBinarySplitting();
    DeviceBinarySplitting(const DeviceBinarySplitting&) = delete;
    DeviceBinarySplitting& operator=(const DeviceBinarySplitting&) = delete;

    // P may be nullptr when it is not needed (the root of a pi computation).
    void compute(unsigned long a, unsigned long b, mpz_ptr P, mpz_ptr Q, mpz_ptr R);
    uint64_t launches() const { return pg_launch_count(ctx_); }

private:
    pg_ctx* ctx_ = nullptr;
    bool owned_ = true;
};

}  // namespace pi
