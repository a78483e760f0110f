// The multiply strategy interface, declared exactly as the reference declares it
// (src/arithmetic/multiplier.h:16-41) so that implementations are interchangeable with
// the reference's GmpMultiplier / GpuNttMultiplier / IntNttMultiplier: same namespace,
// class name, virtual signatures and default square().
#pragma once

#include <memory>

#include "gmp.h"

namespace pi {

class Multiplier {
public:
    virtual ~Multiplier() = default;

    // result = a * b; result must be initialised; result may alias a or b.
    virtual void multiply(mpz_t result, const mpz_t a, const mpz_t b) = 0;

    // result = a * a; the default forwards to multiply(result, a, a).
    virtual void square(mpz_t result, const mpz_t a) { multiply(result, a, a); }
};

using MultiplierPtr = std::unique_ptr<Multiplier>;

// CPU multiply through GMP's mpz_mul (the reference's GmpMultiplier,
// src/arithmetic/gmp_multiplier.cpp:10-19). Used as the routing target for products
// below the GPU threshold and as the CPU arm of comparisons.
class GmpMultiplier : public Multiplier {
public:
    void multiply(mpz_t result, const mpz_t a, const mpz_t b) override { mpz_mul(result, a, b); }
    void square(mpz_t result, const mpz_t a) override { mpz_mul(result, a, a); }
};

}  // namespace pi
