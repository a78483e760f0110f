#include "device_bs.h"

#include <cmath>
#include <stdexcept>
#include <string>

namespace pi {

DeviceBinarySplitting::DeviceBinarySplitting(int device) {
    pg_status s = pg_create(device, &ctx_);
    if (s != PG_OK) throw std::runtime_error("DeviceBinarySplitting: pg_create failed with status " + std::to_string(s));
}

DeviceBinarySplitting::DeviceBinarySplitting(pg_ctx* shared) : ctx_(shared), owned_(false) {}

DeviceBinarySplitting::~DeviceBinarySplitting() {
    if (owned_) pg_destroy(ctx_);
}

void DeviceBinarySplitting::compute(unsigned long a, unsigned long b, mpz_ptr P, mpz_ptr Q, mpz_ptr R) {
    if (b <= a) throw std::invalid_argument("empty range");
    // Upper bound on the limbs of P, Q, R: each term contributes at most 3*log2(b) + 58 bits.
    const double bits_per_term = 3.0 * std::log2((double)b + 2.0) + 60.0;
    const size_t cap = (size_t)((double)(b - a) * bits_per_term / 64.0) + 64;
    mpz_t dummy;
    mpz_init(dummy);
    mpz_ptr outs[3] = {P ? P : dummy, Q, R};
    uint64_t* bufs[3];
    for (int k = 0; k < 3; ++k) bufs[k] = reinterpret_cast<uint64_t*>(mpz_limbs_write(outs[k], (mp_size_t)cap));
    size_t len[3] = {0, 0, 0};
    int sign[3] = {0, 0, 0};
    pg_status s = pg_bs(ctx_, a, b, P ? bufs[0] : nullptr, bufs[1], bufs[2], cap, len, sign);
    if (s != PG_OK) {
        for (int k = 0; k < 3; ++k) mpz_limbs_finish(outs[k], 0);
        mpz_clear(dummy);
        throw std::runtime_error(std::string("DeviceBinarySplitting: ") + pg_last_error(ctx_));
    }
    for (int k = 0; k < 3; ++k) {
        const mp_size_t n = (k == 0 && !P) ? 0 : (mp_size_t)len[k];
        mpz_limbs_finish(outs[k], sign[k] < 0 ? -n : n);
    }
    mpz_clear(dummy);
}

}  // namespace pi
