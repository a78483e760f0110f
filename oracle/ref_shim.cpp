// ORACLE -- test infrastructure only. Compiled together with the reference's own
// sources into oracle/_ref/libpiref.so (see oracle/Makefile); never linked by the product.
//
// C entry points over the reference's classes so tests can read the reference's own
// results:
//   ref_bs        pi::BinarySplitting::compute(a, b) with pi::GmpMultiplier
//                 (src/engine/binary_splitting.cpp:605-644), P/Q/R as hex strings
//   ref_pi        pi::PiEngine::compute(config).digits (src/engine/pi_engine.cpp:207-603)
//   ref_bs_checkpoint  pi::BinarySplitting::compute(a, b) with checkpointing enabled, so the
//                 reference's own save_bs_result writes <dir>/bs_<a>_<b>.ckpt
//                 (src/engine/binary_splitting.cpp:48-71, 104-109, 605-644)
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>

#include "arithmetic/gmp_multiplier.h"
#include "engine/binary_splitting.h"
#include "engine/pi_engine.h"

extern "C" {

static char* dup_str(const std::string& s) {
    char* r = static_cast<char*>(std::malloc(s.size() + 1));
    std::memcpy(r, s.c_str(), s.size() + 1);
    return r;
}

static char* mpz_hex(const mpz_t v) {
    void (*freefunc)(void*, size_t) = nullptr;
    mp_get_memory_functions(nullptr, nullptr, &freefunc);
    char* s = mpz_get_str(nullptr, 16, v);
    std::string out(s);
    freefunc(s, std::strlen(s) + 1);
    return dup_str(out);
}

int ref_bs(unsigned long a, unsigned long b, unsigned int threads, char** P, char** Q, char** R) {
    try {
        pi::GmpMultiplier mult;
        pi::BinarySplitting bs(mult, threads);
        pi::BSResult r = bs.compute(a, b);
        *P = mpz_hex(r.P);
        *Q = mpz_hex(r.Q);
        *R = mpz_hex(r.R);
        return 0;
    } catch (...) {
        return 1;
    }
}

int ref_bs_checkpoint(unsigned long a, unsigned long b, unsigned int threads, const char* dir) {
    try {
        pi::GmpMultiplier mult;
        pi::BinarySplitting bs(mult, threads);
        bs.enable_checkpointing(dir);
        pi::BSResult r = bs.compute(a, b);
        (void)r;
        return 0;
    } catch (...) {
        return 1;
    }
}

char* ref_pi(unsigned long digits, unsigned int threads) {
    try {
        pi::GmpMultiplier mult;
        pi::PiEngine engine(mult);
        pi::PiConfig cfg;
        cfg.digits = digits;
        cfg.num_threads = threads;
        cfg.verbose = false;
        cfg.output_file = "";
        return dup_str(engine.compute(cfg).digits);
    } catch (...) {
        return nullptr;
    }
}

// pi::GmpMultiplier::multiply (src/arithmetic/gmp_multiplier.cpp:10-12) on limb arrays;
// out receives na + nb limbs. Used to time the reference's own CPU product.
void ref_gmp_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out) {
    static pi::GmpMultiplier mult;
    mpz_t x, y, r;
    mpz_init(x);
    mpz_init(y);
    mpz_init(r);
    if (na) mpz_import(x, na, -1, sizeof(uint64_t), 0, 0, a);
    if (nb) mpz_import(y, nb, -1, sizeof(uint64_t), 0, 0, b);
    mult.multiply(r, x, y);
    std::memset(out, 0, (na + nb) * sizeof(uint64_t));
    size_t n = mpz_size(r);
    if (n) std::memcpy(out, mpz_limbs_read(r), n * sizeof(uint64_t));
    mpz_clear(x);
    mpz_clear(y);
    mpz_clear(r);
}

unsigned long ref_terms_needed(unsigned long digits) {
    return pi::BinarySplitting::terms_needed(digits);
}

void ref_free(char* p) { std::free(p); }

}  // extern "C"
