// ORACLE -- test infrastructure only. Compiled with the reference's own sources and
// ref_dropin_factory.cpp into oracle/_ref/libpiref_b200.so (oracle/Makefile); never linked by
// the product.
//
// The drop-in check: the reference's UNCHANGED BinarySplitting (src/engine/binary_splitting.cpp:
// 161-293, 295-394, 605-644) and PiEngine (src/engine/pi_engine.cpp:207-603), driven through its
// own `pi::Multiplier&` seam (src/engine/binary_splitting.h:39, pi_engine.h:34) by the library's
// pi::B200Multiplier, exactly as the reference's main.cpp:128-176 hands them its GPU multipliers.
//   refb_bs   P/Q/R of [a, b) as hex strings
//   refb_pi   "3." + digits of pi
// Both take the multiplier's threshold (products whose smaller operand has fewer limbs go to
// mpz_mul, the reference's should_use_gpu rule) and report how many products the B200 computed.
//
// This translation unit sees the reference's pi::Multiplier declaration; the multiplier object
// comes from ref_dropin_factory.cpp, which sees the library's identical declaration (the two headers
// cannot meet in one translation unit).
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>

#include "engine/binary_splitting.h"
#include "engine/pi_engine.h"

namespace refb {
pi::Multiplier* make_b200_multiplier(size_t threshold, int device);
unsigned long long b200_gpu_calls(pi::Multiplier* m);
}  // namespace refb

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

int refb_bs(unsigned long a, unsigned long b, unsigned int threads, size_t threshold, int device, char** P,
            char** Q, char** R, unsigned long long* gpu_calls) {
    try {
        std::unique_ptr<pi::Multiplier> mult(refb::make_b200_multiplier(threshold, device));
        pi::BinarySplitting bs(*mult, threads);
        pi::BSResult r = bs.compute(a, b);
        *P = mpz_hex(r.P);
        *Q = mpz_hex(r.Q);
        *R = mpz_hex(r.R);
        *gpu_calls = refb::b200_gpu_calls(mult.get());
        return 0;
    } catch (...) {
        return 1;
    }
}

char* refb_pi(unsigned long digits, unsigned int threads, size_t threshold, int device,
              unsigned long long* gpu_calls) {
    try {
        std::unique_ptr<pi::Multiplier> mult(refb::make_b200_multiplier(threshold, device));
        pi::PiEngine engine(*mult);
        pi::PiConfig cfg;
        cfg.digits = digits;
        cfg.num_threads = threads;
        cfg.verbose = false;
        cfg.output_file = "";
        std::string d = engine.compute(cfg).digits;
        *gpu_calls = refb::b200_gpu_calls(mult.get());
        return dup_str(d);
    } catch (...) {
        return nullptr;
    }
}

void refb_free(char* p) { std::free(p); }

}  // extern "C"
