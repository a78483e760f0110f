// Pi engine: binary splitting -> final formula -> decimal string.
//
// Mirrors the reference's PiEngine (src/engine/pi_engine.h:15-43, .cpp:207-603) for the
// parts this project keeps: guard digits (100), terms_needed(digits + 100), the mpf final
// step pi = 426880 * Q * sqrt(10005) / R at digits*3.3219281+64 bits, truncation to an
// integer after scaling by 10^digits, and the "3." + digits output. The binary-splitting
// phase runs either per call through a pi::Multiplier (the drop-in form) or level-batched
// on the device (device_bs.h).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "multiplier.h"

namespace pi {

enum class BSMode { PerCall = 0, Batched = 1 };

// Final formula and decimal conversion: the reference's GMP mpf division/square root and
// mpz_get_str, or integer Newton iterations and divide-and-conquer conversion whose large
// products run on the B200 (newton.h).
enum class FinalMode { Mpf = 0, Newton = 1, Device = 2 };  // Device: pg_pi, every step in HBM

struct PiConfig {
    size_t digits = 1000;
    unsigned int num_threads = 1;   // host threads issuing per-call products / converting digits
    BSMode mode = BSMode::PerCall;
    FinalMode final_mode = FinalMode::Mpf;
    int device = 0;                 // batched mode and the Newton finish
    size_t gpu_threshold = 1024;    // Newton finish: min limbs of the smaller operand for the GPU
    bool verbose = false;
    std::string checkpoint_dir;     // batched device mode: resume from / save checkpoint files here
    // Batched device mode: when set, the digits + 2 output bytes ("3." and the decimals) are written
    // here (for instance into a mapping of the output file) and PiResult::digits stays empty.
    char* digits_out = nullptr;
};

struct PiTimings {
    double bs = 0, final = 0, convert = 0, total = 0;
    uint64_t gpu_launches = 0, gpu_calls = 0, cpu_routed = 0;
};

struct PiResult {
    std::string digits;      // "3." followed by `digits` decimals
    double elapsed_seconds = 0;
    unsigned long terms_used = 0;
    PiTimings t;
};

class PiEngine {
public:
    explicit PiEngine(Multiplier& multiplier);
    PiResult compute(const PiConfig& config);
    std::string compute_digits(size_t digits);

private:
    Multiplier& mult_;
};

// pi_int = floor(pi * 10^digits) from the binary-splitting Q and R, via GMP mpf at the
// reference's precision (pi_engine.cpp:437-491).
void final_formula_mpf(mpz_t pi_int, const mpz_t Q, const mpz_t R, size_t digits);

// "3." + digits decimals of pi_int (reference output format, pi_engine.cpp:556-573).
std::string format_digits(const mpz_t pi_int, size_t digits);

}  // namespace pi
