// B200Multiplier: a pi::Multiplier whose products run on one B200 through the C ABI of
// libpigpu.so (include/pi_b200.h). Drop-in replacement for the reference's
// GpuNttMultiplier / IntNttMultiplier (src/arithmetic/gpu_ntt_multiplier.h:38-103,
// src/arithmetic/int_ntt_multiplier.h).
//
// Differences from the reference bridges, by design:
//   * no digit repacking on the host: the device reads mpz limbs as they are
//     (mpz_limbs_read) and writes the product limbs straight into the result
//     (mpz_limbs_write / mpz_limbs_finish);
//   * products the transform cannot represent exactly raise std::runtime_error; there
//     is no silent CPU fallback (the reference's IntNttMultiplier falls back to mpz_mul,
//     int_ntt_multiplier.cpp:146-151);
//   * routing: a product whose smaller operand has fewer than `threshold` limbs goes to
//     mpz_mul, exactly like GpuNttMultiplier::should_use_gpu (gpu_ntt_multiplier.cpp:67-72).
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <string>

#include "multiplier.h"
#include "pi_b200.h"

namespace pi {

class B200Multiplier : public Multiplier {
public:
    // threshold: minimum limb count of the smaller operand for the GPU path (the
    // reference's --gpu-threshold, default 10000, main.cpp:63).
    explicit B200Multiplier(size_t threshold = 10000, int device = 0);
    // Use an existing context (not destroyed by this multiplier).
    B200Multiplier(size_t threshold, pg_ctx* shared, int device);
    ~B200Multiplier() override;
    B200Multiplier(const B200Multiplier&) = delete;
    B200Multiplier& operator=(const B200Multiplier&) = delete;

    void multiply(mpz_t result, const mpz_t a, const mpz_t b) override;
    void square(mpz_t result, const mpz_t a) override;

    void set_threshold(size_t t) { threshold_ = t; }
    size_t threshold() const { return threshold_; }
    std::string device_name() const;
    pg_ctx* context() const { return ctx_; }

    struct Stats {
        std::atomic<uint64_t> gpu_calls{0};
        std::atomic<uint64_t> cpu_routed_calls{0};
        std::atomic<uint64_t> gpu_ns{0};
        std::atomic<uint64_t> gpu_limbs{0};   // sum of na + nb over GPU calls
    };
    const Stats& stats() const { return stats_; }
    void reset_stats();
    void print_stats() const;

private:
    void product(mpz_t result, const mpz_t a, const mpz_t b, bool square);
    pg_status block_product(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, bool square, uint64_t* out,
                            size_t* len);
    pg_ctx* ctx_ = nullptr;
    bool owned_ = true;
    size_t threshold_;
    int device_;
    mutable Stats stats_;
};

// One context per device for the whole process (tables, workspace and binary-splitting
// buffers are built once and reused by every pi computation). Never destroyed.
pg_ctx* shared_context(int device);

}  // namespace pi
