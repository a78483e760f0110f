/*
 * pi_b200 engine -- C entry points of libpib200.so, the C++17 host library that runs the
 * reference's pi pipeline (binary splitting -> final formula -> decimal string) with its
 * products on the B200 (B200Multiplier over libpigpu.so).
 *
 * The reference has no C API for its engine; its CLI (src/main.cpp:57-211) drives
 * pi::PiEngine::compute (src/engine/pi_engine.cpp:207-603). These entry points expose the
 * same computation to non-C++ callers (tests, benchmarks, FFI bindings).
 */
#ifndef PI_B200_ENGINE_H
#define PI_B200_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Binary-splitting modes. */
#define PIB_MODE_GMP 0        /* products through GMP's mpz_mul (the reference's GmpMultiplier) */
#define PIB_MODE_PER_CALL 1   /* products >= threshold limbs through B200Multiplier, one call at a time */
#define PIB_MODE_BATCHED 2    /* the whole computation on the device (pg_pi): level-batched binary
                                splitting, Newton finish and batched decimal conversion in HBM */
#define PIB_MODE_GMP_NEWTON 3 /* GMP products everywhere, with the Newton finish and conversion
                                (the same integer algorithms as PIB_MODE_BATCHED, on the CPU) */
#define PIB_MODE_BATCHED_HOST_FINISH 4 /* level-batched splitting on the device, Newton finish and
                                conversion on the host with B200 products */

/* Compute pi to `digits` decimals; writes "3." + digits (no terminator) into out, which must
 * have room for digits + 2 bytes. threads = host threads issuing per-call products and
 * converting digits; threshold = min limbs of the smaller operand for the GPU path.
 * stats (may be NULL) receives PIB_NSTATS doubles: seconds of binary splitting, final formula,
 * conversion and total, then the number of GPU kernel launches, GPU product calls and
 * products routed to GMP. Returns 0 on success, non-zero on error (message via pib_last_error). */
#define PIB_NSTATS 8
int pib_pi(size_t digits, int mode, unsigned threads, size_t threshold, int device, char* out, size_t out_cap,
           double* stats);

/* P(a,b), Q(a,b), R(a,b) of the Chudnovsky series as signed little-endian limb arrays.
 * Each output buffer needs `cap` limbs; lengths and signs are written to len[3] and sign[3]. */
int pib_bs(unsigned long a, unsigned long b, int mode, size_t threshold, int device, uint64_t* P, uint64_t* Q,
           uint64_t* R, size_t cap, size_t* len, int* sign);

/* r = a * b through the drop-in pi::B200Multiplier::multiply on mpz_t (threshold routing like the
 * reference's should_use_gpu; products longer than one transform as block products of pg_mul
 * calls). Magnitudes are little-endian limbs with signs sa, sb; out (out_cap limbs) receives |r|,
 * out_len its length and out_sign its sign. Replaces GpuNttMultiplier::multiply
 * (src/arithmetic/gpu_ntt_multiplier.cpp:144-210) for callers outside C++. */
int pib_mul(const uint64_t* a, size_t na, int sa, const uint64_t* b, size_t nb, int sb, size_t threshold, int device,
            uint64_t* out, size_t out_cap, size_t* out_len, int* out_sign);

/* Message of the last failing call in this thread. */
const char* pib_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PI_B200_ENGINE_H */
