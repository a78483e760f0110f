// Device big-integer primitives on little-endian 64-bit limb arrays (sm_100a).
//
// Every operation is batched: job j works on arrays at base + j * stride, all jobs of one
// launch with the same limb count. Carry chains across limbs are resolved exactly with
// generate/propagate pairs: (g, p) of a limb range says "a carry leaves the range" (g, with
// carry-in 0) and "a carry-in passes through it" (p); ranges compose associatively
// (hi o lo = (g_hi | p_hi & g_lo, p_hi & p_lo)). Short numbers (<= 256 limbs) use one warp per
// job and a warp scan; long numbers use 2048-limb segments per block. Plain sums of long numbers
// take one launch: each block publishes its segment's (g, p) and looks back over the job's
// earlier segments for its carry in (a wait on blocks that started before it, bounded: past
// kAddSpinLimit polls it records kErrAddWait in the error word and goes on with carry 0). The
// other forms take three launches (segment transfers, a per-job scan of them, the final sums),
// with no wait.
//
// These kernels carry the host-side mpz arithmetic of the reference's final formula and radix
// conversion (src/engine/pi_engine.cpp:437-491 mpf_sqrt/mpf_div/mpf_mul, and
// src/io/base_converter.cpp:48-147 mpz_tdiv_qr / mpz_get_str) onto the device.
#pragma once
#include <cstdint>

namespace pg {

constexpr int kBigThreads = 256;
constexpr int kBigLimbs = 8;                          // limbs per thread (long form)
constexpr int kBigSeg = kBigThreads * kBigLimbs;      // limbs per block segment
constexpr uint64_t kBigWarpMax = 32 * kBigLimbs;      // longest number for the warp form
constexpr uint32_t kAddSpinLimit = 1u << 22;          // polls of one look-back wait
constexpr uint32_t kErrAddWait = 8;                   // error-word bit: a look-back wait ran out

// Operand fetch of an addition z = u + v + cin, limb i of job j.
//   Plain:    u = x_i ^ mx, v = y_i ^ my (limbs past nx / ny read as 0 before the mask),
//   MulSmall: u = lo(x_i * c), v = hi(x_{i-1} * c)  (z = x * c for a 64-bit c).
enum class AddForm : int { Plain = 0, MulSmall = 1 };

struct AddArgs {
    const uint64_t* x;
    uint64_t sx, nx;
    const uint64_t* y;  // may be null (zero)
    uint64_t sy, ny;
    uint64_t* z;
    uint64_t sz, n;      // z: n limbs per job
    uint64_t mx, my;     // 0 or ~0
    uint64_t c;          // MulSmall multiplier
    uint32_t cin;
    const uint32_t* enable;  // per job: 0 -> z = x unchanged (requires z == x); null: all
    uint32_t* carry_out;     // per job final carry (may be null)
    uint32_t* seg;           // long form: per (job, segment) transfer / status words
    uint64_t njobs;
    uint32_t* err;           // one-pass form: error word (kErrAddWait)
    uint32_t spin_limit;     // one-pass form: polls per wait (0: kAddSpinLimit)
    uint32_t withhold1;      // test hook: segment withhold1 - 1 never publishes its status (0: none)
};

}  // namespace pg
