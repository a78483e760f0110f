// DevArith: signed multi-limb integers in device memory with mpz-like operations, for the
// pieces of the pi pipeline that follow binary splitting (Newton reciprocal, square root,
// final products, radix conversion). Magnitudes are little-endian 64-bit limb arrays in HBM;
// the sign and the limb count are kept on the host. Operations leave an upper bound on the limb
// count without waiting; the exact count is read back (a host wait) only where it is needed:
// bit lengths, comparisons, the sign of a difference, downloads.
//
// Products go through the NTT engine (enqueue_product); additions, shifts, comparisons and
// small multiples through the carry-chain kernels of bigint.cuh.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "ntt_engine.cuh"

namespace pg {

struct DevNum {
    uint64_t* d = nullptr;
    size_t cap = 0;   // limbs allocated
    size_t n = 0;     // limbs in use: exact (top limb non-zero when n > 0), or an upper bound
    int sign = 0;     // -1, 0, +1; with an upper-bound length a zero value may still carry +-1
    size_t slack = 0;   // n may exceed the exact length by at most this many limbs (0: exact)
};

class DevError : public std::runtime_error {
public:
    DevError(int status, const std::string& m) : std::runtime_error(m), status(status) {}
    int status;
};

// Device memory behind DevArith: limb buffers cached by power-of-two size class, scratch and
// flag words, and a pinned word for small reads. Kept by the context across calls, released
// with it (or by trim()). A caller that knows how much a computation will hold can reserve an
// arena first: class buffers are then carved from that one allocation (one cudaMalloc, made
// while the device is busy with other work, instead of one per size class on the critical path).
struct DevPool {
    std::multimap<size_t, uint64_t*> free_;   // free buffers by capacity (limbs)
    std::vector<std::pair<uint64_t*, size_t>> all_;     // buffers of their own cudaMalloc (limbs)
    std::vector<std::pair<uint64_t*, size_t>> carved_;  // buffers carved from an arena (limbs)
    std::vector<void*> arenas_;
    char* arena_next_ = nullptr;
    size_t arena_left_ = 0;                   // bytes
    uint64_t* scratch_ = nullptr;
    size_t scratch_cap_ = 0;
    uint32_t* flags_ = nullptr;
    size_t flags_cap_ = 0;
    uint32_t* seg_ = nullptr;
    size_t seg_cap_ = 0;
    uint64_t* host_word_ = nullptr;           // pinned, 8 words
    uint32_t add_epoch_ = 0;                  // one-pass sums: the last call's epoch (seg_ words)
    ~DevPool() { trim(); }
    void trim();                              // frees everything (no DevNum may be live)
    // Opens an arena of `bytes` unless the open one has that much room left; false (and nothing
    // changed) when the allocation fails.
    bool reserve_arena(size_t bytes);
    // `bytes` (a multiple of 8) from the open arena, 512-byte aligned; nullptr when it has no room.
    uint64_t* carve(size_t bytes);
    size_t held_bytes() const;                // every buffer's capacity, own and carved
};

class DevArith {
public:
    DevArith(const DeviceTables& T, Workspace& W, cudaStream_t st, uint64_t* launches, DevPool& pool);
    ~DevArith();
    DevArith(const DevArith&) = delete;
    DevArith& operator=(const DevArith&) = delete;

    // memory (cached by size class; released with the DevArith)
    void reserve(DevNum& x, size_t limbs);   // capacity >= limbs (contents undefined)
    void release(DevNum& x);
    uint64_t* scratch(size_t limbs);          // temporary, valid until the next scratch call
    cudaStream_t stream() const { return st_; }

    void set_ui(DevNum& x, uint64_t v);
    void set_pow2(DevNum& x, size_t e);
    void copy(DevNum& z, const DevNum& x);
    void upload(DevNum& x, const uint64_t* host, size_t n, int sign);
    void download(const DevNum& x, uint64_t* host);  // x.n limbs (exact length first)
    // Makes x.n exact (and the sign 0 for a zero value), reading the length back from the device
    // when an operation left an upper bound. Products, additions, shifts and small multiples leave
    // upper bounds, so a chain of them runs without host waits; comparisons, bit lengths and
    // downloads call this.
    void exact(DevNum& x) {
        if (x.slack) normalize(x);
    }

    size_t bits(const DevNum& x);             // bit length of |x|
    int cmp_abs(const DevNum& x, const DevNum& y);
    int cmp(const DevNum& x, const DevNum& y);

    void add(DevNum& z, const DevNum& x, const DevNum& y);
    void sub(DevNum& z, const DevNum& x, const DevNum& y);
    void add_si(DevNum& z, const DevNum& x, int64_t v);
    void mul(DevNum& z, const DevNum& x, const DevNum& y);   // any length (block products beyond one transform)
    // z = x * y reduced modulo M = 2^(32 L) - 1, L = 2^logL words: |z| in [0, M] with the
    // product's sign (M itself stands for 0). 2 |x|.n <= L and 2 |y|.n <= L. One L-point
    // transform product instead of the 2 (x.n + y.n)-word one.
    void mul_wrap(DevNum& z, const DevNum& x, const DevNum& y, int logL);
    // z = |x| mod M (M = 2^(32 L) - 1) with x's sign, for |x| < 2^(32 L + 128); M stays M.
    void fold(DevNum& z, const DevNum& x, int logL);
    void sqr(DevNum& z, const DevNum& x);
    void mul_ui(DevNum& z, const DevNum& x, uint64_t c);
    void shl(DevNum& z, const DevNum& x, size_t s);
    void tdiv_q_2exp(DevNum& z, const DevNum& x, size_t s);   // truncate toward zero
    void fdiv_q_2exp(DevNum& z, const DevNum& x, size_t s);   // floor
    void tdiv_r_2exp(DevNum& z, const DevNum& x, size_t s);   // |x| mod 2^s with x's sign

    // Batched kernels for the radix conversion (jobs at base + j * stride, see bigint.cuh).
    void batch_add(const uint64_t* x, uint64_t sx, uint64_t nx, const uint64_t* y, uint64_t sy, uint64_t ny,
                   uint64_t* z, uint64_t sz, uint64_t n, bool subtract, uint32_t cin, const uint32_t* enable,
                   uint64_t njobs);
    void batch_shr(const uint64_t* x, uint64_t sx, uint64_t nx, uint64_t* z, uint64_t sz, uint64_t n, uint64_t s,
                   uint64_t njobs);
    void batch_ge(const uint64_t* x, uint64_t sx, const uint64_t* y, uint64_t sy, uint64_t n, uint32_t* ge,
                  uint64_t njobs);  // ge[j] = (x_j >= y_j), y shared when sy == 0
    // decimal digits of each job into out (device); false when a job has more digits than its
    // slot or the digits below `skip` are not all zero
    bool leaves(const uint64_t* x, uint64_t sx, uint64_t nlimbs, uint64_t njobs, uint64_t digits, char* out,
                uint64_t skip, uint64_t total);


    const DeviceTables& tables() const { return T_; }
    Workspace& workspace() { return W_; }
    void sync();                              // wait and check the product error word
    uint64_t* launches() { return launches_; }

    // out[0 .. na + nb) = a * b for any lengths (b == a allowed): one transform product when it
    // fits split_logL(), otherwise products of blocks of at most half that length each, added
    // into out at their offsets with exact carries.
    void mul_limbs(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out);

private:
    void normalize(DevNum& x);                // exact length (waits)
    void add_mag(DevNum& z, const DevNum& x, const DevNum& y, int sign);          // |z| = |x| + |y|
    void sub_mag(DevNum& z, const DevNum& x, const DevNum& y, int sign_if_pos);   // z = |x| - |y| signed
    void run_add(const struct AddArgs& a, int form);
    uint32_t* flags(size_t n);

    const DeviceTables& T_;
    Workspace& W_;
    cudaStream_t st_;
    uint64_t* launches_;
    DevPool& P_;
    std::multimap<size_t, uint64_t*>& pool_;
    std::vector<std::pair<uint64_t*, size_t>>& all_;
    uint64_t*& scratch_;
    size_t& scratch_cap_;
    uint32_t*& flags_;
    size_t& flags_cap_;
    uint32_t*& seg_;
    size_t& seg_cap_;
    uint64_t*& host_word_;
};

}  // namespace pg
