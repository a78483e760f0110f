// Device engine: twiddle tables, workspace and the launch sequence of one product.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>

#include "dev_alloc.h"
#include "plan.h"
#include "types.cuh"

namespace pg {

// Longest transform (log2 of its length) that one product of the splitting, the device
// arithmetic and the conversion may use: kMaxLogL (26), or less when the environment variable
// PG_MAX_LOGL asks for it (read once; tests lower it to drive the block-product and split-tree
// paths at small sizes). Products beyond it are computed as blocks, and splitting ranges whose
// top merges exceed it are split into subtrees merged with the device arithmetic.
inline int split_logL() {
    static const int v = [] {
        int l = kMaxLogL;
        if (const char* e = std::getenv("PG_MAX_LOGL")) {
            const int x = std::atoi(e);
            if (x >= 10 && x < kMaxLogL) l = x;
        }
        return l;
    }();
    return v;
}

// Threads of a pass kernel's CTA: 256 for tiles of 2^13 residues (4 CTAs per SM), 512 for tiles of
// 2^14 (2 CTAs per SM): 32 resident warps and <= 64 registers per thread either way.
constexpr int pass_threads(int logE) { return logE > kTileLog ? 512 : 256; }

// Launch one forward/inverse pass. Returns cudaGetLastError().
cudaError_t launch_pass(const Plan& plan, int pass, bool inverse, Source src, Fuse fuse, const PassParams& prm,
                        const TwiddleTables& tw, cudaStream_t st);

CrtConsts make_crt_consts(int logL);

// Launch the CRT + carry over `blocks` blocks (jobs * blocks_per_job). max_words, when given, is
// the longest job's word count: jobs of at most 32 * 16 words run one warp each.
cudaError_t launch_crt(const CrtParams& c, uint64_t blocks, cudaStream_t st, uint64_t max_words = 0);

// Launch the wide configuration's CRT + carry over `jobs` jobs of blocks_per_job blocks each (any
// batch form of CrtParams; c.status needs jobs * blocks_per_job words, c.blocks_per_job is set
// here): the blocks, the per-job scan of their carries, the carry application and, for jobs with a
// length slot, the lengths (c.top_ok: a carry out of the top word is dropped instead of reported).
// *launches (if given) counts the kernels.
cudaError_t launch_crt_wide(CrtParams c, uint64_t jobs, uint64_t blocks_per_job, int logL, cudaStream_t st,
                            uint64_t* launches = nullptr, bool three = false);
// Whether a product of na x nb limbs runs in the wide configuration (the context's crossover, or
// PG_WIDE_MIN_LIMBS; 0 = never).
struct DeviceTables;
bool use_wide(const DeviceTables& T, uint64_t na, uint64_t nb);
uint64_t wide_min_limbs(const DeviceTables& T);
// Output words per block of the wide CRT.
uint64_t crt_wide_block_words();

// Stride and four-step block size of pass i.
void set_pass(PassParams& p, const Plan& plan, int i);

struct DeviceTables {
    uint2* base = nullptr;  // one allocation holding every table of the 32-bit configuration
    TwiddleTables tw{};
    uint2* base_wide = nullptr;  // and of the wide one (64-bit coefficients, five primes)
    TwiddleTables tw_wide{};
    bool wide = false;           // tw_wide is built (contexts made by pg_create)
    // Pass splits chosen by the autotuner (pg_tune / pg_tune_load): tuned[logL] = {npass,
    // logN[0..2]}, npass == 0 meaning the built-in make_plan split.
    int8_t tuned[kMaxLogL + 1][4] = {};
    // The same for the wide configuration's transforms (2^6 .. 2^25 points).
    int8_t tuned_wide[kMaxLogL + 1][4] = {};
    Plan plan(int logL) const {
        if (logL >= 0 && logL <= kMaxLogL && tuned[logL][0] > 0) {
            const int n[3] = {tuned[logL][1], tuned[logL][2], tuned[logL][3]};
            return plan_from(logL, tuned[logL][0], n);
        }
        return make_plan(logL);
    }
    Plan plan_wide(int logL) const {
        if (logL >= 0 && logL <= kWideMaxLogL && tuned_wide[logL][0] > 0) {
            const int n[3] = {tuned_wide[logL][1], tuned_wide[logL][2], tuned_wide[logL][3]};
            return plan_from(logL, tuned_wide[logL][0], n);
        }
        return make_plan(logL);
    }
    // Products of at least this many limbs (na + nb) run in the wide configuration when its tables
    // are built (PG_WIDE_MIN_LIMBS overrides it; 0 keeps every product in the 32-bit one).
    uint64_t wide_min_limbs = 1ull << 13;
    cudaError_t build(int device);
    void release();
};

// Growable device workspace for one in-flight product.
struct Workspace {
    uint32_t* a_res = nullptr;   // 3 * L residues
    uint32_t* b_res = nullptr;   // 3 * L residues
    uint64_t res_cap = 0;        // elements per array (3 * L)
    uint64_t* in_a = nullptr;    // staged host operands
    uint64_t* in_b = nullptr;
    uint64_t* outl = nullptr;
    uint64_t limb_cap = 0;       // limbs per staged buffer
    uint32_t* sync = nullptr;    // [0] error, [1] ticket, [2..] look-back status
    uint64_t sync_cap = 0;
    uint64_t* pinned = nullptr;  // pinned host staging (3 * limb_cap limbs)
    cudaError_t ensure_res(uint64_t n);
    cudaError_t ensure_limbs(uint64_t n);
    cudaError_t ensure_sync(uint64_t nblocks);
    // Residues and carry words for an na x nb product (and every smaller one) in one allocation
    // each, instead of growing level by level.
    cudaError_t reserve_for(const DeviceTables& T, size_t na, size_t nb);
    void release();
};

// Enqueue out[0 .. na+nb) = a * b (device pointers; b == nullptr means square).
// *launches (if given) is incremented by the number of kernels enqueued.
cudaError_t enqueue_product(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                            const uint64_t* d_b, size_t nb, uint64_t* d_out, cudaStream_t st,
                            uint64_t* launches = nullptr);

// The residue count per operand array (Workspace::ensure_res) that enqueue_product requests for
// an na x nb product: a caller that knows its largest product can size the workspace once.
uint64_t product_res_elems(const DeviceTables& T, size_t na, size_t nb);

// The same product in a forced configuration (wide: 64-bit coefficients over five primes), for the
// autotuner; cudaErrorInvalidValue when the wide tables are absent or the product is too long for them.
cudaError_t enqueue_product_config(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                                   const uint64_t* d_b, size_t nb, uint64_t* d_out, cudaStream_t st, bool wide);

// Enqueue the wrapped product for a caller-chosen transform length L = 2^logL (2 na <= L and
// 2 nb <= L words; b == nullptr means square): out[0 .. L/2 + 1) receives sum_{i<L} c_i 2^(32 i)
// for the L-point cyclic convolution c of the operands' 32-bit words, a number congruent to
// a * b modulo 2^(32 L) - 1 (fold its words above L to reduce it). Half the transform length
// of the full product when only the product's residue is needed (Newton corrections, division
// remainders).
cudaError_t enqueue_product_wrap(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                                 const uint64_t* d_b, size_t nb, int logL, uint64_t* d_out, cudaStream_t st,
                                 uint64_t* launches = nullptr);

}  // namespace pg
