// Device engine: twiddle tables, workspace and the launch sequence of one product.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "plan.h"
#include "types.cuh"

namespace pg {

constexpr int kPassThreads = 256;

// Launch one forward/inverse pass. Returns cudaGetLastError().
cudaError_t launch_pass(const Plan& plan, int pass, bool inverse, Source src, Fuse fuse, const PassParams& prm,
                        const TwiddleTables& tw, cudaStream_t st);

CrtConsts make_crt_consts(int logL);

// Launch the CRT + carry over `blocks` blocks (jobs * blocks_per_job). max_words, when given, is
// the longest job's word count: jobs of at most 32 * 16 words run one warp each.
cudaError_t launch_crt(const CrtParams& c, uint64_t blocks, cudaStream_t st, uint64_t max_words = 0);

// Stride and four-step block size of pass i.
void set_pass(PassParams& p, const Plan& plan, int i);

struct DeviceTables {
    uint2* base = nullptr;  // one allocation holding every table
    TwiddleTables tw{};
    // Pass splits chosen by the autotuner (pg_tune / pg_tune_load): tuned[logL] = {npass,
    // logN[0..2]}, npass == 0 meaning the built-in make_plan split.
    int8_t tuned[kMaxLogL + 1][4] = {};
    Plan plan(int logL) const {
        if (logL >= 0 && logL <= kMaxLogL && tuned[logL][0] > 0) {
            const int n[3] = {tuned[logL][1], tuned[logL][2], tuned[logL][3]};
            return plan_from(logL, tuned[logL][0], n);
        }
        return make_plan(logL);
    }
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
    void release();
};

// Enqueue out[0 .. na+nb) = a * b (device pointers; b == nullptr means square).
// *launches (if given) is incremented by the number of kernels enqueued.
cudaError_t enqueue_product(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                            const uint64_t* d_b, size_t nb, uint64_t* d_out, cudaStream_t st,
                            uint64_t* launches = nullptr);

}  // namespace pg
