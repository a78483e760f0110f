// pg_mul_noalloc: the product for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code that runs while another
// component owns the device allocator (a framework with its own caching pool, a plugin
// host that forbids allocation inside its callbacks), or code on a path where an
// allocation's implicit device synchronisation is not acceptable. For them this file
// keeps everything the product needs beyond its inputs and outputs in two file-scope
// device arrays of fixed size:
//   g_noalloc_scratch  residues of both operands for transforms up to 2^15 points plus the
//                      carry look-back words: 786,688 bytes;
//   g_noalloc_tables   the twiddle tables (DeviceTables' layout, four-step factor tables only
//                      for the strided passes these sizes use: blocks of 2^14 and 2^15 points
//                      split into sub-transforms of 2^7): 1,966,080 bytes.
// Every GPU that loads libpigpu.so holds these ~2.8 MB until the process exits.
//
// Set-up: the first call on a device (with that device current) looks up the arrays'
// device addresses with cudaGetSymbolAddress and fills the tables with a kernel on the
// caller's stream, then waits for it. Make that first call before any stream capture.
// Every call, the first and all later ones, waits for the caller's stream before it returns:
// it reads the product's error word back with cudaMemcpyAsync and cudaStreamSynchronize.
//
// All calls share the arrays and the arrays keep the previous call's contents: the carry
// look-back words are cleared at the start of every call (the residues are overwritten in
// full). Calls whose work overlaps on the GPU (two host threads, or two streams) race on
// the shared arrays and corrupt each other's results: serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/pi_b200.h"
#include "ntt_engine.cuh"

namespace {

constexpr size_t kNoAllocMaxLimbs = 16384;  // largest na + nb accepted
constexpr int kNoAllocLogL = 15;            // product_logL(na, nb) for na + nb <= 16384
constexpr size_t kResWords = (size_t)pg::kNumPrimes << kNoAllocLogL;  // per operand
constexpr size_t kSyncWords = 64;           // error, ticket, look-back status (<= 8 CRT blocks used)
constexpr size_t kScratchWords = 2 * kResWords + kSyncWords;
constexpr size_t kTableEnt = 1u << pg::kFsLog;
// Four-step factor tables of the strided passes of these sizes (make_plan: L = 2^14 -> 2^7 x 2^7,
// L = 2^15 -> 2^7 x 2^8): block 2^14 or 2^15, sub-transform 2^7.
constexpr int kRowTypes = 2;
constexpr int kRowLogN = 7;
constexpr size_t kTableWords = (3 + kRowTypes) * 2 * pg::kNumPrimes * kTableEnt;

static_assert(kTableEnt == (1u << (pg::kStageLog - 1)), "stage and four-step tables share one length");

constexpr int kMaxDevices = 64;

struct NoAllocDevice {
    bool ready = false;
    uint32_t* scratch = nullptr;
    pg::TwiddleTables tw{};
};

std::mutex g_mu;
NoAllocDevice g_dev[kMaxDevices];

}  // namespace

static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];
static __device__ __align__(256) uint2 g_noalloc_tables[kTableWords];

namespace {

__device__ uint32_t dev_pow_mod(uint32_t b, uint64_t e, uint32_t p) {
    uint64_t r = 1, x = b;
    while (e) {
        if (e & 1) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

// Fills the table array: [type: stage, fs_lo, fs_hi, four-step (2^14, 2^7), four-step (2^15, 2^7)]
// [dir][prime][kTableEnt]; roots[dir][prime] = w_{2^26}^(+-1).
__global__ void fill_tables_kernel(uint2* t, uint32_t r0f, uint32_t r1f, uint32_t r2f, uint32_t r0i, uint32_t r1i,
                                   uint32_t r2i) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= kTableWords) return;
    const uint32_t i = (uint32_t)(idx % kTableEnt);
    const size_t rest = idx / kTableEnt;
    const int j = (int)(rest % pg::kNumPrimes);
    const int dir = (int)((rest / pg::kNumPrimes) % 2);
    const int type = (int)(rest / (2 * pg::kNumPrimes));
    const uint32_t p = pg::kPrime(j);
    const uint32_t root = dir == 0 ? (j == 0 ? r0f : j == 1 ? r1f : r2f) : (j == 0 ? r0i : j == 1 ? r1i : r2i);
    uint64_t e;
    if (type == 0)
        e = (uint64_t)pg::stage_exponent(i) << (pg::kMaxLogL - pg::kStageLog);  // entry h + x = w_{2h}^x
    else if (type == 1)
        e = i;                                                // w_{2^26}^i
    else if (type == 2)
        e = (uint64_t)i << pg::kFsLog;                        // w_{2^26}^(2^13 i)
    else {
        // w_{2^n}^(c bitrev_7(m)) at m * 2^6 + c, n = 14 + (type - 3)
        const uint32_t m = i >> (pg::kTileLog - kRowLogN), c = i & ((1u << (pg::kTileLog - kRowLogN)) - 1);
        const uint32_t k = __brev(m) >> (32 - kRowLogN);
        e = (uint64_t)(c * k) << (pg::kMaxLogL - (pg::kRowLogMin + type - 3));
    }
    const uint32_t w = dev_pow_mod(root, e, p);
    t[idx] = make_uint2(w, (uint32_t)(((uint64_t)w << 32) / p));
}

pg_status setup_device(int dev, cudaStream_t st) {
    NoAllocDevice& d = g_dev[dev];
    if (d.ready) return PG_OK;
    uint32_t* scratch = nullptr;
    uint2* tables = nullptr;
    if (cudaGetSymbolAddress((void**)&scratch, g_noalloc_scratch) != cudaSuccess) return PG_ERR_DEVICE;
    if (cudaGetSymbolAddress((void**)&tables, g_noalloc_tables) != cudaSuccess) return PG_ERR_DEVICE;
    uint32_t rf[pg::kNumPrimes], ri[pg::kNumPrimes];
    for (int j = 0; j < pg::kNumPrimes; ++j) {
        const uint32_t p = pg::kPrime(j);
        rf[j] = pg::pow_mod(pg::kGenerator(j), (uint64_t)(p - 1) >> pg::kMaxLogL, p);
        ri[j] = pg::inv_mod(rf[j], p);
    }
    const unsigned blocks = (unsigned)((kTableWords + 255) / 256);
    fill_tables_kernel<<<blocks, 256, 0, st>>>(tables, rf[0], rf[1], rf[2], ri[0], ri[1], ri[2]);
    if (cudaGetLastError() != cudaSuccess) return PG_ERR_DEVICE;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PG_ERR_DEVICE;
    for (int dir = 0; dir < 2; ++dir)
        for (int j = 0; j < pg::kNumPrimes; ++j) {
            d.tw.stage[dir][j] = tables + ((0 * 2 + dir) * pg::kNumPrimes + j) * kTableEnt;
            d.tw.fs_lo[dir][j] = tables + ((1 * 2 + dir) * pg::kNumPrimes + j) * kTableEnt;
            d.tw.fs_hi[dir][j] = tables + ((2 * 2 + dir) * pg::kNumPrimes + j) * kTableEnt;
        }
    d.tw.row = tables + (size_t)3 * 2 * pg::kNumPrimes * kTableEnt;
    d.tw.row_layout = 1;
    d.tw.nprimes = pg::kNumPrimes;
    d.tw.root_log = pg::kMaxLogL;
    d.scratch = scratch;
    d.ready = true;
    return PG_OK;
}

}  // namespace

// Every failure of a CUDA call leaves through here: the runtime's sticky last error is read
// (and so cleared), so that it does not surface later in the caller's own error checks.
static pg_status device_failure(cudaError_t e) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? PG_ERR_OOM : PG_ERR_DEVICE;
}

extern "C" pg_status pg_mul_noalloc(const uint64_t* d_a, size_t na, const uint64_t* d_b, size_t nb,
                                    uint64_t* d_out, void* stream) {
    // each operand on its own, so that na + nb cannot wrap around
    if (na > kNoAllocMaxLimbs || nb > kNoAllocMaxLimbs - na) return PG_ERR_TOO_LARGE;
    if (!d_out || (na && !d_a) || (nb && !d_b)) return PG_ERR_BAD_ARG;
    if (((uintptr_t)d_a | (uintptr_t)d_b | (uintptr_t)d_out) & 15) return PG_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(g_mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return device_failure(e);
    if (dev < 0 || dev >= kMaxDevices) return PG_ERR_DEVICE;
    if (na == 0 || nb == 0) {
        if (na + nb && (e = cudaMemsetAsync(d_out, 0, (na + nb) * 8, st)) != cudaSuccess) return device_failure(e);
        e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? PG_OK : device_failure(e);
    }
    pg_status s = setup_device(dev, st);
    if (s != PG_OK) {
        cudaGetLastError();
        return s;
    }
    const NoAllocDevice& d = g_dev[dev];
    // A workspace view over the static scratch; its capacities cover every accepted size, so
    // the launch sequence below never reaches an allocation. It is never released.
    pg::Workspace w;
    w.a_res = d.scratch;
    w.b_res = d.scratch + kResWords;
    w.res_cap = kResWords;
    w.sync = d.scratch + 2 * kResWords;
    w.sync_cap = kSyncWords;
    pg::DeviceTables t;
    t.tw = d.tw;
    if ((e = cudaMemsetAsync(w.sync, 0, 4, st)) != cudaSuccess) return device_failure(e);  // error word
    if ((e = pg::enqueue_product(t, w, d_a, na, d_b, nb, d_out, st)) != cudaSuccess) return device_failure(e);
    uint32_t err = 0;
    if ((e = cudaMemcpyAsync(&err, w.sync, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return device_failure(e);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return device_failure(e);
    if (err == 1) return PG_ERR_TIMEOUT;
    if (err != 0) return PG_ERR_INTERNAL;
    return PG_OK;
}
