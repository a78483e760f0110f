// Device engine implementation: twiddle tables, pass dispatch, CRT constants and
// the per-product launch sequence.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

#include "crt_carry.cuh"
#include "ntt_engine.cuh"
#include "ntt_pass.cuh"

namespace pg {

// ---------------------------------------------------------------- host modular helpers
uint32_t pow_mod(uint32_t b, uint64_t e, uint32_t p) {
    uint64_t r = 1, x = b % p;
    while (e) {
        if (e & 1) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}
uint32_t inv_mod(uint32_t a, uint32_t p) { return pow_mod(a, p - 2, p); }
uint32_t shoup_companion(uint32_t w, uint32_t p) { return (uint32_t)(((uint64_t)w << 32) / p); }

// ---------------------------------------------------------------- tables
// Layout of the single table allocation, in uint2 entries:
//   [dir][prime] stage  (2^14 each): entry h + x = w_{2h}^x for h = 2^k, x < h (entry 0 unused)
//   [dir][prime] fs_lo  (2^13 each): w_{2^26}^j
//   [dir][prime] fs_hi  (2^13 each): w_{2^26}^(2^13 j)
//   [n][l][dir][prime] row (2^13 each): w_{2^n}^(c bitrev_l(m)) at m * 2^(13-l) + c, for four-step
//                       blocks of 2^n points (n = 14..26) and strided sub-transforms of 2^l points
//                       (l = 5..10, tiles of 2^13)
//   [n][l][dir][prime] row_big (2^14 each): the same for l = 11, 12 in tiles of 2^14 (m * 2^(14-l) + c)
// The host computes the stage and fs tables (1.5 MB); a kernel derives every row table from fs_lo and
// fs_hi on the device (w_{2^26}^e = lo[e mod 2^13] * hi[e / 2^13]), so a context's 50 MB of tables
// cost no host arithmetic and no upload.
namespace {
constexpr size_t kFsEnt = 1u << kFsLog;
constexpr size_t kSmallTables = (size_t)2 * kNumPrimes * (kStageEnt + 2 * kFsEnt);  // entries
constexpr size_t kRowEnt = (size_t)kRowTables * 2 * kNumPrimes * kFsEnt;
constexpr size_t kRowBigEnt = (size_t)kRowTablesBig * 2 * kNumPrimes * (1u << 14);

__global__ void fill_row_tables_kernel(uint2* row, uint2* row_big, TwiddleTables tw) {
    const uint64_t total = kRowEnt + kRowBigEnt;
    for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const bool big = idx >= kRowEnt;
        const uint64_t k = big ? idx - kRowEnt : idx;
        const int logE = big ? 14 : 13;
        const uint32_t i = (uint32_t)(k & ((1u << logE) - 1));  // entry in its table
        const uint64_t t = k >> logE;                            // ((n, l) * 2 + dir) * primes + prime
        const int j = (int)(t % kNumPrimes);
        const int dir = (int)((t / kNumPrimes) & 1);
        const uint64_t nl = t / (2 * kNumPrimes);
        const int nls = big ? (kRowNBigMax - kRowNBigMin + 1) : (kRowNMax - kRowNMin + 1);
        const int n = kRowLogMin + (int)(nl / nls);
        const int l = (big ? kRowNBigMin : kRowNMin) + (int)(nl % nls);
        const uint32_t m = i >> (logE - l), c = i & ((1u << (logE - l)) - 1);
        const uint32_t kr = __brev(m) >> (32 - l);  // bitrev_l(m)
        const uint32_t e = (c * kr) << (kMaxLogL - n);  // c * kr < 2^logE <= 2^n: e < 2^26
        const uint32_t p = kPrime(j);
        const uint2 a = tw.fs_lo[dir][j][e & (kFsEnt - 1)];
        const uint2 b = tw.fs_hi[dir][j][e >> kFsLog];
        const uint32_t w = mul_shoup(a.x, b.x, b.y, p);
        (big ? row_big : row)[k] = make_uint2(w, shoup_companion_dev(w, p, kRecip64(j)));
    }
}
}  // namespace

static cudaError_t allow_big_tiles();

cudaError_t DeviceTables::build(int device) {
    (void)device;
    std::vector<uint2> h(kSmallTables);
    auto stage_at = [&](int dir, int j) { return h.data() + (size_t)(dir * kNumPrimes + j) * kStageEnt; };
    auto fs_at = [&](int which, int dir, int j) {
        return h.data() + (size_t)2 * kNumPrimes * kStageEnt + ((size_t)(which * 2 + dir) * kNumPrimes + j) * kFsEnt;
    };
    for (int dir = 0; dir < 2; ++dir)
        for (int j = 0; j < kNumPrimes; ++j) {
            const uint32_t p = kPrime(j);
            uint32_t w26 = pow_mod(kGenerator(j), (uint64_t)(p - 1) >> kMaxLogL, p);  // primitive 2^26-th root
            if (dir == 1) w26 = inv_mod(w26, p);
            const uint32_t w14 = pow_mod(w26, 1ull << (kMaxLogL - kStageLog), p);
            const uint32_t w26hi = pow_mod(w26, 1ull << kFsLog, p);
            uint2* st = stage_at(dir, j);
            uint2* lo = fs_at(0, dir, j);
            uint2* hi = fs_at(1, dir, j);
            // stage entries by level: entry 2^k + x = w_{2^(k+1)}^x = w14^(x 2^(13-k))
            st[0] = make_uint2(1, shoup_companion(1, p));
            for (int k = 0; k < kStageLog; ++k) {
                const uint64_t step = pow_mod(w14, 1ull << (kStageLog - 1 - k), p);
                uint64_t r = 1;
                for (uint32_t x = 0; x < (1u << k); ++x) {
                    st[(1u << k) + x] = make_uint2((uint32_t)r, shoup_companion((uint32_t)r, p));
                    r = r * step % p;
                }
            }
            uint64_t b = 1, c = 1;
            for (size_t i = 0; i < kFsEnt; ++i) {
                lo[i] = make_uint2((uint32_t)b, shoup_companion((uint32_t)b, p));
                hi[i] = make_uint2((uint32_t)c, shoup_companion((uint32_t)c, p));
                b = b * w26 % p;
                c = c * w26hi % p;
            }
        }
    cudaError_t e = pg::dev_malloc(&base, (kSmallTables + kRowEnt + kRowBigEnt) * sizeof(uint2));
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(base, h.data(), h.size() * sizeof(uint2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    for (int dir = 0; dir < 2; ++dir)
        for (int j = 0; j < kNumPrimes; ++j) {
            tw.stage[dir][j] = base + (size_t)(dir * kNumPrimes + j) * kStageEnt;
            tw.fs_lo[dir][j] = base + (size_t)2 * kNumPrimes * kStageEnt + ((size_t)(0 * 2 + dir) * kNumPrimes + j) * kFsEnt;
            tw.fs_hi[dir][j] = base + (size_t)2 * kNumPrimes * kStageEnt + ((size_t)(1 * 2 + dir) * kNumPrimes + j) * kFsEnt;
        }
    uint2* row = base + kSmallTables;
    uint2* row_big = row + kRowEnt;
    tw.row = row;
    tw.row_big = row_big;
    tw.row_layout = 0;
    e = allow_big_tiles();
    if (e != cudaSuccess) return e;
    fill_row_tables_kernel<<<148 * 8, 256>>>(row, row_big, tw);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e;
}

void DeviceTables::release() {
    if (base) cudaFree(base);
    base = nullptr;
}

// ---------------------------------------------------------------- workspace
static cudaError_t grow(void** ptr, uint64_t bytes) {
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    return pg::dev_malloc(ptr, bytes);
}

cudaError_t Workspace::ensure_res(uint64_t n) {
    if (n <= res_cap) return cudaSuccess;
    n = std::max(n, res_cap + res_cap / 2);  // geometric growth: products grow level by level
    cudaError_t e = grow((void**)&a_res, n * 4);
    if (e == cudaSuccess) e = grow((void**)&b_res, n * 4);
    res_cap = (e == cudaSuccess) ? n : 0;
    return e;
}

cudaError_t Workspace::ensure_limbs(uint64_t n) {
    if (n <= limb_cap) return cudaSuccess;
    n = std::max<uint64_t>({n, 1024, limb_cap + limb_cap / 2});  // pinned allocations are slow: grow geometrically
    cudaError_t e = grow((void**)&in_a, n * 8);
    if (e == cudaSuccess) e = grow((void**)&in_b, n * 8);
    if (e == cudaSuccess) e = grow((void**)&outl, n * 8);
    if (e == cudaSuccess) {
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        e = cudaMallocHost((void**)&pinned, 3 * n * 8);
    }
    limb_cap = (e == cudaSuccess) ? n : 0;
    return e;
}

cudaError_t Workspace::ensure_sync(uint64_t nblocks) {
    if (nblocks + 2 <= sync_cap) return cudaSuccess;
    uint64_t n = nblocks + 2 < 4096 ? 4096 : nblocks + 2;
    // Carry an error recorded by an earlier (asynchronous) product over to the new buffer.
    uint32_t old_err = 0;
    if (sync) cudaMemcpy(&old_err, sync, 4, cudaMemcpyDeviceToHost);
    cudaError_t e = grow((void**)&sync, n * 4);
    if (e == cudaSuccess) e = cudaMemset(sync, 0, n * 4);
    if (e == cudaSuccess && old_err) e = cudaMemcpy(sync, &old_err, 4, cudaMemcpyHostToDevice);
    sync_cap = (e == cudaSuccess) ? n : 0;
    return e;
}

void Workspace::release() {
    if (a_res) cudaFree(a_res);
    if (b_res) cudaFree(b_res);
    if (in_a) cudaFree(in_a);
    if (in_b) cudaFree(in_b);
    if (outl) cudaFree(outl);
    if (sync) cudaFree(sync);
    if (pinned) cudaFreeHost(pinned);
    *this = Workspace{};
}

// ---------------------------------------------------------------- pass dispatch
// Dynamic shared memory of a pass: the tile, plus the four-step row factors of a strided tile.
template <Layout LAY, int LOGN>
constexpr size_t pass_smem() {
    return ((size_t)4 << tile_log(LAY == Layout::Strided, LOGN)) + (LAY == Layout::Strided ? ((size_t)8 << LOGN) : 0);
}

template <Layout LAY, int LOGN, bool INV, Source SRC, Fuse FUSE>
static cudaError_t run_pass(const PassParams& prm, const TwiddleTables& tw, cudaStream_t st) {
    constexpr int LOGE = tile_log(LAY == Layout::Strided, LOGN);
    constexpr int NT = pass_threads(LOGE);
    uint64_t tiles;
    if constexpr (LAY == Layout::Strided) {
        tiles = (uint64_t)prm.njobs << (prm.logL - LOGE);
    } else {
        const uint64_t rows = (uint64_t)prm.njobs << (prm.logL - LOGN);
        const uint64_t per = 1ull << (LOGE - LOGN);
        tiles = (rows + per - 1) / per;
    }
    auto kern = ntt_pass_kernel<LAY, LOGN, LOGE, NT, INV, SRC, FUSE>;
    constexpr size_t smem = pass_smem<LAY, LOGN>();
    dim3 grid((unsigned)tiles, kNumPrimes);
    kern<<<grid, NT, smem, st>>>(prm, tw);
    return cudaGetLastError();
}

// Kernels whose tiles need more than the default 48 KB of dynamic shared memory opt in on the
// current device; done for every such kernel when a context's tables are built, so that no
// attribute is set in the middle of a stream capture.
template <Layout LAY, int LOGN, bool INV, Source SRC, Fuse FUSE>
static cudaError_t allow_smem() {
    constexpr int LOGE = tile_log(LAY == Layout::Strided, LOGN);
    constexpr size_t smem = pass_smem<LAY, LOGN>();
    if constexpr (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(ntt_pass_kernel<LAY, LOGN, LOGE, pass_threads(LOGE), INV, SRC, FUSE>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int N>
static cudaError_t allow_smem_contig() {
    cudaError_t e = allow_smem<Layout::Contig, N, true, Source::Residues, Fuse::Combine>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, true, Source::Residues, Fuse::None>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Limbs, Fuse::None>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Limbs, Fuse::MulInverse>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Limbs, Fuse::SqrInverse>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::None>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::MulInverse>();
    if (e == cudaSuccess) e = allow_smem<Layout::Contig, N, false, Source::Residues, Fuse::SqrInverse>();
    return e;
}

template <int N>
static cudaError_t allow_smem_strided() {
    cudaError_t e = allow_smem<Layout::Strided, N, true, Source::Residues, Fuse::None>();
    if (e == cudaSuccess) e = allow_smem<Layout::Strided, N, false, Source::Limbs, Fuse::None>();
    if (e == cudaSuccess) e = allow_smem<Layout::Strided, N, false, Source::Residues, Fuse::None>();
    return e;
}

static cudaError_t allow_big_tiles() {
    cudaError_t e = allow_smem_contig<14>();
    if (e == cudaSuccess) e = allow_smem_strided<11>();
    if (e == cudaSuccess) e = allow_smem_strided<12>();
    return e;
}

#define PG_CONTIG_CASE(N)                                                                                    \
    case N:                                                                                                  \
        if (inverse && fuse == Fuse::Combine)                                                                \
            return run_pass<Layout::Contig, N, true, Source::Residues, Fuse::Combine>(prm, tw, st);          \
        if (inverse) return run_pass<Layout::Contig, N, true, Source::Residues, Fuse::None>(prm, tw, st);   \
        if (src == Source::Limbs) {                                                                          \
            if (fuse == Fuse::None) return run_pass<Layout::Contig, N, false, Source::Limbs, Fuse::None>(prm, tw, st); \
            if (fuse == Fuse::MulInverse) return run_pass<Layout::Contig, N, false, Source::Limbs, Fuse::MulInverse>(prm, tw, st); \
            return run_pass<Layout::Contig, N, false, Source::Limbs, Fuse::SqrInverse>(prm, tw, st);        \
        } else {                                                                                             \
            if (fuse == Fuse::None) return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::None>(prm, tw, st); \
            if (fuse == Fuse::MulInverse) return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::MulInverse>(prm, tw, st); \
            return run_pass<Layout::Contig, N, false, Source::Residues, Fuse::SqrInverse>(prm, tw, st);     \
        }

#define PG_STRIDED_CASE(N)                                                                                   \
    case N:                                                                                                  \
        if (inverse) return run_pass<Layout::Strided, N, true, Source::Residues, Fuse::None>(prm, tw, st);  \
        if (src == Source::Limbs) return run_pass<Layout::Strided, N, false, Source::Limbs, Fuse::None>(prm, tw, st); \
        return run_pass<Layout::Strided, N, false, Source::Residues, Fuse::None>(prm, tw, st);

cudaError_t launch_pass(const Plan& plan, int pass, bool inverse, Source src, Fuse fuse, const PassParams& prm0,
                        const TwiddleTables& tw, cudaStream_t st) {
    const int logN = plan.logN[pass];
    const bool contig = (pass == plan.npass - 1);
    PassParams prm = prm0;
    if (!contig) {
        prm.rowB = row_table(tw, plan.logN[pass] + plan.logS[pass], logN, inverse ? 1 : 0);
        if (!prm.rowB) return cudaErrorInvalidValue;  // no four-step table for this split
    }
    if (contig) {
        if (inverse && (src != Source::Residues || (fuse != Fuse::None && fuse != Fuse::Combine)))
            return cudaErrorInvalidValue;
        switch (logN) {
            PG_CONTIG_CASE(6)
            PG_CONTIG_CASE(7)
            PG_CONTIG_CASE(8)
            PG_CONTIG_CASE(9)
            PG_CONTIG_CASE(10)
            PG_CONTIG_CASE(11)
            PG_CONTIG_CASE(12)
            PG_CONTIG_CASE(13)
            PG_CONTIG_CASE(14)
            default:
                return cudaErrorInvalidValue;
        }
    } else {
        switch (logN) {
            PG_STRIDED_CASE(5)
            PG_STRIDED_CASE(6)
            PG_STRIDED_CASE(7)
            PG_STRIDED_CASE(8)
            PG_STRIDED_CASE(9)
            PG_STRIDED_CASE(10)
            PG_STRIDED_CASE(11)
            PG_STRIDED_CASE(12)
            default:
                return cudaErrorInvalidValue;
        }
    }
}

// Test hooks of the look-back wait, read on every launch so that a test can set and clear them
// around one product: PG_TEST_CRT_SPIN_LIMIT=n ends each wait after n polls, and
// PG_TEST_CRT_WITHHOLD=b keeps the block with ticket b from publishing its carry, so that the
// next block's wait runs out (PG_ERR_TIMEOUT, no GPU fault). Unset: the built-in limit, no hook.
static void crt_test_hooks(CrtParams& c) {
    if (const char* e = std::getenv("PG_TEST_CRT_SPIN_LIMIT")) c.spin_limit = (uint32_t)std::strtoul(e, nullptr, 10);
    if (const char* e = std::getenv("PG_TEST_CRT_WITHHOLD")) c.withhold1 = (uint32_t)std::strtoul(e, nullptr, 10) + 1;
}

cudaError_t launch_crt(const CrtParams& c0, uint64_t blocks, cudaStream_t st, uint64_t max_words) {
    CrtParams c = c0;
    crt_test_hooks(c);
    if (max_words && max_words <= kCrtWarpWords && c.blocks_per_job == 1) {
        // blocks == jobs here: one warp per job
        crt_warp_kernel<<<(unsigned)((blocks * 32 + 255) / 256), 256, 0, st>>>(c, blocks);
        return cudaGetLastError();
    }
    crt_carry_kernel<<<(unsigned)blocks, kCrtThreads, 0, st>>>(c);
    return cudaGetLastError();
}

void set_pass(PassParams& p, const Plan& plan, int i) {
    p.logS = plan.logS[i];
    p.logNp = plan.logN[i] + plan.logS[i];
}

// ---------------------------------------------------------------- CRT constants
static void shoup_pair(uint32_t v, uint32_t p, uint32_t& w, uint32_t& wp) {
    w = v % p;
    wp = shoup_companion(w, p);
}

CrtConsts make_crt_consts(int logL) {
    const uint32_t p0 = kPrime(0), p1 = kPrime(1), p2 = kPrime(2);
    // scale f_j = L^-1 * 2^32 mod p_j (unnormalised inverse + Montgomery pointwise factor)
    auto scale = [&](uint32_t p) {
        uint64_t linv = inv_mod(pow_mod(2, (uint64_t)logL, p), p);
        uint64_t r32 = pow_mod(2, 32, p);
        return (uint32_t)(linv * r32 % p);
    };
    const uint64_t f0 = scale(p0), f1 = scale(p1), f2 = scale(p2);
    const uint64_t i01 = inv_mod(p0 % p1, p1);          // p0^-1 mod p1
    const uint64_t i02 = inv_mod(p0 % p2, p2);          // p0^-1 mod p2
    const uint64_t i12 = inv_mod(p1 % p2, p2);          // p1^-1 mod p2
    CrtConsts k;
    shoup_pair((uint32_t)f0, p0, k.c00, k.c00p);
    shoup_pair((uint32_t)(f1 * i01 % p1), p1, k.c11, k.c11p);
    shoup_pair((uint32_t)i01, p1, k.k01, k.k01p);
    shoup_pair((uint32_t)(f2 * i02 % p2 * i12 % p2), p2, k.c22, k.c22p);
    shoup_pair((uint32_t)(i02 * i12 % p2), p2, k.k02, k.k02p);
    shoup_pair((uint32_t)i12, p2, k.k12, k.k12p);
    k.p01 = (uint64_t)p0 * p1;
    // floor(P/2) in Garner digits: P/2 = (p0 p1 p2 - 1)/2; digits by repeated division
    const unsigned __int128 P = (unsigned __int128)p0 * p1 * p2;
    const unsigned __int128 H = P / 2;
    k.h0 = (uint32_t)(H % p0);
    k.h1 = (uint32_t)((H / p0) % p1);
    k.h2 = (uint32_t)(H / ((unsigned __int128)p0 * p1));
    k.P_lo = (uint64_t)P;
    k.P_hi = (uint64_t)(P >> 64);
    return k;
}

// ---------------------------------------------------------------- one product
static cudaError_t enqueue_impl(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                                const uint64_t* d_b, size_t nb, int logL, uint64_t nwords, uint64_t* d_out,
                                cudaStream_t st, uint64_t* launches) {
    const bool square = (d_b == nullptr);
    if (square) nb = na;
    const Plan plan = T.plan(logL);
    const uint64_t L = 1ull << logL;
    cudaError_t e = W.ensure_res(3 * L);
    if (e != cudaSuccess) return e;
    const uint64_t crt_blocks = (nwords + kCrtThreads * kCrtWords - 1) / (kCrtThreads * kCrtWords);
    e = W.ensure_sync(crt_blocks);
    if (e != cudaSuccess) return e;

    auto base = [&](uint32_t* data, const uint64_t* limbs, uint64_t ncoef) {
        PassParams p{};
        p.data = data;
        p.out = data;
        p.other = nullptr;
        p.other_stride = 3 * L;
        p.words_stride = 0;
        p.words = reinterpret_cast<const uint32_t*>(limbs);
        p.ncoef = ncoef;
        p.L = L;
        p.logL = logL;
        p.job_stride = 3 * L;
        p.njobs = 1;
        p.merge = 0;
        return p;
    };
    auto set_pass = [&](PassParams& p, int i) { pg::set_pass(p, plan, i); };

    const int last = plan.npass - 1;
    // Operand a: full forward transform (all but the last pass when squaring).
    {
        PassParams p = base(W.a_res, d_a, 2ull * na);
        const int upto = square ? last : plan.npass;
        for (int i = 0; i < upto; ++i) {
            set_pass(p, i);
            Fuse f = Fuse::None;
            e = launch_pass(plan, i, false, i == 0 ? Source::Limbs : Source::Residues, f, p, T.tw, st);
            if (e != cudaSuccess) return e;
        }
        if (square) {
            set_pass(p, last);
            e = launch_pass(plan, last, false, last == 0 ? Source::Limbs : Source::Residues, Fuse::SqrInverse, p,
                            T.tw, st);
            if (e != cudaSuccess) return e;
        }
    }
    uint32_t* prod = W.a_res;
    if (!square) {
        PassParams p = base(W.b_res, d_b, 2ull * nb);
        for (int i = 0; i < last; ++i) {
            set_pass(p, i);
            e = launch_pass(plan, i, false, i == 0 ? Source::Limbs : Source::Residues, Fuse::None, p, T.tw, st);
            if (e != cudaSuccess) return e;
        }
        set_pass(p, last);
        p.other = W.a_res;
        e = launch_pass(plan, last, false, last == 0 ? Source::Limbs : Source::Residues, Fuse::MulInverse, p, T.tw,
                        st);
        if (e != cudaSuccess) return e;
        prod = W.b_res;
    }
    // Inverse strided passes, last strided pass first.
    {
        PassParams p = base(prod, nullptr, 0);
        for (int i = last - 1; i >= 0; --i) {
            set_pass(p, i);
            e = launch_pass(plan, i, true, Source::Residues, Fuse::None, p, T.tw, st);
            if (e != cudaSuccess) return e;
        }
    }
    // CRT + carry.
    e = cudaMemsetAsync(W.sync + 1, 0, (crt_blocks + 1) * 4, st);
    if (e != cudaSuccess) return e;
    CrtParams c{};
    c.res = prod;
    c.L = L;
    c.nwords = nwords;
    c.out = reinterpret_cast<uint32_t*>(d_out);
    c.ticket = W.sync + 1;
    c.status = W.sync + 2;
    c.error = W.sync;
    c.blocks_per_job = crt_blocks;
    c.merge = 0;
    c.k = make_crt_consts(logL);
    e = launch_crt(c, crt_blocks, st, nwords);
    if (e != cudaSuccess) return e;
    if (launches) *launches += (square ? plan.npass : 2 * plan.npass) + (plan.npass - 1) + 1;
    return cudaGetLastError();
}

cudaError_t enqueue_product(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                            const uint64_t* d_b, size_t nb, uint64_t* d_out, cudaStream_t st,
                            uint64_t* launches) {
    const size_t mb = d_b ? nb : na;
    return enqueue_impl(T, W, d_a, na, d_b, nb, product_logL(na, mb), 2ull * (na + mb), d_out, st, launches);
}

cudaError_t enqueue_product_wrap(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                                 const uint64_t* d_b, size_t nb, int logL, uint64_t* d_out, cudaStream_t st,
                                 uint64_t* launches) {
    if (logL < kMinLogL || logL > kMaxLogL) return cudaErrorInvalidValue;
    const uint64_t L = 1ull << logL;
    if (2ull * na > L || (d_b && 2ull * nb > L)) return cudaErrorInvalidValue;
    // the L-point transform wraps the product: coefficient i sums a_j b_k over j + k = i mod L,
    // at most L terms of < 2^64 (< 2^90 <= the CRT range for L <= 2^26); their weighted sum
    // over i < L is below 2^(32 (L - 1) + 91), i.e. it fits in L + 2 words
    return enqueue_impl(T, W, d_a, na, d_b, nb, logL, L + 2, d_out, st, launches);
}

}  // namespace pg
