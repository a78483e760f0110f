// Device engine implementation: twiddle tables, pass dispatch, CRT constants and
// the per-product launch sequence.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

#include "crt_carry.cuh"
#include "radix3.cuh"
#include "ntt_engine.cuh"
#include "pass_launch.cuh"

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
// One table allocation per configuration (NP = 3 primes with roots w_{2^26}, NP = 5 with w_{2^25}),
// in uint2 entries:
//   [dir][prime] stage  (2^14 each): entry h + x = w_{2h}^x for h = 2^k, x < h (entry 0 unused)
//   [dir][prime] fs_lo  (2^13 each): w_{2^root}^j
//   [dir][prime] fs_hi  (2^13 each): w_{2^root}^(2^13 j)
//   [n][l][dir][prime] row (2^13 each): w_{2^n}^(c bitrev_l(m)) at m * 2^(13-l) + c, for four-step
//                       blocks of 2^n points (n = 14..root) and strided sub-transforms of 2^l points
//                       (l = 5..10, tiles of 2^13)
//   [n][l][dir][prime] row_big (2^14 each): the same for l = 11, 12 in tiles of 2^14 (m * 2^(14-l) + c)
// The host computes the stage and fs tables (2.5 MB); a kernel derives every row table from fs_lo and
// fs_hi on the device (w_{2^root}^e = lo[e mod 2^13] * hi[e / 2^13]), so a context's tables cost no
// host arithmetic and no upload beyond those.
namespace {
constexpr size_t kFsEnt = 1u << kFsLog;
// the wide configuration's radix-3 tables: [lo, hi][dir][prime], 2^13 entries each
constexpr size_t t3_entries(int np) { return np == kWidePrimes ? (size_t)2 * 2 * np * kFsEnt : 0; }
constexpr size_t small_entries(int np) { return (size_t)2 * np * (kStageEnt + 2 * kFsEnt) + t3_entries(np); }
constexpr size_t row_entries(int np) { return (size_t)kRowTables * 2 * np * kFsEnt; }
constexpr size_t row_big_entries(int np) { return (size_t)kRowTablesBig * 2 * np * (1u << 14); }

template <int NP>
__global__ void fill_row_tables_kernel(uint2* row, uint2* row_big, TwiddleTables tw) {
    constexpr uint64_t kRowEnt = row_entries(NP), kRowBigEnt = row_big_entries(NP);
    constexpr int root = root_log_of(NP);
    const uint64_t total = kRowEnt + kRowBigEnt;
    for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const bool big = idx >= kRowEnt;
        const uint64_t k = big ? idx - kRowEnt : idx;
        const int logE = big ? 14 : 13;
        const uint32_t i = (uint32_t)(k & ((1u << logE) - 1));  // entry in its table
        const uint64_t t = k >> logE;                            // ((n, l) * 2 + dir) * primes + prime
        const int j = (int)(t % NP);
        const int dir = (int)((t / NP) & 1);
        const uint64_t nl = t / (2 * NP);
        const int nls = big ? (kRowNBigMax - kRowNBigMin + 1) : (kRowNMax - kRowNMin + 1);
        const int n = kRowLogMin + (int)(nl / nls);
        if (n > root) continue;  // blocks longer than the configuration's transforms: never used
        const int l = (big ? kRowNBigMin : kRowNMin) + (int)(nl % nls);
        const uint32_t m = i >> (logE - l), c = i & ((1u << (logE - l)) - 1);
        const uint32_t kr = __brev(m) >> (32 - l);  // bitrev_l(m)
        const uint32_t e = (c * kr) << (root - n);  // c * kr < 2^logE <= 2^n: e < 2^root
        const uint32_t p = prime_of(NP, j);
        const uint2 a = tw.fs_lo[dir][j][e & (kFsEnt - 1)];
        const uint2 b = tw.fs_hi[dir][j][e >> kFsLog];
        const uint32_t w = mul_shoup(a.x, b.x, b.y, p);
        (big ? row_big : row)[k] = make_uint2(w, shoup_companion_dev(w, p, recip64_of(NP, j)));
    }
}

// Builds the tables of the configuration with NP primes into one allocation (*base).
template <int NP>
cudaError_t build_tables(uint2*& base, TwiddleTables& tw) {
    constexpr int root = root_log_of(NP);
    std::vector<uint2> h(small_entries(NP));
    auto stage_at = [&](int dir, int j) { return h.data() + (size_t)(dir * NP + j) * kStageEnt; };
    auto fs_at = [&](int which, int dir, int j) {
        return h.data() + (size_t)2 * NP * kStageEnt + ((size_t)(which * 2 + dir) * NP + j) * kFsEnt;
    };
    for (int dir = 0; dir < 2; ++dir)
        for (int j = 0; j < NP; ++j) {
            const uint32_t p = prime_of(NP, j);
            uint32_t wr = pow_mod(generator_of(NP, j), (uint64_t)(p - 1) >> root, p);  // primitive 2^root-th root
            if (dir == 1) wr = inv_mod(wr, p);
            const uint32_t w14 = pow_mod(wr, 1ull << (root - kStageLog), p);
            const uint32_t wrhi = pow_mod(wr, 1ull << kFsLog, p);
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
                b = b * wr % p;
                c = c * wrhi % p;
            }
            if (t3_entries(NP)) {
                // W of order 3 * 2^root (3 and 2^root both divide p - 1 for every wide prime)
                uint32_t W = pow_mod(generator_of(NP, j), (uint64_t)(p - 1) / (3ull << root), p);
                if (dir == 1) W = inv_mod(W, p);
                const uint32_t Whi = pow_mod(W, 1ull << kFsLog, p);
                uint2* l3 = h.data() + (size_t)2 * NP * (kStageEnt + 2 * kFsEnt) + ((size_t)(0 * 2 + dir) * NP + j) * kFsEnt;
                uint2* h3 = h.data() + (size_t)2 * NP * (kStageEnt + 2 * kFsEnt) + ((size_t)(1 * 2 + dir) * NP + j) * kFsEnt;
                uint64_t x = 1, y = 1;
                for (size_t i = 0; i < kFsEnt; ++i) {
                    l3[i] = make_uint2((uint32_t)x, shoup_companion((uint32_t)x, p));
                    h3[i] = make_uint2((uint32_t)y, shoup_companion((uint32_t)y, p));
                    x = x * W % p;
                    y = y * Whi % p;
                }
            }
        }
    cudaError_t e = pg::dev_malloc(&base, (small_entries(NP) + row_entries(NP) + row_big_entries(NP)) * sizeof(uint2));
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(base, h.data(), h.size() * sizeof(uint2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    tw = TwiddleTables{};
    tw.nprimes = NP;
    tw.root_log = root;
    for (int dir = 0; dir < 2; ++dir)
        for (int j = 0; j < NP; ++j) {
            tw.stage[dir][j] = base + (size_t)(dir * NP + j) * kStageEnt;
            tw.fs_lo[dir][j] = base + (size_t)2 * NP * kStageEnt + ((size_t)(0 * 2 + dir) * NP + j) * kFsEnt;
            tw.fs_hi[dir][j] = base + (size_t)2 * NP * kStageEnt + ((size_t)(1 * 2 + dir) * NP + j) * kFsEnt;
        }
    if (t3_entries(NP)) {
        for (int dir = 0; dir < 2; ++dir)
            for (int j = 0; j < NP; ++j) {
                const uint32_t p = prime_of(NP, j);
                tw.t3_lo[dir][j] = base + (size_t)2 * NP * (kStageEnt + 2 * kFsEnt) + ((size_t)(0 * 2 + dir) * NP + j) * kFsEnt;
                tw.t3_hi[dir][j] = base + (size_t)2 * NP * (kStageEnt + 2 * kFsEnt) + ((size_t)(1 * 2 + dir) * NP + j) * kFsEnt;
                // w3 = W^(2^root) of order 3 (the inverse direction's is its inverse)
                uint32_t W = pow_mod(generator_of(NP, j), (uint64_t)(p - 1) / (3ull << root), p);
                if (dir == 1) W = inv_mod(W, p);
                const uint64_t w3 = pow_mod(W, 1ull << root, p), w3sq = w3 * w3 % p;
                const uint64_t half = (p + 1) / 2;
                const uint32_t cc = (uint32_t)((w3 + p - w3sq) % p * half % p);
                tw.t3_c[dir][j] = make_uint2(cc, shoup_companion(cc, p));
                if (dir == 0) tw.t3_h[j] = make_uint2((uint32_t)half, shoup_companion((uint32_t)half, p));
            }
    }
    uint2* row = base + small_entries(NP);
    uint2* row_big = row + row_entries(NP);
    tw.row = row;
    tw.row_big = row_big;
    tw.row_layout = 0;
    fill_row_tables_kernel<NP><<<148 * 8, 256>>>(row, row_big, tw);
    return cudaGetLastError();
}
}  // namespace

static cudaError_t allow_big_tiles();

cudaError_t DeviceTables::build(int device) {
    (void)device;
    cudaError_t e = allow_big_tiles();
    if (e == cudaSuccess) e = build_tables<kNumPrimes>(base, tw);
    if (e == cudaSuccess) e = build_tables<kWidePrimes>(base_wide, tw_wide);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) wide = true;
    return e;
}

void DeviceTables::release() {
    if (base) dev_free(base);
    base = nullptr;
    if (base_wide) dev_free(base_wide);
    base_wide = nullptr;
    wide = false;
}

// ---------------------------------------------------------------- workspace
static cudaError_t grow(void** ptr, uint64_t bytes) {
    if (*ptr) dev_free(*ptr);
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
        if (pinned) pinned_free(pinned);
        pinned = nullptr;
        e = pinned_malloc(&pinned, 3 * n * 8);
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

cudaError_t Workspace::reserve_for(const DeviceTables& T, size_t na, size_t nb) {
    cudaError_t e = ensure_res(product_res_elems(T, na, nb));
    const uint64_t nwords = 2ull * (na + nb);
    const uint64_t bw = std::min<uint64_t>((uint64_t)kWideThreads * kWideWords, (uint64_t)kCrtThreads * kCrtWords);
    if (e == cudaSuccess) e = ensure_sync((nwords + bw - 1) / bw);
    return e;
}

void Workspace::release() {
    if (a_res) dev_free(a_res);
    if (b_res) dev_free(b_res);
    if (in_a) dev_free(in_a);
    if (in_b) dev_free(in_b);
    if (outl) dev_free(outl);
    if (sync) dev_free(sync);
    if (pinned) pinned_free(pinned);
    *this = Workspace{};
}

// ---------------------------------------------------------------- pass dispatch
cudaError_t launch_pass(const Plan& plan, int pass, bool inverse, Source src, Fuse fuse, const PassParams& prm,
                        const TwiddleTables& tw, cudaStream_t st) {
    if (tw.nprimes == kWidePrimes) return launch_pass_wide(plan, pass, inverse, src, fuse, prm, tw, st);
    return launch_pass_np<kNumPrimes>(plan, pass, inverse, src, fuse, prm, tw, st);
}

static cudaError_t allow_big_tiles() {
    cudaError_t e = allow_big_tiles_np<kNumPrimes>();
    if (e == cudaSuccess) e = allow_big_tiles_wide();
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(crt_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kFixMaxBlocks * sizeof(uint32_t)));
    return e;
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
// Garner constants of the wide configuration for transforms of 2^logL points (see crt5).
// three: the transform has 3 * 2^logL points (its 1/L includes 1/3).
static CrtWideConsts make_crt_wide_consts(int logL, bool three = false) {
    CrtWideConsts K{};
    uint32_t q[kWidePrimes];
    for (int i = 0; i < kWidePrimes; ++i) q[i] = prime_of(kWidePrimes, i);
    // P_m = q_0 ... q_{m-1} as 32-bit words, and P_m mod q_k
    uint32_t Pw[kWidePrimes][kWidePrimes] = {};
    Pw[0][0] = 1;
    for (int m = 1; m < kWidePrimes; ++m) {
        uint64_t carry = 0;
        for (int w = 0; w < kWidePrimes; ++w) {
            const uint64_t t = (uint64_t)Pw[m - 1][w] * q[m - 1] + carry;
            Pw[m][w] = (uint32_t)t;
            carry = t >> 32;
        }
    }
    auto pmod = [&](int m, uint32_t p) {  // P_m mod p, Horner over the words
        uint64_t r = 0;
        for (int w = kWidePrimes - 1; w >= 0; --w) r = ((r << 32) + Pw[m][w]) % p;
        return (uint32_t)r;
    };
    for (int kk = 0; kk < kWidePrimes; ++kk) {
        const uint32_t p = q[kk];
        const uint64_t linv = inv_mod((uint32_t)((uint64_t)pow_mod(2, (uint64_t)logL, p) * (three ? 3 : 1) % p), p);
        const uint64_t scale = linv * pow_mod(2, 32, p) % p;  // 1/L and the 2^-32 of the pointwise product
        const uint64_t pkinv = inv_mod(pmod(kk, p), p);
        K.c[kk] = (uint32_t)(scale * pkinv % p);
        K.cp[kk] = shoup_companion(K.c[kk], p);
        for (int m = 0; m < kk; ++m) {
            K.k[m][kk] = (uint32_t)((uint64_t)pmod(m, p) * pkinv % p);
            K.kp[m][kk] = shoup_companion(K.k[m][kk], p);
        }
    }
    for (int m = 0; m < kWidePrimes; ++m)
        for (int w = 0; w < kWidePrimes - 1; ++w) K.Pw[m][w] = Pw[m][w];
    // P_5 = P_4 q_4 (five words), floor(P_5 / 2) and its Garner digits (remainders of successive
    // divisions by q_0 .. q_4)
    uint32_t P5[kWidePrimes] = {};
    {
        uint64_t carry = 0;
        for (int w = 0; w < kWidePrimes; ++w) {
            const uint64_t t = (uint64_t)Pw[kWidePrimes - 1][w] * q[kWidePrimes - 1] + carry;
            P5[w] = (uint32_t)t;
            carry = t >> 32;
        }
    }
    uint32_t half[kWidePrimes];
    for (int w = 0; w < kWidePrimes; ++w)
        half[w] = (P5[w] >> 1) | (w + 1 < kWidePrimes ? (P5[w + 1] << 31) : 0u);
    for (int kk = 0; kk < kWidePrimes; ++kk) {
        uint64_t r = 0;
        for (int w = kWidePrimes - 1; w >= 0; --w) {
            const uint64_t cur = (r << 32) | half[w];
            half[w] = (uint32_t)(cur / q[kk]);
            r = cur % q[kk];
        }
        K.h[kk] = (uint32_t)r;
    }
    for (int w = 0; w < kWidePrimes; ++w) K.Pi[w] = P5[w];
    return K;
}

uint64_t crt_wide_block_words() { return (uint64_t)kWideThreads * kWideWords; }

// Wide CRT: every block independently (words with carry-in 0, block transfer functions into
// c.status), then a scan per job and the carries applied.
cudaError_t launch_crt_wide(CrtParams c, uint64_t jobs, uint64_t bpj, int logL, cudaStream_t st, uint64_t* launches,
                            bool three) {
    const bool top_ok = c.top_ok != 0;
    if (!jobs || !bpj) return cudaSuccess;
    if (bpj > kFixMaxBlocks) return cudaErrorInvalidValue;
    c.blocks_per_job = bpj;
    const uint64_t blocks = jobs * bpj;
    crt_wide_kernel<<<(unsigned)blocks, kWideThreads, 0, st>>>(c, make_crt_wide_consts(logL, three));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (bpj <= kScanWarpMax)
        crt_scan_warp_kernel<<<(unsigned)((jobs * 32 + 255) / 256), 256, 0, st>>>(c.status, bpj, jobs, c.error,
                                                                                 top_ok ? 1 : 0);
    else
        crt_scan_kernel<<<(unsigned)jobs, kFixThreads, bpj * sizeof(uint32_t), st>>>(c.status, bpj, c.error,
                                                                                    top_ok ? 1 : 0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    crt_apply_kernel<<<(unsigned)((blocks + kApplyWarps - 1) / kApplyWarps), 32 * kApplyWarps, 0, st>>>(
        c, blocks, crt_wide_block_words());
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    uint64_t n = 3;
    if (c.merge == 1 || (c.merge == 0 && c.dlen)) {
        crt_len_kernel<<<(unsigned)((jobs * 32 + 255) / 256), 256, 0, st>>>(c, jobs, crt_wide_block_words());
        e = cudaGetLastError();
        ++n;
    }
    if (launches) *launches += n;
    return e;
}

// The product's launch sequence in one configuration: 32-bit coefficients over three primes, or
// (wide) 64-bit coefficients over five primes with the tables T.tw_wide.
static cudaError_t enqueue_impl(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                                const uint64_t* d_b, size_t nb, int logL, uint64_t nwords, uint64_t* d_out,
                                cudaStream_t st, uint64_t* launches, bool wide = false) {
    const bool square = (d_b == nullptr);
    if (square) nb = na;
    const int np = wide ? kWidePrimes : kNumPrimes;
    const TwiddleTables& tw = wide ? T.tw_wide : T.tw;
    const Source limbs = wide ? Source::Limbs64 : Source::Limbs;
    const uint64_t coef_per_limb = wide ? 1 : 2;
    const Plan plan = wide ? T.plan_wide(logL) : T.plan(logL);
    const uint64_t L = 1ull << logL;
    cudaError_t e = W.ensure_res(np * L);
    if (e != cudaSuccess) return e;
    const uint64_t block_words = wide ? (uint64_t)kWideThreads * kWideWords : (uint64_t)kCrtThreads * kCrtWords;
    const uint64_t crt_blocks = (nwords + block_words - 1) / block_words;
    e = W.ensure_sync(crt_blocks);
    if (e != cudaSuccess) return e;

    auto base = [&](uint32_t* data, const uint64_t* limbs, uint64_t ncoef) {
        PassParams p{};
        p.data = data;
        p.out = data;
        p.other = nullptr;
        p.other_stride = np * L;
        p.words_stride = 0;
        p.words = reinterpret_cast<const uint32_t*>(limbs);
        p.ncoef = ncoef;
        p.L = L;
        p.logL = logL;
        p.job_stride = np * L;
        p.njobs = 1;
        p.merge = 0;
        p.error = W.sync;  // the product's error word (also the CRT's)
        return p;
    };
    auto set_pass = [&](PassParams& p, int i) { pg::set_pass(p, plan, i); };

    const int last = plan.npass - 1;
    // Operand a: full forward transform (all but the last pass when squaring).
    {
        PassParams p = base(W.a_res, d_a, coef_per_limb * na);
        const int upto = square ? last : plan.npass;
        for (int i = 0; i < upto; ++i) {
            set_pass(p, i);
            Fuse f = Fuse::None;
            e = launch_pass(plan, i, false, i == 0 ? limbs : Source::Residues, f, p, tw, st);
            if (e != cudaSuccess) return e;
        }
        if (square) {
            set_pass(p, last);
            e = launch_pass(plan, last, false, last == 0 ? limbs : Source::Residues, Fuse::SqrInverse, p,
                            tw, st);
            if (e != cudaSuccess) return e;
        }
    }
    uint32_t* prod = W.a_res;
    if (!square) {
        PassParams p = base(W.b_res, d_b, coef_per_limb * nb);
        for (int i = 0; i < last; ++i) {
            set_pass(p, i);
            e = launch_pass(plan, i, false, i == 0 ? limbs : Source::Residues, Fuse::None, p, tw, st);
            if (e != cudaSuccess) return e;
        }
        set_pass(p, last);
        p.other = W.a_res;
        e = launch_pass(plan, last, false, last == 0 ? limbs : Source::Residues, Fuse::MulInverse, p, tw,
                        st);
        if (e != cudaSuccess) return e;
        prod = W.b_res;
    }
    // Inverse strided passes, last strided pass first.
    {
        PassParams p = base(prod, nullptr, 0);
        for (int i = last - 1; i >= 0; --i) {
            set_pass(p, i);
            e = launch_pass(plan, i, true, Source::Residues, Fuse::None, p, tw, st);
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
    if (wide) {
        e = launch_crt_wide(c, 1, crt_blocks, logL, st);
    } else {
        c.k = make_crt_consts(logL);
        e = launch_crt(c, crt_blocks, st, nwords);
    }
    if (e != cudaSuccess) return e;
    if (launches) *launches += (square ? plan.npass : 2 * plan.npass) + (plan.npass - 1) + (wide ? 3 : 1);
    return cudaGetLastError();
}

// The smallest na + nb (limbs) that runs in the wide configuration: the context's value, or the
// environment's PG_WIDE_MIN_LIMBS (read on every call, so that tests can move the boundary).
uint64_t wide_min_limbs(const DeviceTables& T) {
    if (const char* e = std::getenv("PG_WIDE_MIN_LIMBS")) return std::strtoull(e, nullptr, 10);
    return T.wide_min_limbs;
}

bool use_wide(const DeviceTables& T, uint64_t na, uint64_t nb) {
    const uint64_t wmin = T.wide ? wide_min_limbs(T) : 0;
    return wmin && na + nb >= wmin && product_logL_wide(na, nb) <= kWideMaxLogL;
}

// A wide product as a transform of L = 3 * 2^m points: a radix-3 step from the limbs into three rows
// of 2^m points (rows as jobs: [row][prime][2^m]), the 2^m-point passes of the tuned wide plan over the
// three rows (the pointwise product fused into b's last forward pass as usual), their inverse, the
// inverse radix-3 step into [prime][3 * 2^m] and the CRT with 1/L = 1/(3 * 2^m). Transforms of this
// length use roots of order 3 * 2^25, which every wide prime has.
static cudaError_t enqueue_impl3(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                                 const uint64_t* d_b, size_t nb, int logM, uint64_t nwords, uint64_t* d_out,
                                 cudaStream_t st, uint64_t* launches) {
    const bool square = (d_b == nullptr);
    if (square) nb = na;
    constexpr int np = kWidePrimes;
    const TwiddleTables& tw = T.tw_wide;
    if (!tw.t3_lo[0][0] || logM < kMinLogL || logM > kWideMaxLogL - 1) return cudaErrorInvalidValue;
    const Plan plan = T.plan_wide(logM);
    const uint64_t M = 1ull << logM, L3 = 3 * M, rows_stride = (uint64_t)np * M;
    cudaError_t e = W.ensure_res(np * L3);
    if (e != cudaSuccess) return e;
    const uint64_t block_words = (uint64_t)kWideThreads * kWideWords;
    const uint64_t crt_blocks = (nwords + block_words - 1) / block_words;
    e = W.ensure_sync(crt_blocks);
    if (e != cudaSuccess) return e;
    const unsigned r3_grid = (unsigned)(((M / 4 + kR3Threads - 1) / kR3Threads) * np);
    auto rows = [&](uint32_t* data) {
        PassParams p{};
        p.data = data;
        p.out = data;
        p.L = M;
        p.logL = logM;
        p.job_stride = rows_stride;
        p.other_stride = rows_stride;
        p.njobs = 3;
        p.merge = 0;
        p.error = W.sync;
        return p;
    };
    const int last = plan.npass - 1;
    uint64_t n = 0;
    // a: radix-3 step from the limbs, then the 2^m-point forward passes (the last fused with the
    // squaring when b is a)
    radix3_fwd_kernel<np><<<r3_grid, kR3Threads, 0, st>>>(reinterpret_cast<const uint32_t*>(d_a), na, W.a_res, M, logM,
                                                         rows_stride, tw);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    ++n;
    {
        PassParams p = rows(W.a_res);
        for (int i = 0; i < plan.npass; ++i) {
            set_pass(p, plan, i);
            const Fuse f = (square && i == last) ? Fuse::SqrInverse : Fuse::None;
            if ((e = launch_pass(plan, i, false, Source::Residues, f, p, tw, st)) != cudaSuccess) return e;
            ++n;
        }
    }
    uint32_t* prod = W.a_res;
    if (!square) {
        radix3_fwd_kernel<np><<<r3_grid, kR3Threads, 0, st>>>(reinterpret_cast<const uint32_t*>(d_b), nb, W.b_res, M,
                                                             logM, rows_stride, tw);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        ++n;
        PassParams p = rows(W.b_res);
        for (int i = 0; i < plan.npass; ++i) {
            set_pass(p, plan, i);
            if (i == last) p.other = W.a_res;
            const Fuse f = i == last ? Fuse::MulInverse : Fuse::None;
            if ((e = launch_pass(plan, i, false, Source::Residues, f, p, tw, st)) != cudaSuccess) return e;
            ++n;
        }
        prod = W.b_res;
    }
    {
        PassParams p = rows(prod);
        for (int i = last - 1; i >= 0; --i) {
            set_pass(p, plan, i);
            if ((e = launch_pass(plan, i, true, Source::Residues, Fuse::None, p, tw, st)) != cudaSuccess) return e;
            ++n;
        }
    }
    // inverse radix-3 step into the other buffer ([prime][3M], natural order), then the CRT
    uint32_t* coef = (prod == W.a_res) ? W.b_res : W.a_res;
    radix3_inv_kernel<np><<<r3_grid, kR3Threads, 0, st>>>(prod, coef, M, logM, rows_stride, tw);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    ++n;
    e = cudaMemsetAsync(W.sync + 1, 0, (crt_blocks + 1) * 4, st);
    if (e != cudaSuccess) return e;
    CrtParams c{};
    c.res = coef;
    c.L = L3;
    c.nwords = nwords;
    c.out = reinterpret_cast<uint32_t*>(d_out);
    c.ticket = W.sync + 1;
    c.status = W.sync + 2;
    c.error = W.sync;
    c.merge = 0;
    e = launch_crt_wide(c, 1, crt_blocks, logM, st, &n, true);
    if (launches) *launches += n;
    return e;
}

// Whether a wide product of n = na + nb - 1 coefficients takes a 3 * 2^m-point transform: when that
// length (3/4 of the next power of two) holds it, for m >= kR3MinLog (PG_RADIX3=0: never). Measured
// on a B200 (the multiply sweep): 2-7% faster from m = 20 on, slower below (at m = 17-19 the two
// radix-3 steps, which cost about one transform pass each, outweigh the quarter of the points saved).
constexpr int kR3MinLog = 20;
// PG_RADIX3=k (k >= kMinLogL) moves the threshold to m >= k (tests use it to reach the path at small
// sizes).
static int radix3_logM(uint64_t ncoef) {
    int mmin = kR3MinLog;
    if (const char* e = std::getenv("PG_RADIX3")) {
        const long v = std::strtol(e, nullptr, 10);
        if (v == 0) return -1;
        if (v >= kMinLogL) mmin = (int)v;
    }
    const int l2 = ceil_log2(ncoef);
    const int m = l2 - 2;
    if (m < mmin || m > kWideMaxLogL - 1) return -1;
    return (3ull << m) >= ncoef ? m : -1;
}

cudaError_t enqueue_product_config(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                                   const uint64_t* d_b, size_t nb, uint64_t* d_out, cudaStream_t st, bool wide) {
    const size_t mb = d_b ? nb : na;
    if (wide) {
        if (!T.wide || product_logL_wide(na, mb) > kWideMaxLogL) return cudaErrorInvalidValue;
        return enqueue_impl(T, W, d_a, na, d_b, nb, product_logL_wide(na, mb), 2ull * (na + mb), d_out, st, nullptr,
                            true);
    }
    return enqueue_impl(T, W, d_a, na, d_b, nb, product_logL(na, mb), 2ull * (na + mb), d_out, st, nullptr);
}

cudaError_t enqueue_product(const DeviceTables& T, Workspace& W, const uint64_t* d_a, size_t na,
                            const uint64_t* d_b, size_t nb, uint64_t* d_out, cudaStream_t st,
                            uint64_t* launches) {
    const size_t mb = d_b ? nb : na;
    // Configuration from the proven bound: the wide one holds every product of up to 2^25 limbs
    // (min(na, nb) (2^64 - 1)^2 < q0 ... q4 for min(na, nb) < 2^25.35) in half the transform length.
    const uint64_t wmin = T.wide ? wide_min_limbs(T) : 0;
    if (wmin && na + mb >= wmin && product_logL_wide(na, mb) <= kWideMaxLogL) {
        const int m3 = radix3_logM((uint64_t)(na + mb) - 1);
        if (m3 >= 0) return enqueue_impl3(T, W, d_a, na, d_b, nb, m3, 2ull * (na + mb), d_out, st, launches);
        return enqueue_impl(T, W, d_a, na, d_b, nb, product_logL_wide(na, mb), 2ull * (na + mb), d_out, st, launches,
                            true);
    }
    return enqueue_impl(T, W, d_a, na, d_b, nb, product_logL(na, mb), 2ull * (na + mb), d_out, st, launches);
}

uint64_t product_res_elems(const DeviceTables& T, size_t na, size_t nb) {
    const uint64_t wmin = T.wide ? wide_min_limbs(T) : 0;
    if (wmin && na + nb >= wmin && product_logL_wide(na, nb) <= kWideMaxLogL) {
        const int m3 = radix3_logM((uint64_t)(na + nb) - 1);
        if (m3 >= 0) return (uint64_t)kWidePrimes * 3 * (1ull << m3);
        return (uint64_t)kWidePrimes << product_logL_wide(na, nb);
    }
    return (uint64_t)kNumPrimes << product_logL(na, nb);
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
