// Device-resident finish of the pi computation: the final formula and the decimal
// conversion with every operand in HBM (DevArith, devnum.h), products on the NTT engine.
//
//   final formula   pi 10^d = floor(426880 Q sqrt(10005) 10^d / R)  (reference:
//                   src/engine/pi_engine.cpp:437-491, mpf_sqrt / mpf_div / mpf_mul at
//                   d * log2(10) + 64 bits). Here: Newton reciprocal of R and Newton inverse
//                   square root of 10005 at doubling precision, each finished by an exact
//                   integer correction, 5^d by squaring, three truncated products, and a floor
//                   that is accepted only when the rigorous error bound keeps it away from an
//                   integer (otherwise the guard grows and the formula reruns).
//   conversion      the decimal digits of an integer < 10^n (reference: src/io/base_converter.cpp
//                   PowerTree::build + parallel_convert, :48-147): the number is split in
//                   halves of 2^j digits by q = floor(c * inv / 2^(2K)) with inv = floor(2^(2K)
//                   / 10^(2^j)), r = c - q 10^(2^j) and at most two corrections; every level
//                   of the split runs batched over all chunks of that level (two shared-operand
//                   batched products, a shift, a subtraction, the corrections), down to
//                   1024-digit chunks written as ASCII by one thread each.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <exception>
#include <functional>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <dirent.h>
#include <sys/stat.h>
#include <unistd.h>

#include <set>

#include "../../include/pi_b200.h"
#include "bigint.cuh"
#include "ckpt_io.h"
#include "devnum.h"
#include "host_div.h"

namespace pg {

const DeviceTables& ctx_tables(pg_ctx* c);
Workspace& ctx_workspace(pg_ctx* c);
cudaStream_t ctx_stream(pg_ctx* c);
std::mutex& ctx_mutex(pg_ctx* c);
uint64_t* ctx_launches(pg_ctx* c);
void ctx_set_error(pg_ctx* c, const std::string& msg);
int ctx_device(pg_ctx* c);
pg_status bs_run_locked(pg_ctx* ctx, unsigned long a, unsigned long b, LevelView& root, uint32_t hl[3],
                        bool need_P = true, const std::function<void()>* while_running = nullptr);
bool trace_on();

// ------------------------------------------------------------------ batched shared-operand product
// out_j[0 .. na + nb) = a_j * b for j < njobs; a_j at a + j * sa (na limbs), out_j at
// out + j * so. The shared operand is transformed once; the batch's last forward pass fuses the
// pointwise product with it (other_stride 0) and the CRT writes every job's words.
struct SharedProduct {
    uint32_t* res = nullptr;
    uint64_t res_cap = 0;
    uint32_t* bres = nullptr;
    uint64_t bres_cap = 0;
    uint32_t* sync = nullptr;
    uint64_t sync_cap = 0;
    uint32_t* errw = nullptr;
    uint32_t* flags = nullptr;  // per-chunk flags of the conversion, kept across calls
    uint64_t flags_cap = 0;
    char* digits = nullptr;     // the conversion's ASCII output, kept across calls
    uint64_t digits_cap = 0;

    ~SharedProduct() {
        if (res) dev_free(res);
        if (bres) dev_free(bres);
        if (sync) dev_free(sync);
        if (errw) dev_free(errw);
        if (flags) dev_free(flags);
        if (digits) dev_free(digits);
    }

    static void grow(uint32_t** p, uint64_t& cap, uint64_t words, cudaStream_t st) {
        if (words <= cap) return;
        cudaStreamSynchronize(st);
        const uint64_t want = std::max(words, cap + cap / 2);
        if (*p) dev_free(*p);
        *p = nullptr;
        cap = 0;
        cudaError_t e = pg::dev_malloc((void**)p, want * 4);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw DevError(e == cudaErrorMemoryAllocation ? PG_ERR_OOM : PG_ERR_DEVICE, "batched product buffers");
        }
        cap = want;
    }

    // out[j] = a[j] * b for njobs operands a[j] (a + j sa, na limbs each) and one shared b: b is
    // transformed once; the jobs run in chunks of the residue budget, in the configuration the
    // product's size selects (use_wide). With cyc = 2^c limbs (na, nb <= cyc) the product is
    // cyclic instead: out[j] receives cyc limbs, a[j] b modulo 2^(64 cyc) - 1 up to the carries
    // near its bottom and top (a middle product: the wrapped-around part lands in the low limbs,
    // and the carry out of the top is dropped).
    void run(const DeviceTables& T, cudaStream_t st, uint64_t* launches, const uint64_t* a, uint64_t sa, uint64_t na,
             uint64_t njobs, const uint64_t* b, uint64_t nb, uint64_t* out, uint64_t so, uint64_t cyc = 0) {
        if (!njobs) return;
        // a cyclic product's length is its own: the wide configuration holds it up to 2^25 limbs
        const uint64_t wmin = T.wide ? wide_min_limbs(T) : 0;
        const bool wide = cyc ? (wmin && na + nb >= wmin && ceil_log2(cyc) <= kWideMaxLogL) : use_wide(T, na, nb);
        if (cyc && (na > cyc || nb > cyc || (cyc & (cyc - 1))))
            throw DevError(PG_ERR_INTERNAL, "cyclic product operands longer than its length");
        if (!wide && (cyc ? ceil_log2(2 * cyc) : product_logL(na, nb)) > split_logL())
            throw DevError(PG_ERR_TOO_LARGE, "batched product too long");
        if ((sa | so) & 1) throw DevError(PG_ERR_INTERNAL, "batched product strides must be even");
        if (!errw) {
            if (pg::dev_malloc((void**)&errw, 4) != cudaSuccess) throw DevError(PG_ERR_OOM, "error word");
            cudaMemsetAsync(errw, 0, 4, st);
        }
        const int logL = cyc ? std::max(ceil_log2(wide ? cyc : 2 * cyc), kMinLogL)
                             : (wide ? product_logL_wide(na, nb) : product_logL(na, nb));
        const Plan plan = wide ? T.plan_wide(logL) : T.plan(logL);
        const TwiddleTables& tw = wide ? T.tw_wide : T.tw;
        const Source limbs = wide ? Source::Limbs64 : Source::Limbs;
        const uint64_t per_limb = wide ? 1 : 2;  // transform coefficients per limb
        const int last = plan.npass - 1;
        const uint64_t L = 1ull << logL, per = (wide ? kWidePrimes : kNumPrimes) * L;
        auto check = [](cudaError_t e) {
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw DevError(PG_ERR_DEVICE, std::string("batched product: ") + cudaGetErrorString(e));
            }
        };
        // shared operand: full forward transform
        grow(&bres, bres_cap, per, st);
        {
            PassParams p{};
            p.data = bres;
            p.out = bres;
            p.words = reinterpret_cast<const uint32_t*>(b);
            p.ncoef = per_limb * nb;
            p.error = errw;
            p.L = L;
            p.logL = logL;
            p.job_stride = per;
            p.other_stride = per;
            p.njobs = 1;
            for (int i = 0; i < plan.npass; ++i) {
                set_pass(p, plan, i);
                check(launch_pass(plan, i, false, i == 0 ? limbs : Source::Residues, Fuse::None, p, tw, st));
                ++*launches;
            }
        }
        const uint64_t budget = 256ull << 20;  // residue words per chunk of jobs
        const uint64_t m_max = std::max<uint64_t>(1, budget / per);
        const uint64_t nwords = cyc ? 2 * cyc : 2 * (na + nb);
        const uint64_t block_words = wide ? crt_wide_block_words() : (uint64_t)kCrtThreads * kCrtWords;
        const uint64_t bpj = (nwords + block_words - 1) / block_words;
        for (uint64_t j0 = 0; j0 < njobs; j0 += m_max) {
            const uint64_t m = std::min(m_max, njobs - j0);
            grow(&res, res_cap, m * per, st);
            PassParams p{};
            p.data = res;
            p.out = res;
            p.words = reinterpret_cast<const uint32_t*>(a + j0 * sa);
            p.words_stride = 2 * sa;
            p.ncoef = per_limb * na;
            p.error = errw;
            p.L = L;
            p.logL = logL;
            p.job_stride = per;
            p.other = bres;
            p.other_stride = 0;
            p.njobs = (uint32_t)m;
            for (int i = 0; i < plan.npass; ++i) {
                set_pass(p, plan, i);
                check(launch_pass(plan, i, false, i == 0 ? limbs : Source::Residues,
                                  i == last ? Fuse::MulInverse : Fuse::None, p, tw, st));
                ++*launches;
            }
            for (int i = last - 1; i >= 0; --i) {
                set_pass(p, plan, i);
                check(launch_pass(plan, i, true, Source::Residues, Fuse::None, p, tw, st));
                ++*launches;
            }
            CrtParams c{};
            c.res = res;
            c.res_stride = per;
            c.L = L;
            c.nwords = nwords;
            c.out = reinterpret_cast<uint32_t*>(out + j0 * so);
            c.out_stride = 2 * so;
            c.error = errw;
            c.merge = 0;
            c.top_ok = cyc ? 1 : 0;
            if (wide) {
                grow(&sync, sync_cap, m * bpj, st);
                c.status = sync;
                check(launch_crt_wide(c, m, bpj, logL, st, launches));
            } else {
                grow(&sync, sync_cap, m + m * bpj, st);
                check(cudaMemsetAsync(sync, 0, (m + m * bpj) * 4, st));
                c.ticket = sync;
                c.status = sync + m;
                c.blocks_per_job = bpj;
                c.k = make_crt_consts(logL);
                check(launch_crt(c, m * bpj, st, nwords));
                ++*launches;
            }
        }
    }

    uint32_t error(cudaStream_t st) {
        uint32_t h = 0;
        if (!errw) return 0;
        cudaMemcpyAsync(&h, errw, 4, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        return h;
    }
};

// Pinned host staging for checkpoint files: two buffers, so that the copy of one chunk runs
// while the other is read from or written to the file.
struct CkptStaging {
    static constexpr size_t kChunk = (size_t)32 << 20;  // bytes per buffer
    char* buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~CkptStaging() {
        for (int i = 0; i < 2; ++i) {
            if (buf[i]) pinned_free(buf[i]);
            if (ev[i]) cudaEventDestroy(ev[i]);
        }
    }
    void ensure() {
        for (int i = 0; i < 2; ++i) {
            if (!buf[i] && pinned_malloc(&buf[i], kChunk) != cudaSuccess)
                throw DevError(PG_ERR_OOM, "checkpoint staging buffer");
            if (!ev[i] && cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess)
                throw DevError(PG_ERR_DEVICE, "checkpoint staging event");
        }
    }
};

// Per-context state of the device finish, kept across calls: the arithmetic pool, the
// batched-product buffers and the checkpoint staging; and a second stream with its own product
// workspace and pool, on which a helper thread computes what does not depend on the series
// (sqrt(10005), powers of ten) while the splitting and the reciprocal run.
struct FinishState {
    DevPool pool;
    SharedProduct sp;
    CkptStaging stage;
    DevPool pool2;
    Workspace ws2;
    cudaStream_t st2 = nullptr;
    ~FinishState() {
        ws2.release();
        if (st2) cudaStreamDestroy(st2);
    }
};
// The trace's high-water marks of the finish's buffers (bytes held at the end of a call).
void trace_buffers(pg_ctx* ctx, FinishState& fs) {
    auto pool_bytes = [](const DevPool& p) {
        size_t b = 0;
        for (const auto& x : p.all_) b += x.second * 8;
        return std::make_pair(p.all_.size(), b);
    };
    const Workspace& w = ctx_workspace(ctx);
    const auto p1 = pool_bytes(fs.pool), p2 = pool_bytes(fs.pool2);
    FreeList& f = free_list();
    size_t pend = 0;
    {
        std::lock_guard<std::mutex> lk(f.mu);
        pend = f.pending_bytes;
    }
    std::fprintf(stderr,
                 "[pi_device] buffers: workspace %.1f MB residues + %.1f MB limbs, helper workspace %.1f MB residues, "
                 "shared product %.1f + %.1f MB, pool %zu numbers %.1f MB, helper pool %zu numbers %.1f MB, "
                 "deferred frees %.1f MB\n",
                 2e-6 * 4 * w.res_cap, 3e-6 * 8 * w.limb_cap, 2e-6 * 4 * fs.ws2.res_cap, 4e-6 * fs.sp.res_cap,
                 4e-6 * fs.sp.bres_cap, p1.first, 1e-6 * p1.second, p2.first, 1e-6 * p2.second, 1e-6 * pend);
}

FinishState* finish_state_new() { return new FinishState; }
void finish_state_delete(FinishState* f) { delete f; }
FinishState* ctx_finish(pg_ctx* c);

namespace {

typedef unsigned __int128 u128;

// A DevNum released when it goes out of scope.
struct Num {
    DevArith& A;
    DevNum v;
    explicit Num(DevArith& a) : A(a) {}
    ~Num() { A.release(v); }
    Num(const Num&) = delete;
    Num& operator=(const Num&) = delete;
    operator DevNum&() { return v; }
};

// Allocation counters of the process (dev_alloc.h), for the trace.
struct AllocSnap {
    uint64_t n, bytes, ns, frees, free_ns, pinned, pinned_ns;
    static AllocSnap now() {
        const AllocStats& s = alloc_stats();
        return {s.allocs.load(), s.alloc_bytes.load(), s.alloc_ns.load(), s.frees.load(), s.free_ns.load(),
                s.pinned.load(), s.pinned_ns.load()};
    }
};

// " (N cudaMalloc, X MB, T ms; ...)" for the allocations made since `a`, or "" when none.
std::string alloc_delta(const AllocSnap& a) {
    const AllocSnap b = AllocSnap::now();
    if (b.n == a.n && b.frees == a.frees && b.pinned == a.pinned) return "";
    char buf[192];
    std::snprintf(buf, sizeof buf, " (%llu cudaMalloc, %.1f MB, %.3f ms; %llu cudaFree, %.3f ms; %llu pinned, %.3f ms)",
                  (unsigned long long)(b.n - a.n), (double)(b.bytes - a.bytes) / 1e6, (double)(b.ns - a.ns) / 1e6,
                  (unsigned long long)(b.frees - a.frees), (double)(b.free_ns - a.free_ns) / 1e6,
                  (unsigned long long)(b.pinned - a.pinned), (double)(b.pinned_ns - a.pinned_ns) / 1e6);
    return buf;
}

struct Timer {
    const char* what;
    std::chrono::steady_clock::time_point t0;
    AllocSnap a0;
    explicit Timer(const char* w) : what(w), t0(std::chrono::steady_clock::now()), a0(AllocSnap::now()) {}
    double ms() const { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); }
    ~Timer() {
        if (trace_on()) std::fprintf(stderr, "[pi_device] %s: %.3f ms%s\n", what, ms(), alloc_delta(a0).c_str());
    }
};

void upload_u128(DevArith& A, DevNum& x, u128 v) {
    uint64_t w[2] = {(uint64_t)v, (uint64_t)(v >> 64)};
    A.upload(x, w, 2, 1);
}

u128 download_u128(DevArith& A, const DevNum& x) {
    A.exact(const_cast<DevNum&>(x));
    if (x.n > 2) throw DevError(PG_ERR_INTERNAL, "download_u128: value too long");
    uint64_t w[2] = {0, 0};
    if (x.n) A.download(x, w);
    return ((u128)w[1] << 64) | w[0];
}

u128 isqrt128(u128 v) {
    if (v == 0) return 0;
    const int bl = (v >> 64) ? 128 - __builtin_clzll((uint64_t)(v >> 64)) : 64 - __builtin_clzll((uint64_t)v);
    u128 x = (u128)1 << ((bl + 1) / 2);  // > sqrt(v): v < 2^bl
    for (;;) {                           // Newton from above decreases to floor(sqrt(v))
        const u128 y = (x + v / x) / 2;
        if (y >= x) break;
        x = y;
    }
    while (x > v / x) --x;                // x^2 > v, without overflow
    while (x + 1 <= v / (x + 1)) ++x;     // (x+1)^2 <= v
    return x;
}

// Z = floor(2^(2k) / R), k = bits(R) (R > 0). Newton doubling: Zh = floor(2^(2h) / Rh) for the
// top h = k/2 + 32 bits of R, Z0 = Zh 2^(k-h), one Newton step, then the exact correction
// 0 <= 2^(2k) - R Z < R.
// Transform length (log2 of L words) of a wrapped product whose modulus M = 2^(32 L) - 1
// leaves room for a value of `bits` bits and a sign (32 L >= bits + 2), with operands of na, nb
// limbs fitting the transform; 0 when that is not shorter than the full product's transform.
int wrap_logL(size_t bits, size_t na, size_t nb) {
    // below 2^17 points the product is cheaper than the fold's and centring's extra host waits
    if (product_logL(na, nb) <= 17) return 0;
    int l = kMinLogL;
    while (((uint64_t)32 << l) < (uint64_t)bits + 2 || ((uint64_t)1 << l) < 2 * (uint64_t)std::max(na, nb)) ++l;
    if (l > split_logL() || l >= product_logL(na, nb)) return 0;
    return l;
}

// e from its representative in (-M, M), M = 2^(32 L) - 1, when the value itself has
// |e| < 2^(32 L - 2): a representative with 32 L - 1 or more bits is off by M.
void centre(DevArith& A, DevNum& e, int logL) {
    const size_t lbits = (size_t)32 << logL;
    if (A.bits(e) + 1 < lbits) return;
    Num M(A);
    A.set_pow2(M, lbits);
    A.add_si(M, M, -1);
    if (e.sign > 0)
        A.sub(e, e, M);
    else
        A.add(e, e, M);
}

// e = 2^p - x (|e| < 2^(bits)) with x a product known modulo M = 2^(32 L) - 1 (xm in [0, M]).
void residue_diff(DevArith& A, DevNum& e, size_t p, const DevNum& xm, int logL) {
    A.set_pow2(e, p % ((size_t)32 << logL));  // 2^(32 L) = 1 mod M
    A.sub(e, e, xm);
    centre(A, e, logL);
}

// Z = floor(2^(2k) / R), k = bits(R). With exact == false the top step's correction is skipped:
// then |Z - 2^(2k)/R| < 2. The ideal Newton update Z0 + Z0 E / 2^(2k) has error eps^2 / z* with
// eps = z* - Z0, |eps| <= 2^(k-h+2) and z* = 2^(2k)/R > 2^k, i.e. below 2^(k - 2h + 4) = 2^-60;
// dropping E's low bits costs < 1/2 and the floor < 1 (the lower levels stay exact).
// Reciprocals of up to this many bits are divided on the host (exact): the Newton levels below it
// (k -> k/2 + 32 down to 64 bits, a dozen of them) would cost more in launches and host waits.
// Knuth's division takes ~110 us at 12288 bits on one host core, a device level of 5-10 kbits
// 0.3-0.7 ms while the helper stream's long kernels share the device.
constexpr size_t kHostRecipBits = 12288;

void recip_floor(DevArith& A, DevNum& Z, const DevNum& R, bool exact = true) {
    const size_t k = A.bits(R);
    if (k == 0 || R.sign < 0) throw DevError(PG_ERR_BAD_ARG, "recip_floor: R must be positive");
    if (k > 64 && k <= kHostRecipBits) {
        std::vector<uint64_t> r((k + 63) / 64);
        A.download(R, r.data());
        const std::vector<uint64_t> z = host_pow2_div(2 * k, r);
        A.upload(Z, z.data(), z.size(), 1);
        return;
    }
    if (k <= 64) {
        const uint64_t r = (uint64_t)download_u128(A, R);
        u128 z;
        if ((r & (r - 1)) == 0)
            z = (u128)1 << (k + 1);  // r = 2^(k-1)
        else
            z = (k == 64 ? ~(u128)0 : ((u128)1 << (2 * k))) / r;  // r odd part > 1: 2^128 / r = (2^128 - 1) / r
        upload_u128(A, Z, z);
        return;
    }
    const size_t h = k / 2 + 32;
    Num Rh(A), Zh(A), Z0(A), T(A), E(A), D(A);
    A.tdiv_q_2exp(Rh, R, k - h);
    // the trace times each level of at least 2^16 bits apart from the ones below it (waiting for
    // the stream around them)
    const bool tr = trace_on() && k >= (1u << 16);
    std::chrono::steady_clock::time_point tl0, tl1;
    if (tr) {
        A.sync();
        tl0 = std::chrono::steady_clock::now();
    }
    // The half-precision reciprocal without its exact correction: within c <= 2 units of
    // 2^(2h)/Rh (the bound this step keeps, below), which saves a product and its host waits at
    // every level of the recursion.
    recip_floor(A, Zh, Rh, false);
    if (tr) {
        A.sync();
        tl1 = std::chrono::steady_clock::now();
    }
    struct LevelTrace {
        DevArith& A;
        bool on;
        size_t k;
        std::chrono::steady_clock::time_point t0, t1;
        ~LevelTrace() {
            if (!on) return;
            cudaStreamSynchronize(A.stream());  // no throw from a destructor
            const auto t2 = std::chrono::steady_clock::now();
            std::fprintf(stderr, "[pi_device]   reciprocal level %zu bits: %.3f ms (levels below %.3f ms)\n", k,
                         std::chrono::duration<double, std::milli>(t2 - t1).count(),
                         std::chrono::duration<double, std::milli>(t1 - t0).count());
        }
    } ltrace{A, tr, k, tl0, tl1};
    A.shl(Z0, Zh, k - h);
    // E = 2^(2k) - R Z0. With R = 2^(k-h) (Rh + f), 0 <= f < 1, and Rh >= 2^(h-1):
    // |2^(2k)/R - Z0| <= (c + 4) 2^(k-h), so |E| < (c + 4) 2^(2k-h) < 2^(2k-h+3): E follows from
    // R Z0 modulo 2^(32 L) - 1 for a transform about 3/4 the length of the full product's. The
    // Newton step leaves (c + 4)^2 2^(k-2h+1) < 2^-57 of error, plus the truncations below (under
    // 2 units), so this level's result is within 2 units as well.
    const int lw = wrap_logL(2 * k - h + 3, R.n, Z0.v.n);
    if (lw) {
        A.mul_wrap(T, R, Z0, lw);
        residue_diff(A, E, 2 * k, T, lw);
    } else {
        A.mul(T, R, Z0);
        A.set_pow2(E, 2 * k);
        A.sub(E, E, T);
    }
    // D = floor(Z0 E / 2^(2k)) = floor(Zh E / 2^(k+h)) from E's top bits: dropping the low
    // s = k - 2 bits of E lowers Zh E / 2^(k+h) by less than Zh 2^s / 2^(k+h) <= 1/2
    // (Zh <= 2^(h+1)), so D is exact or one low; the final correction absorbs that.
    const size_t s = k - 2;
    A.fdiv_q_2exp(T, E, s);
    A.mul(D, Zh, T);
    A.fdiv_q_2exp(D, D, k + h - s);
    A.add(Z, Z0, D);
    if (!exact) return;
    A.mul(T, R, D);
    A.sub(E, E, T);                 // E = 2^(2k) - R Z
    int steps = 0;
    while (E.v.sign < 0) {
        A.add_si(Z, Z, -1);
        A.add(E, E, R);
        if (++steps > 64) throw DevError(PG_ERR_INTERNAL, "recip_floor: correction did not converge");
    }
    while (A.cmp(E, R) >= 0) {
        A.add_si(Z, Z, 1);
        A.sub(E, E, R);
        if (++steps > 64) throw DevError(PG_ERR_INTERNAL, "recip_floor: correction did not converge");
    }
}

// u ~= 2^q / sqrt(a) within a few units (Newton on the inverse square root).
void rsqrt_approx(DevArith& A, DevNum& u, uint64_t a, size_t q) {
    if (q <= 64) {
        // 2^128 - 1 stands in for 2^128 at q = 64: the estimate may be one unit low
        const u128 t = (q == 64 ? ~(u128)0 : ((u128)1 << (2 * q))) / a;
        upload_u128(A, u, isqrt128(t));
        return;
    }
    const size_t qh = q / 2 + 32;
    Num uh(A), u0(A), T(A), e(A), D(A);
    rsqrt_approx(A, uh, a, qh);
    A.shl(u0, uh, q - qh);
    // e = 2^(2q) - a u0^2 = a (v + u0)(v - u0), v = 2^q / sqrt(a): with uh within c units of
    // 2^qh / sqrt(a), |e| <= 2 c sqrt(a) 2^(2q - qh) (plus a far smaller square term); c <= 2^4
    // and a < 2^64 give |e| < 2^(2q - qh + 38)
    const int lw = wrap_logL(2 * q - qh + 38, u0.v.n, u0.v.n);
    if (lw) {
        A.mul_wrap(T, u0, u0, lw);
        A.mul_ui(T, T, a);
        A.fold(T, T, lw);
        residue_diff(A, e, 2 * q, T, lw);
    } else {
        A.sqr(T, u0);
        A.mul_ui(T, T, a);
        A.set_pow2(e, 2 * q);
        A.sub(e, e, T);
    }
    // D = floor(u0 e / 2^(2q+1)) = floor(uh e / 2^(q + qh + 1)) from e's top bits: dropping
    // s = q - 1 low bits lowers it by less than uh 2^s / 2^(q + qh + 1) < 1/4 (uh < 2^qh)
    const size_t s = q - 1;
    A.fdiv_q_2exp(T, e, s);
    A.mul(D, uh, T);
    A.fdiv_q_2exp(D, D, q + qh + 1 - s);
    A.add(u, u0, D);
}

// S = floor(sqrt(a) 2^s), exactly; with exact == false |S - sqrt(a) 2^s| < 2 (u is within a few
// units of 2^q / sqrt(a), so a u / 2^(q-s) is within a few a / 2^64 units of sqrt(a) 2^s, plus the
// floor) and the square check is skipped.
void sqrt_scaled(DevArith& A, DevNum& S, uint64_t a, size_t s, bool exact = true) {
    const size_t q = s + 64;
    Num u(A), N(A), V(A), t(A);
    rsqrt_approx(A, u, a, q);
    A.mul_ui(S, u, a);              // a 2^q / sqrt(a)
    A.tdiv_q_2exp(S, S, q - s);
    if (!exact) return;
    // V = N - S^2 with N = a 2^(2s); S is within a few units of sqrt(N), so |V| is about
    // 2 S c < 2^(s + 40) for a < 2^64: S^2 modulo 2^(32 L) - 1 is enough
    const int lw = wrap_logL(s + 40, S.n, S.n);
    if (lw) {
        A.mul_wrap(t, S, S, lw);
        A.set_pow2(N, (2 * s) % ((size_t)32 << lw));
        A.mul_ui(N, N, a);
        A.fold(N, N, lw);
        A.sub(V, N, t);
        centre(A, V, lw);
    } else {
        A.set_pow2(N, 2 * s);
        A.mul_ui(N, N, a);
        A.sqr(t, S);
        A.sub(V, N, t);             // V = N - S^2
    }
    int steps = 0;
    while (V.v.sign < 0) {          // (S-1)^2 = S^2 - 2S + 1
        A.add(V, V, S);
        A.add(V, V, S);
        A.add_si(V, V, -1);
        A.add_si(S, S, -1);
        if (++steps > 64) throw DevError(PG_ERR_INTERNAL, "sqrt_scaled: correction did not converge");
    }
    for (;;) {                      // (S+1)^2 = S^2 + 2S + 1 <= N ?
        A.shl(t, S, 1);
        A.add_si(t, t, 1);
        if (A.cmp(V, t) < 0) break;
        A.sub(V, V, t);
        A.add_si(S, S, 1);
        if (++steps > 64) throw DevError(PG_ERR_INTERNAL, "sqrt_scaled: correction did not converge");
    }
}

void pow5(DevArith& A, DevNum& F, size_t n) {
    A.set_ui(F, 1);
    if (n == 0) return;
    int top = 63;
    while (!((n >> top) & 1)) --top;
    for (int b = top; b >= 0; --b) {
        A.sqr(F, F);
        if ((n >> b) & 1) A.mul_ui(F, F, 5);
    }
}

// pi_int = floor(pi 10^digits) from the series root Q, R (both > 0).
void final_formula(DevArith& A, DevNum& pi_int, const DevNum& Q, const DevNum& R, size_t digits) {
    if (Q.sign <= 0 || R.sign <= 0) throw DevError(PG_ERR_BAD_ARG, "final formula needs Q, R > 0");
    const size_t bQ = A.bits(Q), bR = A.bits(R);
    for (size_t guard = 128; guard <= 128 + 4 * 256; guard += 256) {
        const size_t P = (size_t)std::ceil((double)digits * 3.3219280948873623) + 2 + guard;
        const size_t k = P + 64;
        Num Qt(A), Rt(A), Z(A), S(A), F(A), X(A), t(A);
        const long long eQ = (long long)bQ - (long long)k;
        const long long eR = (long long)bR - (long long)k;
        if (eQ >= 0) A.tdiv_q_2exp(Qt, Q, (size_t)eQ); else A.shl(Qt, Q, (size_t)-eQ);
        if (eR >= 0) A.tdiv_q_2exp(Rt, R, (size_t)eR); else A.shl(Rt, R, (size_t)-eR);
        {
            Timer tm("reciprocal of R");
            recip_floor(A, Z, Rt, false);  // 2^(2k) / Rt within 2 units
        }
        {
            Timer tm("sqrt(10005)");
            sqrt_scaled(A, S, 10005, k, false);  // within 2 units
        }
        {
            Timer tm("5^digits");
            pow5(A, F, digits);
        }
        Timer tm("three truncated products and the floor");
        A.mul_ui(X, Qt, 426880);
        long long e = eQ - eR - 3 * (long long)k + (long long)digits;
        auto mul_trunc = [&](const DevNum& y) {
            A.mul(t, X, y);
            const long long over = (long long)A.bits(t) - (long long)k;
            if (over > 0) {
                A.tdiv_q_2exp(X, t, (size_t)over);
                e += over;
            } else {
                A.copy(X, t);
            }
        };
        mul_trunc(S);
        mul_trunc(Z);
        mul_trunc(F);
        if (e >= 0) throw DevError(PG_ERR_INTERNAL, "final formula: no fraction bits");
        const size_t fb = (size_t)(-e);
        // Z and S are within 2 units of their exact values (>= 2^(k-1)), the truncations of Qt,
        // Rt and the three products within 1 unit each: the relative error is below
        // 16 * 2^-(k-1) = 2^(5-k). With V = X / 2^fb < 2^ib the absolute error is below
        // 2^-eb, eb = k - 5 - ib (for pi 10^d < 2^(P - guard): eb >= guard + 59). The floor is
        // certain when the computed fraction lies at least 2^-tw, tw = eb - 2, from an integer;
        // each larger guard narrows that window, so a value closer to an integer than one
        // guard resolves is settled by the next.
        const size_t xb = A.bits(X);
        const size_t ib = xb > fb ? xb - fb : 0;
        if (k < ib + 5 + 64 + 2 || k - 5 - ib - 2 > fb)
            throw DevError(PG_ERR_INTERNAL, "final formula: not enough fraction bits");
        const size_t tw = k - 5 - ib - 2;
        // fr = X mod 2^fb: below <=> fr < 2^(fb-tw); above <=> 2^fb - fr < 2^(fb-tw)
        Num fr(A), c(A);
        A.tdiv_r_2exp(fr, X, fb);
        const bool below = A.bits(fr) <= fb - tw;
        A.set_pow2(c, fb);
        A.sub(c, c, fr);
        const bool above = A.bits(c) <= fb - tw;
        if (!below && !above) {
            A.tdiv_q_2exp(pi_int, X, fb);
            return;
        }
    }
    throw DevError(PG_ERR_INTERNAL, "final formula: the result stayed within the error bound of an integer");
}

// ------------------------------------------------------------------ decimal conversion
constexpr int kLeafLog = 10;  // 1024-digit leaves (56-limb chunks, one thread each)

// *out |= 1 if any flag is set (the conversion's remainders must all be below the split power).
__global__ void flag_any_kernel(const uint32_t* f, uint64_t n, uint32_t* out) {
    bool any = false;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        any |= f[i] != 0;
    if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) atomicOr(out, 1u);
}

// Decimal digits of x (0 <= x < 10^nd) into host out[0 .. nd).
void to_decimal(DevArith& A, SharedProduct& sp, const DevNum& x, size_t nd, char* out) {
    cudaStream_t st = A.stream();
    if (nd == 0) return;
    if (x.n == 0) {
        std::memset(out, '0', nd);
        return;
    }
    int J = kLeafLog;
    while (((size_t)1 << J) < nd) ++J;
    const size_t total = (size_t)1 << J, skip = total - nd;
    // the digit buffer stays with the context: a 100 MB cudaMalloc / cudaFree per call costs a
    // device synchronisation each and, now and then, tens of milliseconds
    if (nd > sp.digits_cap) {
        A.sync();
        if (sp.digits) dev_free(sp.digits);
        sp.digits = nullptr;
        sp.digits_cap = 0;
        if (pg::dev_malloc((void**)&sp.digits, nd) != cudaSuccess) throw DevError(PG_ERR_OOM, "digit buffer");
        sp.digits_cap = nd;
    }
    char* d_out = sp.digits;
    cudaMemsetAsync(d_out, '0', nd, st);
    // powers P[j] = 10^(2^j) and reciprocals for j = kLeafLog .. J-1
    std::vector<Num*> P, inv;
    std::vector<size_t> K;
    struct Owner {
        std::vector<Num*>& a;
        std::vector<Num*>& b;
        ~Owner() {
            for (auto* p : a) delete p;
            for (auto* p : b) delete p;
        }
    } own{P, inv};
    {
        Timer tm("power tree and reciprocals");
        Num p(A);
        A.set_ui(p, 10);
        for (int j = 0; j < J; ++j) {
            if (j >= kLeafLog) {
                P.push_back(new Num(A));
                K.push_back(A.bits(p));  // makes p's length exact before the copy
                A.copy(*P.back(), p);
                inv.push_back(new Num(A));
            }
            if (j + 1 < J) A.sqr(p, p);
        }
        // The top reciprocal by Newton; every lower one from the one above it:
        // with Y = floor(2^(2K') / P^2) (K' = bits(P^2)), floor(P Y / 2^(2K' - 2K)) undershoots
        // floor(2^(2K) / P) by at most one (the error P 2^(2K - 2K') is below 2^(2 - K)), so one
        // exact check 0 <= 2^(2K) - P Z < P finishes it (two with Y's low bits dropped, below).
        const int top = J - 1;
        if (top >= kLeafLog) recip_floor(A, inv[top - kLeafLog]->v, P[top - kLeafLog]->v);
        Num T(A), E(A);
        for (int j = top - 1; j >= kLeafLog; --j) {
            DevNum& Pj = P[j - kLeafLog]->v;
            DevNum& Z = inv[j - kLeafLog]->v;
            const size_t k = K[j - kLeafLog], k2 = K[j + 1 - kLeafLog];
            // Z from the top bits of the reciprocal above: dropping its low s = sh - k - 1 bits
            // lowers P Y / 2^sh by less than P 2^s / 2^sh < 1/2, so Z undershoots by at most 2
            const size_t sh = 2 * k2 - 2 * k;
            const size_t s = sh > k + 1 ? sh - k - 1 : 0;
            A.tdiv_q_2exp(E, inv[j + 1 - kLeafLog]->v, s);
            A.mul(T, Pj, E);
            A.tdiv_q_2exp(Z, T, sh - s);
            // E = 2^(2K) - P Z lies in [0, 3P): P Z modulo 2^(32 L) - 1 suffices
            const int lw = wrap_logL(k + 3, Pj.n, Z.n);
            if (lw) {
                A.mul_wrap(T, Pj, Z, lw);
                residue_diff(A, E, 2 * k, T, lw);
            } else {
                A.mul(T, Pj, Z);
                A.set_pow2(E, 2 * k);
                A.sub(E, E, T);
            }
            int steps = 0;
            while (E.v.sign < 0) {
                A.add_si(Z, Z, -1);
                A.add(E, E, Pj);
                if (++steps > 4) throw DevError(PG_ERR_INTERNAL, "to_decimal: reciprocal step did not converge");
            }
            while (A.cmp(E, Pj) >= 0) {
                A.add_si(Z, Z, 1);
                A.sub(E, E, Pj);
                if (++steps > 4) throw DevError(PG_ERR_INTERNAL, "to_decimal: reciprocal step did not converge");
            }
        }
    }
    auto pw = [&](int j) -> DevNum& { return P[j - kLeafLog]->v; };
    auto iv = [&](int j) -> DevNum& { return inv[j - kLeafLog]->v; };
    auto kb = [&](int j) { return K[j - kLeafLog]; };
    auto even = [](size_t n) { return (n + 1) & ~(size_t)1; };
    // capacity (limbs, even) of a chunk < 10^(2^j): bits(10^(2^j)) / 64 + 1
    auto cap_of = [&](int j) { return even(kb(j) / 64 + 2); };

    // the level's products with one shared operand: one batch, or (chunks too long for one
    // transform, the top levels beyond ~300M digits) a block product per chunk
    auto shared_mul = [&](const uint64_t* a, uint64_t sa, uint64_t na, uint64_t njobs, const uint64_t* b, uint64_t nb,
                          uint64_t* out, uint64_t so) {
        if (product_logL(na, nb) <= split_logL()) {
            sp.run(A.tables(), st, A.launches(), a, sa, na, njobs, b, nb, out, so);
            return;
        }
        for (uint64_t j = 0; j < njobs; ++j) A.mul_limbs(a + j * sa, na, b, nb, out + j * so);
    };

    Timer tm("divide-and-conquer levels and leaves");
    const uint64_t* cur = x.d;
    size_t cur_s = even(std::max<size_t>(x.n, 1)), cur_n = x.n;
    // the top chunk needs an even stride: copy when x.n is odd (only the layout matters)
    Num xcopy(A), lvl_a(A), lvl_b(A), Tbuf(A), Ubuf(A), Rbuf(A), Ppad(A);
    if (x.n & 1) {
        A.reserve(xcopy, cur_s);
        cudaMemsetAsync(xcopy.v.d, 0, cur_s * 8, st);
        cudaMemcpyAsync(xcopy.v.d, x.d, x.n * 8, cudaMemcpyDeviceToDevice, st);
        cur = xcopy.v.d;
    }
    DevNum* next = &lvl_a.v;
    DevNum* spare = &lvl_b.v;
    // chunk flags (grown in the context's state) and one word for "a remainder stayed >= P"
    uint32_t* bad = nullptr;
    {
        const uint64_t most = (uint64_t)1 << (J - kLeafLog);
        if (most + 1 > sp.flags_cap) {
            A.sync();
            if (sp.flags) dev_free(sp.flags);
            sp.flags = nullptr;
            sp.flags_cap = 0;
            if (pg::dev_malloc((void**)&sp.flags, (most + 1) * 4) != cudaSuccess) throw DevError(PG_ERR_OOM, "flags");
            sp.flags_cap = most + 1;
        }
        bad = sp.flags + most;
        cudaMemsetAsync(bad, 0, 4, st);
    }
    uint32_t* ge = sp.flags;
    for (int t = 0; J - t > kLeafLog; ++t) {
        const auto tl0 = std::chrono::steady_clock::now();
        const int j = J - t - 1;  // split power 10^(2^j)
        const uint64_t njobs = 1ull << t;
        const size_t cap = cap_of(j);             // next level's chunk capacity
        const DevNum& Pj = pw(j);
        const DevNum& Ij = iv(j);
        const size_t ni = Ij.n, np = Pj.n;
        if (cur_n == 0) cur_n = 1;
        // T = (c >> 64 s) * inv, q = T >> (2K - 64 s) into the even slots of the next level. The
        // chunk's low 64 s <= K - 2 bits are dropped (an even limb count, so the operand stays
        // 16-byte aligned): that lowers c inv / 2^(2K) by less than 2^(64 s + 1 - K) <= 1/2, so q
        // undershoots floor(c / P) by at most 3 and the product is about 2K bits, not 3K.
        const size_t s64 = std::min<size_t>(kb(j) >= 66 ? ((kb(j) - 2) / 64) & ~(size_t)1 : 0, (cur_n - 1) & ~(size_t)1);
        const size_t nct = cur_n - s64;
        const size_t sT = even(nct + ni);
        A.reserve(Tbuf, sT * njobs);
        shared_mul(cur + s64, cur_s, nct, njobs, Ij.d, ni, Tbuf.v.d, sT);
        A.reserve(*next, 2 * cap * njobs);
        A.batch_shr(Tbuf.v.d, sT, nct + ni, next->d, 2 * cap, cap, 2 * kb(j) - 64 * s64, njobs);
        // U = q * P, r = c - U (< 3 P) into the odd slots
        const size_t sU = even(cap + np);
        A.reserve(Ubuf, sU * njobs);
        shared_mul(next->d, 2 * cap, cap, njobs, Pj.d, np, Ubuf.v.d, sU);
        A.reserve(Rbuf, cur_s * njobs);
        A.batch_add(cur, cur_s, cur_n, Ubuf.v.d, sU, std::min(cap + np, cur_n), Rbuf.v.d, cur_s, cur_n, true, 0,
                    nullptr, njobs);
        A.batch_shr(Rbuf.v.d, cur_s, cur_n, next->d + cap, 2 * cap, cap, 0, njobs);
        // corrections: while r >= P: r -= P, q += 1 (at most three times)
        A.reserve(Ppad, cap);
        cudaMemsetAsync(Ppad.v.d, 0, cap * 8, st);
        cudaMemcpyAsync(Ppad.v.d, Pj.d, np * 8, cudaMemcpyDeviceToDevice, st);
        for (int round = 0; round < 3; ++round) {
            A.batch_ge(next->d + cap, 2 * cap, Ppad.v.d, 0, cap, ge, njobs);
            A.batch_add(next->d + cap, 2 * cap, cap, Ppad.v.d, 0, np, next->d + cap, 2 * cap, cap, true, 0, ge, njobs);
            A.batch_add(next->d, 2 * cap, cap, nullptr, 0, 0, next->d, 2 * cap, cap, false, 1, ge, njobs);
        }
        // a third check must find every remainder below P (read once, after the last level)
        A.batch_ge(next->d + cap, 2 * cap, Ppad.v.d, 0, cap, ge, njobs);
        flag_any_kernel<<<(unsigned)std::min<uint64_t>((njobs + 255) / 256, 148 * 8), 256, 0, st>>>(ge, njobs, bad);
        cur = next->d;
        cur_s = cap;
        cur_n = cap;
        std::swap(next, spare);
        if (trace_on())
            std::fprintf(stderr, "[pi_device] conversion level %2d: %8llu chunks of %zu limbs: %.3f ms\n", t,
                         (unsigned long long)njobs, cur_s,
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tl0).count());
    }
    const auto tw0 = std::chrono::steady_clock::now();
    if (sp.error(st)) throw DevError(PG_ERR_INTERNAL, "to_decimal: product check failed");
    {
        uint32_t hb = 0;
        cudaMemcpyAsync(&hb, bad, 4, cudaMemcpyDeviceToHost, st);
        A.sync();
        if (hb) throw DevError(PG_ERR_INTERNAL, "to_decimal: remainder above the split power");
    }
    if (!A.leaves(cur, cur_s, cur_n, (uint64_t)1 << (J - kLeafLog), (uint64_t)1 << kLeafLog, d_out, skip, total))
        throw DevError(PG_ERR_BAD_ARG, "to_decimal: the number has more digits than requested");
    if (cudaMemcpyAsync(out, d_out, nd, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        throw DevError(PG_ERR_DEVICE, "digit copy");
    A.sync();
    if (trace_on())
        std::fprintf(stderr, "[pi_device] conversion levels drained, leaves, digit copy: %.3f ms\n",
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw0).count());
}

// ------------------------------------------------------------------ pi's digits by a scaled remainder tree
// The n = digits + 1 decimal digits of floor(pi 10^digits) are the first n digits of y = pi / 10
// in (0, 1). Digit positions count from the most significant (position 0 is the "3"), padded on
// the low side to 2^J. A node of the tree covers positions [s, s + m) and holds the fraction
// v = frac(y 10^s), whose first m digits are the node's; its children are (s, m/2) holding v itself
// and (s + m/2, m/2) holding frac(v 10^(m/2)). Each node keeps v to w limbs (v ~= V / 2^(64 w)):
// the high child takes V's top limbs, the low child the top limbs of the low w limbs of
// V * 10^(m/2), a middle product that one cyclic transform of about w limbs gives (the part that
// wraps around lands below the limbs taken). So the conversion is one batched product per level
// (all nodes share 10^(m/2)) and no division; 1024-digit leaves are written by one warp each
// multiplying its fraction by 10^19. Precision: a leaf keeps 1024 log2(10) + 128 bits, and a node
// w(lo) + ceil((m/2) log2(10) / 64) + 1 limbs, so the error of 10^(m/2) v (a few units of V's last
// limb, times 10^(m/2)) stays below one unit of the low child's last limb at every level. A leaf
// whose remaining fraction ends within 2^-128 of 0 or 1 cannot be trusted (the digits next to it
// may carry); it raises a flag and the caller converts exactly instead (expected about once in
// 2^120 leaves).
constexpr int kSrtLeafLog = 10;
constexpr int kSrtGuardBits = 128;
constexpr double kLog2Ten = 3.3219280948873623;

// Children of a level: child j (parent i = j / 2) takes limbs [off, off + wc) of the parent's fraction
// (even j) or of its cyclic product with 10^(m/2) (odd j). Blocks of 256 threads copy 2048 limbs each.
__global__ void srt_children_kernel(const uint64_t* Y, uint64_t wy, const uint64_t* prod, uint64_t wp, uint64_t off,
                                    uint64_t* out, uint64_t wc, uint64_t nchild, uint64_t segs) {
    const uint64_t j = blockIdx.x / segs, seg = blockIdx.x - j * segs;
    if (j >= nchild) return;
    const uint64_t i = j >> 1;
    const uint4* src = reinterpret_cast<const uint4*>(((j & 1) ? prod + i * wp : Y + i * wy) + off);
    uint4* dst = reinterpret_cast<uint4*>(out + j * wc);
    const uint64_t pairs = wc / 2;
    for (uint64_t q = seg * 1024 + threadIdx.x; q < min(pairs, (seg + 1) * 1024); q += blockDim.x) dst[q] = src[q];
}

// One warp per leaf: the fraction V / 2^(64 wl) (wl <= 64 limbs, two per lane) is multiplied by 10^19
// fifty-three times and by 10^17 once; each product's integer part is the next 19 (17) digits. A
// product's limb sums carry between lanes by a warp-wide carry-lookahead (generate / propagate
// ballots). Digits at positions >= n are not written. flag |= 1 when the remaining fraction lies within
// 2^-128 of 0 or 1.
constexpr int kSrtChunks = 54;
__global__ void __launch_bounds__(128) srt_leaves_kernel(const uint64_t* Y, uint64_t wl, uint64_t nleaves,
                                                         uint64_t n, char* out, uint32_t* flag) {
    __shared__ uint64_t s_chunk[4][kSrtChunks];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t leaf = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (leaf >= nleaves) return;  // whole warps
    const int nl = (int)(wl / 2);  // lanes holding limbs
    const uint64_t* y = Y + leaf * wl;
    uint64_t f0 = lane < nl ? y[2 * lane] : 0, f1 = lane < nl ? y[2 * lane + 1] : 0;
    for (int step = 0; step < kSrtChunks; ++step) {
        const uint64_t M = step < kSrtChunks - 1 ? 10000000000000000000ull : 100000000000000000ull;
        const uint64_t lo0 = f0 * M, hi0 = __umul64hi(f0, M);
        const uint64_t lo1 = f1 * M, hi1 = __umul64hi(f1, M);
        uint64_t hp = __shfl_up_sync(0xffffffffu, hi1, 1);
        if (lane == 0) hp = 0;
        const uint64_t s0 = lo0 + hp;
        const uint32_t c0 = s0 < lo0;
        const uint64_t s1 = lo1 + hi0;
        const uint32_t c1 = s1 < lo1;
        const uint64_t s1b = s1 + c0;
        const uint32_t g = c1 | (c0 & (s1b == 0));
        const uint32_t pr = (s0 == ~0ull) & (s1b == ~0ull);
        const uint32_t G = __ballot_sync(0xffffffffu, g), P = __ballot_sync(0xffffffffu, pr);
        const uint32_t a = G | P;
        const uint32_t cm = (a + G) ^ a ^ G;  // bit l: carry into lane l
        const uint32_t cin = (cm >> lane) & 1u;
        const uint64_t r0 = s0 + cin;
        const uint32_t cr0 = cin & (r0 == 0);
        f0 = r0;
        f1 = s1b + cr0;
        // the integer part: the top limb's high word plus the carry out of the top lane
        if (lane == nl - 1) s_chunk[warp][step] = hi1 + ((cm >> nl) & 1u);
    }
    if (lane == nl - 1 && ((f1 == 0 && f0 == 0) || (f1 == ~0ull && f0 == ~0ull))) atomicOr(flag, 1u);
    __syncwarp();
    const uint64_t base = leaf << kSrtLeafLog;
    for (int c = lane; c < kSrtChunks; c += 32) {
        uint64_t v = s_chunk[warp][c];
        const int nd = c < kSrtChunks - 1 ? 19 : 17;
        const uint64_t p0 = base + 19ull * c;
        for (int d = nd - 1; d >= 0; --d) {
            const uint64_t q = v / 10;
            if (p0 + d < n) out[p0 + d] = (char)('0' + (v - q * 10));
            v = q;
        }
    }
}

// Limbs per node at each level (t = 0 .. J - kSrtLeafLog, the last the leaves) and live nodes, for n
// digit positions padded to 2^J.
struct SrtPlan {
    int J = 0;
    uint64_t n = 0;
    std::vector<uint64_t> w, live;
};

uint64_t srt_peel_limbs(uint64_t m) {  // limbs 10^(m/2) can span: ceil((m/2) log2(10) / 64)
    return (uint64_t)std::ceil((double)(m / 2) * kLog2Ten / 64.0) + 1;
}

// w of the node (s, m): its kept digits min(m, n - s) and its live children decide it.
uint64_t srt_node_limbs(uint64_t s, uint64_t m, uint64_t n, uint64_t wleaf) {
    if (m <= (1ull << kSrtLeafLog)) return wleaf;
    const uint64_t wh = srt_node_limbs(s, m / 2, n, wleaf);
    if (s + m / 2 >= n) return wh;
    const uint64_t wl = srt_node_limbs(s + m / 2, m / 2, n, wleaf);
    uint64_t w = std::max(wh, wl + srt_peel_limbs(m) + 1);
    return (w + 1) & ~1ull;  // even: 16-byte aligned nodes
}

SrtPlan srt_plan(uint64_t n) {
    SrtPlan P;
    P.n = n;
    P.J = kSrtLeafLog;
    while ((1ull << P.J) < n) ++P.J;
    const uint64_t wleaf = ((uint64_t)std::ceil(((1ull << kSrtLeafLog) * kLog2Ten + kSrtGuardBits) / 64.0) + 1) & ~1ull;
    for (int t = 0; t <= P.J - kSrtLeafLog; ++t) {
        const uint64_t m = 1ull << (P.J - t);
        // the first node of a level is full, or (at the top) the only live one: it needs the most
        P.w.push_back(srt_node_limbs(0, m, n, wleaf));
        P.live.push_back((n + m - 1) / m);
    }
    return P;
}

// y = pi / 10 to w limbs, V ~= y 2^(64 w) within a few units, from the series root Q, R: the final
// formula's truncated reciprocal, square root and products, 42688 sqrt(10005) Q / R.
size_t pi_tenth_bits(uint64_t w) { return 64 * w + 64; }

// Whether every level of the tree fits one transform of the batched product.
bool srt_fits(const SrtPlan& P) {
    for (size_t t = 0; t + 1 < P.w.size(); ++t)
        if (ceil_log2(2 * P.w[t] + 64) > kWideMaxLogL + 1) return false;
    return true;
}

// out[0 .. n) = the first n digits of V / 2^(64 w[0]) (V: the root's fraction). Returns false if a
// leaf's digits could not be trusted (the caller then converts exactly).
// powers 10^(2^j), j = kSrtLeafLog .. J - 1, into pw (owned by the caller, made on A)
void srt_powers(DevArith& A, int J, std::vector<Num*>& pw) {
    Timer tm("power tree");
    Num p(A);
    A.set_ui(p, 10);
    for (int j = 0; j < J; ++j) {
        if (j >= kSrtLeafLog) {
            pw.push_back(new Num(A));
            A.exact(p);
            A.copy(*pw.back(), p);
        }
        if (j + 1 < J) A.sqr(p, p);
    }
}

bool srt_digits(DevArith& A, SharedProduct& sp, const SrtPlan& P, DevNum& V, char* out,
                const std::vector<Num*>* pw_pre = nullptr) {
    cudaStream_t st = A.stream();
    const int levels = (int)P.w.size() - 1;  // product levels; P.w[levels] is the leaves'
    const uint64_t n = P.n;
    if (n > sp.digits_cap) {
        A.sync();
        if (sp.digits) dev_free(sp.digits);
        sp.digits = nullptr;
        sp.digits_cap = 0;
        if (pg::dev_malloc((void**)&sp.digits, n) != cudaSuccess) throw DevError(PG_ERR_OOM, "digit buffer");
        sp.digits_cap = n;
    }
    // powers 10^(2^j), j = kSrtLeafLog .. J - 1 (given, or made here)
    std::vector<Num*> own_pw;
    struct Owner {
        std::vector<Num*>& a;
        ~Owner() {
            for (auto* p : a) delete p;
        }
    } own{own_pw};
    if (!pw_pre) srt_powers(A, P.J, own_pw);
    const std::vector<Num*>& pw = pw_pre ? *pw_pre : own_pw;
    // level t peels 10^(2^(J - t - 1)), t < levels = J - kSrtLeafLog
    auto power = [&](int t) -> DevNum& { return pw[(size_t)(P.J - t - 1 - kSrtLeafLog)]->v; };
    Timer tm("tree levels and leaves");
    Num lv0(A), lv1(A), prod(A);
    DevNum* cur = &lv0.v;
    DevNum* nxt = &lv1.v;
    A.reserve(*cur, P.w[0]);
    // the root: V's w[0] limbs (V < 2^(64 w[0]); shorter V is padded with zeros)
    A.exact(V);
    if (V.n > P.w[0]) throw DevError(PG_ERR_INTERNAL, "pi digits: root fraction longer than its precision");
    cudaMemsetAsync(cur->d, 0, P.w[0] * 8, st);
    if (V.n) cudaMemcpyAsync(cur->d, V.d, V.n * 8, cudaMemcpyDeviceToDevice, st);
    for (int t = 0; t < levels; ++t) {
        const uint64_t m = 1ull << (P.J - t), wt = P.w[t], wc = P.w[t + 1];
        const uint64_t kids = P.live[t + 1];
        const uint64_t klo = n > m / 2 ? (n - m / 2 + m - 1) / m : 0;  // parents with a live low child
        const DevNum& T = power(t);
        uint64_t cyc = 1;
        while (cyc < std::max(wt, T.n + wc + 8)) cyc <<= 1;
        if (klo) {
            A.reserve(prod, klo * cyc);
            sp.run(A.tables(), st, A.launches(), cur->d, wt, wt, klo, T.d, T.n, prod.v.d, cyc, cyc);
        }
        A.reserve(*nxt, kids * wc);
        const uint64_t segs = (wc / 2 + 1023) / 1024;
        srt_children_kernel<<<(unsigned)(kids * segs), 256, 0, st>>>(cur->d, wt, prod.v.d, cyc, wt - wc, nxt->d, wc,
                                                                    kids, segs);
        ++*A.launches();
        std::swap(cur, nxt);
    }
    uint32_t* flag = sp.flags;
    if (!flag || sp.flags_cap < 1) {
        A.sync();
        if (sp.flags) dev_free(sp.flags);
        sp.flags = nullptr;
        sp.flags_cap = 0;
        if (pg::dev_malloc((void**)&sp.flags, 4) != cudaSuccess) throw DevError(PG_ERR_OOM, "flags");
        sp.flags_cap = 1;
        flag = sp.flags;
    }
    cudaMemsetAsync(flag, 0, 4, st);
    const uint64_t leaves = P.live[levels];
    srt_leaves_kernel<<<(unsigned)((leaves * 32 + 127) / 128), 128, 0, st>>>(cur->d, P.w[levels], leaves, n, sp.digits,
                                                                           flag);
    ++*A.launches();
    if (sp.error(st)) throw DevError(PG_ERR_INTERNAL, "pi digits: product check failed");
    uint32_t hf = 0;
    cudaMemcpyAsync(&hf, flag, 4, cudaMemcpyDeviceToHost, st);
    A.sync();
    if (hf) return false;
    if (cudaMemcpyAsync(out, sp.digits, n, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        throw DevError(PG_ERR_DEVICE, "digit copy");
    A.sync();
    return true;
}

// Whether pi's digits for `digits` take the scaled remainder tree (every level in one transform;
// PG_EXACT_CONVERSION unset).
bool pi_tree_path(size_t digits) { return srt_fits(srt_plan(digits + 1)) && !std::getenv("PG_EXACT_CONVERSION"); }

// The status and message of a workspace error word (bits set by the kernels: 1 a carry look-back
// wait ran out, 2 a carry out of the top word, 4 a tile load wait ran out, 8 a sum's look-back
// wait ran out).
pg_status workspace_error_status(uint32_t err, const char*& what) {
    if (err & kErrAddWait) {
        what = "sum look-back wait ran out of iterations";
        return PG_ERR_TIMEOUT;
    }
    if (err & 4) {
        what = "tile load wait ran out of iterations";
        return PG_ERR_TIMEOUT;
    }
    if (err == 1) {
        what = "carry look-back wait ran out of iterations";
        return PG_ERR_TIMEOUT;
    }
    what = "carry out of the top word";
    return PG_ERR_INTERNAL;
}

// Throws (after clearing it) when a workspace's error word is set; waits for the stream.
void throw_workspace_error(const Workspace& W, cudaStream_t st, const char* where) {
    uint32_t err = 0;
    if (W.sync) cudaMemcpyAsync(&err, W.sync, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) throw DevError(PG_ERR_DEVICE, std::string(where) + ": device error");
    if (!err) return;
    cudaMemsetAsync(W.sync, 0, 4, st);
    cudaStreamSynchronize(st);
    const char* what = "";
    const pg_status s = workspace_error_status(err, what);
    throw DevError(s, std::string(where) + ": " + what);
}

// Buffers of a pi run's finish sized before it starts, so that a fresh process does not grow
// them step by step (each growth a cudaMalloc on the critical path; a process's first run made
// some 450 of them): the product workspace for the largest product (two k-bit factors, k the
// final formula's precision) and an arena of `units` buffers of the k-bit size class for the
// numbers. The arena is opened only while the pool holds less (a later run finds its buffers
// cached). Failures are left to the steps themselves, which allocate as before.
void presize_finish(const DeviceTables& T, Workspace& W, DevPool& pool, size_t digits, size_t units) {
    const SrtPlan P = srt_plan(digits + 1);
    const size_t n = (pi_tenth_bits(P.w[0]) + 63) / 64 + 2;
    if (W.reserve_for(T, n, n) != cudaSuccess) cudaGetLastError();
    size_t cls = 2;
    while (cls < n) cls <<= 1;
    const size_t want = units * cls * 8, held = pool.held_bytes();
    if (held < want) pool.reserve_arena(want - held);
}

// Arena sizes in k-bit size classes: what the two finishes hold at the end of a 100M-digit run
// (the caller's pool 17 classes, the helper's 12).
constexpr size_t kFinishArenaUnits = 16;
constexpr size_t kHelperArenaUnits = 12;

// sqrt(10005) 2^k and the tree's powers of ten, computed by a helper host thread on the finish
// state's second stream (its own product workspace and pool) while the caller's stream runs the
// splitting and the reciprocal; join() waits for it and rethrows its error.
struct PiHelper {
    FinishState& fs;
    const DeviceTables& T;
    int device;
    uint64_t* ctx_launches;  // the helper's kernels are added here when it is done
    uint64_t launches = 0;
    std::unique_ptr<DevArith> A;
    std::unique_ptr<Num> S;
    std::vector<Num*> pw;
    std::exception_ptr err;
    std::thread th;
    PiHelper(FinishState& f, const DeviceTables& t, int dev, uint64_t* cl) : fs(f), T(t), device(dev), ctx_launches(cl) {}
    void start(size_t digits) {
        if (!fs.st2) {
            // default priority: the finish on the device's highest-priority stream instead sped up
            // the reciprocal's small levels but slowed the helper's powers of ten as much (final
            // formula 20.0 against 19.4 ms at 100M digits)
            if (cudaStreamCreateWithFlags(&fs.st2, cudaStreamNonBlocking) != cudaSuccess) {
                cudaGetLastError();
                fs.st2 = nullptr;
                throw DevError(PG_ERR_DEVICE, "helper stream");
            }
        }
        const SrtPlan P = srt_plan(digits + 1);
        const size_t k = pi_tenth_bits(P.w[0]);
        const int J = P.J;
        A.reset(new DevArith(T, fs.ws2, fs.st2, &launches, fs.pool2));
        th = std::thread([this, k, J, digits] {
            try {
                cudaSetDevice(device);
                {
                    Timer tm("helper buffers");
                    presize_finish(T, fs.ws2, fs.pool2, digits, kHelperArenaUnits);
                }
                S.reset(new Num(*A));
                {
                    Timer tm("sqrt(10005), helper stream");
                    sqrt_scaled(*A, S->v, 10005, k, false);
                }
                srt_powers(*A, J, pw);
                A->sync();
                throw_workspace_error(fs.ws2, fs.st2, "helper stream");
            } catch (...) {
                err = std::current_exception();
            }
        });
    }
    // Second task, once the first is done: X1 = 42688 Qt sqrt(10005) 2^k truncated to k bits (over1:
    // the bits dropped), on the helper stream after `ev` (recorded once Qt is on the caller's
    // stream), while the caller computes the reciprocal of R.
    std::unique_ptr<Num> X1;
    long long over1 = 0;
    void start_first_product(const DevNum* Qt, cudaEvent_t ev, size_t k) {
        std::thread prev = std::move(th);
        th = std::thread([this, Qt, ev, k, prev = std::move(prev)]() mutable {
            if (prev.joinable()) prev.join();
            if (err) return;
            try {
                cudaSetDevice(device);
                if (cudaStreamWaitEvent(fs.st2, ev, 0) != cudaSuccess) throw DevError(PG_ERR_DEVICE, "helper stream wait");
                Timer tm("42688 Q sqrt(10005), helper stream");
                X1.reset(new Num(*A));
                Num t(*A);
                A->mul_ui(*X1, *Qt, 42688);
                A->mul(t, *X1, S->v);
                const long long over = (long long)A->bits(t) - (long long)k;
                if (over > 0) {
                    A->tdiv_q_2exp(*X1, t, (size_t)over);
                    over1 = over;
                } else {
                    A->copy(*X1, t);
                    over1 = 0;
                }
                A->sync();
                throw_workspace_error(fs.ws2, fs.st2, "helper stream");
            } catch (...) {
                err = std::current_exception();
            }
        });
    }
    void join() {
        if (th.joinable()) th.join();
        if (err) std::rethrow_exception(err);
    }
    ~PiHelper() {
        if (th.joinable()) th.join();
        X1.reset();
        for (auto* p : pw) delete p;
        S.reset();
        A.reset();
        if (ctx_launches) *ctx_launches += launches;
    }
};

// y = pi / 10 to w limbs, V ~= y 2^(64 w) within a few units, from the series root Q, R: the final
// formula's truncated reciprocal, square root and products, 42688 sqrt(10005) Q / R. With a helper,
// sqrt(10005) comes from it and so does the first product, 42688 Q sqrt(10005), computed on its
// stream while this one computes the reciprocal of R.
void pi_tenth_fraction(DevArith& A, DevNum& V, const DevNum& Q, const DevNum& R, uint64_t w, PiHelper* helper) {
    if (Q.sign <= 0 || R.sign <= 0) throw DevError(PG_ERR_BAD_ARG, "final formula needs Q, R > 0");
    const size_t k = pi_tenth_bits(w);  // relative error 2^(5 - k): below 2^-59 of V's last unit
    const size_t bQ = A.bits(Q), bR = A.bits(R);
    Num Qt(A), Rt(A), Z(A), S(A), t(A);
    const long long eQ = (long long)bQ - (long long)k;
    const long long eR = (long long)bR - (long long)k;
    if (eQ >= 0) A.tdiv_q_2exp(Qt, Q, (size_t)eQ); else A.shl(Qt, Q, (size_t)-eQ);
    cudaEvent_t ev = nullptr;
    if (helper) {
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventRecord(ev, A.stream()) != cudaSuccess) {
            cudaGetLastError();
            if (ev) cudaEventDestroy(ev);
            throw DevError(PG_ERR_DEVICE, "final formula: event");
        }
        helper->start_first_product(&Qt.v, ev, k);
    }
    struct EventGuard {
        cudaEvent_t e;
        ~EventGuard() {
            if (e) cudaEventDestroy(e);
        }
    } eg{ev};
    if (eR >= 0) A.tdiv_q_2exp(Rt, R, (size_t)eR); else A.shl(Rt, R, (size_t)-eR);
    {
        Timer tm("reciprocal of R");
        recip_floor(A, Z, Rt, false);
    }
    long long e = eQ - eR - 3 * (long long)k;  // pi / 10 = V 2^e (before the truncations below)
    auto mul_trunc = [&](const DevNum& x, const DevNum& y) {
        A.mul(t, x, y);
        const long long over = (long long)A.bits(t) - (long long)k;
        if (over > 0) {
            A.tdiv_q_2exp(V, t, (size_t)over);
            e += over;
        } else {
            A.copy(V, t);
        }
    };
    if (helper) {
        helper->join();  // X1 = 42688 Qt S, truncated
        e += helper->over1;
        Timer tm("truncated product by the reciprocal");
        mul_trunc(helper->X1->v, Z);
    } else {
        {
            Timer tm("sqrt(10005)");
            sqrt_scaled(A, S, 10005, k, false);
        }
        Timer tm("two truncated products");
        A.mul_ui(V, Qt, 42688);
        mul_trunc(V, S);
        mul_trunc(V, Z);
    }
    const long long sh = e + 64 * (long long)w;  // V 2^e = (V 2^sh) / 2^(64 w)
    if (sh >= 0) A.shl(V, V, (size_t)sh); else A.fdiv_q_2exp(V, V, (size_t)-sh);
}

// "3." and `digits` digits of pi into out from the series root Q, R: the scaled remainder tree when
// every level fits one transform and no leaf is in doubt, otherwise the exact final formula and
// divide-and-conquer conversion. helper (optional, started for these digits) supplies sqrt(10005)
// and the powers of ten.
void pi_digits(DevArith& A, SharedProduct& sp, const DevNum& Q, const DevNum& R, size_t digits, char* out,
               double* t_final, PiHelper* helper = nullptr) {
    const auto t0 = std::chrono::steady_clock::now();
    const SrtPlan P = srt_plan(digits + 1);
    const bool tree = srt_fits(P) && !std::getenv("PG_EXACT_CONVERSION");
    char* body = out + 1;  // the integer's digits: "3" then the fraction digits
    if (tree) {
        Num V(A);
        pi_tenth_fraction(A, V, Q, R, P.w[0], helper);
        A.sync();
        if (t_final) *t_final = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (srt_digits(A, sp, P, V, body, helper ? &helper->pw : nullptr)) {
            out[0] = body[0];
            out[1] = '.';
            return;
        }
    }
    Num X(A);
    final_formula(A, X, Q, R, digits);
    A.sync();
    if (t_final && !tree) *t_final = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    to_decimal(A, sp, X, digits + 1, body);
    out[0] = body[0];
    out[1] = '.';
}

// ------------------------------------------------------------------ checkpoints
// Writes one integer held in HBM in the checkpoint format (ckpt_io.h): the header, then its
// bytes streamed through the pinned staging buffers.
bool write_dev(ckpt::File& f, DevArith& A, CkptStaging& S, const DevNum& x, bool with_sign) {
    cudaStream_t st = A.stream();
    S.ensure();
    size_t n = x.n;
    uint64_t top = 0;
    while (n) {  // the top limb (lengths are normalised; a zero top limb is only skipped)
        cudaMemcpyAsync(S.buf[0], x.d + n - 1, 8, cudaMemcpyDeviceToHost, st);
        A.sync();
        std::memcpy(&top, S.buf[0], 8);
        if (top) break;
        --n;
    }
    const size_t count = ckpt::byte_count(n, top);
    if (!ckpt::put_header(f, with_sign, n ? (x.sign < 0 ? -1 : 1) : 0, count)) return false;
    const char* src = reinterpret_cast<const char*>(x.d);
    auto issue = [&](size_t o, int b) {
        cudaMemcpyAsync(S.buf[b], src + o, std::min(CkptStaging::kChunk, count - o), cudaMemcpyDeviceToHost, st);
        cudaEventRecord(S.ev[b], st);
    };
    if (count) issue(0, 0);
    int b = 0;
    for (size_t o = 0; o < count; o += CkptStaging::kChunk, b ^= 1) {
        if (o + CkptStaging::kChunk < count) issue(o + CkptStaging::kChunk, b ^ 1);
        if (cudaEventSynchronize(S.ev[b]) != cudaSuccess) throw DevError(PG_ERR_DEVICE, "checkpoint copy");
        if (!f.put(S.buf[b], std::min(CkptStaging::kChunk, count - o))) {
            A.sync();
            return false;
        }
    }
    return true;
}

// Reads one integer of the checkpoint format into x (HBM); false when the file is short.
bool read_dev(ckpt::File& f, DevArith& A, CkptStaging& S, DevNum& x, bool with_sign) {
    cudaStream_t st = A.stream();
    S.ensure();
    int sign = 1;
    size_t count = 0;
    if (!ckpt::get_header(f, with_sign, sign, count)) return false;
    const size_t nl = (count + 7) / 8;
    A.reserve(x, std::max<size_t>(nl, 1));
    if (nl) cudaMemsetAsync(x.d + nl - 1, 0, 8, st);  // the partial top limb
    char* dst = reinterpret_cast<char*>(x.d);
    size_t used = 0;  // bytes up to the last nonzero byte
    bool ok = true;
    int b = 0;
    for (size_t o = 0; o < count; o += CkptStaging::kChunk, b ^= 1) {
        const size_t len = std::min(CkptStaging::kChunk, count - o);
        if (cudaEventSynchronize(S.ev[b]) != cudaSuccess) throw DevError(PG_ERR_DEVICE, "checkpoint copy");
        if (!f.get(S.buf[b], len)) {
            ok = false;
            break;
        }
        for (size_t k = len; k > 0; --k)
            if (S.buf[b][k - 1]) {
                used = o + k;
                break;
            }
        cudaMemcpyAsync(dst + o, S.buf[b], len, cudaMemcpyHostToDevice, st);
        cudaEventRecord(S.ev[b], st);
    }
    A.sync();
    if (!ok) return false;
    x.n = (used + 7) / 8;
    x.sign = x.n ? (sign < 0 ? -1 : 1) : 0;
    x.slack = 0;
    return true;
}

// P, Q, R of one splitting node in HBM.
struct Node {
    Num P, Q, R;
    explicit Node(DevArith& A) : P(A), Q(A), R(A) {}
    DevNum& at(int k) { return k == 0 ? P.v : (k == 1 ? Q.v : R.v); }
};

bool save_node(const std::string& path, DevArith& A, CkptStaging& S, Node& x) {
    ckpt::File f(path, "wb");
    if (!f) return false;
    for (int k = 0; k < 3; ++k)
        if (!write_dev(f, A, S, x.at(k), true)) return false;
    return f.close();
}

bool load_node(const std::string& path, DevArith& A, CkptStaging& S, Node& x) {
    ckpt::File f(path, "rb");
    if (!f) return false;
    for (int k = 0; k < 3; ++k)
        if (!read_dev(f, A, S, x.at(k), true)) return false;
    return true;
}

// The splitting of [a, b) resumed from the checkpoint files of a directory, as the reference's
// BinarySplitting::compute / compute_parallel / compute_sequential do with checkpointing on
// (src/engine/binary_splitting.cpp:295-302, 350-360, 605-644): a node of the tree (split point
// m = a + (b - a) / 2) whose bs_<a>_<b>.ckpt loads is taken from the file. Otherwise, when a
// file lies on a node below it, its halves are resolved and merged on the device
// (P = Pl Pr, Q = Ql Qr, R = Qr Rl + Pl Rr, binary_splitting.cpp:161-293); otherwise the whole
// range is one level-batched device splitting. A file that does not load (short or unreadable)
// counts as absent, as in the reference's load_bs_result. A range whose top merges need
// transforms longer than split_logL() is split the same way (with no directory this is how
// pi beyond ~300M digits runs: level-batched subtrees below, block products above).
class CkptSplit {
public:
    CkptSplit(pg_ctx* ctx, DevArith& A, CkptStaging& S, const std::string& dir, pg_ckpt_report& rep)
        : ctx_(ctx), A_(A), S_(S), dir_(dir), rep_(rep) {
        if (DIR* d = dir.empty() ? nullptr : opendir(dir.c_str())) {
            while (dirent* e = readdir(d)) {
                unsigned long fa = 0, fb = 0;
                int used = 0;
                if (std::sscanf(e->d_name, "bs_%lu_%lu.ckpt%n", &fa, &fb, &used) == 2 &&
                    e->d_name[used] == '\0' && fb > fa &&
                    std::string(e->d_name) == ckpt::bs_path("", fa, fb).substr(1))
                    files_.insert({fa, fb});
            }
            closedir(d);
        }
    }

    // Resolves [a, b) into x; true when x came from the file bs_<a>_<b>.ckpt itself.
    bool resolve(unsigned long a, unsigned long b, Node& x) {
        if (files_.count({a, b}) && load_node(ckpt::bs_path(dir_, a, b), A_, S_, x)) {
            ++rep_.nodes_loaded;
            return true;
        }
        if (b - a > 1 && has_inner(a, b)) {
            merge_halves(a, b, x);
            return false;
        }
        LevelView root;
        uint32_t hl[3];
        const pg_status s = bs_run_locked(ctx_, a, b, root, hl);
        if (s == PG_ERR_TOO_LARGE && b - a > 1) {
            // the top merges of [a, b) need longer transforms than one product may use: its
            // halves, merged with the device arithmetic (block products)
            ctx_set_error(ctx_, "");
            merge_halves(a, b, x);
            return false;
        }
        if (s != PG_OK) throw DevError(s, pg_last_error(ctx_));
        // signs over the series: P(a,b) = (-1)^(#k >= 1), Q > 0, R(a,b) has the sign of R(a, a+1)
        const unsigned long neg_terms = (b - a) - (a == 0 ? 1 : 0);
        const int sg[3] = {(neg_terms & 1) ? -1 : 1, 1, a == 0 ? 1 : -1};
        for (int k = 0; k < 3; ++k) {
            DevNum& v = x.at(k);
            A_.reserve(v, std::max<uint32_t>(hl[k], 1));
            if (hl[k]) cudaMemcpyAsync(v.d, root.X[k], (size_t)hl[k] * 8, cudaMemcpyDeviceToDevice, A_.stream());
            v.n = hl[k];
            v.sign = hl[k] ? sg[k] : 0;
            v.slack = 0;
        }
        ++rep_.subtrees_computed;
        return false;
    }

private:
    void merge_halves(unsigned long a, unsigned long b, Node& x) {
        const unsigned long m = a + (b - a) / 2;
        Node L(A_), Rn(A_);
        resolve(a, m, L);
        resolve(m, b, Rn);
        A_.mul(x.P, L.P, Rn.P);
        A_.mul(x.Q, L.Q, Rn.Q);
        Num t(A_), u(A_);
        A_.mul(t, Rn.Q, L.R);
        A_.mul(u, L.P, Rn.R);
        A_.add(x.R, t, u);
        ++rep_.merges;
    }

    // Is [fa, fb) a node of the tree rooted at [a, b)?
    static bool is_node(unsigned long a, unsigned long b, unsigned long fa, unsigned long fb) {
        while (true) {
            if (a == fa && b == fb) return true;
            if (b - a < 2) return false;
            const unsigned long m = a + (b - a) / 2;
            if (fb <= m)
                b = m;
            else if (fa >= m)
                a = m;
            else
                return false;
        }
    }
    // A file on a node strictly below [a, b)?
    bool has_inner(unsigned long a, unsigned long b) const {
        for (auto it = files_.lower_bound({a, 0}); it != files_.end() && it->first < b; ++it)
            if (it->second <= b && !(it->first == a && it->second == b) && is_node(a, b, it->first, it->second))
                return true;
        return false;
    }

    pg_ctx* ctx_;
    DevArith& A_;
    CkptStaging& S_;
    std::string dir_;
    pg_ckpt_report& rep_;
    std::set<std::pair<unsigned long, unsigned long>> files_;
};

// The reference's BinarySplitting::compute(a, b) with checkpointing on: resume from the
// directory, and save bs_<a>_<b>.ckpt at the end unless it was loaded, removing the two
// children's files (save_checkpoint, binary_splitting.cpp:121-135; compute always saves its
// final result, :639-641).
void split_checkpointed(pg_ctx* ctx, DevArith& A, CkptStaging& S, const std::string& dir, unsigned long a,
                        unsigned long b, Node& x, pg_ckpt_report& rep) {
    mkdir(dir.c_str(), 0755);  // enable_checkpointing (binary_splitting.cpp:104-109)
    CkptSplit split(ctx, A, S, dir, rep);
    if (split.resolve(a, b, x)) {
        rep.root_loaded = 1;
        return;
    }
    if (save_node(ckpt::bs_path(dir, a, b), A, S, x)) {
        rep.root_saved = 1;
        if (b - a > 1) {
            const unsigned long m = a + (b - a) / 2;
            std::remove(ckpt::bs_path(dir, a, m).c_str());
            std::remove(ckpt::bs_path(dir, m, b).c_str());
        }
    }
}

pg_status fail(pg_ctx* c, pg_status s, const std::string& m) {
    ctx_set_error(c, m);
    return s;
}

// Reads and clears the product engine's error word.
pg_status product_errors(pg_ctx* ctx) {
    Workspace& W = ctx_workspace(ctx);
    cudaStream_t st = ctx_stream(ctx);
    uint32_t err = 0;
    if (W.sync) cudaMemcpyAsync(&err, W.sync, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(ctx, PG_ERR_DEVICE, "device error");
    if (err) {
        cudaMemsetAsync(W.sync, 0, 4, st);
        cudaStreamSynchronize(st);
        const char* what = "";
        const pg_status s = workspace_error_status(err, what);
        return fail(ctx, s, what);
    }
    return PG_OK;
}

// Runs f, then reports the kernels' error word; when f throws, an error the kernels recorded
// (a wait that ran out, say) is reported first: it is the cause, the throw its consequence.
template <class F>
pg_status guarded(pg_ctx* ctx, F&& f) {
    try {
        f();
    } catch (const DevError& e) {
        const std::string what = e.what();
        const pg_status k = product_errors(ctx);
        return k != PG_OK ? k : fail(ctx, e.status, what);
    } catch (const std::exception& e) {
        const std::string what = e.what();
        const pg_status k = product_errors(ctx);
        return k != PG_OK ? k : fail(ctx, PG_ERR_INTERNAL, what);
    }
    return product_errors(ctx);
}

}  // namespace

pg_status bs_split_to_host(pg_ctx* ctx, unsigned long a, unsigned long b, uint64_t* P, uint64_t* Q, uint64_t* R,
                           size_t cap, size_t* len, int* sign) {
    return guarded(ctx, [&] {
        FinishState& fs = *ctx_finish(ctx);
        DevArith A(ctx_tables(ctx), ctx_workspace(ctx), ctx_stream(ctx), ctx_launches(ctx), fs.pool);
        Node x(A);
        pg_ckpt_report rep{};
        CkptSplit split(ctx, A, fs.stage, "", rep);
        split.resolve(a, b, x);
        uint64_t* dst[3] = {P, Q, R};
        for (int k = 0; k < 3; ++k) A.exact(x.at(k));
        for (int k = 0; k < 3; ++k)
            if (dst[k] && x.at(k).n > cap) throw DevError(PG_ERR_BAD_ARG, "output buffers smaller than the result");
        for (int k = 0; k < 3; ++k) {
            len[k] = x.at(k).n;
            sign[k] = x.at(k).sign;
            if (dst[k]) A.download(x.at(k), dst[k]);
        }
    });
}

}  // namespace pg

extern "C" {

pg_status pg_recip_floor(pg_ctx* ctx, const uint64_t* r, size_t nr, uint64_t* z, size_t zcap, size_t* zlen) {
    if (!ctx || !r || !z || !zlen || nr == 0) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaSetDevice(pg::ctx_device(ctx));
    return pg::guarded(ctx, [&] {
        pg::FinishState& fs = *pg::ctx_finish(ctx);
        pg::DevArith A(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_stream(ctx), pg::ctx_launches(ctx), fs.pool);
        pg::Num R(A), Z(A);
        A.upload(R, r, nr, 1);
        if (R.v.sign == 0) throw pg::DevError(PG_ERR_BAD_ARG, "pg_recip_floor: R is zero");
        pg::recip_floor(A, Z, R);
        A.exact(Z);
        if (Z.v.n > zcap) throw pg::DevError(PG_ERR_BAD_ARG, "pg_recip_floor: output buffer too small");
        A.download(Z, z);
        *zlen = Z.v.n;
    });
}

pg_status pg_mul_wrap(pg_ctx* ctx, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, int logL, uint64_t* out,
                      size_t cap, size_t* len) {
    if (!ctx || !out || !len || (na && !a) || (nb && !b) || logL < pg::kMinLogL || logL > pg::kMaxLogL)
        return PG_ERR_BAD_ARG;
    const size_t half = (size_t)1 << (logL - 1);
    if (na > half || nb > half) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaSetDevice(pg::ctx_device(ctx));
    return pg::guarded(ctx, [&] {
        pg::FinishState& fs = *pg::ctx_finish(ctx);
        pg::DevArith A(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_stream(ctx), pg::ctx_launches(ctx), fs.pool);
        pg::Num X(A), Y(A), Z(A);
        A.upload(X, a, na, 1);
        A.upload(Y, b, nb, 1);
        A.mul_wrap(Z, X, Y, logL);
        A.exact(Z);
        if (Z.v.n > cap) throw pg::DevError(PG_ERR_BAD_ARG, "pg_mul_wrap: output buffer too small");
        A.download(Z, out);
        *len = Z.v.n;
    });
}

pg_status pg_sqrt_scaled(pg_ctx* ctx, uint64_t a, size_t s, uint64_t* out, size_t cap, size_t* len) {
    if (!ctx || !out || !len || a < 1) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaSetDevice(pg::ctx_device(ctx));
    return pg::guarded(ctx, [&] {
        pg::FinishState& fs = *pg::ctx_finish(ctx);
        pg::DevArith A(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_stream(ctx), pg::ctx_launches(ctx), fs.pool);
        pg::Num S(A);
        pg::sqrt_scaled(A, S, a, s);
        A.exact(S);
        if (S.v.n > cap) throw pg::DevError(PG_ERR_BAD_ARG, "pg_sqrt_scaled: output buffer too small");
        A.download(S, out);
        *len = S.v.n;
    });
}

pg_status pg_to_decimal(pg_ctx* ctx, const uint64_t* x, size_t nx, size_t ndigits, char* out) {
    if (!ctx || (nx && !x) || (ndigits && !out)) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaSetDevice(pg::ctx_device(ctx));
    return pg::guarded(ctx, [&] {
        pg::FinishState& fs = *pg::ctx_finish(ctx);
        pg::DevArith A(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_stream(ctx), pg::ctx_launches(ctx), fs.pool);
        pg::Num X(A);
        A.upload(X, x, nx, 1);
        // x < 10^ndigits is required: check by bit length against 10^ndigits's (upper bound)
        if ((double)A.bits(X) > (double)ndigits * 3.3219280948873623 + 1)
            throw pg::DevError(PG_ERR_BAD_ARG, "pg_to_decimal: x has more than ndigits digits");
        pg::to_decimal(A, fs.sp, X, ndigits, out);
    });
}

pg_status pg_pi_finish(pg_ctx* ctx, const uint64_t* q, size_t nq, const uint64_t* r, size_t nr, size_t digits,
                       char* out) {
    if (!ctx || !q || !r || !out || nq == 0 || nr == 0) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    pg::DeferFrees defer;  // no cudaFree (a wait for the idle device) until the call returns
    cudaSetDevice(pg::ctx_device(ctx));
    return pg::guarded(ctx, [&] {
        pg::FinishState& fs = *pg::ctx_finish(ctx);
        pg::DevArith A(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_stream(ctx), pg::ctx_launches(ctx), fs.pool);
        std::unique_ptr<pg::PiHelper> helper;
        if (pg::pi_tree_path(digits)) {
            helper.reset(new pg::PiHelper(fs, pg::ctx_tables(ctx), pg::ctx_device(ctx), pg::ctx_launches(ctx)));
            helper->start(digits);
        }
        pg::Num Q(A), R(A);
        A.upload(Q, q, nq, 1);
        A.upload(R, r, nr, 1);
        pg::pi_digits(A, fs.sp, Q, R, digits, out, nullptr, helper.get());
    });
}

pg_status pg_pi(pg_ctx* ctx, size_t digits, char* out, double* seconds) {
    if (!ctx || !out || digits == 0) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    pg::DeferFrees defer;  // no cudaFree (a wait for the idle device) until the call returns
    cudaSetDevice(pg::ctx_device(ctx));
    const auto t0 = std::chrono::steady_clock::now();
    auto secs = [](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
    };
    // terms as the reference's PiEngine: terms_needed(digits + 100) (pi_engine.cpp:214-220,
    // binary_splitting.cpp terms_needed); each term adds log10(151931373056000) ~= 14.18 digits
    const unsigned long terms = (unsigned long)std::ceil((double)(digits + 100) / 14.1816474627) + 1;
    // sqrt(10005) and the powers of ten on the helper stream, alongside the splitting
    std::unique_ptr<pg::PiHelper> helper;
    if (pg::pi_tree_path(digits)) {
        try {
            helper.reset(new pg::PiHelper(*pg::ctx_finish(ctx), pg::ctx_tables(ctx), pg::ctx_device(ctx),
                                          pg::ctx_launches(ctx)));
            helper->start(digits);
        } catch (...) {
            helper.reset();  // no helper: pi_digits computes both itself
        }
    }
    pg::LevelView root;
    uint32_t hl[3];
    std::unique_ptr<pg::Timer> tbs(new pg::Timer("binary splitting"));
    // while the splitting runs: the finish's buffers (tree path)
    std::function<void()> presize;
    if (helper)
        presize = [&] {
            pg::Timer tm("finish buffers, during the splitting");
            pg::presize_finish(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_finish(ctx)->pool, digits,
                               pg::kFinishArenaUnits);
        };
    pg_status s = pg::bs_run_locked(ctx, 0, terms, root, hl, false, &presize);  // the root's P is not used
    tbs.reset();
    const bool big = (s == PG_ERR_TOO_LARGE);  // split into subtrees below, merged on the device
    if (s != PG_OK && !big) return s;
    if (big) pg::ctx_set_error(ctx, "");
    double t_bs = secs(t0), t_final = 0;
    auto t1 = std::chrono::steady_clock::now();
    s = pg::guarded(ctx, [&] {
        pg::FinishState& fs = *pg::ctx_finish(ctx);
        pg::DevArith A(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_stream(ctx), pg::ctx_launches(ctx), fs.pool);
        // Q, R of the root (both positive for a = 0)
        pg::Num Q(A), R(A);
        if (big) {
            pg::Node x(A);
            pg_ckpt_report rep{};
            pg::CkptSplit split(ctx, A, fs.stage, "", rep);
            split.resolve(0, terms, x);
            std::swap(Q.v, x.Q.v);
            std::swap(R.v, x.R.v);
            A.sync();
            t_bs = secs(t0);
            t1 = std::chrono::steady_clock::now();
        } else {  // copied out of the splitting buffers
            A.reserve(Q, hl[1]);
            A.reserve(R, hl[2]);
            cudaMemcpyAsync(Q.v.d, root.X[1], (size_t)hl[1] * 8, cudaMemcpyDeviceToDevice, A.stream());
            cudaMemcpyAsync(R.v.d, root.X[2], (size_t)hl[2] * 8, cudaMemcpyDeviceToDevice, A.stream());
            Q.v.n = hl[1];
            Q.v.sign = hl[1] ? 1 : 0;
            R.v.n = hl[2];
            R.v.sign = hl[2] ? 1 : 0;
            Q.v.slack = R.v.slack = 0;
        }
        {
            pg::Timer tf("final formula and digits");
            pg::pi_digits(A, fs.sp, Q, R, digits, out, &t_final, helper.get());
        }
        if (pg::trace_on()) pg::trace_buffers(ctx, fs);
    });
    if (seconds) {
        seconds[0] = t_bs;
        seconds[1] = t_final;
        seconds[2] = secs(t1) - t_final;
        seconds[3] = secs(t0);
    }
    return s;
}

pg_status pg_bs_checkpointed(pg_ctx* ctx, unsigned long a, unsigned long b, const char* dir, uint64_t* P, uint64_t* Q,
                             uint64_t* R, size_t cap, size_t* len, int* sign, pg_ckpt_report* report) {
    if (!ctx || !dir || !*dir || !Q || !R || !len || !sign || b <= a) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    cudaSetDevice(pg::ctx_device(ctx));
    pg_ckpt_report rep{};
    const pg_status s = pg::guarded(ctx, [&] {
        pg::FinishState& fs = *pg::ctx_finish(ctx);
        pg::DevArith A(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_stream(ctx), pg::ctx_launches(ctx), fs.pool);
        pg::Node x(A);
        pg::split_checkpointed(ctx, A, fs.stage, dir, a, b, x, rep);
        uint64_t* dst[3] = {P, Q, R};
        for (int k = 0; k < 3; ++k) A.exact(x.at(k));
        for (int k = 0; k < 3; ++k)
            if (dst[k] && x.at(k).n > cap) throw pg::DevError(PG_ERR_BAD_ARG, "output buffers smaller than the result");
        for (int k = 0; k < 3; ++k) {
            len[k] = x.at(k).n;
            sign[k] = x.at(k).sign;
            if (dst[k]) A.download(x.at(k), dst[k]);
        }
    });
    if (report) *report = rep;
    return s;
}

pg_status pg_pi_checkpointed(pg_ctx* ctx, size_t digits, const char* dir, char* out, double* seconds,
                             pg_ckpt_report* report) {
    if (!ctx || !out || !dir || !*dir || digits == 0) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    pg::DeferFrees defer;  // no cudaFree (a wait for the idle device) until the call returns
    cudaSetDevice(pg::ctx_device(ctx));
    const auto t0 = std::chrono::steady_clock::now();
    auto secs = [](std::chrono::steady_clock::time_point t) {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
    };
    const unsigned long terms = (unsigned long)std::ceil((double)(digits + 100) / 14.1816474627) + 1;
    pg_ckpt_report rep{};
    double t_bs = 0, t_final = 0, t_conv = 0;
    const pg_status s = pg::guarded(ctx, [&] {
        pg::FinishState& fs = *pg::ctx_finish(ctx);
        pg::DevArith A(pg::ctx_tables(ctx), pg::ctx_workspace(ctx), pg::ctx_stream(ctx), pg::ctx_launches(ctx), fs.pool);
        pg::Num X(A);
        {
            // the splitting first, resumed or not, then the pi_int file: the reference's order
            // (pi_engine.cpp:245, then 263-284)
            pg::Node root(A);
            pg::split_checkpointed(ctx, A, fs.stage, dir, 0, terms, root, rep);
            t_bs = secs(t0);
            const auto t1 = std::chrono::steady_clock::now();
            const std::string path = pg::ckpt::pi_int_path(dir, digits);
            bool loaded = false;
            {
                pg::ckpt::File f(path, "rb");
                loaded = f && pg::read_dev(f, A, fs.stage, X.v, false) && X.v.n > 0;
            }
            if (loaded) {
                rep.pi_int_loaded = 1;
            } else {
                pg::final_formula(A, X, root.Q, root.R, digits);
                pg::ckpt::File f(path, "wb");
                if (f && pg::write_dev(f, A, fs.stage, X.v, false) && f.close()) rep.pi_int_saved = 1;
            }
            t_final = secs(t1);
        }
        const auto t2 = std::chrono::steady_clock::now();
        char* body = out + 1;
        pg::to_decimal(A, fs.sp, X, digits + 1, body);
        out[0] = body[0];
        out[1] = '.';
        t_conv = secs(t2);
    });
    if (report) *report = rep;
    if (seconds) {
        seconds[0] = t_bs;
        seconds[1] = t_final;
        seconds[2] = t_conv;
        seconds[3] = secs(t0);
    }
    return s;
}

}  // extern "C"
