// Level-batched, device-resident Chudnovsky binary splitting.
//
// Replaces the reference's recursive BinarySplitting (src/engine/binary_splitting.cpp:295-394,
// 605-644) for the GPU: the same tree (range [a, b) split at m = a + (b - a)/2, so every
// P/Q/R equals the reference's) is evaluated bottom-up one depth at a time, every merge of a
// depth in the same launches, with all operands resident in HBM:
//
//   depth D-1 (D = ceil(log2(b - a)))   nodes of 1 or 2 terms: one thread each, leaf formulas
//                                       (binary_splitting.cpp:137-159) and one merge in registers
//   small depths                        one warp per merge, schoolbook products in shared memory
//   larger depths                       batched NTT: forward transforms of Pl Ql Rl Pr Qr Rr for every
//                                       merge, one pointwise pass producing P^ = Pl^Pr^, Q^ = Ql^Qr^ and
//                                       R^ = Qr^Rl^ + s Pl^Rr^, three inverse transforms, one CRT+carry
//                                       launch for all outputs (signed lift for R when s = -1)
//
// Node i of depth d merges nodes 2i and 2i+1 of depth d+1 (every depth above D-1 is full).
// Magnitudes only are stored; signs follow from the node range (see merge_r_sign).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <functional>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pi_b200.h"
#include "ntt_engine.cuh"
#include "series.cuh"

namespace pg {

// ------------------------------------------------------------------ small multi-limb helpers
typedef unsigned __int128 u128;

// out[0 .. nx+ny) = x * y (schoolbook, 64-bit limbs).
__device__ __forceinline__ void sb_mul(const uint64_t* x, int nx, const uint64_t* y, int ny, uint64_t* out) {
    for (int i = 0; i < nx + ny; ++i) out[i] = 0;
    for (int i = 0; i < nx; ++i) {
        uint64_t carry = 0;
        for (int k = 0; k < ny; ++k) {
            u128 t = (u128)x[i] * y[k] + out[i + k] + carry;
            out[i + k] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
        out[i + ny] = carry;
    }
}

__device__ __forceinline__ int sb_len(const uint64_t* x, int n) {
    while (n > 0 && x[n - 1] == 0) --n;
    return n;
}

// x[0..n) += s * y[0..ny) (s = +1 or -1); for s = -1 the result must be non-negative.
__device__ __forceinline__ void sb_addsub(uint64_t* x, int n, const uint64_t* y, int ny, int s) {
    if (s > 0) {
        uint64_t c = 0;
        for (int i = 0; i < n; ++i) {
            u128 t = (u128)x[i] + (i < ny ? y[i] : 0) + c;
            x[i] = (uint64_t)t;
            c = (uint64_t)(t >> 64);
        }
    } else {
        uint64_t br = 0;
        for (int i = 0; i < n; ++i) {
            const uint64_t yi = i < ny ? y[i] : 0;
            const uint64_t d = x[i] - yi - br;
            br = (x[i] < yi) || (x[i] - yi < br);
            x[i] = d;
        }
    }
}

// Carry resolution of n <= G * K limbs across a group of G lanes (G a power of two <= 32; the
// groups tile the warp and every lane of the warp calls this together): limb i's value before
// carries is v(i), a signed 128-bit number in (-2^65, 3 * 2^64); the carries between limbs lie in
// {-1, 0, 1, 2}. Each lane takes K consecutive limbs, tabulates its carry transfer function (carry
// in -> carry out, four two-bit entries of carry + 1), and a scan of the functions over the group
// gives every lane its carry in. Writes dst[0 .. n) and returns the length without leading zero
// limbs (in every lane of the group). Every lane reads its v(i) before any lane writes dst.
template <int K, int G, class V>
__device__ __forceinline__ int group_resolve(V v, int n, uint64_t* dst) {
    typedef __int128 i128;
    const int gl = threadIdx.x & (G - 1);
    const int c0 = gl * K;
    i128 val[K];
#pragma unroll
    for (int i = 0; i < K; ++i) val[i] = c0 + i < n ? v(c0 + i) : 0;
    auto apply = [](uint32_t f, uint32_t u) { return (f >> (2 * u)) & 3u; };
    auto compose = [&](uint32_t g, uint32_t f) {  // g after f
        return apply(g, apply(f, 0)) | (apply(g, apply(f, 1)) << 2) | (apply(g, apply(f, 2)) << 4) |
               (apply(g, apply(f, 3)) << 6);
    };
    uint32_t f = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        long long c = u - 1;
#pragma unroll
        for (int i = 0; i < K; ++i) c = (long long)((val[i] + c) >> 64);
        const long long uo = c + 1 < 0 ? 0 : (c + 1 > 3 ? 3 : c + 1);  // out of range only off the real path
        f |= (uint32_t)uo << (2 * u);
    }
    uint32_t incl = f;
#pragma unroll
    for (int off = 1; off < G; off <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, off, G);
        if (gl >= off) incl = compose(incl, x);
    }
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1, G);
    if (gl == 0) excl = 0u | (1u << 2) | (2u << 4) | (3u << 6);
    long long c = (long long)apply(excl, 1u) - 1;
    int top = -1;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        if (c0 + i < n) {
            const i128 t = val[i] + c;
            dst[c0 + i] = (uint64_t)t;
            if ((uint64_t)t) top = c0 + i;
            c = (long long)(t >> 64);
        }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) top = max(top, __shfl_xor_sync(0xffffffffu, top, off, G));
    return top + 1;
}

// Leaf magnitudes of term k (binary_splitting.cpp:137-159): |P| = (6k-5)(2k-1)(6k-1),
// Q = k^3 * 640320^3/24, |R| = |P| * (13591409 + 545140134 k); k = 0: 1, 1, 13591409.
__device__ void leaf_values(uint64_t k, uint64_t P[2], int& nP, uint64_t Q[3], int& nQ, uint64_t R[3], int& nR) {
    if (k == 0) {
        P[0] = 1; P[1] = 0; nP = 1;
        Q[0] = 1; Q[1] = Q[2] = 0; nQ = 1;
        R[0] = 13591409; R[1] = R[2] = 0; nR = 1;
        return;
    }
    const u128 p = (u128)(6 * k - 5) * (2 * k - 1) * (6 * k - 1);   // < 2^100 for k < 2^32
    P[0] = (uint64_t)p; P[1] = (uint64_t)(p >> 64);
    nP = sb_len(P, 2);
    const u128 k3 = (u128)k * k * k;                                   // < 2^96
    const uint64_t C = 10939058860032000ull;                           // 640320^3 / 24
    const u128 lo = (u128)(uint64_t)k3 * C;
    const u128 hi = (u128)(uint64_t)(k3 >> 64) * C + (uint64_t)(lo >> 64);
    Q[0] = (uint64_t)lo; Q[1] = (uint64_t)hi; Q[2] = (uint64_t)(hi >> 64);
    nQ = sb_len(Q, 3);
    const uint64_t lin = 13591409ull + 545140134ull * k;               // < 2^62
    const u128 r0 = (u128)P[0] * lin;
    const u128 r1 = (u128)P[1] * lin + (uint64_t)(r0 >> 64);
    R[0] = (uint64_t)r0; R[1] = (uint64_t)r1; R[2] = (uint64_t)(r1 >> 64);
    nR = sb_len(R, 3);
}


// Depth D-1: node i covers 1 or 2 terms. Caps: P 4, Q 6, R 8 limbs (7 needed, kept even).
__global__ void bs_pair_kernel(LevelView out, uint64_t nodes, uint64_t a0, uint64_t b0, int depth) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    uint64_t a, b;
    node_range(a0, b0, depth, i, a, b);
    uint64_t* P = out.X[0] + i * out.cap[0];
    uint64_t* Q = out.X[1] + i * out.cap[1];
    uint64_t* R = out.X[2] + i * out.cap[2];
    uint64_t Pl[2], Ql[3], Rl[3];
    int nPl, nQl, nRl;
    leaf_values(a, Pl, nPl, Ql, nQl, Rl, nRl);
    int nP, nQ, nR;
    if (b - a == 1) {
        for (int t = 0; t < 2; ++t) P[t] = Pl[t];
        for (int t = 0; t < 3; ++t) Q[t] = Ql[t], R[t] = Rl[t];
        nP = nPl; nQ = nQl; nR = nRl;
    } else {
        uint64_t Pr[2], Qr[3], Rr[3];
        int nPr, nQr, nRr;
        leaf_values(a + 1, Pr, nPr, Qr, nQr, Rr, nRr);
        uint64_t x[7], y[7];
        sb_mul(Pl, nPl, Pr, nPr, x);
        nP = sb_len(x, nPl + nPr);
        for (int t = 0; t < 4; ++t) P[t] = t < nPl + nPr ? x[t] : 0;
        sb_mul(Ql, nQl, Qr, nQr, x);
        nQ = sb_len(x, nQl + nQr);
        for (int t = 0; t < 6; ++t) Q[t] = t < nQl + nQr ? x[t] : 0;
        for (int t = 0; t < 7; ++t) x[t] = y[t] = 0;
        sb_mul(Qr, nQr, Rl, nRl, x);
        sb_mul(Pl, nPl, Rr, nRr, y);
        sb_addsub(x, 7, y, 7, merge_r_sign(a, b));
        nR = sb_len(x, 7);
        for (int t = 0; t < 7; ++t) R[t] = x[t];
    }
    out.len[3 * i + 0] = nP;
    out.len[3 * i + 1] = nQ;
    out.len[3 * i + 2] = nR;
}

// One thread per merge for children of at most MAXC limbs (schoolbook in thread-local arrays):
// the bottom depths have millions of merges of a few limbs each.
template <int MAXC>
__global__ void __launch_bounds__(128) bs_thread_merge_kernel(LevelView in, LevelView out, uint64_t merges,
                                                              uint64_t a0, uint64_t b0, int depth) {
    const uint64_t m = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= merges) return;
    uint64_t op[6][MAXC];
    int n[6];
#pragma unroll
    for (int o = 0; o < 6; ++o) {
        const uint64_t child = 2 * m + (o >= 3 ? 1 : 0);
        const int k = o % 3;
        n[o] = (int)in.len[3 * child + k];
        const uint64_t* src = in.X[k] + child * in.cap[k];
        for (int t = 0; t < n[o]; ++t) op[o][t] = src[t];
    }
    uint64_t a, b;
    node_range(a0, b0, depth, m, a, b);
    const int sgn = merge_r_sign(a, b);
    uint64_t r0[2 * MAXC + 1], r1[2 * MAXC];
    auto emit = [&](int k, const uint64_t* v, int nv) {
        uint64_t* dst = out.X[k] + m * out.cap[k];
        const int l = sb_len(v, nv < (int)out.cap[k] ? nv : (int)out.cap[k]);
        for (int t = 0; t < (int)out.cap[k]; ++t) dst[t] = t < l ? v[t] : 0;
        out.len[3 * m + k] = l;
    };
    // P = Pl * Pr
    if (n[0] && n[3]) {
        sb_mul(op[0], n[0], op[3], n[3], r0);
        emit(0, r0, n[0] + n[3]);
    } else {
        emit(0, r0, 0);
    }
    // Q = Ql * Qr
    sb_mul(op[1], n[1], op[4], n[4], r0);
    emit(1, r0, n[1] + n[4]);
    // R = Qr * Rl + s * Pl * Rr
    const int lx = n[4] + n[2], ly = n[0] + n[5];
    sb_mul(op[4], n[4], op[2], n[2], r0);
    if (n[0] && n[5]) {
        sb_mul(op[0], n[0], op[5], n[5], r1);
    }
    const int nr = (lx > ly ? lx : ly) + 1;
    for (int t = lx; t < nr; ++t) r0[t] = 0;
    if (n[0] && n[5]) sb_addsub(r0, nr, r1, ly, sgn);
    emit(2, r0, nr);
}

// A group of G lanes per merge with operands of at most MAXC limbs (shared-memory schoolbook),
// 128 / G merges per block: the lanes of a group take the product's columns in turn, each column
// summed in two independent 192-bit chains, and resolve the carries together (group_resolve).
// Groups sized to the operands keep every lane busy from the bottom depths (millions of merges of
// a few limbs) up to 64-limb children, with no per-thread arrays in local memory. Every lane of a
// warp runs every step (the shuffles need them all): a group past the last merge computes zeros
// and stores nothing.
template <int MAXC, int G>
__global__ void __launch_bounds__(128) bs_group_merge_kernel(LevelView in, LevelView out, uint64_t merges,
                                                             uint64_t a0, uint64_t b0, int depth) {
    constexpr int NG = 128 / G;  // merges per block
    __shared__ uint64_t s_op[NG][6][MAXC];
    __shared__ uint64_t s_col[NG][3][2 * MAXC];  // 192-bit column sums: lo, mid, hi
    __shared__ uint64_t s_res[NG][2][2 * MAXC + 1];
    const int g = threadIdx.x / G, gl = threadIdx.x & (G - 1);
    const uint64_t m = (uint64_t)blockIdx.x * NG + g;
    const bool live = m < merges;
    if (!__any_sync(0xffffffffu, live)) return;  // whole warps past the end
    // load Pl Ql Rl Pr Qr Rr
    int n[6];
    for (int o = 0; o < 6; ++o) {
        const uint64_t child = 2 * m + (o >= 3 ? 1 : 0);
        const int k = o % 3;
        n[o] = live ? (int)in.len[3 * child + k] : 0;
        const uint64_t* src = in.X[k] + child * in.cap[k];
        for (int t = gl; t < MAXC; t += G) s_op[g][o][t] = t < n[o] ? src[t] : 0;
    }
    __syncwarp();
    uint64_t a = 0, b = 0;
    if (live) node_range(a0, b0, depth, m, a, b);
    const int sgn = live ? merge_r_sign(a, b) : 1;

    // product helper: column sums, then the group's carry resolution into dst (nx + ny limbs);
    // an empty operand gives 0
    constexpr int KR = (2 * MAXC + 1 + G - 1) / G;
    auto product = [&](int ox, int oy, uint64_t* dst) -> int {
        const int nx = n[ox], ny = n[oy];
        const uint64_t* x = s_op[g][ox];
        const uint64_t* y = s_op[g][oy];
        const int ncol = nx + ny - 1;
        auto acc = [](uint64_t& lo, uint64_t& mid, uint64_t& hi, u128 t) {
            const u128 s = (u128)lo + (uint64_t)t;
            lo = (uint64_t)s;
            const u128 s2 = (u128)mid + (uint64_t)(t >> 64) + (uint64_t)(s >> 64);
            mid = (uint64_t)s2;
            hi += (uint64_t)(s2 >> 64);
        };
        for (int c = gl; c < ncol; c += G) {
            uint64_t lo = 0, mid = 0, hi = 0, lo2 = 0, mid2 = 0, hi2 = 0;
            const int i0 = c - ny + 1 > 0 ? c - ny + 1 : 0;
            const int i1 = c < nx - 1 ? c : nx - 1;
            int i = i0;
            for (; i + 1 <= i1; i += 2) {
                acc(lo, mid, hi, (u128)x[i] * y[c - i]);
                acc(lo2, mid2, hi2, (u128)x[i + 1] * y[c - i - 1]);
            }
            if (i <= i1) acc(lo, mid, hi, (u128)x[i] * y[c - i]);
            acc(lo, mid, hi, lo2);
            acc(lo, mid, hi, (u128)mid2 << 64);
            hi += hi2;
            s_col[g][0][c] = lo;
            s_col[g][1][c] = mid;
            s_col[g][2][c] = hi;
        }
        __syncwarp();
        // limb c = lo_c + mid_{c-1} + hi_{c-2} (each < 2^64; column sums < MAXC 2^128, so hi < MAXC)
        const uint64_t* cl = s_col[g][0];
        const uint64_t* cm = s_col[g][1];
        const uint64_t* ch = s_col[g][2];
        const int len = group_resolve<KR, G>(
            [&](int c) {
                __int128 t = c < ncol ? cl[c] : 0;
                if (c >= 1 && c - 1 < ncol) t += cm[c - 1];
                if (c >= 2 && c - 2 < ncol) t += ch[c - 2];
                return t;
            },
            nx + ny, dst);
        __syncwarp();
        return len;
    };
    auto store = [&](int k, const uint64_t* v, int l, int lenv) {
        if (live) {
            uint64_t* dst = out.X[k] + m * out.cap[k];
            for (int t = gl; t < (int)out.cap[k]; t += G) dst[t] = t < l ? v[t] : 0;
            if (gl == 0) out.len[3 * m + k] = lenv;
        }
        __syncwarp();
    };

    // P = Pl * Pr
    {
        const int l = product(0, 3, s_res[g][0]);
        store(0, s_res[g][0], l, l);
    }
    // Q = Ql * Qr
    {
        const int l = product(1, 4, s_res[g][0]);
        store(1, s_res[g][0], l, l);
    }
    // R = Qr * Rl + s * Pl * Rr
    {
        const int lx = product(4, 2, s_res[g][0]);
        const int ly = product(0, 5, s_res[g][1]);
        // |R| < 2 max(|Qr Rl|, |Pl Rr|): max(lx, ly) + 1 limbs; limb i = x_i + sgn y_i before carries
        const int nr = (lx > ly ? lx : ly) + 1;
        const uint64_t* x = s_res[g][0];
        const uint64_t* y = s_res[g][1];
        uint64_t* r = s_res[g][0];  // in place over x: every lane reads its limbs before any writes
        const int lr = group_resolve<KR, G>(
            [&](int i) {
                const __int128 xi = i < lx ? x[i] : 0, yi = i < ly ? y[i] : 0;
                return sgn > 0 ? xi + yi : xi - yi;
            },
            nr, r);
        __syncwarp();
        store(2, r, nr, lr < (int)out.cap[2] ? lr : (int)out.cap[2]);
    }
}

// ------------------------------------------------------------------ host side
namespace {

int bitlen128(u128 x) {
    const uint64_t hi = (uint64_t)(x >> 64), lo = (uint64_t)x;
    if (hi) return 128 - __builtin_clzll(hi);
    return lo ? 64 - __builtin_clzll(lo) : 0;
}

}  // namespace

bool trace_on() {
    static const bool on = [] {
        const char* e = std::getenv("PI_B200_TRACE");
        return e && *e && *e != '0';
    }();
    return on;
}

namespace {

// Exact bit lengths of the leaf magnitudes of term k.
void leaf_bits(uint64_t k, int& bp, int& bq, int& br) {
    if (k == 0) {
        bp = 1;
        bq = 1;
        br = 24;
        return;
    }
    const u128 p = (u128)(6 * k - 5) * (2 * k - 1) * (6 * k - 1);
    bp = bitlen128(p);
    const u128 k3 = (u128)k * k * k;
    const u128 lo = (u128)(uint64_t)k3 * 10939058860032000ull;
    const u128 hi = (u128)(uint64_t)(k3 >> 64) * 10939058860032000ull + (uint64_t)(lo >> 64);
    bq = hi ? 64 + bitlen128(hi) : bitlen128(lo);
    const u128 lin = 13591409ull + (u128)545140134ull * k;
    br = bp + bitlen128(lin);  // upper bound
}

struct DepthPlan {
    uint64_t nodes;
    uint32_t cap[3];  // limbs
    int kind;         // 0 pair, 1 warp schoolbook, 2 ntt
    int logL;         // ntt
    bool wide;        // ntt in the wide configuration (64-bit coefficients, five primes)
};

constexpr uint32_t kWarpMaxC = 64;

}  // namespace

struct DeviceBS {
    const DeviceTables* T = nullptr;
    cudaStream_t st = nullptr;
    uint64_t* launches = nullptr;
    // owned buffers
    uint64_t* lev[2][3] = {{nullptr}};
    uint64_t lev_cap[2][3] = {{0}};
    uint32_t* lev_len[2] = {nullptr, nullptr};
    uint64_t lev_len_cap[2] = {0, 0};
    uint32_t* res = nullptr;
    uint64_t res_cap = 0;
    uint32_t* sync = nullptr;     // look-back tickets and status words (grows)
    uint64_t sync_cap = 0;
    uint32_t* errw = nullptr;     // device error word, allocated once and never moved
    uint64_t errw_cap = 0;
    // CUDA graph of the last range's launch sequence (replayed when the same range comes back
    // and no buffer moved since it was captured)
    uint64_t moves = 0;           // buffer reallocations so far
    cudaGraphExec_t gexec = nullptr;  // captured for [g_a0, g_b0); destroyed when a buffer moves
    uint64_t g_a0 = ~0ull, g_b0 = 0;
    uint64_t g_wmin = 0;              // the wide configuration's crossover the graph was planned with
    bool g_skip = false;              // the graph leaves out the rightmost nodes' P
    LevelView groot{};
    uint64_t glaunches = 0;

    ~DeviceBS() {
        if (gexec) cudaGraphExecDestroy(gexec);
        release();
    }
    void release() {
        for (int s = 0; s < 2; ++s) {
            for (int k = 0; k < 3; ++k)
                if (lev[s][k]) dev_free(lev[s][k]), lev[s][k] = nullptr, lev_cap[s][k] = 0;
            if (lev_len[s]) dev_free(lev_len[s]), lev_len[s] = nullptr, lev_len_cap[s] = 0;
        }
        if (res) dev_free(res), res = nullptr, res_cap = 0;
        if (sync) dev_free(sync), sync = nullptr, sync_cap = 0;
        if (errw) dev_free(errw), errw = nullptr, errw_cap = 0;
    }
    cudaError_t grow(void** p, uint64_t& cap, uint64_t need) {
        if (need <= cap) return cudaSuccess;
        ++moves;
        if (gexec) {  // the graph refers to the buffer about to be freed
            cudaGraphExecDestroy(gexec);
            gexec = nullptr;
        }
        if (*p) dev_free(*p);
        *p = nullptr;
        cap = 0;
        cudaError_t e = pg::dev_malloc(p, need);
        if (e == cudaSuccess) cap = need;
        return e;
    }

    // run() through a CUDA graph: the range is planned and every buffer sized first (host work
    // and allocations, outside any capture), then its launch sequence is captured and replayed; a
    // later call on the same range, with no buffer moved since, replays the graph alone.
    cudaError_t run_graph(uint64_t a0, uint64_t b0, LevelView& root, std::string& err, bool skipP) {
        if (trace_on()) return run(a0, b0, root, err, skipP);  // tracing waits between depths
        const uint64_t wmin = T->wide ? wide_min_limbs(*T) : 0;
        if (gexec && g_a0 == a0 && g_b0 == b0 && g_wmin == wmin && g_skip == skipP) {  // no buffer moved since
            root = groot;
            if (launches) *launches += glaunches;
            return cudaGraphLaunch(gexec, st);
        }
        if (gexec) {
            cudaGraphExecDestroy(gexec);
            gexec = nullptr;
        }
        std::vector<DepthPlan> dp;
        int D = 0;
        cudaError_t e = prepare(a0, b0, dp, D, err);
        if (e != cudaSuccess) return e;
        uint64_t* saved = launches;
        uint64_t counted = 0;
        launches = &counted;
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
        if (e != cudaSuccess) {
            launches = saved;
            cudaGetLastError();
            return enqueue(a0, b0, dp, D, root, skipP);  // run directly instead
        }
        const uint64_t m0 = moves;
        cudaError_t er = enqueue(a0, b0, dp, D, root, skipP);
        e = cudaStreamEndCapture(st, &g);
        launches = saved;
        if (er != cudaSuccess || e != cudaSuccess || moves != m0) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return enqueue(a0, b0, dp, D, root, skipP);
        }
        e = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            gexec = nullptr;
            cudaGetLastError();
            return enqueue(a0, b0, dp, D, root, skipP);
        }
        groot = root;
        g_a0 = a0;
        g_b0 = b0;
        g_wmin = wmin;
        g_skip = skipP;
        glaunches = counted;
        if (launches) *launches += counted;
        return cudaGraphLaunch(gexec, st);
    }

    std::vector<DepthPlan> plan(uint64_t a0, uint64_t b0, int& D, std::string& err) {
        std::vector<DepthPlan> dp;
        const uint64_t n = b0 - a0;
        D = 0;
        while ((1ull << D) < n) ++D;
        // Quick rejection before the pass over all terms: q(k) = 10939058860032000 k^3 > 2^53 k^3,
        // so Q(a0, b0) has more than 53 (b0 - lo) + 3 (b0 - mid) floor(log2 mid) bits (lo =
        // max(a0, 1), mid = the middle of [lo, b0)), and the root merge's Q product needs a
        // transform of at least that many bits / 32 points.
        if (n >= 2) {
            const uint64_t lo = std::max<uint64_t>(a0, 1), mid = lo + (b0 - lo) / 2;
            int lg = 0;
            while ((2ull << lg) <= mid) ++lg;
            const uint64_t qmin = 53 * (b0 - lo) + 3 * (b0 - mid) * (uint64_t)lg;
            if (qmin / 32 > (1ull << split_logL())) {
                err = "binary-splitting product exceeds the transform range";
                return {};
            }
        }
        // rightmost node at each depth: [b0 - s_d, b0)
        std::vector<uint64_t> s(D + 1);
        {
            uint64_t lo = a0, hi = b0;
            for (int d = 0; d <= D; ++d) {
                s[d] = hi - lo;
                if (hi - lo > 1) lo = lo + (hi - lo) / 2;
            }
        }
        // Bit sums over the rightmost node of each depth. The nodes are nested, so the terms
        // [b0 - s[0], b0) split into disjoint segments [b0 - s[d], b0 - s[d+1]) (d < D) and
        // [b0 - s[D], b0); one pass over the terms (spread over host threads) sums each segment,
        // and depth d's sum is the suffix sum of segments d..D.
        std::vector<uint64_t> sp(D + 1), sq(D + 1);
        {
            std::vector<uint64_t> lo(D + 1);
            for (int d = 0; d <= D; ++d) lo[d] = b0 - s[d];  // non-decreasing in d
            const uint64_t first = lo[0];
            const uint64_t nterms = b0 - first;
            const unsigned nt = (unsigned)std::max<uint64_t>(
                1, std::min<uint64_t>(std::max(1u, std::thread::hardware_concurrency()), nterms / 65536 + 1));
            std::vector<std::vector<uint64_t>> segp(nt, std::vector<uint64_t>(D + 1, 0)),
                segq(nt, std::vector<uint64_t>(D + 1, 0));
            auto work = [&](unsigned t) {
                const uint64_t k0 = first + nterms * t / nt, k1 = first + nterms * (t + 1) / nt;
                int seg = 0;
                while (seg < D && lo[seg + 1] <= k0) ++seg;
                for (uint64_t k = k0; k < k1; ++k) {
                    while (seg < D && lo[seg + 1] <= k) ++seg;
                    int bp, bq, br;
                    leaf_bits(k, bp, bq, br);
                    segp[t][seg] += (uint64_t)bp;
                    segq[t][seg] += (uint64_t)bq;
                }
            };
            std::vector<std::thread> th;
            for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
            work(0);
            for (auto& x : th) x.join();
            uint64_t accp = 0, accq = 0;
            for (int d = D; d >= 0; --d) {
                for (unsigned t = 0; t < nt; ++t) {
                    accp += segp[t][d];
                    accq += segq[t][d];
                }
                sp[d] = accp;
                sq[d] = accq;
            }
        }
        dp.resize(D);
        // depth D-1: pair nodes
        if (D >= 1) {
            dp[D - 1].nodes = 1ull << (D - 1);
            dp[D - 1].cap[0] = 4;
            dp[D - 1].cap[1] = 6;
            dp[D - 1].cap[2] = 8;  // 7 limbs rounded up to even
            dp[D - 1].kind = 0;
        }
        uint64_t rbits = 0;  // running R bound (bits) of the child depth
        {
            int p, q, r;
            leaf_bits(b0 - 1, p, q, r);
            // pair level R bound: max(q + r, p + r) + 1 over two leaves of the largest terms
            rbits = (uint64_t)(q + r + 1);
        }
        for (int d = D - 2; d >= 0; --d) {
            DepthPlan& P = dp[d];
            P.nodes = 1ull << d;
            const uint64_t pb = sp[d], qb = sq[d];
            // children's bounds (depth d + 1)
            const uint64_t cqb = sq[d + 1], cpb = sp[d + 1];
            const uint64_t rb = std::max(cqb + rbits, cpb + rbits) + 1;
            // limbs, +1 spare, rounded up to even so every slot starts on a 16-byte boundary
            P.cap[0] = (uint32_t)(((pb + 63) / 64 + 2) & ~1ull);
            P.cap[1] = (uint32_t)(((qb + 63) / 64 + 2) & ~1ull);
            P.cap[2] = (uint32_t)(((rb + 63) / 64 + 2) & ~1ull);
            rbits = rb;
            const DepthPlan& C = dp[d + 1];
            const uint32_t cmax = std::max({C.cap[0], C.cap[1], C.cap[2]});
            if (cmax <= kWarpMaxC) {
                P.kind = 1;
                P.logL = 0;
            } else {
                P.kind = 2;
                const uint64_t conv =
                    2ull * std::max({C.cap[1] + C.cap[1], C.cap[1] + C.cap[2], C.cap[0] + C.cap[2], C.cap[0] + C.cap[0]});
                int l = 0;
                while ((1ull << l) < conv) ++l;
                P.logL = std::max(l, kMinLogL);
                if (P.logL > split_logL()) {
                    err = "binary-splitting product exceeds the transform range";
                    return {};
                }
                // CRT exactness: R^ sums two convolutions, lifted to (-P/2, P/2]:
                // (min(2capQ, 2capR) + min(2capP, 2capR)) * (2^32 - 1)^2 < p0 p1 p2 / 2
                const double bound = (double)(2.0 * std::min(C.cap[1], C.cap[2]) + 2.0 * std::min(C.cap[0], C.cap[2])) *
                                     18446744065119617025.0;
                const double half = 2013265921.0 * 1811939329.0 * 469762049.0 / 2.0;
                if (bound >= half) {
                    err = "binary-splitting merge exceeds the proven CRT bound";
                    return {};
                }
                // The wide configuration (the crossover of single products, applied to the level's
                // longest product) when its bound holds: R^'s two convolutions of 64-bit
                // coefficients, (min(capQ, capR) + min(capP, capR)) (2^64 - 1)^2 < q0 ... q4 / 2.
                const uint64_t convl = conv / 2;
                const double wbound = (double)(std::min(C.cap[1], C.cap[2]) + std::min(C.cap[0], C.cap[2])) *
                                      3.402823669209385e38;  // (2^64 - 1)^2 rounded up
                const double whalf =
                    2113929217.0 * 2013265921.0 * 1811939329.0 * 1711276033.0 * 1107296257.0 / 2.0 * (1.0 - 1e-12);
                P.wide = false;
                if (use_wide(*T, convl - convl / 2, convl / 2) && wbound < whalf) {
                    P.wide = true;
                    P.logL = std::max(ceil_log2(convl), kMinLogL);
                }
            }
        }
        return dp;
    }

    // skipP: the level's last merge needs no P (nor its right child's P): its Pr slot and P^ output,
    // the last of the batch's operands and outputs, are left out.
    cudaError_t launch_ntt_level(const DepthPlan& P, const DepthPlan& C, const LevelView& in, const LevelView& out,
                                 uint64_t a0, uint64_t b0, int depth, bool skipP) {
        const Plan plan = P.wide ? T->plan_wide(P.logL) : T->plan(P.logL);
        const TwiddleTables& tw = P.wide ? T->tw_wide : T->tw;
        const Source limbs = P.wide ? Source::Limbs64 : Source::Limbs;
        const uint64_t L = 1ull << P.logL;
        const uint64_t M = P.nodes;
        const uint64_t stride = (P.wide ? kWidePrimes : kNumPrimes) * L;
        cudaError_t e = grow((void**)&res, res_cap, 6 * M * stride * 4);
        if (e != cudaSuccess) return e;
        // forward transforms of all 6M operands
        PassParams p{};
        p.error = errw;
        p.data = res;
        p.out = res;
        p.L = L;
        p.logL = P.logL;
        p.job_stride = stride;
        p.njobs = (uint32_t)(6 * M - (skipP ? 1 : 0));
        p.merge = 1;
        for (int k = 0; k < 3; ++k) {
            p.ms.X[k] = in.X[k];
            p.ms.cap[k] = in.cap[k];
        }
        p.ms.len = in.len;
        for (int i = 0; i < plan.npass; ++i) {
            set_pass(p, plan, i);
            e = launch_pass(plan, i, false, i == 0 ? limbs : Source::Residues, Fuse::None, p, tw, st);
            if (e != cudaSuccess) return e;
            if (launches) ++*launches;
        }
        // inverse transforms of the 3M outputs, one launch per pass over all of them: output k of
        // merge m (P^ = Pl Pr, Q^ = Ql Qr, R^ = Qr Rl +- Pl Rr) is formed on load by the first
        // (contiguous) inverse pass and written over operand slot comb_out_slot(k) (Ql, Rr, Pr),
        // which no other output reads, so the three outputs need no order among themselves (no
        // separate pointwise kernel and no pass over the products).
        {
            PassParams q{};
            q.error = errw;
            q.data = res;
            q.out = res;
            q.L = L;
            q.logL = P.logL;
            q.job_stride = 0;
            q.njobs = (uint32_t)(3 * M - (skipP ? 1 : 0));
            q.merge = 0;
            q.comb3 = 1;
            q.comb_slot = stride;
            q.comb_a0 = a0;
            q.comb_b0 = b0;
            q.comb_depth = depth;
            for (int i = plan.npass - 1; i >= 0; --i) {
                set_pass(q, plan, i);
                e = launch_pass(plan, i, true, Source::Residues, i == plan.npass - 1 ? Fuse::Combine : Fuse::None, q,
                                tw, st);
                if (e != cudaSuccess) return e;
                if (launches) ++*launches;
            }
        }
        // CRT + carry for all 3M outputs
        uint64_t maxw = 2ull * std::max({out.cap[0], out.cap[1], out.cap[2]});
        const uint64_t jobs = 3 * M - (skipP ? 1 : 0);
        if (P.wide) {
            const uint64_t bpj = (maxw + crt_wide_block_words() - 1) / crt_wide_block_words();
            CrtParams c{};
            c.L = L;
            c.error = errw;
            c.status = sync;
            c.merge = 1;
            c.res = res;
            c.res_stride = stride;
            for (int k = 0; k < 3; ++k) {
                c.dst[k] = out.X[k];
                c.dcap[k] = out.cap[k];
            }
            c.dlen = out.len;
            c.a0 = a0;
            c.b0 = b0;
            c.depth = depth;
            return launch_crt_wide(c, jobs, bpj, P.logL, st, launches);
        }
        const uint64_t bpj = (maxw + kCrtThreads * kCrtWords - 1) / (kCrtThreads * kCrtWords);
        e = grow((void**)&sync, sync_cap, (jobs + jobs * bpj) * 4);
        if (e != cudaSuccess) return e;
        e = cudaMemsetAsync(sync, 0, (jobs + jobs * bpj) * 4, st);
        if (e != cudaSuccess) return e;
        e = cudaMemsetAsync(out.len, 0, 3 * M * 4, st);
        if (e != cudaSuccess) return e;
        CrtParams c{};
        c.L = L;
        c.error = errw;
        c.ticket = sync;
        c.status = sync + jobs;
        c.blocks_per_job = bpj;
        c.k = make_crt_consts(P.logL);
        c.merge = 1;
        c.res = res;
        c.res_stride = stride;
        for (int k = 0; k < 3; ++k) {
            c.dst[k] = out.X[k];
            c.dcap[k] = out.cap[k];
        }
        c.dlen = out.len;
        c.a0 = a0;
        c.b0 = b0;
        c.depth = depth;
        e = launch_crt(c, jobs * bpj, st, maxw);
        if (launches) ++*launches;
        (void)C;
        return e;
    }

    // Computes P, Q, R of [a0, b0); results stay in the final level buffers (root = node 0).
    // Plans [a0, b0) and sizes every buffer for it (allocations and host work only, nothing enqueued).
    cudaError_t prepare(uint64_t a0, uint64_t b0, std::vector<DepthPlan>& dp, int& D, std::string& err) {
        D = 0;
        const bool tr = trace_on();
        auto tp0 = std::chrono::steady_clock::now();
        dp = plan(a0, b0, D, err);
        if (tr)
            std::fprintf(stderr, "[pg_bs] plan %.3f ms, %d depths\n",
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp0).count(), D);
        if (!err.empty()) return cudaErrorInvalidValue;
        cudaError_t e = grow((void**)&errw, errw_cap, 256);
        if (e != cudaSuccess) return e;
        if (D == 0) {
            // single term: the root is a leaf; treat it as a "pair level" of one node of size 1
            dp.resize(1);
            dp[0].nodes = 1;
            dp[0].cap[0] = 4;
            dp[0].cap[1] = 6;
            dp[0].cap[2] = 8;
            dp[0].kind = 0;
            D = 1;
        }
        // Every buffer at its largest size for this range before the first launch: growing them
        // depth by depth would free and reallocate (each cudaFree waits for the device) up to the
        // root on a range's first run.
        {
            uint64_t lev_need[2][3] = {{0}}, len_need[2] = {0, 0}, res_need = 0, sync_need = 0;
            for (int d = D - 1; d >= 0; --d) {
                const DepthPlan& P = dp[d];
                const int s = (D - 1 - d) & 1;
                for (int k = 0; k < 3; ++k) lev_need[s][k] = std::max<uint64_t>(lev_need[s][k], P.nodes * P.cap[k] * 8);
                len_need[s] = std::max<uint64_t>(len_need[s], P.nodes * 3 * 4);
                if (P.kind == 2) {
                    const uint64_t L = 1ull << P.logL, M = P.nodes;
                    res_need = std::max<uint64_t>(res_need, 6 * M * (P.wide ? kWidePrimes : kNumPrimes) * L * 4);
                    const uint64_t maxw = 2ull * std::max({P.cap[0], P.cap[1], P.cap[2]});
                    const uint64_t bw = P.wide ? crt_wide_block_words() : (uint64_t)kCrtThreads * kCrtWords;
                    const uint64_t bpj = (maxw + bw - 1) / bw;
                    sync_need = std::max<uint64_t>(sync_need, (3 * M + 3 * M * bpj) * 4);
                }
            }
            for (int s = 0; s < 2; ++s) {
                for (int k = 0; k < 3; ++k)
                    if (lev_need[s][k] && (e = grow((void**)&lev[s][k], lev_cap[s][k], lev_need[s][k])) != cudaSuccess)
                        return e;
                if (len_need[s] && (e = grow((void**)&lev_len[s], lev_len_cap[s], len_need[s])) != cudaSuccess) return e;
            }
            if (res_need && (e = grow((void**)&res, res_cap, res_need)) != cudaSuccess) return e;
            if (sync_need && (e = grow((void**)&sync, sync_cap, sync_need)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    // Enqueues the splitting of [a0, b0) planned and sized by prepare(): kernels and memsets only
    // (no allocation, no host wait), so it may run inside a stream capture.
    cudaError_t enqueue(uint64_t a0, uint64_t b0, std::vector<DepthPlan>& dp, int D, LevelView& root, bool skipP) {
        const bool tr = trace_on();
        cudaError_t e = cudaMemsetAsync(errw, 0, 4, st);
        if (e != cudaSuccess) return e;
        auto view = [&](int slot, const DepthPlan& P) {
            LevelView v;
            for (int k = 0; k < 3; ++k) {
                v.X[k] = lev[slot][k];
                v.cap[k] = P.cap[k];
            }
            v.len = lev_len[slot];
            return v;
        };
        auto alloc = [&](int slot, const DepthPlan& P) -> cudaError_t {
            for (int k = 0; k < 3; ++k) {
                cudaError_t r = grow((void**)&lev[slot][k], lev_cap[slot][k], P.nodes * P.cap[k] * 8);
                if (r != cudaSuccess) return r;
            }
            return grow((void**)&lev_len[slot], lev_len_cap[slot], P.nodes * 3 * 4);
        };
        int slot = 0;
        // depth D-1
        {
            const DepthPlan& P = dp[D - 1];
            e = alloc(slot, P);
            if (e != cudaSuccess) return e;
            LevelView v = view(slot, P);
            const int depth = (b0 - a0 == 1) ? 0 : D - 1;
            bs_pair_kernel<<<(unsigned)((P.nodes + 127) / 128), 128, 0, st>>>(v, P.nodes, a0, b0, depth);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            if (launches) ++*launches;
        }
        for (int d = D - 2; d >= 0; --d) {
            const DepthPlan& C = dp[d + 1];
            const DepthPlan& P = dp[d];
            const int oslot = slot ^ 1;
            e = alloc(oslot, P);
            if (e != cudaSuccess) return e;
            LevelView in = view(slot, C), out = view(oslot, P);
            auto tl0 = std::chrono::steady_clock::now();
            if (P.kind == 1) {
                // children's largest slot decides the kernel: a thread per merge up to 16 limbs
                // (measured faster there than lane groups, whose carry resolution outweighs such
                // small products), 16 lanes per merge up to 32, a warp per merge up to 64
                const uint32_t cmax = std::max({C.cap[0], C.cap[1], C.cap[2]});
                if (cmax <= 8)
                    bs_thread_merge_kernel<8><<<(unsigned)((P.nodes + 127) / 128), 128, 0, st>>>(in, out, P.nodes, a0,
                                                                                                 b0, d);
                else if (cmax <= 16)
                    bs_thread_merge_kernel<16><<<(unsigned)((P.nodes + 127) / 128), 128, 0, st>>>(in, out, P.nodes,
                                                                                                  a0, b0, d);
                else if (cmax <= 20)
                    bs_thread_merge_kernel<20><<<(unsigned)((P.nodes + 127) / 128), 128, 0, st>>>(in, out, P.nodes,
                                                                                                  a0, b0, d);
                else if (cmax <= 32)
                    bs_group_merge_kernel<32, 16><<<(unsigned)((P.nodes + 7) / 8), 128, 0, st>>>(in, out, P.nodes, a0,
                                                                                                 b0, d);
                else
                    bs_group_merge_kernel<kWarpMaxC, 32><<<(unsigned)((P.nodes + 3) / 4), 128, 0, st>>>(
                        in, out, P.nodes, a0, b0, d);
                e = cudaGetLastError();
                if (launches) ++*launches;
            } else {
                e = launch_ntt_level(P, C, in, out, a0, b0, d, skipP);
            }
            if (e != cudaSuccess) return e;
            if (tr) {
                cudaStreamSynchronize(st);
                std::fprintf(stderr, "[pg_bs] depth %2d: %8llu merges, caps %u/%u/%u limbs, %s L=2^%d: %.3f ms\n", d,
                             (unsigned long long)P.nodes, P.cap[0], P.cap[1], P.cap[2],
                             P.kind == 1 ? "warp" : (P.wide ? "wide" : "ntt "), P.logL,
                             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tl0).count());
            }
            slot = oslot;
        }
        root = view(slot, dp[0]);
        return cudaSuccess;
    }

    cudaError_t run(uint64_t a0, uint64_t b0, LevelView& root, std::string& err, bool skipP) {
        std::vector<DepthPlan> dp;
        int D = 0;
        cudaError_t e = prepare(a0, b0, dp, D, err);
        if (e != cudaSuccess) return e;
        return enqueue(a0, b0, dp, D, root, skipP);
    }
};

}  // namespace pg

// ------------------------------------------------------------------ C ABI
struct pg_ctx;
namespace pg {
// defined in pg_api.cu
const DeviceTables& ctx_tables(pg_ctx* c);
cudaStream_t ctx_stream(pg_ctx* c);
std::mutex& ctx_mutex(pg_ctx* c);
uint64_t* ctx_launches(pg_ctx* c);
void ctx_set_error(pg_ctx* c, const std::string& msg);
int ctx_device(pg_ctx* c);
DeviceBS* ctx_bs(pg_ctx* c);
// defined in pi_device.cu: [a, b) as subtrees merged on the device, into host buffers like pg_bs
pg_status bs_split_to_host(pg_ctx* ctx, unsigned long a, unsigned long b, uint64_t* P, uint64_t* Q, uint64_t* R,
                           size_t cap, size_t* len, int* sign);
DeviceBS* bs_state_new() { return new DeviceBS; }
void bs_state_delete(DeviceBS* b) { delete b; }
}  // namespace pg

namespace pg {
// Runs the level-batched splitting of [a, b) with the context lock held by the caller. On
// PG_OK the root's P, Q, R stay in the context's level buffers (root.X[k], hl[k] limbs) until
// the next splitting on this context. while_running (optional) is called once the splitting is
// enqueued, before the wait for it: host work (allocations for the next steps) that then
// overlaps the device's.
pg_status bs_run_locked(pg_ctx* ctx, unsigned long a, unsigned long b, LevelView& root, uint32_t hl[3], bool need_P,
                        const std::function<void()>* while_running = nullptr) {
    cudaSetDevice(ctx_device(ctx));
    DeviceBS& bs = *ctx_bs(ctx);  // buffers persist in the context across calls
    bs.T = &ctx_tables(ctx);
    bs.st = ctx_stream(ctx);
    bs.launches = ctx_launches(ctx);
    std::string err;
    cudaError_t e = bs.run_graph(a, b, root, err, !need_P);
    if (!err.empty()) {
        ctx_set_error(ctx, err);
        return PG_ERR_TOO_LARGE;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx_set_error(ctx, std::string("pg_bs: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PG_ERR_OOM : PG_ERR_DEVICE;
    }
    if (while_running && *while_running) (*while_running)();
    uint32_t herr = 0;
    hl[0] = hl[1] = hl[2] = 0;
    e = cudaMemcpyAsync(hl, root.len, 12, cudaMemcpyDeviceToHost, bs.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, bs.errw, 4, cudaMemcpyDeviceToHost, bs.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(bs.st);
    if (!need_P) hl[0] = 0;  // not computed
    if (e != cudaSuccess) {
        ctx_set_error(ctx, std::string("pg_bs: ") + cudaGetErrorString(e));
        return PG_ERR_DEVICE;
    }
    if (herr) {
        const bool tmo = herr == 1 || (herr & 4);
        ctx_set_error(ctx, herr == 1 ? "carry look-back wait ran out of iterations"
                                     : (herr & 4) ? "tile load wait ran out of iterations" : "carry out of the top word");
        return tmo ? PG_ERR_TIMEOUT : PG_ERR_INTERNAL;
    }
    return PG_OK;
}
}  // namespace pg

extern "C" pg_status pg_bs(pg_ctx* ctx, unsigned long a, unsigned long b, uint64_t* P, uint64_t* Q, uint64_t* R,
                           size_t cap, size_t* len, int* sign) {
    if (!ctx || !Q || !R || !len || !sign || b <= a) return PG_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lock(pg::ctx_mutex(ctx));
    pg::LevelView root;
    uint32_t hl[3];
    pg_status s = pg::bs_run_locked(ctx, a, b, root, hl, P != nullptr);
    if (s == PG_ERR_TOO_LARGE && b - a > 1) {  // subtrees merged with block products
        pg::ctx_set_error(ctx, "");
        return pg::bs_split_to_host(ctx, a, b, P, Q, R, cap, len, sign);
    }
    if (s != PG_OK) return s;
    cudaStream_t st = pg::ctx_stream(ctx);
    auto tc0 = std::chrono::steady_clock::now();
    if (hl[1] > cap || hl[2] > cap || (P && hl[0] > cap)) {
        pg::ctx_set_error(ctx, "output buffers smaller than the result");
        return PG_ERR_BAD_ARG;
    }
    uint64_t* dsts[3] = {P, Q, R};
    for (int k = 0; k < 3; ++k) {
        len[k] = hl[k];
        if (dsts[k] && hl[k]) cudaMemcpyAsync(dsts[k], root.X[k], hl[k] * 8, cudaMemcpyDeviceToHost, st);
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return PG_ERR_DEVICE;
    if (pg::trace_on())
        std::fprintf(stderr, "[pg_bs] copy-out of P/Q/R: %.3f ms\n",
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc0).count());
    // signs over the series: P(a,b) = (-1)^(#k >= 1), Q > 0, R(a,b) has the sign of R(a, a+1)
    const unsigned long neg_terms = (b - a) - (a == 0 ? 1 : 0);
    sign[0] = hl[0] ? ((neg_terms & 1) ? -1 : 1) : 0;
    sign[1] = hl[1] ? 1 : 0;
    sign[2] = hl[2] ? (a == 0 ? 1 : -1) : 0;
    return PG_OK;
}
