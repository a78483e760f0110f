// Host-side transform planning and constant generation (no CUDA types).
#pragma once
#include <cstddef>
#include <cstdint>

namespace pg {

constexpr int kTileLog = 13;        // E = 2^13 residues per CTA tile (32 KB of shared memory) ...
constexpr int kTileLogBig = 14;     // ... or 2^14 (64 KB) for the longest sub-transforms
constexpr int kMinLogL = 6;         // smallest transform (64 points)
constexpr int kMaxStridedLog = 12;  // strided passes keep >= 4 adjacent columns per tile
constexpr int kMaxContigLog = 14;   // contiguous passes hold whole sub-transforms of up to 2^14 points

// Tile of a pass: 2^13 residues, or 2^14 for strided sub-transforms of 2^11 and 2^12 points (8 and 4
// columns of 16 and 32 bytes, coalesced with the neighbouring tile in L2) and contiguous ones of 2^14.
// The large tiles make 2^24..2^26-point transforms two passes instead of three.
constexpr int tile_log(bool strided, int logN) {
    return strided ? (logN <= 10 ? kTileLog : kTileLogBig) : (logN <= kTileLog ? kTileLog : kTileLogBig);
}

struct Plan {
    int logL = 0;
    int npass = 0;
    int logN[3] = {0, 0, 0};   // sub-transform length of each pass, first = largest stride
    int logS[3] = {0, 0, 0};   // element stride of each pass
};

// Pass split for L = 2^logL: one contiguous pass up to 2^13, two passes above (a contiguous last
// pass of 2^13 points up to 2^23, of 2^14 points from 2^24 to 2^26).
inline Plan make_plan(int logL) {
    Plan p;
    p.logL = logL;
    if (logL <= kTileLog) {
        p.npass = 1;
        p.logN[0] = logL;
    } else if (logL <= 20) {
        p.npass = 2;
        p.logN[0] = logL / 2;
        p.logN[1] = logL - logL / 2;
    } else if (logL <= kTileLog + 10) {
        p.npass = 2;
        p.logN[0] = logL - kTileLog;
        p.logN[1] = kTileLog;
    } else {
        p.npass = 2;
        p.logN[0] = logL - kMaxContigLog;
        p.logN[1] = kMaxContigLog;
    }
    int s = logL;
    for (int i = 0; i < p.npass; ++i) {
        s -= p.logN[i];
        p.logS[i] = s;
    }
    return p;
}

// Whether a pass split can run: one contiguous last pass of 2^6..2^14 points, strided passes of
// 2^5..2^12 points whose tiles (2^(tile_log - N) columns) fit in their stride, every strided pass's
// four-step block at least 2^14 points (the row power tables' range), lengths summing to logL.
inline bool plan_valid(const Plan& p) {
    if (p.npass < 1 || p.npass > 3) return false;
    int sum = 0;
    for (int i = 0; i < p.npass; ++i) sum += p.logN[i];
    if (sum != p.logL) return false;
    const int last = p.npass - 1;
    if (p.logN[last] < kMinLogL || p.logN[last] > kMaxContigLog) return false;
    int s = p.logL;
    for (int i = 0; i < last; ++i) {
        s -= p.logN[i];  // stride of pass i
        if (p.logN[i] < 5 || p.logN[i] > kMaxStridedLog) return false;
        if (s < tile_log(true, p.logN[i]) - p.logN[i]) return false;  // C columns <= S
        if (p.logN[i] + s < 14) return false;                          // four-step block >= 2^14
    }
    return true;
}

// Plan with the given pass lengths (strides filled in).
inline Plan plan_from(int logL, int npass, const int* n) {
    Plan p;
    p.logL = logL;
    p.npass = npass;
    int s = logL;
    for (int i = 0; i < npass; ++i) {
        p.logN[i] = n[i];
        s -= n[i];
        p.logS[i] = s;
    }
    return p;
}

inline int ceil_log2(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) ++l;
    return l;
}

// Transform length for an na x nb limb product with 32-bit coefficients.
inline int product_logL(size_t na, size_t nb) {
    uint64_t conv = 2ull * (na + nb) - 1;  // coefficients of the linear convolution
    int l = ceil_log2(conv);
    return l < kMinLogL ? kMinLogL : l;
}

// Transform length for an na x nb limb product with 64-bit coefficients (the wide configuration):
// na + nb - 1 coefficients.
inline int product_logL_wide(size_t na, size_t nb) {
    int l = ceil_log2((uint64_t)(na + nb) - 1);
    return l < kMinLogL ? kMinLogL : l;
}

uint32_t pow_mod(uint32_t b, uint64_t e, uint32_t p);
uint32_t inv_mod(uint32_t a, uint32_t p);
uint32_t shoup_companion(uint32_t w, uint32_t p);

}  // namespace pg
