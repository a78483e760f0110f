// Chudnovsky binary-splitting tree: node ranges and the sign rule of the R merge.
#pragma once
#include <cstdint>

namespace pg {

// Range [a, b) of node `idx` at `depth` below the root range [a0, b0) (split a + (b-a)/2).
__device__ __forceinline__ void node_range(uint64_t a0, uint64_t b0, int depth, uint64_t idx, uint64_t& a,
                                           uint64_t& b) {
    a = a0;
    b = b0;
    for (int t = depth - 1; t >= 0; --t) {
        const uint64_t mid = a + (b - a) / 2;
        if ((idx >> t) & 1)
            a = mid;
        else
            b = mid;
    }
}

// Sign s of R = Qr*Rl + s*Pl*Rr on magnitudes for the merge of [a, b): s = sgn(Rl)sgn(Pl)sgn(Rr).
// Over the Chudnovsky series sgn(P(x,y)) = (-1)^(#terms k >= 1 in [x,y)) and
// sgn(R(x,y)) = sgn(R(x,x+1)) (+1 for x = 0, -1 otherwise), so with m the split point
// s = (-1)^(m-a) for a >= 1 and (-1)^m for a = 0.
__device__ __forceinline__ int merge_r_sign(uint64_t a, uint64_t b) {
    const uint64_t m = a + (b - a) / 2;
    const uint64_t e = (a >= 1) ? (m - a) : m;
    return (e & 1) ? -1 : 1;
}

}  // namespace pg
