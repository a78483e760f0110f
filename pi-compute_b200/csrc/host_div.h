// Host long division for the smallest Newton levels: floor(2^e / v) for a v of a few dozen limbs,
// by Knuth's Algorithm D (The Art of Computer Programming, vol. 2, 4.3.1) in base 2^64 with 128-bit
// partial products. Exact; used where a device Newton level would cost more in launches and host
// waits than the arithmetic itself.
#pragma once
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <vector>

namespace pg {

// q = floor(2^e / v); v (little-endian limbs, top limb non-zero) at least two limbs long.
inline std::vector<uint64_t> host_pow2_div(size_t e, std::vector<uint64_t> v) {
    typedef unsigned __int128 u128;
    const size_t n = v.size();
    if (n < 2 || v[n - 1] == 0) throw std::invalid_argument("host_pow2_div: divisor must have >= 2 limbs");
    // normalise: the divisor's top bit set
    int s = 0;
    while (!((v[n - 1] << s) >> 63)) ++s;
    if (s) {
        for (size_t i = n - 1; i > 0; --i) v[i] = (v[i] << s) | (v[i - 1] >> (64 - s));
        v[0] <<= s;
    }
    // dividend 2^(e + s): m + n limbs plus one for the top digit step
    const size_t bit = e + (size_t)s;
    const size_t ulimbs = bit / 64 + 1;
    if (ulimbs < n) return {0};
    std::vector<uint64_t> u(ulimbs + 1, 0);
    u[bit / 64] = (uint64_t)1 << (bit % 64);
    const size_t m = ulimbs - n;  // quotient has m + 1 limbs
    std::vector<uint64_t> q(m + 1, 0);
    const uint64_t v1 = v[n - 1], v2 = v[n - 2];
    for (size_t jj = m + 1; jj-- > 0;) {
        const u128 num = ((u128)u[jj + n] << 64) | u[jj + n - 1];
        u128 qhat = num / v1;
        u128 rhat = num % v1;
        while (qhat >> 64 || (u128)(uint64_t)qhat * v2 > ((rhat << 64) | u[jj + n - 2])) {
            --qhat;
            rhat += v1;
            if (rhat >> 64) break;
        }
        // u[jj .. jj + n] -= qhat * v
        uint64_t borrow = 0, carry = 0;
        for (size_t i = 0; i < n; ++i) {
            const u128 p = (u128)(uint64_t)qhat * v[i] + carry;
            carry = (uint64_t)(p >> 64);
            const uint64_t pl = (uint64_t)p;
            const uint64_t ui = u[jj + i];
            const uint64_t d = ui - pl - borrow;
            borrow = (ui < pl) || (ui - pl < borrow);
            u[jj + i] = d;
        }
        const uint64_t top = u[jj + n];
        const uint64_t d = top - carry - borrow;
        const bool neg = (top < carry) || (top - carry < borrow);
        u[jj + n] = d;
        if (neg) {  // qhat was one too large: add v back
            --qhat;
            uint64_t c = 0;
            for (size_t i = 0; i < n; ++i) {
                const u128 t = (u128)u[jj + i] + v[i] + c;
                u[jj + i] = (uint64_t)t;
                c = (uint64_t)(t >> 64);
            }
            u[jj + n] += c;
        }
        q[jj] = (uint64_t)qhat;
    }
    while (q.size() > 1 && q.back() == 0) q.pop_back();
    return q;
}

}  // namespace pg
