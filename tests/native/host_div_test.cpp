// Host test driver of pi-compute_b200/csrc/host_div.h (floor(2^e / v) by Knuth's Algorithm D).
// Reads cases from stdin, one per line: e, n, then the n little-endian 64-bit limbs of v in hex;
// prints each quotient's limbs in hex, least significant first, one line per case.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "host_div.h"

int main() {
    unsigned long long e = 0, n = 0;
    while (std::scanf("%llu %llu", &e, &n) == 2) {
        std::vector<uint64_t> v(n);
        for (auto& x : v) {
            unsigned long long t = 0;
            if (std::scanf("%llx", &t) != 1) return 2;
            x = t;
        }
        const std::vector<uint64_t> q = pg::host_pow2_div((size_t)e, v);
        for (size_t i = 0; i < q.size(); ++i) std::printf(i ? " %llx" : "%llx", (unsigned long long)q[i]);
        std::printf("\n");
    }
    return 0;
}
