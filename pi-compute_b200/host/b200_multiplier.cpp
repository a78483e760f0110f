#include "b200_multiplier.h"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <vector>

namespace pi {

B200Multiplier::B200Multiplier(size_t threshold, int device) : threshold_(threshold), device_(device) {
    pg_status s = pg_create(device, &ctx_);
    if (s != PG_OK) throw std::runtime_error("B200Multiplier: pg_create failed with status " + std::to_string(s));
}

B200Multiplier::B200Multiplier(size_t threshold, pg_ctx* shared, int device)
    : ctx_(shared), owned_(false), threshold_(threshold), device_(device) {}

B200Multiplier::~B200Multiplier() {
    if (owned_) pg_destroy(ctx_);
}

pg_ctx* shared_context(int device) {
    static std::mutex mu;
    static std::map<int, pg_ctx*> ctxs;
    std::lock_guard<std::mutex> lock(mu);
    auto it = ctxs.find(device);
    if (it != ctxs.end()) return it->second;
    pg_ctx* c = nullptr;
    pg_status s = pg_create(device, &c);
    if (s != PG_OK) throw std::runtime_error("pg_create failed with status " + std::to_string(s));
    ctxs[device] = c;
    return c;
}

std::string B200Multiplier::device_name() const {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device_) != cudaSuccess) return "unknown";
    return prop.name;
}

void B200Multiplier::product(mpz_t result, const mpz_t a, const mpz_t b, bool sq) {
    const size_t na = mpz_size(a), nb = mpz_size(b);
    const int sign = mpz_sgn(a) * mpz_sgn(b);
    if (std::min(na, nb) < threshold_ || sign == 0) {
        // Routing (not a fallback): small products stay on GMP like the reference's
        // should_use_gpu (gpu_ntt_multiplier.cpp:67-72); zero needs no device work.
        stats_.cpu_routed_calls.fetch_add(1);
        mpz_mul(result, a, b);
        return;
    }
    auto t0 = std::chrono::steady_clock::now();
    // result may alias a or b: mpz_limbs_write could move their storage, so write into a
    // fresh integer in that case and swap.
    const bool alias = (result == a) || (result == b);
    mpz_t tmp;
    mpz_ptr dst = result;
    if (alias) {
        mpz_init(tmp);
        dst = tmp;
    }
    mp_limb_t* out = mpz_limbs_write(dst, (mp_size_t)(na + nb));
    size_t len = 0;
    pg_status s;
    const uint64_t* ap = reinterpret_cast<const uint64_t*>(mpz_limbs_read(a));
    const uint64_t* bp = reinterpret_cast<const uint64_t*>(mpz_limbs_read(b));
    if (na + nb > pg_mul_max_limbs())
        s = block_product(ap, na, bp, nb, sq, reinterpret_cast<uint64_t*>(out), &len);
    else if (sq)
        s = pg_sqr(ctx_, ap, na, reinterpret_cast<uint64_t*>(out), na + nb, &len);
    else
        s = pg_mul(ctx_, ap, na, bp, nb, reinterpret_cast<uint64_t*>(out), na + nb, &len);
    if (s != PG_OK) {
        mpz_limbs_finish(dst, 0);
        if (alias) mpz_clear(tmp);
        throw std::runtime_error(std::string("B200Multiplier: ") + pg_last_error(ctx_) + " (status " +
                                 std::to_string(s) + ")");
    }
    mpz_limbs_finish(dst, sign < 0 ? -(mp_size_t)len : (mp_size_t)len);
    if (alias) {
        mpz_swap(result, tmp);
        mpz_clear(tmp);
    }
    stats_.gpu_calls.fetch_add(1);
    stats_.gpu_limbs.fetch_add(na + nb);
    stats_.gpu_ns.fetch_add(
        (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count());
}

// A product longer than one transform (pg_mul_max_limbs): products of blocks of at most half that
// many limbs each, one pg_mul call per pair, added into out at their limb offsets.
pg_status B200Multiplier::block_product(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, bool sq,
                                        uint64_t* out, size_t* len) {
    const size_t cap = pg_mul_max_limbs() / 2;
    const size_t ka = (na + cap - 1) / cap, kb = (nb + cap - 1) / cap;
    const size_t Ba = (na + ka - 1) / ka, Bb = (nb + kb - 1) / kb, total = na + nb;
    std::fill(out, out + total, (uint64_t)0);
    std::vector<uint64_t> buf(Ba + Bb);
    for (size_t i = 0; i < ka && i * Ba < na; ++i) {
        const size_t la = std::min(Ba, na - i * Ba);
        for (size_t j = sq ? i : 0; j < kb && j * Bb < nb; ++j) {
            const size_t lb = std::min(Bb, nb - j * Bb);
            size_t n = 0;
            const pg_status s = (sq && i == j) ? pg_sqr(ctx_, a + i * Ba, la, buf.data(), la + lb, &n)
                                               : pg_mul(ctx_, a + i * Ba, la, b + j * Bb, lb, buf.data(), la + lb, &n);
            if (s != PG_OK) return s;
            for (int rep = 0; rep < ((sq && i != j) ? 2 : 1); ++rep) {  // off-diagonal blocks of a square twice
                unsigned __int128 c = 0;
                size_t k = i * Ba + j * Bb;
                for (size_t t = 0; t < n; ++t, ++k) {
                    c += (unsigned __int128)out[k] + buf[t];
                    out[k] = (uint64_t)c;
                    c >>= 64;
                }
                for (; c && k < total; ++k) {
                    c += out[k];
                    out[k] = (uint64_t)c;
                    c >>= 64;
                }
            }
        }
    }
    size_t n = total;
    while (n && out[n - 1] == 0) --n;
    *len = n;
    return PG_OK;
}

void B200Multiplier::multiply(mpz_t result, const mpz_t a, const mpz_t b) { product(result, a, b, a == b); }

void B200Multiplier::square(mpz_t result, const mpz_t a) { product(result, a, a, true); }

void B200Multiplier::reset_stats() {
    stats_.gpu_calls = 0;
    stats_.cpu_routed_calls = 0;
    stats_.gpu_ns = 0;
    stats_.gpu_limbs = 0;
}

void B200Multiplier::print_stats() const {
    std::printf("  B200 Multiplier Stats:\n    GPU multiply calls:    %llu\n    CPU routed calls:      %llu\n"
                "    GPU path time:         %.3fs\n",
                (unsigned long long)stats_.gpu_calls.load(), (unsigned long long)stats_.cpu_routed_calls.load(),
                stats_.gpu_ns.load() / 1e9);
}

}  // namespace pi
