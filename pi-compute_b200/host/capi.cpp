// C entry points of libpib200.so (declarations in include/pi_b200_engine.h).
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "b200_multiplier.h"
#include "binary_splitting.h"
#include "device_bs.h"
#include "pi_b200_engine.h"
#include "pi_engine.h"

namespace {
thread_local std::string g_err;

std::unique_ptr<pi::Multiplier> make_multiplier(int mode, size_t threshold, int device) {
    if (mode == PIB_MODE_GMP) return std::make_unique<pi::GmpMultiplier>();
    if (mode == PIB_MODE_PER_CALL) return std::make_unique<pi::B200Multiplier>(threshold, device);
    throw std::invalid_argument("unknown binary-splitting mode " + std::to_string(mode));
}

void export_signed(const mpz_t v, uint64_t* out, size_t cap, size_t* len, int* sign) {
    size_t n = mpz_size(v);
    if (n > cap) throw std::length_error("output buffer too small");
    if (n) std::memcpy(out, mpz_limbs_read(v), n * 8);
    *len = n;
    *sign = mpz_sgn(v);
}
}  // namespace

extern "C" {

int pib_pi(size_t digits, int mode, unsigned threads, size_t threshold, int device, char* out, size_t out_cap,
           double* stats) {
    try {
        if (!out || out_cap < digits + 2) throw std::invalid_argument("output buffer smaller than digits + 2");
        if (mode == PIB_MODE_BATCHED) {
            // the whole computation on the device, digits written straight into the caller's buffer
            pg_ctx* ctx = pi::shared_context(device);
            const uint64_t l0 = pg_launch_count(ctx);
            double sec[4] = {0, 0, 0, 0};
            const pg_status st = pg_pi(ctx, digits, out, sec);
            if (st != PG_OK)
                throw std::runtime_error(std::string("pg_pi: ") + pg_last_error(ctx) + " (status " +
                                         std::to_string(st) + ")");
            if (stats) {
                for (int i = 0; i < 4; ++i) stats[i] = sec[i];
                stats[4] = (double)(pg_launch_count(ctx) - l0);
                stats[5] = stats[6] = stats[7] = 0;
            }
            return 0;
        }
        pi::PiConfig cfg;
        cfg.digits = digits;
        cfg.num_threads = threads ? threads : 1;
        cfg.device = device;
        const bool batched = mode == PIB_MODE_BATCHED || mode == PIB_MODE_BATCHED_HOST_FINISH;
        cfg.mode = batched ? pi::BSMode::Batched : pi::BSMode::PerCall;
        cfg.final_mode = mode == PIB_MODE_BATCHED ? pi::FinalMode::Device
                         : (batched || mode == PIB_MODE_GMP_NEWTON) ? pi::FinalMode::Newton
                                                                    : pi::FinalMode::Mpf;
        std::unique_ptr<pi::Multiplier> m =
            make_multiplier((batched || mode == PIB_MODE_GMP_NEWTON) ? PIB_MODE_GMP : mode, threshold, device);
        pi::PiEngine eng(*m);
        pi::PiResult r = eng.compute(cfg);
        std::memcpy(out, r.digits.data(), r.digits.size());
        if (stats) {
            stats[0] = r.t.bs;
            stats[1] = r.t.final;
            stats[2] = r.t.convert;
            stats[3] = r.t.total;
            stats[4] = (double)r.t.gpu_launches;
            stats[5] = (double)r.t.gpu_calls;
            stats[6] = (double)r.t.cpu_routed;
            stats[7] = 0;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int pib_bs(unsigned long a, unsigned long b, int mode, size_t threshold, int device, uint64_t* P, uint64_t* Q,
           uint64_t* R, size_t cap, size_t* len, int* sign) {
    try {
        if (b <= a) throw std::invalid_argument("empty range");
        pi::BSResult r;
        if (mode == PIB_MODE_BATCHED) {
            pi::DeviceBinarySplitting dbs(device);
            dbs.compute(a, b, r.P, r.Q, r.R);
        } else {
            std::unique_ptr<pi::Multiplier> m = make_multiplier(mode, threshold, device);
            pi::BinarySplitting bs(*m, 1);
            r = bs.compute(a, b);
        }
        export_signed(r.P, P, cap, &len[0], &sign[0]);
        export_signed(r.Q, Q, cap, &len[1], &sign[1]);
        export_signed(r.R, R, cap, &len[2], &sign[2]);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int pib_mul(const uint64_t* a, size_t na, int sa, const uint64_t* b, size_t nb, int sb, size_t threshold, int device,
            uint64_t* out, size_t out_cap, size_t* out_len, int* out_sign) {
    try {
        if ((na && !a) || (nb && !b) || !out || !out_len || !out_sign) throw std::invalid_argument("null argument");
        pi::B200Multiplier m(threshold, device);
        mpz_t x, y, r;
        mpz_init(x);
        mpz_init(y);
        mpz_init(r);
        if (na) mpz_import(x, na, -1, sizeof(uint64_t), 0, 0, a);
        if (nb) mpz_import(y, nb, -1, sizeof(uint64_t), 0, 0, b);
        if (sa < 0) mpz_neg(x, x);
        if (sb < 0) mpz_neg(y, y);
        try {
            m.multiply(r, x, y);
            export_signed(r, out, out_cap, out_len, out_sign);
        } catch (...) {
            mpz_clear(x);
            mpz_clear(y);
            mpz_clear(r);
            throw;
        }
        mpz_clear(x);
        mpz_clear(y);
        mpz_clear(r);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

const char* pib_last_error(void) { return g_err.c_str(); }

}  // extern "C"
