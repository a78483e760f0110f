#include "pi_engine.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>

#include "b200_multiplier.h"
#include "binary_splitting.h"
#include "device_bs.h"
#include "newton.h"

namespace pi {

using Clock = std::chrono::steady_clock;
static double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

PiEngine::PiEngine(Multiplier& m) : mult_(m) {}

void final_formula_mpf(mpz_t pi_int, const mpz_t Q, const mpz_t R, size_t digits) {
    const size_t precision = digits + 100;
    const mp_bitcnt_t bits = static_cast<mp_bitcnt_t>(precision * 3.3219281) + 64;
    mpf_t s, num, den, pv, scale;
    mpf_init2(s, bits);
    mpf_set_prec(s, bits);
    mpf_set_ui(s, 10005);
    mpf_sqrt(s, s);
    mpz_t t;
    mpz_init(t);
    mpz_mul_ui(t, Q, 426880);
    mpf_init2(num, bits);
    mpf_init2(den, bits);
    mpf_init2(pv, bits);
    mpf_set_z(num, t);
    mpf_set_z(den, R);
    mpf_mul(pv, num, s);
    mpf_div(pv, pv, den);
    mpz_ui_pow_ui(t, 10, digits);
    mpf_init2(scale, bits);
    mpf_set_z(scale, t);
    mpf_mul(pv, pv, scale);
    mpz_set_f(pi_int, pv);
    mpz_clear(t);
    mpf_clear(s);
    mpf_clear(num);
    mpf_clear(den);
    mpf_clear(pv);
    mpf_clear(scale);
}

std::string format_digits(const mpz_t pi_int, size_t digits) {
    void (*freefunc)(void*, size_t) = nullptr;
    mp_get_memory_functions(nullptr, nullptr, &freefunc);
    char* s = mpz_get_str(nullptr, 10, pi_int);
    size_t n = std::strlen(s);
    std::string out;
    out.reserve(digits + 2);
    out.push_back(s[0]);
    out.push_back('.');
    out.append(s + 1, std::min(n - 1, digits));
    freefunc(s, n + 1);
    return out;
}

PiResult PiEngine::compute(const PiConfig& cfg) {
    auto t0 = Clock::now();
    PiResult res;
    const size_t precision = cfg.digits + 100;
    const unsigned long terms = BinarySplitting::terms_needed(precision);
    res.terms_used = terms;
    mpz_t Q, R, pi_int;
    mpz_init(Q);
    mpz_init(R);
    mpz_init(pi_int);
    if (cfg.mode == BSMode::Batched && cfg.final_mode == FinalMode::Device) {
        // The whole computation on the device (pg_pi): splitting, final formula, conversion.
        pg_ctx* ctx = shared_context(cfg.device);
        const uint64_t l0 = pg_launch_count(ctx);
        std::string s;
        if (!cfg.digits_out) s.assign(cfg.digits + 2, '0');
        char* out = cfg.digits_out ? cfg.digits_out : &s[0];
        double sec[4] = {0, 0, 0, 0};
        pg_ckpt_report rep{};
        const bool ckpt = !cfg.checkpoint_dir.empty();
        const pg_status st = ckpt ? pg_pi_checkpointed(ctx, cfg.digits, cfg.checkpoint_dir.c_str(), out, sec, &rep)
                                  : pg_pi(ctx, cfg.digits, out, sec);
        if (st != PG_OK)
            throw std::runtime_error(std::string(ckpt ? "pg_pi_checkpointed: " : "pg_pi: ") + pg_last_error(ctx) +
                                     " (status " + std::to_string(st) + ")");
        if (ckpt && cfg.verbose)
            std::printf("  Checkpoints in %s: splitting %s, %zu node(s) loaded, %zu subtree(s) computed, %zu merge(s);"
                        " pi_int %s\n",
                        cfg.checkpoint_dir.c_str(), rep.root_loaded ? "resumed" : (rep.root_saved ? "saved" : "not saved"),
                        rep.nodes_loaded, rep.subtrees_computed, rep.merges,
                        rep.pi_int_loaded ? "resumed" : (rep.pi_int_saved ? "saved" : "not saved"));
        res.digits.swap(s);
        res.t.gpu_launches += pg_launch_count(ctx) - l0;
        res.t.bs = sec[0];
        res.t.final = sec[1];
        res.t.convert = sec[2];
        res.t.total = secs(t0, Clock::now());
        res.elapsed_seconds = res.t.total;
        if (cfg.verbose || std::getenv("PI_B200_TRACE"))
            std::printf("  Terms: %lu\n  Binary splitting: %.3fs\n  Final computation: %.3fs\n"
                        "  String conversion: %.3fs\n  Total: %.3fs\n",
                        terms, res.t.bs, res.t.final, res.t.convert, res.t.total);
        mpz_clear(Q);
        mpz_clear(R);
        mpz_clear(pi_int);
        return res;
    }
    if (cfg.mode == BSMode::Batched) {
        pg_ctx* ctx = shared_context(cfg.device);
        const uint64_t l0 = pg_launch_count(ctx);
        DeviceBinarySplitting dbs(ctx);
        dbs.compute(0, terms, nullptr, Q, R);  // P(0, N) is not needed (pi_engine.cpp:257-258)
        res.t.gpu_launches += pg_launch_count(ctx) - l0;
    } else {
        BinarySplitting bs(mult_, cfg.num_threads);
        BSResult r = bs.compute(0, terms);
        mpz_swap(Q, r.Q);
        mpz_swap(R, r.R);
        if (auto* b = dynamic_cast<B200Multiplier*>(&mult_)) {
            res.t.gpu_launches += pg_launch_count(b->context());
            res.t.gpu_calls += b->stats().gpu_calls.load();
            res.t.cpu_routed += b->stats().cpu_routed_calls.load();
        }
    }
    auto t1 = Clock::now();
    Clock::time_point t2, t3;
    if (cfg.final_mode == FinalMode::Newton) {
        // Products of the finish: the B200 when the splitting ran there, else the engine's multiplier.
        std::unique_ptr<B200Multiplier> gpu;
        uint64_t l0 = 0;
        if (cfg.mode == BSMode::Batched) {
            pg_ctx* ctx = shared_context(cfg.device);
            l0 = pg_launch_count(ctx);
            gpu = std::make_unique<B200Multiplier>(cfg.gpu_threshold, ctx, cfg.device);
        }
        Multiplier& fm = gpu ? static_cast<Multiplier&>(*gpu) : mult_;
        final_formula_newton(pi_int, Q, R, cfg.digits, fm);
        t2 = Clock::now();
        std::string d = to_decimal(pi_int, cfg.digits + 1, fm, cfg.num_threads);
        if (gpu) {
            res.t.gpu_launches += pg_launch_count(gpu->context()) - l0;
            res.t.gpu_calls += gpu->stats().gpu_calls.load();
            res.t.cpu_routed += gpu->stats().cpu_routed_calls.load();
        }
        res.digits.reserve(cfg.digits + 2);
        res.digits.push_back(d[0]);
        res.digits.push_back('.');
        res.digits.append(d, 1, std::string::npos);
        t3 = Clock::now();
    } else {
        final_formula_mpf(pi_int, Q, R, cfg.digits);
        t2 = Clock::now();
        res.digits = format_digits(pi_int, cfg.digits);
        t3 = Clock::now();
    }
    res.t.bs = secs(t0, t1);
    res.t.final = secs(t1, t2);
    res.t.convert = secs(t2, t3);
    res.t.total = secs(t0, t3);
    res.elapsed_seconds = res.t.total;
    if (cfg.verbose || std::getenv("PI_B200_TRACE")) {
        std::printf("  Terms: %lu\n  Binary splitting: %.3fs\n  Final computation: %.3fs\n"
                    "  String conversion: %.3fs\n  Total: %.3fs\n",
                    terms, res.t.bs, res.t.final, res.t.convert, res.t.total);
    }
    mpz_clear(Q);
    mpz_clear(R);
    mpz_clear(pi_int);
    return res;
}

std::string PiEngine::compute_digits(size_t digits) {
    PiConfig c;
    c.digits = digits;
    return compute(c).digits;
}

}  // namespace pi
