#include "newton.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <future>
#include <stdexcept>
#include <thread>
#include <vector>

namespace pi {
namespace {

struct Mpz {
    mpz_t v;
    Mpz() { mpz_init(v); }
    ~Mpz() { mpz_clear(v); }
    Mpz(const Mpz&) = delete;
    Mpz& operator=(const Mpz&) = delete;
    operator mpz_ptr() { return v; }
    operator mpz_srcptr() const { return v; }
};

size_t bits(mpz_srcptr x) { return mpz_sgn(x) == 0 ? 0 : mpz_sizeinbase(x, 2); }

void pow2(mpz_ptr r, size_t e) {
    mpz_set_ui(r, 1);
    mpz_mul_2exp(r, r, e);
}

constexpr size_t kSmallBits = 4096;  // below this, GMP's own division/root on the host

// Phase timer printed to stderr when PI_B200_TRACE is set.
struct Trace {
    const char* what;
    std::chrono::steady_clock::time_point t0;
    static bool on() {
        static const bool v = [] {
            const char* e = std::getenv("PI_B200_TRACE");
            return e && *e && *e != '0';
        }();
        return v;
    }
    explicit Trace(const char* w) : what(w), t0(std::chrono::steady_clock::now()) {}
    ~Trace() {
        if (on())
            std::fprintf(stderr, "[newton] %s: %.3f ms\n", what,
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
};

}  // namespace

void recip_floor(mpz_t Z, const mpz_t R, Multiplier& mul) {
    const size_t k = bits(R);
    if (k == 0 || mpz_sgn(R) < 0) throw std::invalid_argument("recip_floor: R must be positive");
    if (k <= kSmallBits) {
        Mpz t;
        pow2(t, 2 * k);
        mpz_tdiv_q(Z, t, R);
        return;
    }
    // Half precision: Zh = floor(2^(2h) / Rh) for the top h bits of R.
    const size_t h = k / 2 + 64;
    Mpz Rh, Zh, Z0, T, E, D;
    mpz_tdiv_q_2exp(Rh, R, k - h);
    recip_floor(Zh, Rh, mul);
    mpz_mul_2exp(Z0, Zh, k - h);
    // One Newton step: Z = Z0 + Z0 (2^(2k) - R Z0) / 2^(2k) (relative error squares).
    mul.multiply(T, R, Z0);
    pow2(E, 2 * k);
    mpz_sub(E, E, T);                 // E = 2^(2k) - R Z0 (may be slightly negative)
    mul.multiply(D, Zh, E);           // Z0 E / 2^(2k) = Zh E / 2^(k+h)
    mpz_fdiv_q_2exp(D, D, k + h);
    mpz_add(Z, Z0, D);
    // Exact correction: E <- 2^(2k) - R Z = E - R D, then 0 <= E < R.
    mul.multiply(T, R, D);
    mpz_sub(E, E, T);
    int steps = 0;
    while (mpz_sgn(E) < 0) {
        mpz_sub_ui(Z, Z, 1);
        mpz_add(E, E, R);
        if (++steps > 64) throw std::runtime_error("recip_floor: Newton correction did not converge");
    }
    while (mpz_cmp(E, R) >= 0) {
        mpz_add_ui(Z, Z, 1);
        mpz_sub(E, E, R);
        if (++steps > 64) throw std::runtime_error("recip_floor: Newton correction did not converge");
    }
}

namespace {

// u ~= 2^q / sqrt(a) to within a few units (Newton on the inverse square root).
void rsqrt_approx(mpz_ptr u, unsigned long a, size_t q, Multiplier& mul) {
    if (q <= kSmallBits) {
        Mpz t, av;
        pow2(t, 2 * q);
        mpz_set_ui(av, a);
        mpz_tdiv_q(t, t, av);  // floor(2^(2q) / a)
        mpz_sqrt(u, t);        // floor(sqrt(floor(X))) = floor(sqrt(X))
        return;
    }
    const size_t qh = q / 2 + 64;
    Mpz uh, u0, T, e, D;
    rsqrt_approx(uh, a, qh, mul);
    mpz_mul_2exp(u0, uh, q - qh);
    // u = u0 + u0 (2^(2q) - a u0^2) / 2^(2q+1)
    mul.square(T, u0);
    mpz_mul_ui(T, T, a);
    pow2(e, 2 * q);
    mpz_sub(e, e, T);
    mul.multiply(D, uh, e);          // u0 e / 2^(2q+1) = uh e / 2^(q + qh + 1)
    mpz_fdiv_q_2exp(D, D, q + qh + 1);
    mpz_add(u, u0, D);
}

// F = 5^n by squaring (products through `mul`).
void pow5(mpz_ptr F, size_t n, Multiplier& mul) {
    mpz_set_ui(F, 1);
    if (n == 0) return;
    int top = 63;
    while (!((n >> top) & 1)) --top;
    Mpz t;
    for (int b = top; b >= 0; --b) {
        mul.square(t, F);
        mpz_swap(F, t);
        if ((n >> b) & 1) mpz_mul_ui(F, F, 5);
    }
}

}  // namespace

void sqrt_scaled(mpz_t S, unsigned long a, size_t s, Multiplier& mul) {
    const size_t q = s + 64;
    Mpz u, N, V, t;
    rsqrt_approx(u, a, q, mul);
    mpz_mul_ui(S, u, a);                 // a * 2^q / sqrt(a) = sqrt(a) 2^q
    mpz_fdiv_q_2exp(S, S, q - s);
    // Exact correction: S^2 <= N = a 2^(2s) < (S+1)^2.
    pow2(N, 2 * s);
    mpz_mul_ui(N, N, a);
    mul.square(t, S);
    mpz_sub(V, N, t);                    // V = N - S^2
    int steps = 0;
    while (mpz_sgn(V) < 0) {             // (S-1)^2 = S^2 - 2S + 1
        mpz_add(V, V, S);
        mpz_add(V, V, S);
        mpz_sub_ui(V, V, 1);
        mpz_sub_ui(S, S, 1);
        if (++steps > 64) throw std::runtime_error("sqrt_scaled: correction did not converge");
    }
    for (;;) {                           // (S+1)^2 = S^2 + 2S + 1 <= N ?
        mpz_set(t, S);
        mpz_mul_2exp(t, t, 1);
        mpz_add_ui(t, t, 1);
        if (mpz_cmp(V, t) < 0) break;
        mpz_sub(V, V, t);
        mpz_add_ui(S, S, 1);
        if (++steps > 64) throw std::runtime_error("sqrt_scaled: correction did not converge");
    }
}

void final_formula_newton(mpz_t pi_int, const mpz_t Q, const mpz_t R, size_t digits, Multiplier& mul) {
    if (mpz_sgn(Q) <= 0 || mpz_sgn(R) <= 0) throw std::invalid_argument("final formula needs Q, R > 0");
    for (size_t guard = 128; guard <= 128 + 4 * 256; guard += 256) {
        // P bits cover the integer part of pi * 10^digits plus the guard.
        const size_t P = (size_t)std::ceil((double)digits * 3.3219280948873623) + 2 + guard;
        const size_t k = P + 64;
        Mpz Qt, Rt, Z, S, F, X;
        long long e = 0;
        // Qt, Rt: exactly k bits (truncate or shift up); Q = Qt 2^eQ (1 + d), |d| < 2^-(k-1).
        const long long eQ = (long long)bits(Q) - (long long)k;
        const long long eR = (long long)bits(R) - (long long)k;
        if (eQ >= 0) mpz_tdiv_q_2exp(Qt, Q, (size_t)eQ); else mpz_mul_2exp(Qt, Q, (size_t)-eQ);
        if (eR >= 0) mpz_tdiv_q_2exp(Rt, R, (size_t)eR); else mpz_mul_2exp(Rt, R, (size_t)-eR);
        {
            Trace t("reciprocal of R");
            recip_floor(Z, Rt, mul);          // 2^(2k) / Rt
        }
        {
            Trace t("sqrt(10005)");
            sqrt_scaled(S, 10005, k, mul);    // sqrt(10005) 2^k
        }
        {
            Trace t("5^digits");
            pow5(F, digits, mul);             // 10^digits = 5^digits 2^digits
        }
        Trace tprod("three truncated products");
        // pi 10^digits = 426880 Q sqrt(10005) 10^digits / R ~= X 2^e
        mpz_mul_ui(X, Qt, 426880);
        e = eQ - eR - 2 * (long long)k - (long long)k + (long long)digits;
        Mpz t;
        auto mul_trunc = [&](mpz_srcptr y) {
            mul.multiply(t, X, y);
            const long long over = (long long)bits(t) - (long long)k;
            if (over > 0) {
                mpz_tdiv_q_2exp(X, t, (size_t)over);
                e += over;
            } else {
                mpz_swap(X, t);
            }
        };
        mul_trunc(S);
        mul_trunc(Z);
        mul_trunc(F);
        if (e >= -160) throw std::runtime_error("final formula: not enough fraction bits");
        const size_t fb = (size_t)(-e);
        // Total relative error < 8 * 2^-(k-1) and pi 10^digits < 2^(P - guard), so the absolute
        // error is below 2^(P - guard + 4 - k) < 2^-(guard + 60) <= 2^-188: the floor is certain
        // unless the fraction lies within 2^-100 of an integer.
        Mpz fr, lim;
        mpz_tdiv_q_2exp(pi_int, X, fb);
        mpz_tdiv_r_2exp(fr, X, fb);
        pow2(lim, fb - 100);
        Mpz hi;
        pow2(hi, fb);
        mpz_sub(hi, hi, lim);
        if (mpz_cmp(fr, lim) >= 0 && mpz_cmp(fr, hi) <= 0) return;
    }
    throw std::runtime_error("final formula: the result stayed within the error bound of an integer");
}

// ------------------------------------------------------------------ radix conversion
namespace {

void write_leaf(mpz_srcptr n, char* dst, size_t D) {
    if (mpz_sgn(n) == 0) return;  // already '0'
    void (*freefunc)(void*, size_t) = nullptr;
    mp_get_memory_functions(nullptr, nullptr, &freefunc);
    char* s = mpz_get_str(nullptr, 10, n);
    const size_t len = std::strlen(s);
    if (len > D) {
        freefunc(s, len + 1);
        throw std::runtime_error("to_decimal: chunk has more digits than its slot");
    }
    std::memcpy(dst + (D - len), s, len);
    freefunc(s, len + 1);
}

struct Converter {
    Multiplier& mul;
    char* out;
    size_t leaf;
    std::vector<Mpz*> pw;    // pw[j] = 10^(2^j)
    std::vector<Mpz*> inv;   // inv[j] = floor(2^(2K) / pw[j]), K = bits(pw[j]) (large j only)
    std::vector<size_t> K;

    ~Converter() {
        for (auto* p : pw) delete p;
        for (auto* p : inv) delete p;
    }

    void divmod(mpz_ptr q, mpz_ptr r, mpz_srcptr n, int j) {
        mpz_srcptr P = *pw[j];
        if (inv[j] == nullptr) {
            mpz_tdiv_qr(q, r, n, P);
            return;
        }
        Mpz T;
        mul.multiply(T, n, *inv[j]);
        mpz_fdiv_q_2exp(q, T, 2 * K[j]);   // <= floor(n / P), at most 2 below
        mul.multiply(T, q, P);
        mpz_sub(r, n, T);
        int steps = 0;
        while (mpz_sgn(r) < 0) {
            mpz_sub_ui(q, q, 1);
            mpz_add(r, r, P);
            if (++steps > 8) throw std::runtime_error("to_decimal: quotient correction did not converge");
        }
        while (mpz_cmp(r, P) >= 0) {
            mpz_add_ui(q, q, 1);
            mpz_sub(r, r, P);
            if (++steps > 8) throw std::runtime_error("to_decimal: quotient correction did not converge");
        }
    }

    // Digits of n (< 10^D) into out[off, off + D).
    void rec(mpz_srcptr n, size_t D, size_t off, int j, int depth) {
        if (D <= leaf || j < 0) {
            write_leaf(n, out + off, D);
            return;
        }
        while (j >= 0 && ((size_t)1 << j) >= D) --j;
        if (j < 0) {
            write_leaf(n, out + off, D);
            return;
        }
        const size_t lo = (size_t)1 << j, hi = D - lo;
        Mpz q, r;
        divmod(q, r, n, j);
        if (depth > 0) {
            auto f = std::async(std::launch::async, [&] { rec(r, lo, off + hi, j - 1, depth - 1); });
            rec(q, hi, off, j - 1, depth - 1);
            f.get();
        } else {
            rec(q, hi, off, j - 1, 0);
            rec(r, lo, off + hi, j - 1, 0);
        }
    }
};

}  // namespace

std::string to_decimal(const mpz_t x, size_t ndigits, Multiplier& mul, unsigned threads, size_t leaf_digits) {
    if (mpz_sgn(x) < 0) throw std::invalid_argument("to_decimal: negative input");
    std::string out(ndigits, '0');
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    Converter c{mul, &out[0], std::max<size_t>(leaf_digits, 64), {}, {}, {}};
    // power tree 10^(2^j) for 2^j < ndigits
    int J = -1;
    while (((size_t)1 << (J + 1)) < ndigits) ++J;
    {
        Trace t("power tree and reciprocals");
        for (int j = 0; j <= J; ++j) {
            Mpz* p = new Mpz;
            if (j == 0)
                mpz_set_ui(*p, 10);
            else
                mul.square(*p, *c.pw[j - 1]);
            c.pw.push_back(p);
            c.K.push_back(bits(*p));
            // reciprocals for the divisions done above the leaves
            if (((size_t)1 << j) * 2 > c.leaf && c.K.back() > kSmallBits) {
                Mpz* z = new Mpz;
                recip_floor(*z, *p, mul);
                c.inv.push_back(z);
            } else {
                c.inv.push_back(nullptr);
            }
        }
    }
    {
        Trace t("divide-and-conquer splits and leaves");
        int depth = 0;
        for (unsigned th = threads; th > 1; th >>= 1) ++depth;
        c.rec(x, ndigits, 0, J, depth);
    }
    return out;
}

}  // namespace pi
