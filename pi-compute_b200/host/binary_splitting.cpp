#include "binary_splitting.h"

#include <cmath>
#include <future>

namespace pi {

BSResult::BSResult() {
    mpz_init(P);
    mpz_init(Q);
    mpz_init(R);
}
BSResult::~BSResult() {
    mpz_clear(P);
    mpz_clear(Q);
    mpz_clear(R);
}
BSResult::BSResult(BSResult&& o) noexcept {
    mpz_init(P);
    mpz_init(Q);
    mpz_init(R);
    mpz_swap(P, o.P);
    mpz_swap(Q, o.Q);
    mpz_swap(R, o.R);
}
BSResult& BSResult::operator=(BSResult&& o) noexcept {
    if (this != &o) {
        mpz_swap(P, o.P);
        mpz_swap(Q, o.Q);
        mpz_swap(R, o.R);
    }
    return *this;
}

BinarySplitting::BinarySplitting(Multiplier& m, unsigned int n) : mult_(m), threads_(n == 0 ? 1 : n) {}

unsigned long BinarySplitting::terms_needed(size_t digits) {
    return static_cast<unsigned long>(std::ceil(static_cast<double>(digits) / 14.1816474627)) + 1;
}

void BinarySplitting::leaf(unsigned long a, mpz_t P, mpz_t Q, mpz_t R) {
    if (a == 0) {
        mpz_set_ui(P, 1);
        mpz_set_ui(Q, 1);
        mpz_set_ui(R, 13591409);
        return;
    }
    // P = -(6a-5)(2a-1)(6a-1); Q = a^3 * 640320^3 / 24; R = P * (13591409 + 545140134 a)
    mpz_set_ui(P, 6 * a - 5);
    mpz_mul_ui(P, P, 2 * a - 1);
    mpz_mul_ui(P, P, 6 * a - 1);
    mpz_neg(P, P);
    mpz_set_ui(Q, a);
    mpz_mul_ui(Q, Q, a);
    mpz_mul_ui(Q, Q, a);
    mpz_mul_ui(Q, Q, 10939058860032000UL);
    mpz_t t;
    mpz_init_set_ui(t, a);
    mpz_mul_ui(t, t, 545140134UL);
    mpz_add_ui(t, t, 13591409UL);
    mpz_mul(R, P, t);
    mpz_clear(t);
}

BSResult BinarySplitting::merge(BSResult& l, BSResult& r, bool concurrent) {
    BSResult out;
    mpz_t x;
    mpz_init(x);
    if (concurrent) {
        // Four products at once, like the reference's tier-2 merge (binary_splitting.cpp:178-201).
        auto f1 = std::async(std::launch::async, [&] { mult_.multiply(x, r.Q, l.R); });
        auto f2 = std::async(std::launch::async, [&] { mult_.multiply(out.R, l.P, r.R); });
        auto f3 = std::async(std::launch::async, [&] { mult_.multiply(out.P, l.P, r.P); });
        mult_.multiply(out.Q, l.Q, r.Q);
        f1.get();
        f2.get();
        f3.get();
    } else {
        mult_.multiply(x, r.Q, l.R);
        mult_.multiply(out.R, l.P, r.R);
        mult_.multiply(out.P, l.P, r.P);
        mult_.multiply(out.Q, l.Q, r.Q);
    }
    mpz_add(out.R, out.R, x);
    mpz_clear(x);
    return out;
}

BSResult BinarySplitting::rec(unsigned long a, unsigned long b, int depth) {
    if (b - a == 1) {
        BSResult r;
        leaf(a, r.P, r.Q, r.R);
        return r;
    }
    unsigned long m = a + (b - a) / 2;
    BSResult left, right;
    if (depth > 0 && b - a >= 64) {
        auto fr = std::async(std::launch::async, [&] { return rec(m, b, depth - 1); });
        left = rec(a, m, depth - 1);
        right = fr.get();
    } else {
        left = rec(a, m, depth);
        right = rec(m, b, depth);
    }
    size_t mx = mpz_size(left.Q) > mpz_size(right.Q) ? mpz_size(left.Q) : mpz_size(right.Q);
    return merge(left, right, threads_ > 1 && mx > 1000);
}

BSResult BinarySplitting::compute(unsigned long a, unsigned long b) {
    int depth = 0;
    for (unsigned int t = threads_; t > 1; t >>= 1) ++depth;
    return rec(a, b, depth);
}

}  // namespace pi
