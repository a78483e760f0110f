/*
 * ORACLE -- test infrastructure only (see oracle.h).
 *
 * Chudnovsky binary splitting restated over GMP integers, following the
 * reference's BinarySplitting:
 *   leaves        src/engine/binary_splitting.cpp:137-159
 *                 P(a,a+1) = -(6a-5)(2a-1)(6a-1), Q = a^3 * C^3/24, R = P*(13591409 + 545140134 a);
 *                 a = 0: P = Q = 1, R = 13591409
 *   merge         src/engine/binary_splitting.cpp:161-293
 *                 P = Pl*Pr, Q = Ql*Qr, R = Qr*Rl + Pl*Rr
 *   recursion     src/engine/binary_splitting.cpp:295-348, split m = a + (b-a)/2
 *   terms_needed  src/engine/binary_splitting.cpp:100-102
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gmp.h"
#include "oracle.h"

struct oracle_int {
    mpz_t v;
};

oracle_int* oracle_int_new(void) {
    oracle_int* x = (oracle_int*)malloc(sizeof(oracle_int));
    mpz_init(x->v);
    return x;
}
void oracle_int_free(oracle_int* x) {
    if (!x) return;
    mpz_clear(x->v);
    free(x);
}
int oracle_int_sign(const oracle_int* x) { return mpz_sgn(x->v); }
size_t oracle_int_size(const oracle_int* x) { return mpz_size(x->v); }
void oracle_int_get_limbs(const oracle_int* x, uint64_t* out) {
    size_t n = mpz_size(x->v);
    if (n) memcpy(out, mpz_limbs_read(x->v), n * sizeof(uint64_t));
}
void oracle_int_set_limbs(oracle_int* x, const uint64_t* limbs, size_t n, int sign) {
    mpz_set_ui(x->v, 0);
    if (n) mpz_import(x->v, n, -1, sizeof(uint64_t), 0, 0, limbs);
    if (sign < 0) mpz_neg(x->v, x->v);
}

unsigned long oracle_terms_needed(size_t digits) {
    return (unsigned long)ceil((double)digits / 14.1816474627) + 1;
}

static const char* C3_OVER_24 = "10939058860032000"; /* 640320^3 / 24 */

static void leaf(unsigned long a, mpz_ptr P, mpz_ptr Q, mpz_ptr R) {
    if (a == 0) {
        mpz_set_ui(P, 1);
        mpz_set_ui(Q, 1);
        mpz_set_ui(R, 13591409);
        return;
    }
    mpz_t t;
    mpz_init(t);
    mpz_set_ui(P, 6 * a - 5);
    mpz_mul_ui(P, P, 2 * a - 1);
    mpz_mul_ui(P, P, 6 * a - 1);
    mpz_neg(P, P);
    mpz_set_str(Q, C3_OVER_24, 10);
    mpz_ui_pow_ui(t, a, 3);
    mpz_mul(Q, Q, t);
    mpz_set_ui(t, 545140134);
    mpz_mul_ui(t, t, a);
    mpz_add_ui(t, t, 13591409);
    mpz_mul(R, P, t);
    mpz_clear(t);
}

static void merge(mpz_srcptr Pl, mpz_srcptr Ql, mpz_srcptr Rl, mpz_srcptr Pr, mpz_srcptr Qr, mpz_srcptr Rr,
                  mpz_ptr P, mpz_ptr Q, mpz_ptr R) {
    mpz_t t1, t2;
    mpz_init(t1);
    mpz_init(t2);
    mpz_mul(t1, Qr, Rl);
    mpz_mul(t2, Pl, Rr);
    mpz_add(R, t1, t2);
    mpz_mul(P, Pl, Pr);
    mpz_mul(Q, Ql, Qr);
    mpz_clear(t1);
    mpz_clear(t2);
}

static void bs_rec(unsigned long a, unsigned long b, mpz_ptr P, mpz_ptr Q, mpz_ptr R) {
    if (b - a == 1) {
        leaf(a, P, Q, R);
        return;
    }
    unsigned long m = a + (b - a) / 2;
    mpz_t P1, Q1, R1, P2, Q2, R2;
    mpz_init(P1); mpz_init(Q1); mpz_init(R1);
    mpz_init(P2); mpz_init(Q2); mpz_init(R2);
    bs_rec(a, m, P1, Q1, R1);
    bs_rec(m, b, P2, Q2, R2);
    merge(P1, Q1, R1, P2, Q2, R2, P, Q, R);
    mpz_clear(P1); mpz_clear(Q1); mpz_clear(R1);
    mpz_clear(P2); mpz_clear(Q2); mpz_clear(R2);
}

void oracle_bs(unsigned long a, unsigned long b, oracle_int* P, oracle_int* Q, oracle_int* R) {
    bs_rec(a, b, P->v, Q->v, R->v);
}

void oracle_bs_merge(const oracle_int* Pl, const oracle_int* Ql, const oracle_int* Rl,
                     const oracle_int* Pr, const oracle_int* Qr, const oracle_int* Rr,
                     oracle_int* P, oracle_int* Q, oracle_int* R) {
    merge(Pl->v, Ql->v, Rl->v, Pr->v, Qr->v, Rr->v, P->v, Q->v, R->v);
}
