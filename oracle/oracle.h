/*
 * ORACLE -- test infrastructure only. Nothing in the product links or calls this.
 *
 * CPU restatement of the reference's arithmetic on the multiply hot path of
 * f97johan/pi-compute:
 *   - exact limb products (the reference's GmpMultiplier::multiply/square,
 *     src/arithmetic/gmp_multiplier.cpp:10-19, which is one call to GMP's mpz_mul);
 *   - Chudnovsky binary splitting leaves and merges
 *     (src/engine/binary_splitting.cpp:137-159, 161-293, 295-348).
 *
 * The product algorithm lives in a third-party dependency, GMP (the reference
 * pins no version, CMakeLists.txt:27-28; its published runs used 6.2.1; this
 * image carries libgmp.so.10 = GMP 6.3.0). Two independent restatements are
 * provided so each pins the other: a plain-C schoolbook / Karatsuba product
 * (the algorithms of the GMP manual, "Basecase Multiplication" and "Karatsuba
 * Multiplication") and a wrapper over libgmp's mpz_mul itself. Parity is
 * anchored on the reference's known-answer tests (tests/test_gmp_multiplier.cpp,
 * tests/test_binary_splitting.cpp, tests/data/pi_1000.txt).
 */
#ifndef PI_B200_ORACLE_H
#define PI_B200_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Exact product of little-endian 64-bit limb arrays; out has na+nb limbs (zero-padded). */
void oracle_mul_schoolbook(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out);
void oracle_mul_karatsuba(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out);
void oracle_mul_gmp(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out);

/* Opaque signed integer (an mpz_t) for the binary-splitting restatement. */
typedef struct oracle_int oracle_int;
oracle_int* oracle_int_new(void);
void oracle_int_free(oracle_int* x);
int oracle_int_sign(const oracle_int* x);
size_t oracle_int_size(const oracle_int* x);
void oracle_int_get_limbs(const oracle_int* x, uint64_t* out);
void oracle_int_set_limbs(oracle_int* x, const uint64_t* limbs, size_t n, int sign);

/* P(a,b), Q(a,b), R(a,b) of the Chudnovsky series, same split m = a + (b-a)/2. */
void oracle_bs(unsigned long a, unsigned long b, oracle_int* P, oracle_int* Q, oracle_int* R);
/* One merge: P = Pl*Pr, Q = Ql*Qr, R = Qr*Rl + Pl*Rr. */
void oracle_bs_merge(const oracle_int* Pl, const oracle_int* Ql, const oracle_int* Rl,
                     const oracle_int* Pr, const oracle_int* Qr, const oracle_int* Rr,
                     oracle_int* P, oracle_int* Q, oracle_int* R);
unsigned long oracle_terms_needed(size_t digits);

#ifdef __cplusplus
}
#endif
#endif
