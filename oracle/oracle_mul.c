/*
 * ORACLE -- test infrastructure only (see oracle.h).
 *
 * Exact products of little-endian 64-bit limb arrays, restating what the
 * reference's GmpMultiplier::multiply does (src/arithmetic/gmp_multiplier.cpp:10-12:
 * mpz_mul(result, a, b)) on magnitudes:
 *   oracle_mul_schoolbook  the basecase O(na*nb) product;
 *   oracle_mul_karatsuba   Karatsuba's three-half-products recursion over the basecase;
 *   oracle_mul_gmp         libgmp's mpz_mul itself (the reference's actual call).
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

#include "gmp.h"

typedef unsigned __int128 u128;

void oracle_mul_schoolbook(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out) {
    memset(out, 0, (na + nb) * sizeof(uint64_t));
    for (size_t i = 0; i < na; ++i) {
        uint64_t carry = 0;
        for (size_t j = 0; j < nb; ++j) {
            u128 t = (u128)a[i] * b[j] + out[i + j] + carry;
            out[i + j] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
        out[i + nb] = carry;
    }
}

/* r[0..n) += x[0..m), returns carry out of r[n-1]; requires m <= n. */
static uint64_t add_into(uint64_t* r, size_t n, const uint64_t* x, size_t m) {
    uint64_t c = 0;
    size_t i = 0;
    for (; i < m; ++i) {
        u128 t = (u128)r[i] + x[i] + c;
        r[i] = (uint64_t)t;
        c = (uint64_t)(t >> 64);
    }
    for (; c && i < n; ++i) {
        r[i] += 1;
        c = (r[i] == 0);
    }
    return c;
}

/* r[0..n) -= x[0..m), returns borrow; requires m <= n. */
static uint64_t sub_from(uint64_t* r, size_t n, const uint64_t* x, size_t m) {
    uint64_t br = 0;
    size_t i = 0;
    for (; i < m; ++i) {
        uint64_t xi = x[i];
        uint64_t ri = r[i];
        uint64_t d = ri - xi - br;
        br = (ri < xi) || (ri - xi < br);
        r[i] = d;
    }
    for (; br && i < n; ++i) {
        br = (r[i] == 0);
        r[i] -= 1;
    }
    return br;
}

#define KARATSUBA_CUTOFF 32

static void kara_rec(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out) {
    if (na < nb) {
        const uint64_t* t = a; a = b; b = t;
        size_t tn = na; na = nb; nb = tn;
    }
    if (nb < KARATSUBA_CUTOFF) {
        oracle_mul_schoolbook(a, na, b, nb, out);
        return;
    }
    size_t h = na / 2; /* split point; a = a1*B^h + a0 */
    if (nb <= h) {
        /* Unbalanced: out = (a1*b)*B^h + a0*b. */
        uint64_t* t = (uint64_t*)calloc(na - h + nb, sizeof(uint64_t));
        kara_rec(a, h, b, nb, out);
        memset(out + h + nb, 0, (na - h) * sizeof(uint64_t));
        kara_rec(a + h, na - h, b, nb, t);
        add_into(out + h, na + nb - h, t, na - h + nb);
        free(t);
        return;
    }
    const uint64_t *a0 = a, *a1 = a + h, *b0 = b, *b1 = b + h;
    size_t na1 = na - h, nb1 = nb - h;
    /* z0 = a0*b0, z2 = a1*b1, z1 = (a0+a1)(b0+b1) - z0 - z2 */
    size_t ns = (h > na1 ? h : na1) + 1, ms = (h > nb1 ? h : nb1) + 1;
    uint64_t* sa = (uint64_t*)calloc(ns, sizeof(uint64_t));
    uint64_t* sb = (uint64_t*)calloc(ms, sizeof(uint64_t));
    memcpy(sa, a0, h * sizeof(uint64_t));
    add_into(sa, ns, a1, na1);
    memcpy(sb, b0, h * sizeof(uint64_t));
    add_into(sb, ms, b1, nb1);
    uint64_t* z1 = (uint64_t*)calloc(ns + ms, sizeof(uint64_t));
    kara_rec(sa, ns, sb, ms, z1);
    memset(out, 0, (na + nb) * sizeof(uint64_t));
    kara_rec(a0, h, b0, h, out);                 /* z0 in out[0 .. 2h) */
    kara_rec(a1, na1, b1, nb1, out + 2 * h);     /* z2 in out[2h .. na+nb) */
    sub_from(z1, ns + ms, out, 2 * h);
    sub_from(z1, ns + ms, out + 2 * h, na1 + nb1);
    size_t nz = ns + ms;
    while (nz > 0 && z1[nz - 1] == 0) --nz;
    add_into(out + h, na + nb - h, z1, nz);
    free(sa);
    free(sb);
    free(z1);
}

void oracle_mul_karatsuba(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out) {
    if (na == 0 || nb == 0) {
        memset(out, 0, (na + nb) * sizeof(uint64_t));
        return;
    }
    kara_rec(a, na, b, nb, out);
}

void oracle_mul_gmp(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out) {
    mpz_t x, y, r;
    mpz_init(x);
    mpz_init(y);
    mpz_init(r);
    if (na) mpz_import(x, na, -1, sizeof(uint64_t), 0, 0, a);
    if (nb) mpz_import(y, nb, -1, sizeof(uint64_t), 0, 0, b);
    mpz_mul(r, x, y); /* gmp_multiplier.cpp:11 */
    memset(out, 0, (na + nb) * sizeof(uint64_t));
    size_t n = mpz_size(r);
    if (n) memcpy(out, mpz_limbs_read(r), n * sizeof(uint64_t));
    mpz_clear(x);
    mpz_clear(y);
    mpz_clear(r);
}
