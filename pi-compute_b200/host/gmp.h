/*
 * Minimal declaration header for the GNU MP library (libgmp.so.10, GMP 6.x).
 *
 * The container image ships the GMP runtime library but not its development
 * header. This file declares the subset of GMP's documented public API that
 * this project (and the oracle build of the reference's CPU sources) uses:
 * the documented types mpz_t / mpf_t, and each documented function under its
 * exported link name (__gmpz_* / __gmpf_*), mapped to the public name with a
 * macro exactly as the GMP manual describes ("mpz_mul" is the documented
 * name, "__gmpz_mul" the symbol libgmp exports).
 *
 * Only LP64 targets (x86_64, aarch64 Linux) are supported: mp_limb_t is a
 * 64-bit unsigned long there.
 */
#ifndef PI_B200_GMP_DECL_H
#define PI_B200_GMP_DECL_H

#include <stddef.h>
#include <stdio.h>

#if !defined(__LP64__)
#error "this GMP declaration header assumes an LP64 target (64-bit limbs)"
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long mp_limb_t;
typedef long mp_limb_signed_t;
typedef long mp_size_t;
typedef long mp_exp_t;
typedef unsigned long mp_bitcnt_t;

#define GMP_LIMB_BITS 64
#define GMP_NUMB_BITS 64

/* Integer: |_mp_size| limbs at _mp_d, little-endian; the sign of _mp_size is
 * the sign of the integer (GMP manual, "Integer Internals"). */
typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t* _mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct* mpz_ptr;
typedef const __mpz_struct* mpz_srcptr;

/* Float (GMP manual, "Float Internals"). */
typedef struct {
    int _mp_prec;
    int _mp_size;
    mp_exp_t _mp_exp;
    mp_limb_t* _mp_d;
} __mpf_struct;
typedef __mpf_struct mpf_t[1];
typedef __mpf_struct* mpf_ptr;
typedef const __mpf_struct* mpf_srcptr;

extern const char* const __gmp_version;
#define gmp_version __gmp_version

/* ---- mpz: initialisation and assignment ---- */
void __gmpz_init(mpz_ptr);
void __gmpz_init2(mpz_ptr, mp_bitcnt_t);
void __gmpz_clear(mpz_ptr);
void __gmpz_realloc2(mpz_ptr, mp_bitcnt_t);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
void __gmpz_set_si(mpz_ptr, long);
int __gmpz_set_str(mpz_ptr, const char*, int);
void __gmpz_set_f(mpz_ptr, mpf_srcptr);
void __gmpz_swap(mpz_ptr, mpz_ptr);
void __gmpz_init_set(mpz_ptr, mpz_srcptr);
void __gmpz_init_set_ui(mpz_ptr, unsigned long);
void __gmpz_init_set_si(mpz_ptr, long);
int __gmpz_init_set_str(mpz_ptr, const char*, int);

/* ---- mpz: arithmetic ---- */
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul_si(mpz_ptr, mpz_srcptr, long);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_addmul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_neg(mpz_ptr, mpz_srcptr);
void __gmpz_abs(mpz_ptr, mpz_srcptr);
void __gmpz_pow_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_ui_pow_ui(mpz_ptr, unsigned long, unsigned long);
void __gmpz_sqrt(mpz_ptr, mpz_srcptr);
void __gmpz_tdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_tdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_tdiv_qr(mpz_ptr, mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_tdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_tdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);

/* ---- mpz: comparison and inspection ---- */
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long);
int __gmpz_cmp_si(mpz_srcptr, long);
int __gmpz_cmpabs(mpz_srcptr, mpz_srcptr);
size_t __gmpz_size(mpz_srcptr);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
unsigned long __gmpz_get_ui(mpz_srcptr);
mp_bitcnt_t __gmpz_scan1(mpz_srcptr, mp_bitcnt_t);

/* ---- mpz: conversion and raw limb access ---- */
char* __gmpz_get_str(char*, int, mpz_srcptr);
void* __gmpz_export(void*, size_t*, int, size_t, int, size_t, mpz_srcptr);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void*);
const mp_limb_t* __gmpz_limbs_read(mpz_srcptr);
mp_limb_t* __gmpz_limbs_write(mpz_ptr, mp_size_t);
mp_limb_t* __gmpz_limbs_modify(mpz_ptr, mp_size_t);
void __gmpz_limbs_finish(mpz_ptr, mp_size_t);
mpz_srcptr __gmpz_roinit_n(mpz_ptr, const mp_limb_t*, mp_size_t);

/* ---- mpf ---- */
void __gmpf_init2(mpf_ptr, mp_bitcnt_t);
void __gmpf_clear(mpf_ptr);
void __gmpf_set_prec(mpf_ptr, mp_bitcnt_t);
mp_bitcnt_t __gmpf_get_prec(mpf_srcptr);
void __gmpf_set_ui(mpf_ptr, unsigned long);
void __gmpf_set_z(mpf_ptr, mpz_srcptr);
void __gmpf_mul(mpf_ptr, mpf_srcptr, mpf_srcptr);
void __gmpf_div(mpf_ptr, mpf_srcptr, mpf_srcptr);
void __gmpf_sqrt(mpf_ptr, mpf_srcptr);
char* __gmpf_get_str(char*, mp_exp_t*, int, size_t, mpf_srcptr);

/* ---- memory functions (used to free strings returned by get_str) ---- */
void __gmp_get_memory_functions(void* (**)(size_t), void* (**)(void*, size_t, size_t),
                                void (**)(void*, size_t));

#ifdef __cplusplus
}
#endif

#define mpz_init __gmpz_init
#define mpz_init2 __gmpz_init2
#define mpz_clear __gmpz_clear
#define mpz_realloc2 __gmpz_realloc2
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_set_si __gmpz_set_si
#define mpz_set_str __gmpz_set_str
#define mpz_set_f __gmpz_set_f
#define mpz_swap __gmpz_swap
#define mpz_init_set __gmpz_init_set
#define mpz_init_set_ui __gmpz_init_set_ui
#define mpz_init_set_si __gmpz_init_set_si
#define mpz_init_set_str __gmpz_init_set_str
#define mpz_add __gmpz_add
#define mpz_add_ui __gmpz_add_ui
#define mpz_sub __gmpz_sub
#define mpz_sub_ui __gmpz_sub_ui
#define mpz_mul __gmpz_mul
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_mul_si __gmpz_mul_si
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_addmul __gmpz_addmul
#define mpz_neg __gmpz_neg
#define mpz_abs __gmpz_abs
#define mpz_pow_ui __gmpz_pow_ui
#define mpz_ui_pow_ui __gmpz_ui_pow_ui
#define mpz_sqrt __gmpz_sqrt
#define mpz_tdiv_q __gmpz_tdiv_q
#define mpz_tdiv_r __gmpz_tdiv_r
#define mpz_tdiv_qr __gmpz_tdiv_qr
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
#define mpz_tdiv_q_2exp __gmpz_tdiv_q_2exp
#define mpz_tdiv_r_2exp __gmpz_tdiv_r_2exp
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_cmp_si __gmpz_cmp_si
#define mpz_cmpabs __gmpz_cmpabs
#define mpz_size __gmpz_size
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_get_ui __gmpz_get_ui
#define mpz_scan1 __gmpz_scan1
#define mpz_get_str __gmpz_get_str
#define mpz_export __gmpz_export
#define mpz_import __gmpz_import
#define mpz_limbs_read __gmpz_limbs_read
#define mpz_limbs_write __gmpz_limbs_write
#define mpz_limbs_modify __gmpz_limbs_modify
#define mpz_limbs_finish __gmpz_limbs_finish
#define mpz_roinit_n __gmpz_roinit_n
#define mpf_init2 __gmpf_init2
#define mpf_clear __gmpf_clear
#define mpf_set_prec __gmpf_set_prec
#define mpf_get_prec __gmpf_get_prec
#define mpf_set_ui __gmpf_set_ui
#define mpf_set_z __gmpf_set_z
#define mpf_mul __gmpf_mul
#define mpf_div __gmpf_div
#define mpf_sqrt __gmpf_sqrt
#define mpf_get_str __gmpf_get_str
#define mp_get_memory_functions __gmp_get_memory_functions

/* The GMP manual documents mpz_sgn as a macro reading the sign of _mp_size; an inline
 * function with the same result lets C++ wrappers convert to mpz_srcptr implicitly. */
static inline int mpz_sgn(mpz_srcptr z) { return z->_mp_size < 0 ? -1 : z->_mp_size > 0; }

#endif /* PI_B200_GMP_DECL_H */
