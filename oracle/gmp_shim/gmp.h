/* gmp.h -- declarations of the part of GMP's documented mpz interface that
 * the reference's tests use.  This image ships libgmp.so.10 without its
 * header; link against that library.  Test tooling only. */
#ifndef BW_GMP_SHIM_H
#define BW_GMP_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef unsigned long mp_limb_t;
typedef unsigned long mp_bitcnt_t;
typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t* _mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct* mpz_ptr;
typedef const __mpz_struct* mpz_srcptr;

void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
void __gmpz_init_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
unsigned long __gmpz_get_ui(mpz_srcptr);
void __gmpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void*);
void* __gmpz_export(void*, size_t*, int, size_t, int, size_t, mpz_srcptr);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);

#define mpz_init __gmpz_init
#define mpz_clear __gmpz_clear
#define mpz_init_set __gmpz_init_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_add_ui __gmpz_add_ui
#define mpz_get_ui __gmpz_get_ui
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
#define mpz_import __gmpz_import
#define mpz_export __gmpz_export
#define mpz_mul __gmpz_mul
#ifdef __cplusplus
}
#endif
#endif
