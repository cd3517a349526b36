/*
 * Declarations of the subset of the GMP 6 integer API (mpz_*) used by this
 * project and by the CPU transforms it is checked against.
 *
 * The image ships the GMP runtime (libgmp.so.10, GMP 6.3.0) but no development
 * header.  This file declares the documented public API (names, argument types
 * and macro semantics as given in the GMP manual, "Integer Functions") against
 * the exported __gmpz_* symbols.  Link with the runtime by path:
 *   /usr/lib/x86_64-linux-gnu/libgmp.so.10
 *
 * Only the LP64 layout of mpz_t is supported (64-bit limbs).
 */
#ifndef ANNIE_B200_GMP_DECL_H
#define ANNIE_B200_GMP_DECL_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long int mp_limb_t;
typedef long int mp_size_t;
typedef unsigned long int mp_bitcnt_t;
typedef long int mp_exp_t;

typedef struct
{
	int _mp_alloc;
	int _mp_size;   /* |size| = limbs in use, sign = sign of the integer */
	mp_limb_t * _mp_d;
} __mpz_struct;

typedef __mpz_struct mpz_t[1];
typedef __mpz_struct * mpz_ptr;
typedef const __mpz_struct * mpz_srcptr;

#define GMP_LIMB_BITS 64

/* initialisation / assignment */
#define mpz_init __gmpz_init
void mpz_init(mpz_ptr);
#define mpz_inits __gmpz_inits
void mpz_inits(mpz_ptr, ...);
#define mpz_clear __gmpz_clear
void mpz_clear(mpz_ptr);
#define mpz_clears __gmpz_clears
void mpz_clears(mpz_ptr, ...);
#define mpz_set __gmpz_set
void mpz_set(mpz_ptr, mpz_srcptr);
#define mpz_set_ui __gmpz_set_ui
void mpz_set_ui(mpz_ptr, unsigned long int);
#define mpz_set_si __gmpz_set_si
void mpz_set_si(mpz_ptr, signed long int);
#define mpz_set_str __gmpz_set_str
int mpz_set_str(mpz_ptr, const char *, int);
#define mpz_init_set __gmpz_init_set
void mpz_init_set(mpz_ptr, mpz_srcptr);
#define mpz_init_set_ui __gmpz_init_set_ui
void mpz_init_set_ui(mpz_ptr, unsigned long int);
#define mpz_init_set_si __gmpz_init_set_si
void mpz_init_set_si(mpz_ptr, signed long int);

/* conversion */
#define mpz_get_ui __gmpz_get_ui
unsigned long int mpz_get_ui(mpz_srcptr);
#define mpz_get_d_2exp __gmpz_get_d_2exp
double mpz_get_d_2exp(signed long int *, mpz_srcptr);
#define mpz_get_str __gmpz_get_str
char * mpz_get_str(char *, int, mpz_srcptr);
#define mpz_import __gmpz_import
void mpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void *);
#define mpz_export __gmpz_export
void * mpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);

/* arithmetic */
#define mpz_add __gmpz_add
void mpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_add_ui __gmpz_add_ui
void mpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_sub __gmpz_sub
void mpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_sub_ui __gmpz_sub_ui
void mpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_mul __gmpz_mul
void mpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_mul_si __gmpz_mul_si
void mpz_mul_si(mpz_ptr, mpz_srcptr, long int);
#define mpz_mul_ui __gmpz_mul_ui
void mpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_mul_2exp __gmpz_mul_2exp
void mpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_neg __gmpz_neg
void mpz_neg(mpz_ptr, mpz_srcptr);
#define mpz_abs __gmpz_abs
void mpz_abs(mpz_ptr, mpz_srcptr);

/* division */
#define mpz_fdiv_q __gmpz_fdiv_q
void mpz_fdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_fdiv_r __gmpz_fdiv_r
void mpz_fdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
void mpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_fdiv_r_2exp __gmpz_fdiv_r_2exp
void mpz_fdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_tdiv_q_2exp __gmpz_tdiv_q_2exp
void mpz_tdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_mod __gmpz_mod
void mpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_fdiv_ui __gmpz_fdiv_ui
unsigned long int mpz_fdiv_ui(mpz_srcptr, unsigned long int);
#define mpz_divexact_ui __gmpz_divexact_ui
void mpz_divexact_ui(mpz_ptr, mpz_srcptr, unsigned long int);
/* Obsolete names kept by the manual: division rounding toward -infinity. */
#define mpz_div_2exp mpz_fdiv_q_2exp
#define mpz_mod_2exp mpz_fdiv_r_2exp

/* exponentiation, number theory */
#define mpz_powm __gmpz_powm
void mpz_powm(mpz_ptr, mpz_srcptr, mpz_srcptr, mpz_srcptr);
#define mpz_ui_pow_ui __gmpz_ui_pow_ui
void mpz_ui_pow_ui(mpz_ptr, unsigned long int, unsigned long int);
#define mpz_invert __gmpz_invert
int mpz_invert(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_gcd __gmpz_gcd
void mpz_gcd(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_probab_prime_p __gmpz_probab_prime_p
int mpz_probab_prime_p(mpz_srcptr, int);
#define mpz_si_kronecker __gmpz_si_kronecker
int mpz_si_kronecker(long, mpz_srcptr);
#define mpz_jacobi __gmpz_jacobi
int mpz_jacobi(mpz_srcptr, mpz_srcptr);
#define mpz_perfect_square_p __gmpz_perfect_square_p
int mpz_perfect_square_p(mpz_srcptr);
#define mpz_sqrt __gmpz_sqrt
void mpz_sqrt(mpz_ptr, mpz_srcptr);

/* comparison, bits, size */
#define mpz_cmp __gmpz_cmp
int mpz_cmp(mpz_srcptr, mpz_srcptr);
#define mpz_cmp_ui __gmpz_cmp_ui
int mpz_cmp_ui(mpz_srcptr, unsigned long int);
#define mpz_tstbit __gmpz_tstbit
int mpz_tstbit(mpz_srcptr, mp_bitcnt_t);
#define mpz_setbit __gmpz_setbit
void mpz_setbit(mpz_ptr, mp_bitcnt_t);
#define mpz_sizeinbase __gmpz_sizeinbase
size_t mpz_sizeinbase(mpz_srcptr, int);
#define mpz_size __gmpz_size
size_t mpz_size(mpz_srcptr);
#define mpz_getlimbn __gmpz_getlimbn
mp_limb_t mpz_getlimbn(mpz_srcptr, mp_size_t);

/* direct limb access */
#define mpz_limbs_read __gmpz_limbs_read
const mp_limb_t * mpz_limbs_read(mpz_srcptr);
#define mpz_limbs_write __gmpz_limbs_write
mp_limb_t * mpz_limbs_write(mpz_ptr, mp_size_t);
#define mpz_limbs_finish __gmpz_limbs_finish
void mpz_limbs_finish(mpz_ptr, mp_size_t);

/* Macros the manual documents as macros (sign and parity tests). */
#define mpz_sgn(z) ((z)->_mp_size < 0 ? -1 : (z)->_mp_size > 0)
#define mpz_odd_p(z) (((z)->_mp_size != 0) & (int)((z)->_mp_d[0]))
#define mpz_even_p(z) (!mpz_odd_p(z))

#ifdef __cplusplus
}
#endif

#endif
