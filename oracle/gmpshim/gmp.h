/* Minimal declarations of GMP 6.3.0's documented mpz API, written from the
 * GMP manual, so that the reference's C++ sources compile against the system
 * runtime libgmp.so.10 in a container without GMP development headers.
 *
 * TEST INFRASTRUCTURE ONLY (used to build the reference checker under
 * oracle/_ref).  Public names follow the manual; the library exports each
 * mpz_xxx function as __gmpz_xxx. */
#ifndef CUHE_ORACLE_GMP_SHIM_H
#define CUHE_ORACLE_GMP_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long mp_limb_t;
typedef long mp_size_t;
typedef unsigned long mp_bitcnt_t;
#define GMP_NUMB_BITS 64
#define GMP_LIMB_BITS 64

typedef struct {
  int _mp_alloc;
  int _mp_size;
  mp_limb_t* _mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct* mpz_ptr;
typedef const __mpz_struct* mpz_srcptr;

/* random state: seed, algorithm tag, algorithm data */
typedef struct {
  __mpz_struct _mp_seed;
  int _mp_alg;
  union { void* _mp_lc; } _mp_algdata;
} __gmp_randstate_struct;
typedef __gmp_randstate_struct gmp_randstate_t[1];

extern const char* const __gmp_version;
#define gmp_version __gmp_version

#define GMPZ(name) __gmpz_##name
void __gmpz_init(mpz_ptr);
void __gmpz_init_set(mpz_ptr, mpz_srcptr);
void __gmpz_init_set_ui(mpz_ptr, unsigned long);
void __gmpz_init_set_si(mpz_ptr, long);
int __gmpz_init_set_str(mpz_ptr, const char*, int);
void __gmpz_clear(mpz_ptr);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
void __gmpz_set_si(mpz_ptr, long);
int __gmpz_set_str(mpz_ptr, const char*, int);
void __gmpz_swap(mpz_ptr, mpz_ptr);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_ui_sub(mpz_ptr, unsigned long, mpz_srcptr);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul_si(mpz_ptr, mpz_srcptr, long);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_addmul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_submul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_neg(mpz_ptr, mpz_srcptr);
void __gmpz_tdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_tdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_fdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_fdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
unsigned long __gmpz_fdiv_ui(mpz_srcptr, unsigned long);
void __gmpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long);
int __gmpz_cmp_si(mpz_srcptr, long);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
mp_limb_t __gmpz_getlimbn(mpz_srcptr, mp_size_t);
size_t __gmpz_size(mpz_srcptr);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void*);
void* __gmpz_export(void*, size_t*, int, size_t, int, size_t, mpz_srcptr);
int __gmpz_probab_prime_p(mpz_srcptr, int);
char* __gmpz_get_str(char*, int, mpz_srcptr);
unsigned long __gmpz_get_ui(mpz_srcptr);
long __gmpz_get_si(mpz_srcptr);
int __gmpz_fits_ulong_p(mpz_srcptr);
int __gmpz_fits_slong_p(mpz_srcptr);
void __gmpz_urandomb(mpz_ptr, gmp_randstate_t, mp_bitcnt_t);
void __gmpz_urandomm(mpz_ptr, gmp_randstate_t, mpz_srcptr);
void __gmp_randinit_default(gmp_randstate_t);
void __gmp_randseed_ui(gmp_randstate_t, unsigned long);
void __gmp_randclear(gmp_randstate_t);
void __gmp_get_memory_functions(void* (**)(size_t), void* (**)(void*, size_t, size_t), void (**)(void*, size_t));

#define mpz_init __gmpz_init
#define mpz_init_set __gmpz_init_set
#define mpz_init_set_ui __gmpz_init_set_ui
#define mpz_init_set_si __gmpz_init_set_si
#define mpz_init_set_str __gmpz_init_set_str
#define mpz_clear __gmpz_clear
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_set_si __gmpz_set_si
#define mpz_set_str __gmpz_set_str
#define mpz_swap __gmpz_swap
#define mpz_add __gmpz_add
#define mpz_add_ui __gmpz_add_ui
#define mpz_sub __gmpz_sub
#define mpz_sub_ui __gmpz_sub_ui
#define mpz_ui_sub __gmpz_ui_sub
#define mpz_mul __gmpz_mul
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_mul_si __gmpz_mul_si
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_addmul_ui __gmpz_addmul_ui
#define mpz_submul_ui __gmpz_submul_ui
#define mpz_neg __gmpz_neg
#define mpz_tdiv_q __gmpz_tdiv_q
#define mpz_tdiv_r __gmpz_tdiv_r
#define mpz_fdiv_q __gmpz_fdiv_q
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
#define mpz_fdiv_r_2exp __gmpz_fdiv_r_2exp
#define mpz_fdiv_ui __gmpz_fdiv_ui
#define mpz_mod __gmpz_mod
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_cmp_si __gmpz_cmp_si
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_getlimbn __gmpz_getlimbn
#define mpz_size __gmpz_size
#define mpz_import __gmpz_import
#define mpz_export __gmpz_export
#define mpz_probab_prime_p __gmpz_probab_prime_p
#define mpz_get_str __gmpz_get_str
#define mpz_get_ui __gmpz_get_ui
#define mpz_get_si __gmpz_get_si
#define mpz_fits_ulong_p __gmpz_fits_ulong_p
#define mpz_fits_slong_p __gmpz_fits_slong_p
#define mpz_urandomb __gmpz_urandomb
#define mpz_urandomm __gmpz_urandomm
#define gmp_randinit_default __gmp_randinit_default
#define gmp_randseed_ui __gmp_randseed_ui
#define gmp_randclear __gmp_randclear
#define mp_get_memory_functions __gmp_get_memory_functions
#define mpz_sgn(z) ((z)->_mp_size < 0 ? -1 : (z)->_mp_size > 0)
#define mpz_odd_p(z) (((z)->_mp_size != 0) & (int)((z)->_mp_d[0]))
#define mpz_even_p(z) (!mpz_odd_p(z))

#ifdef __cplusplus
}
#endif

#endif
