/*
 * Declaration-only stand-in for <gmp.h>, used solely to compile the
 * reference's own C/CUDA sources for the oracle harness (the image ships the
 * GMP 6.3.0 runtime, libgmp.so.10, but not its development header).
 *
 * It holds public API names and signatures, the public mpz/randstate struct
 * shapes the ABI requires, and the documented mpz_sgn / mpz_odd_p /
 * mpz_even_p semantics.  Every function maps to the exported __gmpz_* /
 * __gmp_* symbol of the runtime library.  Nothing here implements GMP.
 */
#ifndef CCS_GMP_DECL_H
#define CCS_GMP_DECL_H

#include <stdio.h>
#include <stdarg.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long mp_limb_t;
typedef long mp_size_t;
typedef unsigned long mp_bitcnt_t;

typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t* _mp_d;
} __mpz_struct;

typedef __mpz_struct mpz_t[1];
typedef __mpz_struct* mpz_ptr;
typedef const __mpz_struct* mpz_srcptr;

/* random state: public shape, padded generously (the library only writes
 * within its own size) */
typedef struct {
    __mpz_struct _mp_seed;
    int _mp_alg;
    union { void* _mp_lc; } _mp_algdata;
    char _pad[64];
} __gmp_randstate_struct;
typedef __gmp_randstate_struct gmp_randstate_t[1];

void __gmpz_init(mpz_ptr);
void __gmpz_inits(mpz_ptr, ...);
void __gmpz_clear(mpz_ptr);
void __gmpz_clears(mpz_ptr, ...);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
int __gmpz_set_str(mpz_ptr, const char*, int);
void __gmpz_init_set(mpz_ptr, mpz_srcptr);
int __gmpz_init_set_str(mpz_ptr, const char*, int);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long);
int __gmpz_probab_prime_p(mpz_srcptr, int);
unsigned long __gmpz_fdiv_ui(mpz_srcptr, unsigned long);
void __gmpz_fdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
unsigned long __gmpz_fdiv_q_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_cdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_addmul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
size_t __gmpz_out_str(FILE*, int, mpz_srcptr);
int __gmpz_divisible_p(mpz_srcptr, mpz_srcptr);
int __gmp_fprintf(FILE*, const char*, ...);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
void __gmpz_ui_pow_ui(mpz_ptr, unsigned long, unsigned long);
char* __gmpz_get_str(char*, int, mpz_srcptr);
unsigned long __gmpz_get_ui(mpz_srcptr);
double __gmpz_get_d(mpz_srcptr);
void __gmpz_powm(mpz_ptr, mpz_srcptr, mpz_srcptr, mpz_srcptr);
void __gmpz_gcd(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_divexact(mpz_ptr, mpz_srcptr, mpz_srcptr);
int __gmpz_divisible_ui_p(mpz_srcptr, unsigned long);
size_t __gmpz_size(mpz_srcptr);
mp_limb_t __gmpz_getlimbn(mpz_srcptr, mp_size_t);
size_t __gmpz_inp_str(mpz_ptr, FILE*, int);
void __gmpz_urandomm(mpz_ptr, __gmp_randstate_struct*, mpz_srcptr);
void __gmp_randinit_mt(__gmp_randstate_struct*);
void __gmp_randseed_ui(__gmp_randstate_struct*, unsigned long);
void __gmp_randclear(__gmp_randstate_struct*);
int __gmp_snprintf(char*, size_t, const char*, ...);
int __gmp_printf(const char*, ...);

#define mpz_init __gmpz_init
#define mpz_inits __gmpz_inits
#define mpz_clear __gmpz_clear
#define mpz_clears __gmpz_clears
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_set_str __gmpz_set_str
#define mpz_init_set __gmpz_init_set
#define mpz_init_set_str __gmpz_init_set_str
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_probab_prime_p __gmpz_probab_prime_p
#define mpz_fdiv_ui __gmpz_fdiv_ui
#define mpz_fdiv_q __gmpz_fdiv_q
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
#define mpz_fdiv_q_ui __gmpz_fdiv_q_ui
#define mpz_cdiv_q __gmpz_cdiv_q
#define mpz_add __gmpz_add
#define mpz_add_ui __gmpz_add_ui
#define mpz_addmul_ui __gmpz_addmul_ui
#define mpz_sub __gmpz_sub
#define mpz_sub_ui __gmpz_sub_ui
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_mul __gmpz_mul
#define mpz_out_str __gmpz_out_str
#define mpz_divisible_p __gmpz_divisible_p
#define gmp_fprintf __gmp_fprintf
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_ui_pow_ui __gmpz_ui_pow_ui
#define mpz_get_str __gmpz_get_str
#define mpz_get_ui __gmpz_get_ui
#define mpz_get_d __gmpz_get_d
#define mpz_powm __gmpz_powm
#define mpz_gcd __gmpz_gcd
#define mpz_mod __gmpz_mod
#define mpz_divexact __gmpz_divexact
#define mpz_divisible_ui_p __gmpz_divisible_ui_p
#define mpz_size __gmpz_size
#define mpz_getlimbn __gmpz_getlimbn
#define mpz_inp_str __gmpz_inp_str
#define mpz_urandomm __gmpz_urandomm
#define gmp_randinit_mt __gmp_randinit_mt
#define gmp_randseed_ui __gmp_randseed_ui
#define gmp_randclear __gmp_randclear
#define gmp_snprintf __gmp_snprintf
#define gmp_printf __gmp_printf

/* documented value semantics */
#define mpz_sgn(z) ((z)->_mp_size < 0 ? -1 : (z)->_mp_size > 0)
#define mpz_odd_p(z) (((z)->_mp_size != 0) & (int)((z)->_mp_d[0] & 1))
#define mpz_even_p(z) (!mpz_odd_p(z))

#ifdef __cplusplus
}
#endif
#endif
