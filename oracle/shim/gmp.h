/* Declarations of the GMP 6 public functions the reference sources and the
 * host C++ restatement (oracle/pi_cpu.cpp) call (the image ships
 * libgmp.so.10 without its development header).  Names and
 * signatures follow GMP's documented API; the library itself is linked by
 * path.  Used only to build the parity oracle. */
#ifndef GPUPI_ORACLE_GMP_SHIM_H
#define GPUPI_ORACLE_GMP_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef unsigned long mp_limb_t;
typedef unsigned long mp_bitcnt_t;
typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t *_mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

void __gmpz_init(mpz_ptr);
void __gmpz_inits(mpz_ptr, ...);
void __gmpz_clear(mpz_ptr);
void __gmpz_clears(mpz_ptr, ...);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
unsigned long __gmpz_get_ui(mpz_srcptr);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void *);
void *__gmpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_fdiv_qr(mpz_ptr, mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_fdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_divexact_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_ui_pow_ui(mpz_ptr, unsigned long, unsigned long);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long);
void __gmpz_neg(mpz_ptr, mpz_srcptr);
void __gmpz_swap(mpz_ptr, mpz_ptr);
char *__gmpz_get_str(char *, int, mpz_srcptr);
unsigned long __gmpz_fdiv_ui(mpz_srcptr, unsigned long);
int __gmp_printf(const char *, ...);

#define mpz_init __gmpz_init
#define mpz_inits __gmpz_inits
#define mpz_clear __gmpz_clear
#define mpz_clears __gmpz_clears
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_get_ui __gmpz_get_ui
#define mpz_import __gmpz_import
#define mpz_export __gmpz_export
#define mpz_mul __gmpz_mul
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_add __gmpz_add
#define mpz_sub __gmpz_sub
#define mpz_add_ui __gmpz_add_ui
#define mpz_sub_ui __gmpz_sub_ui
#define mpz_sgn(Z) ((Z)->_mp_size < 0 ? -1 : (Z)->_mp_size > 0)
#define mpz_fdiv_qr __gmpz_fdiv_qr
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
#define mpz_fdiv_r_2exp __gmpz_fdiv_r_2exp
#define mpz_divexact_ui __gmpz_divexact_ui
#define mpz_ui_pow_ui __gmpz_ui_pow_ui
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_neg __gmpz_neg
#define mpz_swap __gmpz_swap
#define mpz_get_str __gmpz_get_str
#define mpz_fdiv_ui __gmpz_fdiv_ui
#define gmp_printf __gmp_printf
#ifdef __cplusplus
}
#endif
#endif
