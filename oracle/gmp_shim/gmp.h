/* gmp.h -- declarations of the GMP integer functions that the reference's
 * vendored CGBN host code names (cgbn/cgbn_mpz.h, cgbn/impl_mpz.cc), so that
 * the reference's plain binary (AlphaComplexParallel.cu, which includes
 * <gmp.h> through cgbn/xmp_float.h) compiles where GMP's development headers
 * are not installed.  It links against the system's runtime library
 * libgmp.so.10, whose exported names are the __gmpz_* ones declared here.
 *
 * Checker infrastructure only (oracle/ref_build.sh); written from GMP's
 * documented public interface (types and prototypes of the mpz_ functions).
 * The reference never runs this code on its hot path: its CGBN fallback is
 * dead (it builds a few values and writes nothing).
 */
#ifndef __GMP_H__
#define __GMP_H__

#include <stddef.h>
#include <stdio.h>

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
typedef const __mpz_struct *mpz_srcptr;
typedef __mpz_struct *mpz_ptr;

void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
void __gmpz_set_si(mpz_ptr, long);
void __gmpz_swap(mpz_ptr, mpz_ptr);
unsigned long __gmpz_get_ui(mpz_srcptr);
long __gmpz_get_si(mpz_srcptr);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_ui_sub(mpz_ptr, unsigned long, mpz_srcptr);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_submul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_fdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_fdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_fdiv_qr(mpz_ptr, mpz_ptr, mpz_srcptr, mpz_srcptr);
unsigned long __gmpz_fdiv_q_ui(mpz_ptr, mpz_srcptr, unsigned long);
unsigned long __gmpz_fdiv_r_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_fdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long);
int __gmpz_tstbit(mpz_srcptr, mp_bitcnt_t);
void __gmpz_setbit(mpz_ptr, mp_bitcnt_t);
void __gmpz_clrbit(mpz_ptr, mp_bitcnt_t);
void __gmpz_and(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_ior(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_xor(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sqrt(mpz_ptr, mpz_srcptr);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
int __gmpz_invert(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_gcd(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_powm(mpz_ptr, mpz_srcptr, mpz_srcptr, mpz_srcptr);
mp_bitcnt_t __gmpz_popcount(mpz_srcptr);
mp_bitcnt_t __gmpz_scan1(mpz_srcptr, mp_bitcnt_t);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void *);
void *__gmpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);
size_t __gmpz_out_str(FILE *, int, mpz_srcptr);

#define mpz_init __gmpz_init
#define mpz_clear __gmpz_clear
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_set_si __gmpz_set_si
#define mpz_swap __gmpz_swap
#define mpz_get_ui __gmpz_get_ui
#define mpz_get_si __gmpz_get_si
#define mpz_add __gmpz_add
#define mpz_add_ui __gmpz_add_ui
#define mpz_sub __gmpz_sub
#define mpz_sub_ui __gmpz_sub_ui
#define mpz_ui_sub __gmpz_ui_sub
#define mpz_mul __gmpz_mul
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_submul __gmpz_submul
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_fdiv_q __gmpz_fdiv_q
#define mpz_fdiv_r __gmpz_fdiv_r
#define mpz_fdiv_qr __gmpz_fdiv_qr
#define mpz_fdiv_q_ui __gmpz_fdiv_q_ui
#define mpz_fdiv_r_ui __gmpz_fdiv_r_ui
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
#define mpz_fdiv_r_2exp __gmpz_fdiv_r_2exp
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_tstbit __gmpz_tstbit
#define mpz_setbit __gmpz_setbit
#define mpz_clrbit __gmpz_clrbit
#define mpz_and __gmpz_and
#define mpz_ior __gmpz_ior
#define mpz_xor __gmpz_xor
#define mpz_sqrt __gmpz_sqrt
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_invert __gmpz_invert
#define mpz_gcd __gmpz_gcd
#define mpz_powm __gmpz_powm
#define mpz_popcount __gmpz_popcount
#define mpz_scan1 __gmpz_scan1
#define mpz_import __gmpz_import
#define mpz_export __gmpz_export
#define mpz_out_str __gmpz_out_str
/* sign of z: the sign of its stored limb count */
#define mpz_sgn(z) ((z)->_mp_size < 0 ? -1 : (z)->_mp_size > 0)

#ifdef __cplusplus
}
#endif
#endif /* __GMP_H__ */
