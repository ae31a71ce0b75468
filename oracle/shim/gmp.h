/* Minimal stand-in for <gmp.h>.  Only the string codecs of the reference use GMP;
 * the integer codec path never calls these, so they are inert no-ops that exist
 * only so that bit_write.h compiles. */
#pragma once
#include <stdint.h>
typedef struct { int _unused; } __mpz_struct_stub;
typedef __mpz_struct_stub mpz_t[1];
static inline void mpz_init(mpz_t) {}
static inline void mpz_clear(mpz_t) {}
static inline void mpz_set(mpz_t, const mpz_t) {}
static inline void mpz_set_ui(mpz_t, unsigned long) {}
static inline unsigned long mpz_get_ui(const mpz_t) { return 0; }
static inline int mpz_sgn(const mpz_t) { return 0; }
static inline void mpz_neg(mpz_t, const mpz_t) {}
static inline void mpz_add(mpz_t, const mpz_t, const mpz_t) {}
static inline void mpz_add_ui(mpz_t, const mpz_t, unsigned long) {}
static inline void mpz_sub(mpz_t, const mpz_t, const mpz_t) {}
static inline void mpz_sub_ui(mpz_t, const mpz_t, unsigned long) {}
static inline void mpz_mul_2exp(mpz_t, const mpz_t, unsigned long) {}
static inline void mpz_fdiv_q_2exp(mpz_t, const mpz_t, unsigned long) {}
static inline void mpz_and(mpz_t, const mpz_t, const mpz_t) {}
static inline void mpz_ior(mpz_t, const mpz_t, const mpz_t) {}
static inline void mpz_mod(mpz_t, const mpz_t, const mpz_t) {}
static inline void mpz_div(mpz_t, const mpz_t, const mpz_t) {}
static inline int mpz_cmp(const mpz_t, const mpz_t) { return 0; }
static inline int mpz_cmp_ui(const mpz_t, unsigned long) { return 0; }
static inline void mpz_tdiv_r_2exp(mpz_t, const mpz_t, unsigned long) {}
