/*
 * Oracle (test infrastructure only): KoalaBear prime field and its degree-4
 * binomial extension in plain canonical arithmetic.
 *
 * This file is part of the CPU restatement used by tests/, smoke() and the
 * CPU-baseline leg of bench.py to check the CUDA path. Nothing in the product
 * library includes, links or calls it.
 *
 * Restates (from published mathematics, not from source):
 *   - KoalaBear: p = 2^31 - 2^24 + 1 (Plonky3 p3-koala-bear @ c38eb05, the
 *     field `F` of src/bin/main.rs:28 and benches/whir.rs:21).
 *   - BinomialExtensionField<KoalaBear, 4> (src/bin/main.rs:29): F[X]/(X^4 - W)
 *     with W = 3, the smallest quadratic non-residue mod p (p = 1 mod 4, so
 *     X^4 - W is irreducible exactly when W is a non-residue).
 *   - two_adic_generator(bits) (used at src/whir/parameters.rs:183,381,394):
 *     g^((p-1)/2^bits) with g = 3, the smallest multiplicative generator.
 *
 * Values are always canonical (0 <= x < p). Products use exact 64-bit
 * arithmetic followed by `% p`, deliberately unlike the Montgomery form of
 * the GPU path so that the two implementations share no arithmetic code.
 */
#ifndef WHIR_ORACLE_FIELD_H
#define WHIR_ORACLE_FIELD_H

#include <stdint.h>

#define OR_P 0x7f000001u
#define OR_W 3u
#define OR_TWO_ADICITY 24
#define OR_GEN 3u

static inline uint32_t or_add(uint32_t a, uint32_t b) {
  uint32_t s = a + b;
  return s >= OR_P ? s - OR_P : s;
}
static inline uint32_t or_sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + OR_P - b; }
static inline uint32_t or_neg(uint32_t a) { return a ? OR_P - a : 0; }
static inline uint32_t or_mul(uint32_t a, uint32_t b) {
  return (uint32_t)(((uint64_t)a * (uint64_t)b) % OR_P);
}
static inline uint32_t or_pow(uint32_t a, uint64_t e) {
  uint32_t r = 1;
  while (e) {
    if (e & 1) r = or_mul(r, a);
    a = or_mul(a, a);
    e >>= 1;
  }
  return r;
}
static inline uint32_t or_inv(uint32_t a) { return or_pow(a, OR_P - 2); }
static inline uint32_t or_two_adic_generator(int bits) {
  /* generator of the multiplicative subgroup of order 2^bits */
  return or_pow(OR_GEN, (uint64_t)(OR_P - 1) >> bits);
}

typedef struct {
  uint32_t c[4];
} or_ef;

static inline or_ef or_ef_zero(void) {
  or_ef r = {{0, 0, 0, 0}};
  return r;
}
static inline or_ef or_ef_from(uint32_t a) {
  or_ef r = {{a, 0, 0, 0}};
  return r;
}
static inline int or_ef_eq(or_ef a, or_ef b) {
  return a.c[0] == b.c[0] && a.c[1] == b.c[1] && a.c[2] == b.c[2] && a.c[3] == b.c[3];
}
static inline int or_ef_is_zero(or_ef a) { return (a.c[0] | a.c[1] | a.c[2] | a.c[3]) == 0; }
static inline or_ef or_ef_add(or_ef a, or_ef b) {
  or_ef r;
  for (int i = 0; i < 4; i++) r.c[i] = or_add(a.c[i], b.c[i]);
  return r;
}
static inline or_ef or_ef_sub(or_ef a, or_ef b) {
  or_ef r;
  for (int i = 0; i < 4; i++) r.c[i] = or_sub(a.c[i], b.c[i]);
  return r;
}
static inline or_ef or_ef_double(or_ef a) { return or_ef_add(a, a); }
static inline or_ef or_ef_mul_base(or_ef a, uint32_t b) {
  or_ef r;
  for (int i = 0; i < 4; i++) r.c[i] = or_mul(a.c[i], b);
  return r;
}
static inline or_ef or_ef_mul(or_ef a, or_ef b) {
  /* schoolbook product reduced with X^4 = W */
  uint64_t t[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) t[i + j] = (t[i + j] + (uint64_t)or_mul(a.c[i], b.c[j])) % OR_P;
  or_ef r;
  for (int k = 0; k < 4; k++) {
    uint64_t hi = k + 4 < 7 ? t[k + 4] : 0;
    r.c[k] = (uint32_t)((t[k] + (uint64_t)OR_W * hi) % OR_P);
  }
  return r;
}
static inline or_ef or_ef_square(or_ef a) { return or_ef_mul(a, a); }
static inline or_ef or_ef_pow(or_ef a, uint64_t e) {
  or_ef r = or_ef_from(1);
  while (e) {
    if (e & 1) r = or_ef_mul(r, a);
    a = or_ef_mul(a, a);
    e >>= 1;
  }
  return r;
}

#endif
