// KoalaBear prime field (p = 2^31 - 2^24 + 1) and its degree-4 binomial
// extension (X^4 = 3), for device kernels and for the host-side transcript.
//
// Representation: Montgomery form with R = 2^32, value x stored as x*R mod p
// in [0, p). Reduction follows Montgomery (1985) in its "subtract" form:
// for T < 2^64, m = T_lo * p^-1 mod 2^32 makes T - m*p divisible by 2^32, and
// (T - m*p) / 2^32 = T_hi - mulhi(m, p) exactly (the low words cancel).
// Additions use the unsigned-min trick: with t = a + b - p (wrapping), the
// reduced sum is min(t + p, t), since t wraps to a large value exactly when
// a + b < p. Writing the sum as a three-input addition keeps it on the integer
// ALU pipe (a multiply-add cannot express it), leaving the multiply pipe to
// the Montgomery products.
//
// Reference types this replaces: p3-koala-bear `KoalaBear` and
// p3-field `BinomialExtensionField<KoalaBear, 4>` (src/bin/main.rs:28-29).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define KB_HD __host__ __device__ __forceinline__
#else
#define KB_HD inline
#endif

namespace kb {

constexpr uint32_t P = 0x7f000001u;
constexpr uint32_t P_INV = 0x81000001u;   // p^-1 mod 2^32
constexpr uint32_t R2 = 0x17f7efe4u;      // 2^64 mod p
constexpr uint32_t ONE = 0x01fffffeu;     // 2^32 mod p  (Montgomery form of 1)
constexpr uint32_t W = 3u;                // X^4 = W in the extension
constexpr int TWO_ADICITY = 24;

KB_HD uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

KB_HD uint32_t add(uint32_t a, uint32_t b) {
  uint32_t t = a + b - P;
  return umin32(t + P, t);
}
KB_HD uint32_t sub(uint32_t a, uint32_t b) {
  uint32_t t = a - b + P;
  return umin32(t, t - P);
}
KB_HD uint32_t neg(uint32_t a) { return sub(0u, a); }
KB_HD uint32_t dbl(uint32_t a) { return add(a, a); }

KB_HD uint32_t mulhi(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// Montgomery reduction of T < p * 2^32 (result in [0, p)).
KB_HD uint32_t reduce(uint64_t t) {
  uint32_t lo = (uint32_t)t, hi = (uint32_t)(t >> 32);
  uint32_t m = lo * P_INV;
  uint32_t r = hi - mulhi(m, P) + P;  // in (0, 2p)
  return umin32(r, r - P);
}
// Montgomery reduction of T < 2p * 2^32 (any sum of up to four products < p^2).
// Here hi - mulhi(m, p) lies in (-p, 2p); the two ranges overlap as unsigned
// 32-bit values, so the sign comes from the borrow, not from the value.
KB_HD uint32_t reduce_wide(uint64_t t) {
  uint32_t lo = (uint32_t)t, hi = (uint32_t)(t >> 32);
  uint32_t m = lo * P_INV;
  uint32_t mh = mulhi(m, P);
  uint32_t r = hi - mh + (hi < mh ? P : 0u);  // -> [0, 2p)
  return umin32(r, r - P);                    // -> [0, p)
}

KB_HD uint32_t mul(uint32_t a, uint32_t b) { return reduce((uint64_t)a * b); }
// Product by a constant w < p with Shoup's precomputed quotient (Shoup, NTL;
// Harvey, "Faster arithmetic for number-theoretic transforms", 2014):
// ws = floor(w * 2^32 / p), q = floor(a * ws / 2^32) <= floor(a * w / p) and
// a * w - q * p < 2p for every 32-bit a, so one conditional subtraction
// finishes. Three 32-bit multiplies (a*w, mulhi(a, ws), q*p as a multiply-add)
// instead of Montgomery's four. With a in Montgomery form and w canonical the
// result is the Montgomery form of the product.
KB_HD uint32_t shoup_const(uint32_t w) { return (uint32_t)(((uint64_t)w << 32) / P); }
KB_HD uint32_t mul_shoup(uint32_t a, uint32_t w, uint32_t ws) {
  const uint32_t q = mulhi(a, ws);
  const uint32_t r = a * w - q * P;
  return umin32(r, r - P);
}

KB_HD uint32_t sqr(uint32_t a) { return mul(a, a); }
KB_HD uint32_t to_mont(uint32_t x) { return mul(x, R2); }
KB_HD uint32_t from_mont(uint32_t x) { return reduce((uint64_t)x); }

KB_HD uint32_t pow(uint32_t a, uint64_t e) {
  uint32_t r = ONE;
  while (e) {
    if (e & 1) r = mul(r, a);
    a = mul(a, a);
    e >>= 1;
  }
  return r;
}
KB_HD uint32_t inv(uint32_t a) { return pow(a, P - 2); }

// Montgomery form of the generator of the subgroup of order 2^bits:
// 3^((p-1)/2^bits), 3 being the smallest multiplicative generator.
inline uint32_t two_adic_generator(int bits) { return pow(to_mont(3u), (uint64_t)(P - 1) >> bits); }

struct ef {
  uint32_t c[4];
};

KB_HD ef ef_zero() { return ef{{0u, 0u, 0u, 0u}}; }
KB_HD ef ef_one() { return ef{{ONE, 0u, 0u, 0u}}; }
KB_HD ef ef_from_base(uint32_t a) { return ef{{a, 0u, 0u, 0u}}; }
KB_HD ef ef_add(const ef& a, const ef& b) {
  return ef{{add(a.c[0], b.c[0]), add(a.c[1], b.c[1]), add(a.c[2], b.c[2]), add(a.c[3], b.c[3])}};
}
KB_HD ef ef_sub(const ef& a, const ef& b) {
  return ef{{sub(a.c[0], b.c[0]), sub(a.c[1], b.c[1]), sub(a.c[2], b.c[2]), sub(a.c[3], b.c[3])}};
}
KB_HD ef ef_dbl(const ef& a) { return ef_add(a, a); }
KB_HD ef ef_mul_base(const ef& a, uint32_t b) {
  return ef{{mul(a.c[0], b), mul(a.c[1], b), mul(a.c[2], b), mul(a.c[3], b)}};
}
KB_HD bool ef_eq(const ef& a, const ef& b) {
  return a.c[0] == b.c[0] && a.c[1] == b.c[1] && a.c[2] == b.c[2] && a.c[3] == b.c[3];
}

// Schoolbook product in F[X]/(X^4 - 3). The W-multiples of b are formed by
// additions, so every coefficient is a sum of four products < p^2, which fits
// 64 bits, and is reduced once.
KB_HD ef ef_mul(const ef& a, const ef& b) {
  const uint32_t b1w = add(dbl(b.c[1]), b.c[1]);
  const uint32_t b2w = add(dbl(b.c[2]), b.c[2]);
  const uint32_t b3w = add(dbl(b.c[3]), b.c[3]);
  uint64_t t0 = (uint64_t)a.c[0] * b.c[0] + (uint64_t)a.c[1] * b3w + (uint64_t)a.c[2] * b2w +
                (uint64_t)a.c[3] * b1w;
  uint64_t t1 = (uint64_t)a.c[0] * b.c[1] + (uint64_t)a.c[1] * b.c[0] + (uint64_t)a.c[2] * b3w +
                (uint64_t)a.c[3] * b2w;
  uint64_t t2 = (uint64_t)a.c[0] * b.c[2] + (uint64_t)a.c[1] * b.c[1] + (uint64_t)a.c[2] * b.c[0] +
                (uint64_t)a.c[3] * b3w;
  uint64_t t3 = (uint64_t)a.c[0] * b.c[3] + (uint64_t)a.c[1] * b.c[2] + (uint64_t)a.c[2] * b.c[1] +
                (uint64_t)a.c[3] * b.c[0];
  return ef{{reduce_wide(t0), reduce_wide(t1), reduce_wide(t2), reduce_wide(t3)}};
}
KB_HD ef ef_sqr(const ef& a) { return ef_mul(a, a); }
KB_HD ef ef_pow(ef a, uint64_t e) {
  ef r = ef_one();
  while (e) {
    if (e & 1) r = ef_mul(r, a);
    a = ef_mul(a, a);
    e >>= 1;
  }
  return r;
}

// Accumulator for sums of (extension x base) products with one reduction per
// four terms: each product is < p^2 and four of them fit 64 bits.
struct ef_acc {
  uint64_t t[4];
  int n;
  KB_HD void clear() { t[0] = t[1] = t[2] = t[3] = 0; n = 0; }
  KB_HD void fold(ef& into) {
    into = ef_add(into, ef{{reduce_wide(t[0]), reduce_wide(t[1]), reduce_wide(t[2]), reduce_wide(t[3])}});
    clear();
  }
  KB_HD void mac(const ef& a, uint32_t b, ef& into) {
    t[0] += (uint64_t)a.c[0] * b;
    t[1] += (uint64_t)a.c[1] * b;
    t[2] += (uint64_t)a.c[2] * b;
    t[3] += (uint64_t)a.c[3] * b;
    if (++n == 4) fold(into);
  }
};

}  // namespace kb
