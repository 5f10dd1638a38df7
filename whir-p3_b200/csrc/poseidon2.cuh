// Poseidon2 permutation over KoalaBear, width 16 and 24, S-box x^3.
//
// Structure from the Poseidon2 paper (Grassi, Khovratovich, Schofnegger,
// eprint 2023/323): an initial external linear layer, R_F/2 full rounds,
// R_P partial rounds, R_F/2 full rounds. The external layer is
// circ(2*M, M, ..., M) for a 4x4 block M; the internal layer is
// 1*1^T + diag(mu).
//
// Two choices of the block M (the template parameter MAT of every form below):
//   MAT 0  the circulant [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]]: the block
//          of Plonky3's Monty-31 external layer (`MDSMat4`), which
//          `Poseidon2KoalaBear` applies;
//   MAT 1  the paper's M4 [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]]
//          (Plonky3's `HLMDSMat4`, the Horizen Labs form).
// MAT 0 is the default of the library (the reference's permutation).
//
// Reference types this replaces: p3-koala-bear `Poseidon2KoalaBear<16>` and
// `<24>` (src/bin/main.rs:31-32), used by PaddingFreeSponge (leaf hashing),
// TruncatedPermutation (2-to-1 compression) and DuplexChallenger.
//
// The round constants are run-time data (`P2Consts`, canonical form, passed
// to kernels in the constant bank) so a caller can supply the constants of
// its deployment. The internal diagonal is fixed, as in p3-koala-bear, whose
// internal layer takes only round constants: its entries are small integers
// and signed powers of two, so every diagonal product is a few shifts and
// additions instead of a modular multiplication. The shapes (8 full rounds;
// 20 partial rounds at width 16, 23 at width 24) are compile-time.
//
// The permutation runs on canonical values. On the device the S-box products
// take their quotient from a double-precision estimate (the floating-point
// quotient method of Shoup's NTL MulMod): for a * b < 2^64,
// q = round(a * fl(b / p)) is within one of a * b / p, so r = a * b - q * p,
// computed modulo 2^32, lies in (-p, p) and one signed correction gives the
// residue. This moves the high halves of the products from the integer
// multiply pipe (which also carries every other product of the permutation)
// to the double-precision pipe.
#pragma once
#include "kb.cuh"

namespace p2 {

constexpr int RF = 8;
constexpr int RP16 = 20;
constexpr int RP24 = 23;

// external 4x4 block choices
constexpr int kMatMds = 0;  // Plonky3 MDSMat4 (circulant 2, 3, 1, 1)
constexpr int kMatHl = 1;   // the paper's M4 (Plonky3 HLMDSMat4)

struct P2Consts {
  uint32_t width, rounds_f, rounds_p;
  uint32_t mat;             // kMatMds or kMatHl
  uint32_t ext_rc[8 * 24];  // canonical
  uint32_t int_rc[32];      // canonical
  uint32_t diag_c[24];      // the fixed diagonal, canonical (run-time indexed uses)
  uint32_t diag_s[24];      // kb::shoup_const(diag_c)
  uint32_t ext_rc_m[8 * 24];  // ext_rc in Montgomery form (permutations run on Montgomery words)
  uint32_t int_rc_m[32];      // int_rc in Montgomery form
};

// Internal diagonal codes: an integer v in [-4, 4] \ {0} is v itself;
// 100 + k is 2^-k and 200 + k is -2^-k (1 <= k <= 24).
KB_HD constexpr int diag_code(int width, int i) {
  const int d16[16] = {-2, 1, 2, 101, 3, 4, 201, -3, -4, 108, 103, 124, 208, 203, 204, 224};
  const int d24[24] = {-2, 1,   2,   101, 3,   4,   201, -3,  -4,  108, 102, 103,
                       104, 105, 106, 124, 208, 203, 204, 205, 206, 207, 209, 224};
  return width == 16 ? d16[i] : d24[i];
}

// Canonical value of a diagonal code (2^-k = ((p + 1) / 2)^k).
inline uint32_t diag_value(int code) {
  if (code >= -4 && code <= 4) return code >= 0 ? (uint32_t)code : (uint32_t)((int64_t)kb::P + code);
  const int k = code % 100;
  uint64_t v = 1;
  for (int j = 0; j < k; j++) v = v * ((kb::P + 1) / 2) % kb::P;
  return code < 200 ? (uint32_t)v : (uint32_t)((kb::P - v) % kb::P);
}

// Entry (i, j) of the block M.
template <int MAT>
KB_HD constexpr int m4_entry(int i, int j) {
  const int hl[4][4] = {{5, 7, 1, 3}, {4, 6, 1, 1}, {1, 3, 5, 7}, {1, 1, 4, 6}};
  const int circ[4] = {2, 3, 1, 1};  // row i is this row rotated right by i
  return MAT == kMatHl ? hl[i][j] : circ[(j - i) & 3];
}

// x <- M x.
// MAT 0: with s = x0 + x1 + x2 + x3, a = s + x1 and b = s + x3, the rows are
//   2x0 + 3x1 + x2 + x3 = a + (x0 + x1),   x0 + 2x1 + 3x2 + x3 = a + 2x2,
//   x0 + x1 + 2x2 + 3x3 = b + (x2 + x3),   3x0 + x1 + x2 + 2x3 = b + 2x0:
//   9 additions and 2 doublings.
// MAT 1: the paper's addition chain (8 additions, 6 doublings).
template <int MAT>
KB_HD void m4(uint32_t& x0, uint32_t& x1, uint32_t& x2, uint32_t& x3) {
  using namespace kb;
  if (MAT == kMatHl) {
    const uint32_t t0 = add(x0, x1);
    const uint32_t t1 = add(x2, x3);
    const uint32_t t2 = add(dbl(x1), t1);
    const uint32_t t3 = add(dbl(x3), t0);
    const uint32_t t4 = add(dbl(dbl(t1)), t3);
    const uint32_t t5 = add(dbl(dbl(t0)), t2);
    x0 = add(t3, t5);
    x1 = t5;
    x2 = add(t2, t4);
    x3 = t4;
  } else {
    const uint32_t s01 = add(x0, x1), s23 = add(x2, x3);
    const uint32_t s = add(s01, s23);
    const uint32_t a = add(s, x1), b = add(s, x3);
    const uint32_t y0 = add(a, s01), y1 = add(a, dbl(x2));
    const uint32_t y2 = add(b, s23), y3 = add(b, dbl(x0));
    x0 = y0;
    x1 = y1;
    x2 = y2;
    x3 = y3;
  }
}

// Row 3 of M applied to (x0, x1, x2, x3).
template <int MAT>
KB_HD uint32_t m4_row3(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3) {
  using namespace kb;
  if (MAT == kMatHl) {  // x0 + x1 + 4x2 + 6x3
    const uint32_t t0 = add(x0, x1), t1 = add(x2, x3);
    return add(dbl(dbl(t1)), add(dbl(x3), t0));
  } else {  // 3x0 + x1 + x2 + 2x3
    const uint32_t s = add(add(x0, x1), add(x2, x3));
    return add(add(s, x3), dbl(x0));
  }
}

template <int T, int MAT>
KB_HD void ext_layer(uint32_t (&x)[T]) {
  using namespace kb;
#pragma unroll
  for (int c = 0; c < T; c += 4) m4<MAT>(x[c], x[c + 1], x[c + 2], x[c + 3]);
  uint32_t s0 = x[0], s1 = x[1], s2 = x[2], s3 = x[3];
#pragma unroll
  for (int c = 4; c < T; c += 4) {
    s0 = add(s0, x[c]);
    s1 = add(s1, x[c + 1]);
    s2 = add(s2, x[c + 2]);
    s3 = add(s3, x[c + 3]);
  }
#pragma unroll
  for (int c = 0; c < T; c += 4) {
    x[c] = add(x[c], s0);
    x[c + 1] = add(x[c + 1], s1);
    x[c + 2] = add(x[c + 2], s2);
    x[c + 3] = add(x[c + 3], s3);
  }
}

#ifdef __CUDA_ARCH__
// a as a double (exact: a < 2^53). A single conversion instruction; it was
// measured faster in this permutation than building 2^52 + a from its bit
// pattern and subtracting 2^52 (one instruction instead of two moves and an add).
__device__ __forceinline__ double exact_double(uint32_t a) { return __uint2double_rn(a); }
#endif

// v^3 mod p for any v < 2^32 (not necessarily reduced). On the device: with
// v < 2^32 the estimate of v^2 / p is off by less than 2^-20 before rounding,
// so q is within one of the quotient and t = v^2 - q p lies in (-p, p). t is
// kept signed (no correction): the second product t * v has |t * v| < 2^63,
// its estimate round(t * fl(v / p)) is again within one of the quotient (the
// rounding constant 1.5 * 2^52 leaves q mod 2^32 in the low word for negative
// q too), so t * v - q' p lies in (-p, p) and one correction finishes. On the
// host both products fit 64 bits.
KB_HD uint32_t cube(uint32_t v) {
#ifdef __CUDA_ARCH__
  constexpr double kInvP = 1.0 / 2130706433.0;
  const double vd = exact_double(v);
  const double vp = vd * kInvP;
  const double q = fma(vd, vp, 6755399441055744.0);
  const uint32_t t = v * v - (uint32_t)__double2loint(q) * kb::P;
  const double q2 = fma(__int2double_rn((int)t), vp, 6755399441055744.0);
  const uint32_t r = t * v - (uint32_t)__double2loint(q2) * kb::P;
  return kb::umin32(r, r + kb::P);
#else
  const uint64_t sq = (uint64_t)v * v % kb::P;
  return (uint32_t)(sq * v % kb::P);
#endif
}

// (a + b)^3 mod p for canonical a, b: the sum is below 2p < 2^32 and goes
// into the S-box unreduced.
KB_HD uint32_t cube_sum(uint32_t a, uint32_t b) { return cube(a + b); }

// x / 2, x canonical: (x + p) / 2 for odd x
KB_HD uint32_t halve(uint32_t x) { return (x >> 1) + (x & 1u) * ((kb::P + 1) / 2); }

// s +- x * 2^-k for canonical s, x and 1 <= k <= 24. With x = hi * 2^k + lo,
// x * 2^-k = hi + lo * 2^-k and 2^-k = -127 * 2^(24-k) (mod p), because
// 127 * 2^24 = p - 1; lo * 127 * 2^(24-k) < p.
KB_HD uint32_t add_shr(uint32_t s, uint32_t x, int k) {
  const uint32_t hi = x >> k, lo = x & ((1u << k) - 1u);
  uint32_t u = s + kb::P - lo * (127u << (24 - k));  // (s, s + p]
  u = kb::umin32(u, u - kb::P);
  u += hi;  // < p + p / 2
  return kb::umin32(u, u - kb::P);
}
KB_HD uint32_t sub_shr(uint32_t s, uint32_t x, int k) {
  const uint32_t hi = x >> k, lo = x & ((1u << k) - 1u);
  uint32_t u = s + lo * (127u << (24 - k));  // < 2p
  u = kb::umin32(u, u - kb::P);
  u = u + kb::P - hi;  // (p / 2, 2p)
  return kb::umin32(u, u - kb::P);
}

// s + mu * x for the diagonal code of mu (a compile-time constant after
// unrolling, so the switch folds away)
KB_HD uint32_t diag_axpy(int code, uint32_t s, uint32_t x) {
  using namespace kb;
  switch (code) {
    case 1: return add(s, x);
    case 2: return add(s, dbl(x));
    case 3: return add(s, add(dbl(x), x));
    case 4: return add(s, dbl(dbl(x)));
    case -2: return sub(s, dbl(x));
    case -3: return sub(s, add(dbl(x), x));
    case -4: return sub(s, dbl(dbl(x)));
    case 101: return add(s, halve(x));
    case 201: return sub(s, halve(x));
    default: return code > 200 ? sub_shr(s, x, code - 200) : add_shr(s, x, code - 100);
  }
}

template <int T, int MAT>
KB_HD void full_round(uint32_t (&x)[T], const uint32_t* rc) {
#pragma unroll
  for (int i = 0; i < T; i++) x[i] = cube_sum(x[i], rc[i]);
  ext_layer<T, MAT>(x);
}

// Sum of x[1..T-1] (T even, canonical values) mod p without a reduction per
// addition: pairs of values < p sum below 2^32, the pair sums accumulate in 64
// bits (below 2^36), and the total is reduced once with 2^32 = 2^25 - 2 (mod p).
template <int T>
KB_HD uint32_t sum_rest(const uint32_t (&x)[T]) {
  uint64_t acc = x[T - 1];
#pragma unroll
  for (int i = 1; i + 1 < T; i += 2) acc += (uint64_t)(x[i] + x[i + 1]);
  const uint32_t lo = (uint32_t)acc, hi = (uint32_t)(acc >> 32);
  uint32_t u = kb::umin32(lo, lo - 2u * kb::P);  // lo < 2^32 < 3p
  u = kb::umin32(u, u - kb::P);
  u += hi * 33554430u;  // hi < 2^4: u < p + 2^29
  return kb::umin32(u, u - kb::P);
}

// Internal round: S-box on x[0], then x_i <- sum(x) + mu_i * x_i. The sum of
// the words the S-box does not touch, a, is formed beside the S-box; with
// mu_0 = -2 the next S-box input is s - 2 x0 = a - x0 (s = a + x0), so only
// the S-box and one subtraction lie on the chain from round to round.
template <int T>
KB_HD void partial_round(uint32_t (&x)[T], uint32_t rc) {
  using namespace kb;
  static_assert(diag_code(T, 0) == -2, "the round form needs mu_0 = -2");
  const uint32_t a = sum_rest<T>(x);
  const uint32_t x0 = cube_sum(x[0], rc);
  const uint32_t s = add(a, x0);
  x[0] = sub(a, x0);
#pragma unroll
  for (int i = 1; i < T; i++) x[i] = diag_axpy(diag_code(T, i), s, x[i]);
}

// The permutation on canonical values. The round loops stay rolled: a fully
// unrolled width-24 permutation is about ten thousand instructions, more than
// the instruction cache holds, while one round body is a few hundred. The
// internal rounds are unrolled by two, so that one round's S-box overlaps the
// previous round's diagonal products (measured: 5 % more permutations per
// second at full occupancy, 12 % less latency). Round constants are read by
// index.
template <int T, int RP, int MAT>
KB_HD void permute_canonical(uint32_t (&x)[T], const P2Consts& k) {
  ext_layer<T, MAT>(x);
#pragma unroll 1
  for (int r = 0; r < RF / 2; r++) full_round<T, MAT>(x, k.ext_rc + r * T);
#pragma unroll 2
  for (int r = 0; r < RP; r++) partial_round<T>(x, k.int_rc[r]);
#pragma unroll 1
  for (int r = RF / 2; r < RF; r++) full_round<T, MAT>(x, k.ext_rc + r * T);
}

// The same with the block chosen at run time from k.mat (host-side callers).
template <int T, int RP>
inline void permute_canonical_rt(uint32_t (&x)[T], const P2Consts& k) {
  if (k.mat == (uint32_t)kMatHl) permute_canonical<T, RP, kMatHl>(x, k);
  else permute_canonical<T, RP, kMatMds>(x, k);
}

// Sponge forms of the permutation (PaddingFreeSponge, overwrite mode). FIRST:
// the capacity words (from RATE on) are zero on entry, so the initial external
// layer skips their M blocks and sums; LAST: only the first 8 words (the
// digest) of the output are read, so the final external layer forms only those.
template <int T, int RATE, int MAT>
KB_HD void ext_layer_zero_capacity(uint32_t (&x)[T]) {
  using namespace kb;
#pragma unroll
  for (int c = 0; c < RATE; c += 4) m4<MAT>(x[c], x[c + 1], x[c + 2], x[c + 3]);
  uint32_t s0 = x[0], s1 = x[1], s2 = x[2], s3 = x[3];
#pragma unroll
  for (int c = 4; c < RATE; c += 4) {
    s0 = add(s0, x[c]);
    s1 = add(s1, x[c + 1]);
    s2 = add(s2, x[c + 2]);
    s3 = add(s3, x[c + 3]);
  }
#pragma unroll
  for (int c = 0; c < T; c += 4) {
    x[c] = c < RATE ? add(x[c], s0) : s0;
    x[c + 1] = c < RATE ? add(x[c + 1], s1) : s1;
    x[c + 2] = c < RATE ? add(x[c + 2], s2) : s2;
    x[c + 3] = c < RATE ? add(x[c + 3], s3) : s3;
  }
}
template <int T, int MAT>
KB_HD void ext_layer_digest(uint32_t (&x)[T]) {
  using namespace kb;
#pragma unroll
  for (int c = 0; c < T; c += 4) m4<MAT>(x[c], x[c + 1], x[c + 2], x[c + 3]);
  uint32_t s0 = x[0], s1 = x[1], s2 = x[2], s3 = x[3];
#pragma unroll
  for (int c = 4; c < T; c += 4) {
    s0 = add(s0, x[c]);
    s1 = add(s1, x[c + 1]);
    s2 = add(s2, x[c + 2]);
    s3 = add(s3, x[c + 3]);
  }
#pragma unroll
  for (int c = 0; c < 8; c += 4) {
    x[c] = add(x[c], s0);
    x[c + 1] = add(x[c + 1], s1);
    x[c + 2] = add(x[c + 2], s2);
    x[c + 3] = add(x[c + 3], s3);
  }
}
template <int T, int RP, int RATE, bool FIRST, bool LAST, int MAT>
KB_HD void permute_sponge(uint32_t (&x)[T], const P2Consts& k) {
  if (FIRST) ext_layer_zero_capacity<T, RATE, MAT>(x);
  else ext_layer<T, MAT>(x);
#pragma unroll 1
  for (int r = 0; r < RF / 2; r++) full_round<T, MAT>(x, k.ext_rc + r * T);
#pragma unroll 2
  for (int r = 0; r < RP; r++) partial_round<T>(x, k.int_rc[r]);
#pragma unroll 1
  for (int r = RF / 2; r < RF - 1; r++) full_round<T, MAT>(x, k.ext_rc + r * T);
  const uint32_t* rc = k.ext_rc + (RF - 1) * T;
#pragma unroll
  for (int i = 0; i < T; i++) x[i] = cube_sum(x[i], rc[i]);
  if (LAST) ext_layer_digest<T, MAT>(x);
  else ext_layer<T, MAT>(x);
}

// Proof-of-work check of one candidate w (the duplex challenger's
// check_witness): the width-16 permutation of the sponge state with w at
// position SLOT, of which sample_bits reads only output word 7. The initial
// external layer is linear, so it and the first round's constants fold into
// cp = ext(state with 0 at SLOT) + rc (grind_fold, once per search) plus w
// times column SLOT of circ(2*M, M, M, M), whose entries are small integers;
// the last external layer forms word 7 only.
template <int MAT>
KB_HD constexpr int ext_col16(int slot, int i) {
  return m4_entry<MAT>(i & 3, slot & 3) * ((i >> 2) == (slot >> 2) ? 2 : 1);
}
// the largest entry of circ(2*M, M, M, M), plus one
template <int MAT>
KB_HD constexpr int ext_col_bound() {
  return MAT == kMatHl ? 15 : 7;
}
// state (canonical, 0 at the witness position) -> cp
template <int MAT>
KB_HD void grind_fold(uint32_t (&state)[16], const P2Consts& k) {
  ext_layer<16, MAT>(state);
#pragma unroll
  for (int i = 0; i < 16; i++) state[i] = kb::add(state[i], k.ext_rc[i]);
}
inline void grind_fold_rt(uint32_t (&state)[16], const P2Consts& k) {
  if (k.mat == (uint32_t)kMatHl) grind_fold<kMatHl>(state, k);
  else grind_fold<kMatMds>(state, k);
}
// `stop()` is asked twice, after the first full rounds and after the partial
// rounds; when it answers true the search no longer needs this candidate and
// the form returns 0xffffffff (nonzero in any low bits) without finishing.
struct NeverStop {
  KB_HD bool operator()() const { return false; }
};
template <int SLOT, int MAT, typename Stop = NeverStop>
KB_HD uint32_t grind_word7(uint32_t w, const uint32_t (&cp)[16], const P2Consts& k, Stop stop = Stop()) {
  using namespace kb;
  constexpr int kJ = ext_col_bound<MAT>();
  uint32_t wm[kJ];  // w * j mod p, j < kJ
  wm[0] = 0u;
  wm[1] = w;
#pragma unroll
  for (int j = 2; j < kJ; j++) wm[j] = add(wm[j - 1], w);
  uint32_t x[16];
#pragma unroll
  for (int i = 0; i < 16; i++) x[i] = cube_sum(cp[i], wm[ext_col16<MAT>(SLOT, i)]);
  ext_layer<16, MAT>(x);
#pragma unroll 1
  for (int r = 1; r < RF / 2; r++) full_round<16, MAT>(x, k.ext_rc + r * 16);
  if (stop()) return 0xffffffffu;
#pragma unroll 2
  for (int r = 0; r < RP16; r++) partial_round<16>(x, k.int_rc[r]);
  if (stop()) return 0xffffffffu;
#pragma unroll 1
  for (int r = RF / 2; r < RF - 1; r++) full_round<16, MAT>(x, k.ext_rc + r * 16);
  const uint32_t* rc = k.ext_rc + (RF - 1) * 16;
#pragma unroll
  for (int i = 0; i < 16; i++) x[i] = cube_sum(x[i], rc[i]);
  // word 7 of the external layer: row 3 of M on block 1, plus the sum of
  // row 3 of M over all blocks
  uint32_t r3[4];
#pragma unroll
  for (int b = 0; b < 4; b++) r3[b] = m4_row3<MAT>(x[4 * b], x[4 * b + 1], x[4 * b + 2], x[4 * b + 3]);
  return add(r3[1], add(add(r3[0], r3[1]), add(r3[2], r3[3])));
}

}  // namespace p2
