// Poseidon2 permutation over KoalaBear, width 16 and 24, S-box x^3.
//
// Structure from the Poseidon2 paper (Grassi, Khovratovich, Schofnegger,
// eprint 2023/323): an initial external linear layer, R_F/2 full rounds,
// R_P partial rounds, R_F/2 full rounds. The external layer is
// circ(2*M4, M4, ..., M4) with the paper's 4x4 matrix M4, evaluated with its
// published 8-addition chain; the internal layer is 1*1^T + diag(mu).
//
// Reference types this replaces: p3-koala-bear `Poseidon2KoalaBear<16>` and
// `<24>` (src/bin/main.rs:31-32), used by PaddingFreeSponge (leaf hashing),
// TruncatedPermutation (2-to-1 compression) and DuplexChallenger.
//
// The round constants and diagonal are run-time data (`P2Consts`, Montgomery
// form, passed to kernels in the constant bank) so a caller can supply the
// exact permutation of its deployment; the shapes (8 full rounds; 20 partial
// rounds at width 16, 23 at width 24) are compile-time.
#pragma once
#include "kb.cuh"

namespace p2 {

constexpr int RF = 8;
constexpr int RP16 = 20;
constexpr int RP24 = 23;

struct P2Consts {
  uint32_t width, rounds_f, rounds_p;
  uint32_t ext_rc[8 * 24];
  uint32_t int_rc[32];
  uint32_t diag[24];    // Montgomery form
  uint32_t diag_c[24];  // canonical, the Shoup multiplier
  uint32_t diag_s[24];  // kb::shoup_const(diag_c)
};

// M4 = [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] via the paper's addition chain.
KB_HD void m4(uint32_t& x0, uint32_t& x1, uint32_t& x2, uint32_t& x3) {
  using namespace kb;
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
}

template <int T>
KB_HD void ext_layer(uint32_t (&x)[T]) {
  using namespace kb;
#pragma unroll
  for (int c = 0; c < T; c += 4) m4(x[c], x[c + 1], x[c + 2], x[c + 3]);
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

// v^3 with the square left unreduced: v^2 < 2p, and (v^2) * v < 2p^2 < p * 2^32
KB_HD uint32_t cube(uint32_t v) { return kb::mul(kb::mul_lazy(v, v), v); }

template <int T>
KB_HD void full_round(uint32_t (&x)[T], const uint32_t* rc) {
#pragma unroll
  for (int i = 0; i < T; i++) x[i] = cube(kb::add(x[i], rc[i]));
  ext_layer<T>(x);
}

// Internal round: S-box on x[0], then x_i <- sum(x) + mu_i * x_i, the sum as
// a tree of four-element partial sums and the diagonal products in Shoup form
// (canonical mu_i times a Montgomery-form x_i is the Montgomery form of the
// product).
template <int T>
KB_HD void partial_round(uint32_t (&x)[T], uint32_t rc, const P2Consts& k) {
  using namespace kb;
  x[0] = cube(add(x[0], rc));
  uint32_t part[T / 4];
#pragma unroll
  for (int c = 0; c < T / 4; c++) part[c] = add(add(x[4 * c], x[4 * c + 1]), add(x[4 * c + 2], x[4 * c + 3]));
  uint32_t s = part[0];
#pragma unroll
  for (int c = 1; c < T / 4; c++) s = add(s, part[c]);
#pragma unroll
  for (int i = 0; i < T; i++) x[i] = add(s, mul_shoup(x[i], k.diag_c[i], k.diag_s[i]));
}

// The round loops stay rolled: a fully unrolled width-24 permutation is about
// ten thousand instructions, more than the instruction cache holds, while one
// round body is a few hundred. Round constants are read by index.
template <int T, int RP>
KB_HD void permute(uint32_t (&x)[T], const P2Consts& k) {
  ext_layer<T>(x);
#pragma unroll 1
  for (int r = 0; r < RF / 2; r++) full_round<T>(x, k.ext_rc + r * T);
#pragma unroll 1
  for (int r = 0; r < RP; r++) partial_round<T>(x, k.int_rc[r], k);
#pragma unroll 1
  for (int r = RF / 2; r < RF; r++) full_round<T>(x, k.ext_rc + r * T);
}

}  // namespace p2
