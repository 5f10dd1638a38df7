// Keccak family of the reference's Keccak WHIR configuration
// (src/whir/mod.rs:236-383): MerkleTreeMmcs<F, u64,
// SerializingHasher<PaddingFreeSponge<KeccakF, 25, 17, 4>>,
// CompressionFunctionFromHasher<.., 2, 4>, 4> and
// SerializingChallenger32<F, HashChallenger<u8, Keccak256Hash, 32>>.
//
// Keccak-f[1600] follows FIPS 202 (theta, rho, pi, chi, iota on 25 64-bit
// lanes, lane (x, y) at index x + 5y); its rotation offsets and round
// constants are generated at compile time by the standard's algorithms.
// Keccak256Hash is Keccak-256 with the original padding (0x01 ... 0x80, rate
// 136 bytes). The Merkle hash runs a 64-bit sponge: 17 lanes of rate,
// overwrite mode, a permutation after every full or partial chunk, output
// lanes 0..3; field elements (canonical values) enter it in pairs, v0 | v1 << 32.
// A digest is held as 8 words, word 2i the low and word 2i + 1 the high half
// of lane i, which are also its little-endian bytes.
#pragma once
#include <stdint.h>

#include "kb.cuh"

namespace kk {

KB_HD constexpr int lfsr_rc(int t) {
  // rc(t): output bit of the LFSR x^8 + x^6 + x^5 + x^4 + 1 after t steps
  if (t % 255 == 0) return 1;
  unsigned r = 1u;
  for (int i = 1; i <= t % 255; i++) {
    r <<= 1;
    if (r & 0x100u) r ^= 0x171u;
  }
  return (int)(r & 1u);
}
// iota constant of round ir
KB_HD constexpr uint64_t rc_of(int ir) {
  uint64_t rc = 0;
  for (int j = 0; j <= 6; j++)
    if (lfsr_rc(j + 7 * ir)) rc |= 1ull << ((1 << j) - 1);
  return rc;
}
// rho offset of lane i: the walk (x, y) <- (y, 2x + 3y) from (1, 0), step t
// giving (t + 1)(t + 2) / 2 mod 64
KB_HD constexpr int rho(int i) {
  if (i == 0) return 0;
  int x = 1, y = 0;
  for (int s = 0; s < 24; s++) {
    if (x + 5 * y == i) return ((s + 1) * (s + 2) / 2) % 64;
    const int nx = y, ny = (2 * x + 3 * y) % 5;
    x = nx;
    y = ny;
  }
  return 0;
}
// the lane pi moves lane i = x + 5y to: (y, 2x + 3y)
KB_HD constexpr int pi_dst(int i) { return (i / 5) + 5 * ((2 * (i % 5) + 3 * (i / 5)) % 5); }

#define KK_RC_LIST                                                                                              \
  rc_of(0), rc_of(1), rc_of(2), rc_of(3), rc_of(4), rc_of(5), rc_of(6), rc_of(7), rc_of(8), rc_of(9), rc_of(10), \
      rc_of(11), rc_of(12), rc_of(13), rc_of(14), rc_of(15), rc_of(16), rc_of(17), rc_of(18), rc_of(19),         \
      rc_of(20), rc_of(21), rc_of(22), rc_of(23)
#ifdef __CUDACC__
static __constant__ uint64_t c_rc[24] = {KK_RC_LIST};
#endif
static const uint64_t h_rc[24] = {KK_RC_LIST};
#undef KK_RC_LIST

KB_HD uint64_t rotl64(uint64_t v, int n) { return n == 0 ? v : (v << n) | (v >> (64 - n)); }

// Keccak-f[1600]. Every index is a compile-time constant after unrolling, so
// the 25 lanes stay in registers; the round constant is read from a small
// table by the round index.
KB_HD void keccak_f(uint64_t (&a)[25]) {
#if defined(__CUDA_ARCH__)
#pragma unroll 1
#endif
  for (int ir = 0; ir < 24; ir++) {
    uint64_t c[5], b[25];
#pragma unroll
    for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
#pragma unroll
    for (int x = 0; x < 5; x++) {
      const uint64_t d = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
#pragma unroll
      for (int y = 0; y < 5; y++) a[x + 5 * y] ^= d;
    }
#pragma unroll
    for (int i = 0; i < 25; i++) b[pi_dst(i)] = rotl64(a[i], rho(i));
#pragma unroll
    for (int y = 0; y < 5; y++)
#pragma unroll
      for (int x = 0; x < 5; x++)
        a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
#if defined(__CUDA_ARCH__)
    a[0] ^= c_rc[ir];
#else
    a[0] ^= h_rc[ir];
#endif
  }
}

// Keccak-256 absorbing state: the lanes and the bytes absorbed into the
// current 136-byte block.
struct K256 {
  uint64_t st[25];
  uint32_t pos;
};

KB_HD void k256_init(K256& k) {
  for (int i = 0; i < 25; i++) k.st[i] = 0;
  k.pos = 0;
}
KB_HD void k256_byte(K256& k, uint8_t b) {
  k.st[k.pos >> 3] ^= (uint64_t)b << (8 * (k.pos & 7));
  if (++k.pos == 136) {
    keccak_f(k.st);
    k.pos = 0;
  }
}
KB_HD void k256_update(K256& k, const uint8_t* in, size_t len) {
  for (size_t i = 0; i < len; i++) k256_byte(k, in[i]);
}
KB_HD void k256_word(K256& k, uint32_t v) {
  for (int i = 0; i < 4; i++) k256_byte(k, (uint8_t)(v >> (8 * i)));
}
// the digest of everything absorbed so far (k is left as it was)
KB_HD void k256_final(const K256& k, uint8_t (&out)[32]) {
  uint64_t st[25];
  for (int i = 0; i < 25; i++) st[i] = k.st[i];
  st[k.pos >> 3] ^= (uint64_t)0x01 << (8 * (k.pos & 7));
  st[135 >> 3] ^= (uint64_t)0x80 << (8 * (135 & 7));
  keccak_f(st);
  for (int i = 0; i < 32; i++) out[i] = (uint8_t)(st[i >> 3] >> (8 * (i & 7)));
}

// 2-to-1 compression of two digests (8 words each)
KB_HD void compress(const uint32_t* l, const uint32_t* r, uint32_t* out) {
  uint64_t st[25];
#pragma unroll
  for (int i = 0; i < 25; i++) st[i] = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    st[i] = (uint64_t)l[2 * i] | (uint64_t)l[2 * i + 1] << 32;
    st[4 + i] = (uint64_t)r[2 * i] | (uint64_t)r[2 * i + 1] << 32;
  }
  keccak_f(st);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    out[2 * i] = (uint32_t)st[i];
    out[2 * i + 1] = (uint32_t)(st[i] >> 32);
  }
}

}  // namespace kk
