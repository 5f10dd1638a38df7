/*
 * Oracle (test infrastructure only): Plonky3 primitives restated from their
 * published algorithms, plus the whir-p3 polynomial routines.
 *
 *   Poseidon2 ...... Grassi, Khovratovich, Schofnegger, "Poseidon2: A Faster
 *                    Version of the Poseidon Hash Function", eprint 2023/323.
 *                    S-box x^3, external matrix circ(2*M, M, ...) for a 4x4
 *                    block M, internal matrix 1*1^T + diag(mu). Round counts
 *                    8 full + 20 partial (width 16) and 8 + 23 (width 24) for
 *                    the 31-bit field with x^3. Block M: mat 0 is the circulant
 *                    (2, 3, 1, 1) that Plonky3's Monty-31 external layer uses
 *                    for Poseidon2KoalaBear (MDSMat4); mat 1 is the paper's M4
 *                    (Plonky3's HLMDSMat4).
 *   Constants ...... Poseidon2KoalaBear::new_from_rng_128 on
 *                    rand::rngs::SmallRng::seed_from_u64(1), the width-16 set
 *                    drawn first and the width-24 set after it on the same
 *                    stream (src/bin/main.rs:100-102, benches/whir.rs:66-68).
 *                    SmallRng = xoshiro256++ (Blackman, Vigna 2021) with its
 *                    four state words from SplitMix64 (Steele, Lea, Flood
 *                    2014) of the seed; next_u32 = high half of next_u64.
 *                    KoalaBear sampling: v = next_u32 >> 1, rejected if
 *                    v >= p, and v is the Montgomery word (value v / 2^32).
 *                    Order (p3-poseidon2 new_from_rng): the 4 initial external
 *                    rows, the 4 terminal external rows, then the internal
 *                    constants. These are restated from the published
 *                    algorithms and Plonky3's documented behaviour; no output
 *                    of the reference pins them (parity unpinned).
 *                    The internal diagonal is fixed, not drawn: small integers
 *                    and signed powers of two, the form of p3-koala-bear's
 *                    internal layer (which takes only round constants).
 *   Sponges ........ PaddingFreeSponge (overwrite mode) and
 *                    TruncatedPermutation as used at src/bin/main.rs:35-36.
 *   Challenger ..... DuplexChallenger<F, P16, 16, 8> duplex sponge
 *                    (src/bin/main.rs:37): observe / sample / sample_bits /
 *                    grind / check_witness. grind returns the smallest valid
 *                    witness, the result of a sequential search.
 *   Merkle tree .... MerkleTreeMmcs with one matrix of power-of-two height:
 *                    leaf digest = sponge(row), node = compress(left, right).
 *   DFT ............ Radix2DFTSmallBatch::dft_batch semantics: natural-order
 *                    DFT over the subgroup of order `height` (not a coset).
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "or_field.h"

/* ------------------------------------------------------------------------ */
/* SmallRng and KoalaBear sampling                                           */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint64_t s[4];
} or_rng;

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static void or_rng_seed(or_rng* g, uint64_t seed) {
  for (int i = 0; i < 4; i++) {
    uint64_t z = (seed += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    g->s[i] = z ^ (z >> 31);
  }
}

static uint64_t or_rng_next(or_rng* g) {
  uint64_t* s = g->s;
  const uint64_t out = rotl64(s[0] + s[3], 23) + s[0];
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return out;
}

/* canonical value of the next KoalaBear element */
static uint32_t or_rng_field(or_rng* g) {
  const uint32_t r_inv = 0x3f010000u; /* 2^-32 mod p */
  for (;;) {
    const uint32_t v = (uint32_t)(or_rng_next(g) >> 32) >> 1;
    if (v < OR_P) return or_mul(v, r_inv);
  }
}

void or_rng_fields(uint64_t seed, uint32_t* out, size_t count) {
  or_rng g;
  or_rng_seed(&g, seed);
  for (size_t i = 0; i < count; i++) out[i] = or_rng_field(&g);
}

/* raw generator access for known-answer checks */
void or_rng_seed_state(uint64_t seed, uint64_t* state4) {
  or_rng g;
  or_rng_seed(&g, seed);
  memcpy(state4, g.s, sizeof(g.s));
}
void or_rng_u64_from_state(const uint64_t* state4, uint64_t* out, size_t count) {
  or_rng g;
  memcpy(g.s, state4, sizeof(g.s));
  for (size_t i = 0; i < count; i++) out[i] = or_rng_next(&g);
}

/* ------------------------------------------------------------------------ */
/* Poseidon2                                                                 */
/* ------------------------------------------------------------------------ */

static void p2_fill(or_p2_params* p, uint32_t width, uint32_t rp, uint32_t mat, or_rng* g) {
  memset(p, 0, sizeof(*p));
  p->width = width;
  p->rounds_f = 8;
  p->rounds_p = rp;
  p->mat = mat;
  for (uint32_t r = 0; r < 8; r++)
    for (uint32_t i = 0; i < width; i++) p->ext_rc[r * width + i] = or_rng_field(g);
  for (uint32_t r = 0; r < rp; r++) p->int_rc[r] = or_rng_field(g);
  /* internal diagonal: fixed, drawn from no RNG. Entries are small integers
   * and signed powers of two: width 16
   *   -2, 1, 2, 1/2, 3, 4, -1/2, -3, -4, 2^-8, 2^-3, 2^-24, -2^-8, -2^-3, -2^-4, -2^-24
   * width 24
   *   -2, 1, 2, 1/2, 3, 4, -1/2, -3, -4, 2^-8, 2^-2, 2^-3, 2^-4, 2^-5, 2^-6, 2^-24,
   *   -2^-8, -2^-3, -2^-4, -2^-5, -2^-6, -2^-7, -2^-9, -2^-24 */
  static const int small[9] = {-2, 1, 2, 0, 3, 4, 0, -3, -4}; /* 0 marks +-1/2 */
  static const int pow16[7] = {8, 3, 24, -8, -3, -4, -24};
  static const int pow24[15] = {8, 2, 3, 4, 5, 6, 24, -8, -3, -4, -5, -6, -7, -9, -24};
  const uint32_t half = (OR_P + 1) / 2;
  for (uint32_t i = 0; i < 9; i++) {
    if (small[i] > 0) p->diag[i] = (uint32_t)small[i];
    else if (small[i] < 0) p->diag[i] = OR_P - (uint32_t)(-small[i]);
    else p->diag[i] = i == 3 ? half : OR_P - half;
  }
  const int* pw = width == 16 ? pow16 : pow24;
  for (uint32_t i = 9; i < width; i++) {
    const int e = pw[i - 9] < 0 ? -pw[i - 9] : pw[i - 9];
    uint32_t v = 1;
    for (int j = 0; j < e; j++) v = or_mul(v, half);
    p->diag[i] = pw[i - 9] < 0 ? OR_P - v : v;
  }
}

void or_p2_from_rng(uint64_t seed, uint32_t mat, or_p2_params* p16, or_p2_params* p24) {
  or_rng g;
  or_rng_seed(&g, seed);
  or_p2_params t16, t24;
  p2_fill(&t16, 16, 20, mat, &g);
  p2_fill(&t24, 24, 23, mat, &g);
  if (p16) *p16 = t16;
  if (p24) *p24 = t24;
}

void or_p2_default(or_p2_params* p16, or_p2_params* p24) { or_p2_from_rng(1, 0, p16, p24); }

static void m4(uint32_t* x, uint32_t mat) {
  /* mat 0: circ(2, 3, 1, 1), row i = (2, 3, 1, 1) rotated right by i;
   * mat 1: [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] (eprint 2023/323, sec. 5.1) */
  static const uint64_t circ[4][4] = {{2, 3, 1, 1}, {1, 2, 3, 1}, {1, 1, 2, 3}, {3, 1, 1, 2}};
  static const uint64_t hl[4][4] = {{5, 7, 1, 3}, {4, 6, 1, 1}, {1, 3, 5, 7}, {1, 1, 4, 6}};
  const uint64_t(*m)[4] = mat == 1 ? hl : circ;
  uint64_t y[4];
  for (int i = 0; i < 4; i++) y[i] = (m[i][0] * x[0] + m[i][1] * x[1] + m[i][2] * x[2] + m[i][3] * x[3]) % OR_P;
  for (int i = 0; i < 4; i++) x[i] = (uint32_t)y[i];
}

static void ext_layer(uint32_t* x, uint32_t t, uint32_t mat) {
  for (uint32_t c = 0; c < t; c += 4) m4(x + c, mat);
  uint32_t s[4] = {0, 0, 0, 0};
  for (uint32_t c = 0; c < t; c += 4)
    for (int j = 0; j < 4; j++) s[j] = or_add(s[j], x[c + j]);
  for (uint32_t i = 0; i < t; i++) x[i] = or_add(x[i], s[i & 3]);
}

static inline uint32_t cube(uint32_t v) { return or_mul(or_mul(v, v), v); }

void or_p2_permute(const or_p2_params* prm, uint32_t* x) {
  const uint32_t t = prm->width, hf = prm->rounds_f / 2;
  ext_layer(x, t, prm->mat);
  for (uint32_t r = 0; r < hf; r++) {
    for (uint32_t i = 0; i < t; i++) x[i] = cube(or_add(x[i], prm->ext_rc[r * t + i]));
    ext_layer(x, t, prm->mat);
  }
  for (uint32_t r = 0; r < prm->rounds_p; r++) {
    x[0] = cube(or_add(x[0], prm->int_rc[r]));
    uint32_t s = 0;
    for (uint32_t i = 0; i < t; i++) s = or_add(s, x[i]);
    for (uint32_t i = 0; i < t; i++) x[i] = or_add(s, or_mul(prm->diag[i], x[i]));
  }
  for (uint32_t r = hf; r < prm->rounds_f; r++) {
    for (uint32_t i = 0; i < t; i++) x[i] = cube(or_add(x[i], prm->ext_rc[r * t + i]));
    ext_layer(x, t, prm->mat);
  }
}

/* PaddingFreeSponge<P, WIDTH, RATE, 8>::hash_iter: overwrite the rate part
 * with the next input chunk, permute after every (possibly partial) chunk. */
static void sponge(const or_p2_params* p, uint32_t rate, const uint32_t* in, size_t len,
                   uint32_t* out8) {
  uint32_t st[24];
  memset(st, 0, sizeof(st));
  size_t pos = 0;
  while (pos < len) {
    size_t take = len - pos < rate ? len - pos : rate;
    for (size_t i = 0; i < take; i++) st[i] = in[pos + i];
    pos += take;
    or_p2_permute(p, st);
  }
  memcpy(out8, st, 8 * sizeof(uint32_t));
}

/* TruncatedPermutation<P16, 2, 8, 16>: permute(left || right)[0..8] */
static void compress(const or_p2_params* p16, const uint32_t* l, const uint32_t* r, uint32_t* out) {
  uint32_t st[16];
  memcpy(st, l, 32);
  memcpy(st + 8, r, 32);
  or_p2_permute(p16, st);
  memcpy(out, st, 32);
}

/* ------------------------------------------------------------------------ */
/* Challenger                                                                */
/* ------------------------------------------------------------------------ */

void or_chal_init(or_chal* c) { memset(c, 0, sizeof(*c)); }

static void duplexing(or_chal* c, const or_p2_params* p16) {
  for (int i = 0; i < c->in_len; i++) c->state[i] = c->in[i];
  c->in_len = 0;
  or_p2_permute(p16, c->state);
  memcpy(c->out, c->state, 8 * sizeof(uint32_t));
  c->out_len = 8;
}

void or_chal_observe(or_chal* c, const or_p2_params* p16, uint32_t v) {
  c->out_len = 0;
  c->in[c->in_len++] = v;
  if (c->in_len == 8) duplexing(c, p16);
}

uint32_t or_chal_sample(or_chal* c, const or_p2_params* p16) {
  if (c->in_len > 0 || c->out_len == 0) duplexing(c, p16);
  return c->out[--c->out_len];
}

uint64_t or_chal_sample_bits(or_chal* c, const or_p2_params* p16, int bits) {
  uint32_t v = or_chal_sample(c, p16);
  return (uint64_t)v & ((1ull << bits) - 1);
}

int or_chal_check_witness(or_chal* c, const or_p2_params* p16, int bits, uint32_t w) {
  if (bits == 0) return 1;
  or_chal_observe(c, p16, w);
  return or_chal_sample_bits(c, p16, bits) == 0;
}

uint32_t or_chal_grind(or_chal* c, const or_p2_params* p16, int bits) {
  /* smallest witness w in [0, p) with check_witness(bits, w) */
  const uint32_t chunk = 1u << 16;
  uint32_t found = OR_P;
  for (uint32_t base = 0; base < OR_P && found == OR_P; base += chunk) {
    uint32_t end = base + chunk < OR_P ? base + chunk : OR_P;
    uint32_t best = OR_P;
#pragma omp parallel for schedule(static) reduction(min : best)
    for (uint32_t w = base; w < end; w++) {
      or_chal t = *c;
      if (or_chal_check_witness(&t, p16, bits, w) && w < best) best = w;
    }
    found = best;
  }
  or_chal_check_witness(c, p16, bits, found);
  return found;
}

/* ------------------------------------------------------------------------ */
/* Merkle tree (MerkleTreeMmcs, single power-of-two-height matrix)           */
/* ------------------------------------------------------------------------ */

void or_merkle_build(const or_p2_params* p16, const or_p2_params* p24, int leaf_hash,
                     const uint32_t* rows, int log_height, int row_words, uint32_t* digests,
                     uint32_t* root) {
  const size_t h = (size_t)1 << log_height;
  if (leaf_hash == 2) {
    /* Keccak MMCS (or_keccak.c) */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < h; i++) or_keccak_leaf(rows + i * row_words, row_words, digests + i * 8);
    uint32_t* prev = digests;
    size_t n = h;
    while (n > 1) {
      uint32_t* cur = prev + n * 8;
#pragma omp parallel for schedule(static)
      for (size_t j = 0; j < n / 2; j++) or_keccak_compress(prev + 2 * j * 8, prev + (2 * j + 1) * 8, cur + j * 8);
      prev = cur;
      n /= 2;
    }
    memcpy(root, prev, 32);
    return;
  }
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < h; i++) {
    if (leaf_hash == 0)
      sponge(p24, 16, rows + i * row_words, (size_t)row_words, digests + i * 8);
    else
      sponge(p16, 8, rows + i * row_words, (size_t)row_words, digests + i * 8);
  }
  uint32_t* prev = digests;
  size_t n = h;
  while (n > 1) {
    uint32_t* cur = prev + n * 8;
#pragma omp parallel for schedule(static)
    for (size_t j = 0; j < n / 2; j++) compress(p16, prev + 2 * j * 8, prev + (2 * j + 1) * 8, cur + j * 8);
    prev = cur;
    n /= 2;
  }
  memcpy(root, prev, 32);
}

/* ------------------------------------------------------------------------ */
/* DFT                                                                       */
/* ------------------------------------------------------------------------ */

/* in-place natural-order forward DFT of size 2^log_n over `lanes` interleaved
 * base-field words per element: a[i] <- sum_j a[j] * w^(i*j) */
static void ntt(uint32_t* a, int log_n, int lanes) {
  const size_t n = (size_t)1 << log_n;
  for (size_t i = 1, j = 0; i < n; i++) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j)
      for (int l = 0; l < lanes; l++) {
        uint32_t t = a[i * lanes + l];
        a[i * lanes + l] = a[j * lanes + l];
        a[j * lanes + l] = t;
      }
  }
  for (int s = 1; s <= log_n; s++) {
    const size_t m = (size_t)1 << s, half = m >> 1;
    const uint32_t wm = or_two_adic_generator(s);
    uint32_t* tw = (uint32_t*)malloc(half * sizeof(uint32_t));
    tw[0] = 1;
    for (size_t k = 1; k < half; k++) tw[k] = or_mul(tw[k - 1], wm);
    for (size_t b = 0; b < n; b += m)
      for (size_t k = 0; k < half; k++)
        for (int l = 0; l < lanes; l++) {
          uint32_t u = a[(b + k) * lanes + l];
          uint32_t v = or_mul(a[(b + k + half) * lanes + l], tw[k]);
          a[(b + k) * lanes + l] = or_add(u, v);
          a[(b + k + half) * lanes + l] = or_sub(u, v);
        }
    free(tw);
  }
}

/* transpose & pad & dft_batch (src/whir/committer/writer.rs:70-86,
 * src/whir/prover/mod.rs:166-180): the input is 2^log_width contiguous chunks
 * of 2^log_chunk elements (column j = chunk j), each zero-padded to
 * 2^(log_chunk+log_blowup) and transformed; the output is row-major with
 * 2^log_width elements per row. Elements are 1 (base) or 4 (ext) words. */
void or_dft_batch(const uint32_t* chunks, int log_chunk, int log_width, int log_blowup, int ext,
                  uint32_t* out) {
  const int lanes = ext ? 4 : 1;
  const size_t L = (size_t)1 << log_chunk, W = (size_t)1 << log_width;
  const int log_h = log_chunk + log_blowup;
  const size_t H = (size_t)1 << log_h;
#pragma omp parallel for schedule(dynamic)
  for (size_t j = 0; j < W; j++) {
    uint32_t* col = (uint32_t*)calloc(H * lanes, sizeof(uint32_t));
    memcpy(col, chunks + j * L * lanes, L * lanes * sizeof(uint32_t));
    ntt(col, log_h, lanes);
    for (size_t r = 0; r < H; r++)
      for (int l = 0; l < lanes; l++) out[(r * W + j) * lanes + l] = col[r * lanes + l];
    free(col);
  }
}

/* ------------------------------------------------------------------------ */
/* Polynomial routines (src/poly/evals.rs, src/poly/multilinear.rs)          */
/* ------------------------------------------------------------------------ */

static or_ef ld(const uint32_t* p) {
  or_ef r;
  memcpy(r.c, p, 16);
  return r;
}
static void st(uint32_t* p, or_ef v) { memcpy(p, v.c, 16); }

/* eq table: out[x] = scale * eq(point, x), x in {0,1}^n with point[0] <-> MSB
 * (EvaluationsList::new_from_point, evals.rs:312-320) */
void or_eq_table(const uint32_t* point, int n, const uint32_t* scale, uint32_t* out) {
  st(out, ld(scale));
  for (int i = 0; i < n; i++) {
    /* process coordinates from last to first: bit i of x <-> point[n-1-i] */
    or_ef z = ld(point + 4 * (n - 1 - i));
    size_t half = (size_t)1 << i;
    for (size_t x = 0; x < half; x++) {
      or_ef lo = ld(out + 4 * x);
      or_ef hi = or_ef_mul(lo, z);
      st(out + 4 * (x + half), hi);
      st(out + 4 * x, or_ef_sub(lo, hi));
    }
  }
}

/* repeated first-variable folding: f(z) = fold(...fold(f, z0)..., z_{n-1}) */
void or_eval_base(const uint32_t* evals, int n, const uint32_t* point, uint32_t* out) {
  size_t N = (size_t)1 << n;
  uint32_t* t = (uint32_t*)malloc(N * 16);
  for (size_t i = 0; i < N; i++) st(t + 4 * i, or_ef_from(evals[i]));
  for (int j = 0; j < n; j++) or_fold_ext(t, n - j, point + 4 * j);
  memcpy(out, t, 16);
  free(t);
}

void or_eval_ext(const uint32_t* evals, int n, const uint32_t* point, uint32_t* out) {
  size_t N = (size_t)1 << n;
  uint32_t* t = (uint32_t*)malloc(N * 16);
  memcpy(t, evals, N * 16);
  for (int j = 0; j < n; j++) or_fold_ext(t, n - j, point + 4 * j);
  memcpy(out, t, 16);
  free(t);
}

/* compress (evals.rs:127-148): a[i] += (a[i + N/2] - a[i]) * r, keep lower half */
void or_fold_ext(uint32_t* evals, int n, const uint32_t* r) {
  or_ef rr = ld(r);
  size_t mid = (size_t)1 << (n - 1);
#pragma omp parallel for schedule(static) if (mid > 4096)
  for (size_t i = 0; i < mid; i++) {
    or_ef a0 = ld(evals + 4 * i), a1 = ld(evals + 4 * (i + mid));
    st(evals + 4 * i, or_ef_add(a0, or_ef_mul(or_ef_sub(a1, a0), rr)));
  }
}

/* compress_ext (evals.rs:382-400): base evals folded into extension evals */
void or_fold_base(const uint32_t* evals, int n, const uint32_t* r, uint32_t* out) {
  or_ef rr = ld(r);
  size_t mid = (size_t)1 << (n - 1);
#pragma omp parallel for schedule(static) if (mid > 4096)
  for (size_t i = 0; i < mid; i++)
    st(out + 4 * i, or_ef_add(or_ef_from(evals[i]), or_ef_mul_base(rr, or_sub(evals[i + mid], evals[i]))));
}

/* compress_multi_into_packed (evals.rs:422-447): out[x] = sum_y eq(rs, y) f[y*2^(n-k) + x] */
void or_fold_multi_base(const uint32_t* evals, int n, const uint32_t* rs, int k, uint32_t* out) {
  size_t K = (size_t)1 << k, M = (size_t)1 << (n - k);
  uint32_t* eq = (uint32_t*)malloc(K * 16);
  uint32_t one[4] = {1, 0, 0, 0};
  or_eq_table(rs, k, one, eq);
#pragma omp parallel for schedule(static) if (M > 4096)
  for (size_t x = 0; x < M; x++) {
    or_ef acc = or_ef_zero();
    for (size_t y = 0; y < K; y++) acc = or_ef_add(acc, or_ef_mul_base(ld(eq + 4 * y), evals[y * M + x]));
    st(out + 4 * x, acc);
  }
  free(eq);
}

/* sumcheck_coefficients (evals.rs:493-526) on extension evals and weights */
void or_sumcheck_coeffs(const uint32_t* f, const uint32_t* w, int n, uint32_t* c0, uint32_t* c2) {
  size_t mid = (size_t)1 << (n - 1);
  or_ef a0 = or_ef_zero(), a2 = or_ef_zero();
  for (size_t i = 0; i < mid; i++) {
    or_ef el = ld(f + 4 * i), eh = ld(f + 4 * (i + mid));
    or_ef wl = ld(w + 4 * i), wh = ld(w + 4 * (i + mid));
    a0 = or_ef_add(a0, or_ef_mul(wl, el));
    a2 = or_ef_add(a2, or_ef_mul(or_ef_sub(or_ef_double(wh), wl), or_ef_sub(or_ef_double(eh), el)));
  }
  st(c0, a0);
  st(c2, a2);
}

/* SelectStatement::combine (select.rs:296-380): weights[x] += sum_j gamma_j * var_j^x */
void or_combine_select(uint32_t* weights, int n, const uint32_t* vars, int n_vars,
                       const uint32_t* gamma_pows) {
  size_t N = (size_t)1 << n;
  const size_t blk = 1024;
#pragma omp parallel for schedule(static)
  for (size_t b = 0; b < N; b += blk) {
    for (int j = 0; j < n_vars; j++) {
      uint32_t pw = or_pow(vars[j], b);
      or_ef g = ld(gamma_pows + 4 * j);
      for (size_t x = b; x < b + blk && x < N; x++) {
        st(weights + 4 * x, or_ef_add(ld(weights + 4 * x), or_ef_mul_base(g, pw)));
        pw = or_mul(pw, vars[j]);
      }
    }
  }
}

void or_free(void* p) { free(p); }
