// Merkle tree and proof-of-work kernels, templated on the Poseidon2 external
// block MAT (p2::kMatMds or p2::kMatHl). Each form is instantiated in its own
// translation unit (merkle_mds.cu, merkle_hl.cu); kernels.cu dispatches on the
// context's choice. The kernels have internal linkage in each unit; only the
// launchers at the end are shared.
#pragma once
#include "devutil.cuh"

namespace wk {
namespace {

using kb::ef;
using p2::P2Consts;

// ---------------------------------------------------------------------------
// Merkle tree (MerkleTreeMmcs::commit_matrix, src/whir/committer/writer.rs:89
// and src/whir/prover/mod.rs:182-184): one thread hashes one row with the
// PaddingFreeSponge (overwrite mode), then the CTA compresses its subtree
// level by level in shared memory with TruncatedPermutation<P16>.
// ---------------------------------------------------------------------------

constexpr int MERKLE_CTA = 128;

// TruncatedPermutation<P16, 2, 8, 16> on Montgomery-form digests: the
// permutation runs on canonical values, and only the kept half of the output
// is converted back.
template <int MAT>
__device__ __forceinline__ void compress_mont(uint32_t (&s)[16], const P2Consts& k) {
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = kb::from_mont(s[i]);
  p2::permute_canonical<16, p2::RP16, MAT>(s, k);
#pragma unroll
  for (int i = 0; i < 8; i++) s[i] = kb::to_mont(s[i]);
}

template <int MAT>
__device__ __forceinline__ void compress16(const uint32_t* l, const uint32_t* r, uint32_t* out,
                                           const P2Consts& k) {
  uint32_t s[16];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    s[i] = l[i];
    s[i + 8] = r[i];
  }
  compress_mont<MAT>(s, k);
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = s[i];
}

// Compress `levels` levels above the digests in sh[0 .. count*8), writing each
// level to global; `node0` is this CTA's first node index at the input level.
template <int MAT>
__device__ __forceinline__ void subtree_up(uint32_t* sh, int count, int levels, size_t node0, uint32_t* level_base,
                                           size_t level_size, const P2Consts& comp) {
  size_t off = 0;
  size_t lsz = level_size;
  for (int l = 1; l <= levels; l++) {
    const int act = count >> l;
    uint32_t d[8];
    const int t = threadIdx.x;
    if (t < act) compress16<MAT>(sh + 2 * t * 8, sh + (2 * t + 1) * 8, d, comp);
    __syncthreads();
    off += lsz;
    lsz >>= 1;
    if (t < act) {
      const size_t node = (node0 >> l) + t;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        sh[t * 8 + i] = d[i];
        level_base[(off + node) * 8 + i] = d[i];
      }
    }
    __syncthreads();
  }
}

template <int T, int RP, int RATE, int MAT>
__global__ void __launch_bounds__(MERKLE_CTA) k_merkle_leaves(const uint32_t* __restrict__ rows, int row_words,
                                                               size_t h, int levels, uint32_t* __restrict__ digests,
                                                               const __grid_constant__ P2Consts leaf,
                                                               const __grid_constant__ P2Consts comp) {
  __shared__ uint32_t sh[MERKLE_CTA * 8];
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < h) {
    uint32_t s[T];
#pragma unroll
    for (int k = 0; k < T; k++) s[k] = 0u;
    const uint32_t* row = rows + i * (size_t)row_words;
    for (int pos = 0; pos < row_words; pos += RATE) {
      const int take = row_words - pos < RATE ? row_words - pos : RATE;
      if (take == RATE && (row_words & 3) == 0) {
#pragma unroll
        for (int k = 0; k < RATE; k += 4) {
          uint4 v = __ldg(reinterpret_cast<const uint4*>(row + pos + k));
          s[k] = kb::from_mont(v.x);
          s[k + 1] = kb::from_mont(v.y);
          s[k + 2] = kb::from_mont(v.z);
          s[k + 3] = kb::from_mont(v.w);
        }
      } else {
#pragma unroll
        for (int k = 0; k < RATE; k++)
          if (k < take) s[k] = kb::from_mont(row[pos + k]);
      }
      const bool first = pos == 0, last = pos + RATE >= row_words;
      if (first && last) p2::permute_sponge<T, RP, RATE, true, true, MAT>(s, leaf);
      else if (first) p2::permute_sponge<T, RP, RATE, true, false, MAT>(s, leaf);
      else if (last) p2::permute_sponge<T, RP, RATE, false, true, MAT>(s, leaf);
      else p2::permute_sponge<T, RP, RATE, false, false, MAT>(s, leaf);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      s[k] = kb::to_mont(s[k]);
      sh[threadIdx.x * 8 + k] = s[k];
      digests[i * 8 + k] = s[k];
    }
  }
  __syncthreads();
  subtree_up<MAT>(sh, blockDim.x, levels, (size_t)blockIdx.x * blockDim.x, digests, h, comp);
}

static int ilog2i(size_t v) {
  int r = -1;
  while (v) {
    r++;
    v >>= 1;
  }
  return r;
}

// Leaf digests only (level 0): one thread per row, full occupancy, no barriers.
template <int T, int RP, int RATE, int CTA, int MAT>
__global__ void __launch_bounds__(CTA) k_leaf_digests(const uint32_t* __restrict__ rows, int row_words, size_t h,
                                                       uint32_t* __restrict__ digests,
                                                       const __grid_constant__ P2Consts leaf) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < h; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t s[T];
#pragma unroll
    for (int k = 0; k < T; k++) s[k] = 0u;
    const uint32_t* row = rows + i * (size_t)row_words;
    for (int pos = 0; pos < row_words; pos += RATE) {
      const int take = row_words - pos < RATE ? row_words - pos : RATE;
      if (take == RATE && (row_words & 3) == 0) {
#pragma unroll
        for (int k = 0; k < RATE; k += 4) {
          uint4 v = __ldg(reinterpret_cast<const uint4*>(row + pos + k));
          s[k] = kb::from_mont(v.x);
          s[k + 1] = kb::from_mont(v.y);
          s[k + 2] = kb::from_mont(v.z);
          s[k + 3] = kb::from_mont(v.w);
        }
      } else {
#pragma unroll
        for (int k = 0; k < RATE; k++)
          if (k < take) s[k] = kb::from_mont(row[pos + k]);
      }
      const bool first = pos == 0, last = pos + RATE >= row_words;
      if (first && last) p2::permute_sponge<T, RP, RATE, true, true, MAT>(s, leaf);
      else if (first) p2::permute_sponge<T, RP, RATE, true, false, MAT>(s, leaf);
      else if (last) p2::permute_sponge<T, RP, RATE, false, true, MAT>(s, leaf);
      else p2::permute_sponge<T, RP, RATE, false, false, MAT>(s, leaf);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) s[k] = kb::to_mont(s[k]);
    uint4* d = reinterpret_cast<uint4*>(digests + i * 8);
    d[0] = make_uint4(s[0], s[1], s[2], s[3]);
    d[1] = make_uint4(s[4], s[5], s[6], s[7]);
  }
}

// Two tree levels per launch: each thread compresses four nodes of level l
// into two nodes of level l+1 (written out) and their parent at level l+2.
// SEQ = false keeps both level-(l+1) permutations in flight together (two
// independent chains per thread, about 78 registers); SEQ = true runs them one
// after the other (one chain, fewer registers, more resident warps).
template <int CTA, bool SEQ, int MAT>
__global__ void __launch_bounds__(CTA) k_merkle_two_levels(uint32_t* __restrict__ digests, size_t in_off,
                                                            size_t in_count, const __grid_constant__ P2Consts comp) {
  const size_t out_count = in_count >> 2;
  const size_t mid_off = in_off + in_count, top_off = mid_off + (in_count >> 1);
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < out_count; j += (size_t)gridDim.x * blockDim.x) {
    const uint4* src = reinterpret_cast<const uint4*>(digests + (in_off + 4 * j) * 8);
    uint4* mid = reinterpret_cast<uint4*>(digests + (mid_off + 2 * j) * 8);
    uint32_t c[16];  // the parent's inputs, canonical
    if (SEQ) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        uint32_t a[16];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const uint4 v = src[4 * h + q];
          a[4 * q] = kb::from_mont(v.x);
          a[4 * q + 1] = kb::from_mont(v.y);
          a[4 * q + 2] = kb::from_mont(v.z);
          a[4 * q + 3] = kb::from_mont(v.w);
        }
        p2::permute_canonical<16, p2::RP16, MAT>(a, comp);
#pragma unroll
        for (int k = 0; k < 8; k++) c[8 * h + k] = a[k];
        mid[2 * h] = make_uint4(kb::to_mont(a[0]), kb::to_mont(a[1]), kb::to_mont(a[2]), kb::to_mont(a[3]));
        mid[2 * h + 1] = make_uint4(kb::to_mont(a[4]), kb::to_mont(a[5]), kb::to_mont(a[6]), kb::to_mont(a[7]));
      }
    } else {
      uint32_t a[16], b[16];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint4 va = src[q], vb = src[4 + q];
        a[4 * q] = va.x; a[4 * q + 1] = va.y; a[4 * q + 2] = va.z; a[4 * q + 3] = va.w;
        b[4 * q] = vb.x; b[4 * q + 1] = vb.y; b[4 * q + 2] = vb.z; b[4 * q + 3] = vb.w;
      }
#pragma unroll
      for (int k = 0; k < 16; k++) {
        a[k] = kb::from_mont(a[k]);
        b[k] = kb::from_mont(b[k]);
      }
      p2::permute_canonical<16, p2::RP16, MAT>(a, comp);
      p2::permute_canonical<16, p2::RP16, MAT>(b, comp);
      uint32_t am[8], bm[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        c[k] = a[k];
        c[8 + k] = b[k];
        am[k] = kb::to_mont(a[k]);
        bm[k] = kb::to_mont(b[k]);
      }
      mid[0] = make_uint4(am[0], am[1], am[2], am[3]);
      mid[1] = make_uint4(am[4], am[5], am[6], am[7]);
      mid[2] = make_uint4(bm[0], bm[1], bm[2], bm[3]);
      mid[3] = make_uint4(bm[4], bm[5], bm[6], bm[7]);
    }
    p2::permute_canonical<16, p2::RP16, MAT>(c, comp);
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] = kb::to_mont(c[k]);
    uint4* top = reinterpret_cast<uint4*>(digests + (top_off + j) * 8);
    top[0] = make_uint4(c[0], c[1], c[2], c[3]);
    top[1] = make_uint4(c[4], c[5], c[6], c[7]);
  }
}

// Width-16 Poseidon2 spread over four consecutive lanes (q = lane & 3 holds
// state words 4q .. 4q+3). The M4 blocks are lane-local; the cross-chunk sums
// of the external layer and the full sum of the internal layer take two
// xor-shuffle steps. For the narrow top levels of a tree, where one
// permutation's latency sets the time (measured on B200: 6.5 thousand cycles
// for the canonical-value form of this layout against 12 thousand for a
// one-thread permutation). All 32 lanes of the warp must call it together.
template <int MAT>
__device__ __forceinline__ void coop_ext_layer(uint32_t (&x)[4]) {
  using namespace kb;
  p2::m4<MAT>(x[0], x[1], x[2], x[3]);
  uint32_t s[4] = {x[0], x[1], x[2], x[3]};
#pragma unroll
  for (int m = 1; m <= 2; m <<= 1)
#pragma unroll
    for (int j = 0; j < 4; j++) s[j] = add(s[j], __shfl_xor_sync(0xffffffffu, s[j], m));
#pragma unroll
  for (int j = 0; j < 4; j++) x[j] = add(x[j], s[j]);
}

// The permutation runs on Montgomery words (x * 2^32 mod p) in and out, the
// form the digests are stored in. Every linear step is the same on Montgomery words, the
// round constants come in Montgomery form, and the S-box is two Montgomery
// products (x^3 in Montgomery form): an integer-only dependent chain with no
// conversion at either end. The internal rounds also take the cross-lane sum
// off the dependent chain: with p_j = mu_j x_j the words after a round are
// s + p_j, so the next round's sum of words 1..15 is 15 s + sum_{j>=1} p_j,
// and that sum of products (two shuffles) runs beside the S-box; a round's
// chain is S-box, one addition and the product by 15. ROLLED keeps the round
// loops rolled: a kernel that permutes once or twice (the challenger steps)
// would otherwise spend its time fetching the unrolled code. FROM_SBOX: x
// already holds the first S-box inputs (the initial external layer and the
// first round constants applied, as the proof-of-work search folds them).
__device__ __forceinline__ uint32_t cube_m(uint32_t a) { return kb::mul(kb::mul(a, a), a); }
template <int MAT, bool ROLLED = false, bool FROM_SBOX = false>
__device__ __forceinline__ void coop_permute16_m(uint32_t (&x)[4], int q, const P2Consts& k) {
  using namespace kb;
  static_assert(!(ROLLED && FROM_SBOX), "the search form is unrolled");
  constexpr uint32_t k15s = (uint32_t)((15ull << 32) / P);  // Shoup constant of 15
  if (!FROM_SBOX) coop_ext_layer<MAT>(x);
#pragma unroll(ROLLED ? 1 : p2::RF / 2)
  for (int r = 0; r < p2::RF / 2; r++) {
#pragma unroll
    for (int j = 0; j < 4; j++)
      x[j] = cube_m(FROM_SBOX && r == 0 ? x[j] : add(x[j], k.ext_rc_m[r * 16 + 4 * q + j]));
    coop_ext_layer<MAT>(x);
  }
  // word 0 lives in w0 on every lane; lane 0's x[0] is not read again until
  // the internal rounds end
  uint32_t w0 = __shfl_sync(0xffffffffu, x[0], (threadIdx.x & 31) & ~3);
  uint32_t o = add(add(q == 0 ? 0u : x[0], x[1]), add(x[2], x[3]));  // sum of words 1..15
  o = add(o, __shfl_xor_sync(0xffffffffu, o, 1));
  o = add(o, __shfl_xor_sync(0xffffffffu, o, 2));
#pragma unroll(ROLLED ? 1 : p2::RP16)
  for (int r = 0; r < p2::RP16; r++) {
    uint32_t pj[4];
#pragma unroll
    for (int j = 0; j < 4; j++) pj[j] = mul_shoup(x[j], k.diag_c[4 * q + j], k.diag_s[4 * q + j]);
    uint32_t d = add(add(q == 0 ? 0u : pj[0], pj[1]), add(pj[2], pj[3]));  // sum of p_j, j >= 1
    d = add(d, __shfl_xor_sync(0xffffffffu, d, 1));
    d = add(d, __shfl_xor_sync(0xffffffffu, d, 2));
    const uint32_t y0 = cube_m(add(w0, k.int_rc_m[r]));
    const uint32_t s = add(o, y0);
#pragma unroll
    for (int j = 0; j < 4; j++) x[j] = add(s, pj[j]);
    w0 = p2::diag_axpy(p2::diag_code(16, 0), s, y0);
    o = add(mul_shoup(s, 15u, k15s), d);
  }
  if (q == 0) x[0] = w0;
#pragma unroll(ROLLED ? 1 : p2::RF / 2)
  for (int r = p2::RF / 2; r < p2::RF; r++) {
#pragma unroll
    for (int j = 0; j < 4; j++) x[j] = cube_m(add(x[j], k.ext_rc_m[r * 16 + 4 * q + j]));
    coop_ext_layer<MAT>(x);
  }
}

// Compresses `levels` levels above the `cnt` nodes in sh (8 words each), one
// four-lane group per node pair, writing every new level to global; `base` is
// the first node's index in its level, `off` and `lsz` the level's offset and
// size in `digests` (advanced past the levels done).
template <int MAT>
__device__ __forceinline__ void coop_levels(uint32_t* sh, int cnt, int levels, size_t base, size_t& off, size_t& lsz,
                                            uint32_t* __restrict__ digests, const P2Consts& comp) {
  const int t = threadIdx.x, g = t >> 2, q = t & 3;
  int cur = cnt;
  for (int l = 1; l <= levels; l++) {
    const int act = cur >> 1;
    const bool on = g < act;
    const int src = on ? 16 * g + 4 * q : 0;
    uint32_t x[4];
#pragma unroll
    for (int j = 0; j < 4; j++) x[j] = sh[src + j];
    // a warp holds groups 8w .. 8w+7: warps with none of this level's pairs
    // skip the permutation (warp-uniform, so its shuffles stay full-warp),
    // which leaves the upper levels latency-bound rather than issue-bound
    if ((t >> 5) * 8 < act) coop_permute16_m<MAT>(x, q, comp);
    __syncthreads();
    off += lsz;
    lsz >>= 1;
    if (on && q < 2) {
      const size_t node = (base >> l) + g;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        sh[8 * g + 4 * q + j] = x[j];
        digests[(off + node) * 8 + 4 * q + j] = x[j];
      }
    }
    __syncthreads();
    cur = act;
  }
}

// Two tree levels with four-lane cooperative permutations: one group of four
// lanes per output node (its two children, then the node), for the last,
// narrow two-level step of a tree, where one thread per node leaves the
// launch latency-bound (two dependent single-thread permutations). Lane q
// holds words 4q .. 4q+3 of a state; a child's digest ends on lanes 0 and 1.
// The loop runs per warp so all 32 lanes take every shuffle together.
template <int CTA, int MAT>
__global__ void __launch_bounds__(CTA) k_merkle_two_levels_coop(uint32_t* __restrict__ digests, size_t in_off,
                                                                 size_t in_count, const __grid_constant__ P2Consts comp) {
  const size_t out_count = in_count >> 2;
  const size_t mid_off = in_off + in_count, top_off = mid_off + (in_count >> 1);
  const int lane = threadIdx.x & 31, q = lane & 3;
  const size_t groups = (size_t)gridDim.x * (CTA / 4);
  for (size_t base = (size_t)blockIdx.x * (CTA / 4) + (threadIdx.x >> 5) * 8; base < out_count; base += groups) {
    const size_t jw = base + (lane >> 2);
    const bool on = jw < out_count;
    const size_t j = on ? jw : base;
    uint32_t keep[4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      // children 4j + 2h and 4j + 2h + 1: 16 consecutive words
      const uint4 v = *reinterpret_cast<const uint4*>(digests + (in_off + 4 * j + 2 * h) * 8 + 4 * q);
      uint32_t x[4] = {v.x, v.y, v.z, v.w};
      coop_permute16_m<MAT>(x, q, comp);
      if (on && q < 2)
        *reinterpret_cast<uint4*>(digests + (mid_off + 2 * j + h) * 8 + 4 * q) = make_uint4(x[0], x[1], x[2], x[3]);
      // the parent's state: the first child's digest on lanes 0-1, the
      // second's moved to lanes 2-3
      if (h == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) keep[k] = x[k];
      } else {
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint32_t from_b = __shfl_sync(0xffffffffu, x[k], (lane & ~3) | (q & 1));
          if (q >= 2) keep[k] = from_b;
        }
      }
    }
    coop_permute16_m<MAT>(keep, q, comp);
    if (on && q < 2)
      *reinterpret_cast<uint4*>(digests + (top_off + j) * 8 + 4 * q) = make_uint4(keep[0], keep[1], keep[2], keep[3]);
  }
}

// Top of a tree: each CTA compresses up to 256 nodes of one level into a
// subtree, one four-lane group per node pair, level by level in shared memory.
// With several CTAs (at most 256), the last one to finish (atomic counter, no
// waiting) loads their subtree roots and compresses them to the root in the
// same launch. With `mail` set, the root is posted to that mailbox.
constexpr int TOP_CTA = 512;
constexpr int TOP_NODES = 256;
template <int MAT>
__global__ void __launch_bounds__(TOP_CTA) k_merkle_top_coop(uint32_t* __restrict__ digests, size_t in_off,
                                                              size_t in_count, int levels,
                                                              const __grid_constant__ P2Consts comp,
                                                              unsigned* __restrict__ counter, uint32_t* mail,
                                                              uint32_t seq) {
  __shared__ uint32_t sh[TOP_NODES * 8];
  __shared__ bool s_last;
  const int t = threadIdx.x;
  const size_t base = (size_t)blockIdx.x * TOP_NODES;
  const int cnt = (int)min((size_t)TOP_NODES, in_count - base);
  for (int k = t; k < cnt * 8; k += blockDim.x) sh[k] = digests[(in_off + base) * 8 + k];
  __syncthreads();
  size_t off = in_off, lsz = in_count;
  coop_levels<MAT>(sh, cnt, levels, base, off, lsz, digests, comp);
  if (gridDim.x > 1) {
    if (t == 0) {
      __threadfence();
      s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int n = (int)gridDim.x;  // subtree roots, level `off`
    for (int k = t; k < n * 8; k += blockDim.x) sh[k] = __ldcg(digests + off * 8 + k);
    __syncthreads();
    int top = 0;
    while ((1 << top) < n) top++;
    coop_levels<MAT>(sh, n, top, 0, off, lsz, digests, comp);
    if (t == 0) *counter = 0u;
  }
  if (t == 0 && mail) mail_post(mail, sh, 8, seq);
}

// Top of a tree in one CTA: a level of at most 2 * TOP1_CTA nodes is
// compressed to the root, one thread (one whole permutation) per node pair,
// each new level kept in shared memory for the next and written out.
constexpr int TOP1_CTA = 1024;
template <int MAT>
__global__ void __launch_bounds__(TOP1_CTA) k_merkle_top_cta(uint32_t* __restrict__ digests, size_t in_off,
                                                              int in_count, const __grid_constant__ P2Consts comp,
                                                              uint32_t* mail, uint32_t seq) {
  __shared__ uint4 sh[2 * TOP1_CTA];  // node i at sh[2i], sh[2i + 1]
  const int t = threadIdx.x;
  size_t off = in_off;
  int cnt = in_count;
  for (int level = 0; cnt > 1; level++) {
    const int act = cnt >> 1;
    uint32_t x[16];
    if (t < act) {
      const uint4* src = level == 0 ? reinterpret_cast<const uint4*>(digests + (off + 2 * (size_t)t) * 8) : sh + 4 * t;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint4 v = src[q];
        x[4 * q] = v.x;
        x[4 * q + 1] = v.y;
        x[4 * q + 2] = v.z;
        x[4 * q + 3] = v.w;
      }
      compress_mont<MAT>(x, comp);
    }
    __syncthreads();
    off += cnt;
    if (t < act) {
      const uint4 a = make_uint4(x[0], x[1], x[2], x[3]), b = make_uint4(x[4], x[5], x[6], x[7]);
      sh[2 * t] = a;
      sh[2 * t + 1] = b;
      uint4* dst = reinterpret_cast<uint4*>(digests + (off + t) * 8);
      dst[0] = a;
      dst[1] = b;
    }
    __syncthreads();
    cnt = act;
  }
  if (threadIdx.x == 0 && mail) mail_post(mail, reinterpret_cast<const uint32_t*>(sh), 8, seq);
}

// Trees with at least kLevelPairMin leaves are built as: leaf digests, then
// two levels per launch while a level is wider than the top kernel takes, then
// the top: either cooperative-permutation subtrees (k_merkle_top_coop, node
// shape variant 0, from 2^15 nodes) or one CTA (k_merkle_top_cta, variant 1,
// from 2^11 nodes). Smaller trees hash their leaves with in-CTA subtrees and
// use the same top kernels above those.
constexpr size_t kLevelPairMin = (size_t)kMerkleLevelPairMin;
constexpr size_t kCoopTop = (size_t)1 << 15;
constexpr size_t kCtaTop = (size_t)2 * TOP1_CTA;

template <int T, int RP, int RATE, int MAT>
void launch_leaf_digests(const uint32_t* rows, int row_words, size_t h, uint32_t* digests,
                                const P2Consts& k, Shape sh, cudaStream_t st) {
  const unsigned blocks = grid_shape(h, sh);
  if (sh.threads == 128)
    k_leaf_digests<T, RP, RATE, 128, MAT><<<blocks, 128, 0, st>>>(rows, row_words, h, digests, k);
  else if (sh.threads == 512)
    k_leaf_digests<T, RP, RATE, 512, MAT><<<blocks, 512, 0, st>>>(rows, row_words, h, digests, k);
  else
    k_leaf_digests<T, RP, RATE, 256, MAT><<<blocks, 256, 0, st>>>(rows, row_words, h, digests, k);
}

}  // namespace

template <int MAT>
cudaError_t merkle_leaves_m(const uint32_t* rows, int log_h, int row_words, int leaf_hash, uint32_t* digests,
                            const P2Consts& p16, const P2Consts& p24, Shape leaf, cudaStream_t st) {
  const size_t h = (size_t)1 << log_h;
  if (h >= kLevelPairMin) {
    if ((leaf.threads != 128 && leaf.threads != 256 && leaf.threads != 512) || leaf.per_sm < 0)
      return cudaErrorInvalidValue;
    if (leaf_hash == 0)
      launch_leaf_digests<24, p2::RP24, 16, MAT>(rows, row_words, h, digests, p24, leaf, st);
    else
      launch_leaf_digests<16, p2::RP16, 8, MAT>(rows, row_words, h, digests, p16, leaf, st);
    LAUNCH_DONE();
  }
  const int cta = (int)(h < (size_t)MERKLE_CTA ? h : (size_t)MERKLE_CTA);
  const int lv = ilog2i((size_t)cta);
  const unsigned blocks = (unsigned)(h / cta);
  if (leaf_hash == 0)
    k_merkle_leaves<24, p2::RP24, 16, MAT><<<blocks, cta, 0, st>>>(rows, row_words, h, lv, digests, p24, p16);
  else
    k_merkle_leaves<16, p2::RP16, 8, MAT><<<blocks, cta, 0, st>>>(rows, row_words, h, lv, digests, p16, p16);
  LAUNCH_DONE();
}

template <int MAT>
cudaError_t merkle_upper_m(int log_h, uint32_t* digests, const P2Consts& p16, Shape node, unsigned* counter,
                           uint32_t* mail, uint32_t seq, int* posted, cudaStream_t st) {
  if (posted) *posted = 0;
  const size_t h = (size_t)1 << log_h;
  size_t off = 0, cnt = h;
  // variant bit 0: the top kernel (0 cooperative subtrees, 1 one CTA); bit 1:
  // the two-level kernel with its two permutations one after the other; bit 2:
  // the last two-level step with four-lane cooperative permutations
  if (node.variant < 0 || node.variant > 7) return cudaErrorInvalidValue;
  const bool top_cta = (node.variant & 1) != 0, one_chain = (node.variant & 2) != 0, coop_tail = (node.variant & 4) != 0;
  const size_t top = top_cta ? kCtaTop : kCoopTop;
  if (h >= kLevelPairMin) {
    if ((node.threads != 128 && node.threads != 256) || node.per_sm < 0) return cudaErrorInvalidValue;
    while (cnt > top) {
      const size_t out = cnt >> 2;
      const unsigned blocks = grid_shape(out, node);
      if (coop_tail && (cnt >> 2) <= top) {
        const unsigned cblocks = grid_shape(out * 4, node);
        if (node.threads == 128)
          k_merkle_two_levels_coop<128, MAT><<<cblocks, 128, 0, st>>>(digests, off, cnt, p16);
        else
          k_merkle_two_levels_coop<256, MAT><<<cblocks, 256, 0, st>>>(digests, off, cnt, p16);
      } else if (node.threads == 128 && one_chain)
        k_merkle_two_levels<128, true, MAT><<<blocks, 128, 0, st>>>(digests, off, cnt, p16);
      else if (node.threads == 128)
        k_merkle_two_levels<128, false, MAT><<<blocks, 128, 0, st>>>(digests, off, cnt, p16);
      else if (one_chain)
        k_merkle_two_levels<256, true, MAT><<<blocks, 256, 0, st>>>(digests, off, cnt, p16);
      else
        k_merkle_two_levels<256, false, MAT><<<blocks, 256, 0, st>>>(digests, off, cnt, p16);
      count_launch();
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      off += cnt + (cnt >> 1);
      cnt >>= 2;
    }
  } else {
    const int cta = (int)(h < (size_t)MERKLE_CTA ? h : (size_t)MERKLE_CTA);
    const int lv = ilog2i((size_t)cta);
    for (int l = 0; l < lv; l++) {
      off += cnt;
      cnt >>= 1;
    }
  }
  if (cnt <= 1) return cudaSuccess;
  if (top_cta) {
    k_merkle_top_cta<MAT><<<1, TOP1_CTA, 0, st>>>(digests, off, (int)cnt, p16, mail, seq);
  } else {
    // one launch: subtrees of 256 nodes, then the last CTA joins their roots
    const int c2 = (int)(cnt < (size_t)TOP_NODES ? cnt : (size_t)TOP_NODES);
    const unsigned blocks2 = (unsigned)(cnt / c2);
    if (blocks2 > (unsigned)TOP_NODES || (blocks2 > 1 && !counter)) return cudaErrorInvalidValue;
    k_merkle_top_coop<MAT><<<blocks2, TOP_CTA, 0, st>>>(digests, off, cnt, ilog2i((size_t)c2), p16, counter, mail, seq);
  }
  count_launch();
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && posted && mail) *posted = 1;
  return e;
}

// ---------------------------------------------------------------------------
// Duplex challenger steps on the device (DuplexChallenger observe / sample /
// sample_bits, the transcript calls of SumcheckData::observe_and_sample,
// src/whir/proof.rs:163-193). One warp runs them: lane 0 keeps the input and
// output buffers in shared memory, and a duplexing permutes the sponge state
// with the four-lane permutation (every four-lane group computes it; group
// 0's result is kept). The state is Montgomery words, as the host's. The
// steps run in the tails of the kernels whose results they observe (the last
// CTA of a sumcheck round, the last CTA of a proof-of-work search), so a
// sumcheck stage needs no launch of its own for its transcript.
// ---------------------------------------------------------------------------

namespace {

template <int MAT>
__device__ void dc_duplex(DevChal& c, const P2Consts& k) {
  const int lane = threadIdx.x & 31, q = lane & 3;
  __syncwarp();
  if (lane == 0) {
    for (int i = 0; i < c.in_len; i++) c.st[i] = c.in[i];
    c.in_len = 0;
  }
  __syncwarp();
  uint32_t x[4];
#pragma unroll
  for (int j = 0; j < 4; j++) x[j] = c.st[4 * q + j];
  __syncwarp();
  coop_permute16_m<MAT, true>(x, q, k);
  if (lane < 4) {
#pragma unroll
    for (int j = 0; j < 4; j++) c.st[4 * lane + j] = x[j];
  }
  __syncwarp();
  if (lane == 0) {
    for (int i = 0; i < 8; i++) c.out[i] = c.st[i];
    c.out_len = 8;
  }
  __syncwarp();
}

template <int MAT>
__device__ void dc_observe(DevChal& c, uint32_t v, const P2Consts& k) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0) {
    c.out_len = 0;
    c.in[c.in_len++] = v;
  }
  __syncwarp();
  if (c.in_len == 8) dc_duplex<MAT>(c, k);
}

template <int MAT>
__device__ uint32_t dc_sample(DevChal& c, const P2Consts& k) {
  __syncwarp();
  if (c.in_len > 0 || c.out_len == 0) dc_duplex<MAT>(c, k);
  const uint32_t v = c.out[c.out_len - 1];
  __syncwarp();
  if ((threadIdx.x & 31) == 0) c.out_len--;
  __syncwarp();
  return v;
}

__device__ void dc_load(DevChal& c, const DevChal* g) {
  const uint32_t* src = reinterpret_cast<const uint32_t*>(g);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&c);
  for (int i = threadIdx.x & 31; i < (int)(sizeof(DevChal) / 4); i += 32) dst[i] = __ldcg(src + i);
  __syncwarp();
}
__device__ void dc_store(const DevChal& c, DevChal* g) {
  __syncwarp();
  const uint32_t* src = reinterpret_cast<const uint32_t*>(&c);
  uint32_t* dst = reinterpret_cast<uint32_t*>(g);
  for (int i = threadIdx.x & 31; i < (int)(sizeof(DevChal) / 4); i += 32) dst[i] = src[i];
}

// Observe a round's coefficients c0, c2 (8 words, word i in lane i of cw);
// then, with grind_next, write the folded initial state of the next
// proof-of-work search (16 canonical words) to cp_out, else sample the
// round's challenge into r_out.
template <int MAT>
__device__ void dc_coeffs_step(DevChal& c, uint32_t cw, int grind_next, uint32_t* cp_out, ef* r_out,
                               const P2Consts& k) {
  for (int i = 0; i < 8; i++) dc_observe<MAT>(c, __shfl_sync(0xffffffffu, cw, i), k);
  if (grind_next) {
    // the sponge state with the pending inputs and 0 at the witness position,
    // canonical, through the initial external layer plus the first constants
    if ((threadIdx.x & 31) == 0) {
      uint32_t s[16];
      for (int i = 0; i < 16; i++) s[i] = kb::from_mont(c.st[i]);
      for (int i = 0; i < c.in_len; i++) s[i] = kb::from_mont(c.in[i]);
      s[c.in_len] = 0u;
      p2::grind_fold<MAT>(s, k);
      for (int i = 0; i < 16; i++) cp_out[i] = s[i];
    }
  } else {
    ef r;
    for (int i = 0; i < 4; i++) r.c[i] = dc_sample<MAT>(c, k);
    if ((threadIdx.x & 31) == 0) *r_out = r;
  }
}

// Observe the witness w (canonical; p means none was found), check that
// sample_bits(bits) is 0, then sample the round's challenge into r_out. A
// failed check sets bit 0 (no witness) or bit 1 (check failed) of *err;
// returns false, leaving the transcript as it is, when there is no witness.
template <int MAT>
__device__ bool dc_witness_step(DevChal& c, uint32_t w, int bits, ef* r_out, uint32_t* err, const P2Consts& k) {
  if (w >= kb::P) {
    if ((threadIdx.x & 31) == 0) atomicOr(err, 1u);
    return false;
  }
  dc_observe<MAT>(c, kb::to_mont(w), k);
  const uint32_t v = kb::from_mont(dc_sample<MAT>(c, k));
  if ((v & ((1u << bits) - 1u)) != 0u && (threadIdx.x & 31) == 0) atomicOr(err, 2u);
  ef r;
  for (int i = 0; i < 4; i++) r.c[i] = dc_sample<MAT>(c, k);
  if ((threadIdx.x & 31) == 0) *r_out = r;
  return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// Proof of work (GrindingChallenger::grind on DuplexChallenger, called at
// src/whir/proof.rs:188 and src/whir/prover/mod.rs:224,363). Candidates are
// claimed in increasing chunks; a CTA stops once every remaining chunk starts
// above the best witness found, so the result is the smallest valid witness.
// The loop is bounded by `limit` candidates.
// ---------------------------------------------------------------------------

namespace {
constexpr int GRIND_CTA = 128;  // one warp per SM sub-partition

// Each claim is CLAIM consecutive candidates: one per thread (COOP false), or
// one per four-lane group (COOP true: the four-lane Montgomery permutation,
// whose latency is about 40 % of a one-thread permutation's, for searches
// small enough that one pass's latency sets their time). CTA b's first claim
// is chunk b, later claims come from the counter (chunks gridDim.x,
// gridDim.x + 1, ...). With `ch` set (and res_out), the last CTA's first warp
// also runs the transcript step that follows the search on the device
// challenger (dc_witness_step).
template <int SLOT, int MAT, bool COOP>
__global__ void __launch_bounds__(GRIND_CTA, 10) k_grind(const __grid_constant__ P2Consts p16, uint4 st0, uint4 st1,
                                                      uint4 st2, uint4 st3, int bits, uint64_t limit,
                                                      uint32_t* result, uint32_t* counter, uint32_t* done,
                                                      uint32_t* mail, uint32_t seq, const uint32_t* cp_dev,
                                                      uint32_t* res_out, DevChal* ch, ef* r_out, uint32_t* err) {
  constexpr int CLAIM = COOP ? GRIND_CTA / 4 : GRIND_CTA;
  __shared__ uint64_t s_start;
  __shared__ int s_go;
  __shared__ bool s_last;
  __shared__ uint32_t s_w;
  __shared__ DevChal c;
  const uint32_t mask = (1u << bits) - 1u;
  uint32_t cp[16] = {st0.x, st0.y, st0.z, st0.w, st1.x, st1.y, st1.z, st1.w,
                     st2.x, st2.y, st2.z, st2.w, st3.x, st3.y, st3.z, st3.w};
  if (cp_dev) {
#pragma unroll
    for (int i = 0; i < 16; i++) cp[i] = __ldcg(cp_dev + i);
  }
  // the four-lane form: lane q's words 4q .. 4q+3 of the folded state and of
  // the witness column, in Montgomery form
  uint32_t cpm[4] = {0u, 0u, 0u, 0u}, colm[4] = {0u, 0u, 0u, 0u};
  const int q = threadIdx.x & 3;
  if constexpr (COOP) {
#pragma unroll
    for (int j = 0; j < 4; j++) {
      // word 4q + j of cp, selected without indexing the array by a lane value
      const uint32_t v = q == 0 ? cp[j] : q == 1 ? cp[4 + j] : q == 2 ? cp[8 + j] : cp[12 + j];
      cpm[j] = kb::to_mont(v);
      colm[j] = kb::to_mont((uint32_t)p2::ext_col16<MAT>(SLOT, 4 * q + j));
    }
  }
  for (bool first = true;; first = false) {
    if (threadIdx.x == 0) {
      const uint64_t chunk = first ? (uint64_t)blockIdx.x : (uint64_t)gridDim.x + atomicAdd(counter, 1u);
      const uint64_t start = chunk * CLAIM;
      s_start = start;
      s_go = start < limit && start < (uint64_t)*(volatile uint32_t*)result;
    }
    __syncthreads();
    const uint64_t start = s_start;
    const int go = s_go;
    __syncthreads();
    if (!go) {
      // every atomicMin of this CTA precedes the barriers above; the last CTA
      // to stop holds the final result, posts it to the mailbox with the
      // number of candidates evaluated (the counter's claims times the claim
      // size: every CTA evaluated its first claim and made exactly one claim
      // that it did not evaluate) and resets the search state for the next
      // search (every other CTA has finished with it), which then needs no
      // initialising launch
      if (threadIdx.x == 0) {
        s_last = false;
        if (mail || res_out) {
          __threadfence();
          if (atomicAdd(done, 1u) == gridDim.x - 1) {
            const uint32_t post[2] = {atomicAdd(result, 0u), atomicAdd(counter, 0u) * (uint32_t)CLAIM};
            if (mail) mail_post(mail, post, 2, seq);
            if (res_out) {
              res_out[0] = post[0];
              res_out[1] = post[1];
            }
            *result = kb::P;
            *counter = 0u;
            *done = 0u;
            s_w = post[0];
            s_last = true;
          }
        }
      }
      if (!ch) return;
      __syncthreads();
      if (!s_last || threadIdx.x >= 32) return;
      dc_load(c, ch);
      if (dc_witness_step<MAT>(c, s_w, bits, r_out, err, p16)) dc_store(c, ch);
      return;
    }
    if constexpr (COOP) {
      // every lane runs the permutation (its shuffles take the whole warp);
      // word 7 of the output is lane 1's last word
      const uint64_t w = start + (threadIdx.x >> 2);
      const uint32_t wm = kb::to_mont(w < limit ? (uint32_t)w : 0u);
      uint32_t x[4];
#pragma unroll
      for (int j = 0; j < 4; j++) x[j] = kb::add(cpm[j], kb::mul(wm, colm[j]));
      coop_permute16_m<MAT, false, true>(x, q, p16);
      if (q == 1 && w < limit && (kb::from_mont(x[3]) & mask) == 0u) atomicMin(result, (uint32_t)w);
    } else {
      const uint64_t w = start + threadIdx.x;
      // a witness below this claim's first candidate makes the claim useless,
      // so its threads may stop early; they read the same condition (up to a
      // witness landing between their reads), and a stopped candidate is
      // never one the smallest witness could be
      const auto stop = [result, start] { return (uint64_t)*(volatile uint32_t*)result < start; };
      if (w < limit && (p2::grind_word7<SLOT, MAT>((uint32_t)w, cp, p16, stop) & mask) == 0u)
        atomicMin(result, (uint32_t)w);
    }
  }
}

}  // namespace

template <int MAT>
cudaError_t grind_m(const uint32_t* state, const uint32_t* in, int in_len, int bits, uint64_t limit,
                    uint32_t* result, uint32_t* counter, uint32_t* done, uint32_t* mail, uint32_t seq,
                    const P2Consts& p16, cudaStream_t st, const uint32_t* cp_dev, uint32_t* res_out, DevChal* ch,
                    ef* r_out, uint32_t* err, int window) {
  if (in_len < 0 || in_len > 7 || bits < 0 || bits > 30) return cudaErrorInvalidValue;
  if (ch && (!res_out || !r_out || !err || bits < 1)) return cudaErrorInvalidValue;
  if (limit > kb::P) limit = kb::P;
  // the sponge state with the pending inputs, canonical (a witness w < p is
  // its own canonical value), with 0 at the witness position; then its
  // external layer plus the first round constants (read from cp_dev instead
  // when the device challenger prepared them)
  uint32_t s[16] = {0u};
  if (!cp_dev) {
    for (int i = 0; i < 16; i++) s[i] = kb::from_mont(state[i]);
    for (int i = 0; i < in_len; i++) s[i] = kb::from_mont(in[i]);
    s[in_len] = 0u;
    p2::grind_fold<MAT>(s, p16);
  }
  // with a mailbox or a result slot the previous search left the state reset
  // (grind_reset initialises it once per context)
  if (!mail && !res_out) {
    const cudaError_t e = grind_reset(result, counter, done, st);
    if (e != cudaSuccess) return e;
  }
  uint4 a = make_uint4(s[0], s[1], s[2], s[3]), b = make_uint4(s[4], s[5], s[6], s[7]);
  uint4 c = make_uint4(s[8], s[9], s[10], s[11]), d = make_uint4(s[12], s[13], s[14], s[15]);
  // Candidates in flight: once the smallest witness w is found, every claim
  // already running still completes, so a search costs about w + W
  // permutations for W in flight, while the rate grows with W. Expected cost
  // (2^bits + W) / rate(W), minimised over CTAs per SM with the rates measured
  // for Poseidon2-16 on B200, relative to 16 CTAs of 128 per SM (one CTA per
  // SM: one warp per sub-partition, about 7 us per permutation, 47 % of the
  // full rate; the kernel's registers allow 10 resident CTAs). A search too
  // small to fill the GPU runs one CTA per SM with about 2^(bits+3)
  // candidates in flight: the first pass then holds a witness with
  // probability 1 - e^-8, and the pass costs no more than a narrower one.
  // Searches of up to kCoopGrindBits bits (2^(bits+3) candidates in flight in
  // at most 4 CTAs per SM) run the four-lane form: one pass is a four-lane
  // permutation's latency instead of a one-thread permutation's.
  // With other work sharing the GPU (a batch), evaluated candidates count
  // more than the search's own latency: window bit kGrindLeanSmall keeps about
  // 2^(bits+1) candidates in flight in a four-lane search instead of
  // 2^(bits+3); bit kGrindLeanLarge runs a larger search with one CTA per SM
  // (the smallest window that spans the GPU, at about half the rate the cost
  // model's window reaches on an idle GPU).
  static const int kPerSm[7] = {1, 2, 3, 4, 6, 8, 10};
  static const double kRate[7] = {0.467, 0.703, 0.811, 0.865, 0.911, 0.948, 0.965};
  const double expect = (double)(1ull << bits);
  const bool coop = bits <= kCoopGrindBits;
  const int lead = (window & kGrindLeanSmall) ? 1 : 3;  // 2^(bits+lead) candidates in flight
  if (coop) {
    const unsigned blocks = (unsigned)(((1ull << (bits + lead)) + GRIND_CTA / 4 - 1) / (GRIND_CTA / 4));
    switch (in_len) {
#define WK_GRIND_COOP(S)                                                                                          \
  case S:                                                                                                        \
    k_grind<S, MAT, true><<<blocks, GRIND_CTA, 0, st>>>(p16, a, b, c, d, bits, limit, result, counter, done, mail, \
                                                        seq, cp_dev, res_out, ch, r_out, err);                    \
    break;
      WK_GRIND_COOP(0) WK_GRIND_COOP(1) WK_GRIND_COOP(2) WK_GRIND_COOP(3) WK_GRIND_COOP(4) WK_GRIND_COOP(5)
      WK_GRIND_COOP(6) WK_GRIND_COOP(7)
#undef WK_GRIND_COOP
    }
    LAUNCH_DONE();
  }
  unsigned blocks = (unsigned)(((8ull << bits) + GRIND_CTA - 1) / GRIND_CTA);
  if (window & kGrindLeanLarge) {
    if (blocks > (unsigned)sm_count()) blocks = (unsigned)sm_count();
  } else if (blocks > (unsigned)sm_count()) {
    double best = 0.0;
    unsigned pick = (unsigned)sm_count();
    for (int i = 0; i < 7; i++) {
      const unsigned b = (unsigned)sm_count() * kPerSm[i];
      const double cost = (expect + (double)b * GRIND_CTA) / kRate[i];
      if (i == 0 || cost < best) {
        best = cost;
        pick = b;
      }
    }
    if (pick < blocks) blocks = pick;
  }
  switch (in_len) {
#define WK_GRIND(S) \
  case S:                                                                                                      \
    k_grind<S, MAT, false><<<blocks, GRIND_CTA, 0, st>>>(p16, a, b, c, d, bits, limit, result, counter, done, mail, \
                                                         seq, cp_dev, res_out, ch, r_out, err);                    \
    break;
    WK_GRIND(0) WK_GRIND(1) WK_GRIND(2) WK_GRIND(3) WK_GRIND(4) WK_GRIND(5) WK_GRIND(6) WK_GRIND(7)
#undef WK_GRIND
  }
  LAUNCH_DONE();
}

// ---------------------------------------------------------------------------
// A sumcheck round with its transcript step (sumcheck_round_body, then
// dc_coeffs_step in the first warp of the last CTA): the round's coefficients
// are observed on the device challenger in the same launch. With use_init the
// challenger starts from `init` (the host's challenger at the start of a
// sumcheck stage) and *err is cleared.
// ---------------------------------------------------------------------------

namespace {

template <bool FOLD, int MAT>
__global__ void __launch_bounds__(256) k_sumcheck_round_tr(ef* __restrict__ f, ef* __restrict__ w, size_t q, ef r,
                                                            ef* __restrict__ partials, unsigned* __restrict__ counter,
                                                            ef* __restrict__ out, const ef* __restrict__ r_dev,
                                                            DevChal* ch, const __grid_constant__ DevChal init,
                                                            int use_init, uint32_t* err, int grind_next,
                                                            uint32_t* cp_out, ef* r_out,
                                                            const __grid_constant__ P2Consts k) {
  __shared__ ef sh[2][32];
  __shared__ bool s_last;
  __shared__ ef s_co[2];
  __shared__ DevChal c;
  ef res[2];
  if (!sumcheck_round_body<FOLD>(f, w, q, r, partials, counter, out, r_dev, res, sh, s_last)) return;
  if (threadIdx.x == 0) {
    s_co[0] = res[0];
    s_co[1] = res[1];
  }
  __syncthreads();
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  const uint32_t cw = lane < 8 ? s_co[lane >> 2].c[lane & 3] : 0u;
  if (use_init) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&init);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&c);
    for (int i = lane; i < (int)(sizeof(DevChal) / 4); i += 32) dst[i] = src[i];
    if (lane == 0) *err = 0u;
    __syncwarp();
  } else {
    dc_load(c, ch);
  }
  dc_coeffs_step<MAT>(c, cw, grind_next, cp_out, r_out, k);
  dc_store(c, ch);
}

}  // namespace

template <int MAT>
cudaError_t sumcheck_round_tr_m(ef* f, ef* w, size_t q, int fold, ef r, ef* partials, unsigned* counter, ef* out,
                                const ef* r_dev, DevChal* ch, const DevChal* init, uint32_t* err, int grind_next,
                                uint32_t* cp_out, ef* r_out, const P2Consts& p16, cudaStream_t st) {
  if (q == 0 || !ch || !err || !out || (grind_next ? !cp_out : !r_out)) return cudaErrorInvalidValue;
  DevChal iv{};
  if (init) iv = *init;
  const unsigned b = sumcheck_round_blocks(q);
  if (fold)
    k_sumcheck_round_tr<true, MAT><<<b, 256, 0, st>>>(f, w, q, r, partials, counter, out, r_dev, ch, iv, init ? 1 : 0,
                                                       err, grind_next, cp_out, r_out, p16);
  else
    k_sumcheck_round_tr<false, MAT><<<b, 256, 0, st>>>(f, w, q, r, partials, counter, out, r_dev, ch, iv, init ? 1 : 0,
                                                        err, grind_next, cp_out, r_out, p16);
  LAUNCH_DONE();
}

// ---------------------------------------------------------------------------
// Many independent trees in few launches (merkle_many_m): one leaf launch for
// all trees and one launch per tree level across all trees tall enough to
// have it. The leaf kernel is persistent: its CTAs claim chunks of
// MANY_CTA leaves from one work counter over the trees' concatenated leaves,
// and a table of each tree's first global leaf (binary-searched in shared
// memory) maps a claimed leaf to its tree. A level launch maps its global node
// index to (tree, node) the same way through that level's table.
// ---------------------------------------------------------------------------

constexpr int MANY_CTA = 256;

namespace {

// the largest i < count with first[i] <= g (first strictly increasing, first[0] = 0)
__device__ __forceinline__ int tree_of(const unsigned long long* first, int count, unsigned long long g) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int T, int RP, int RATE, int MAT>
__global__ void __launch_bounds__(MANY_CTA) k_leaves_many(const TreeDesc* __restrict__ desc, int count,
                                                          int row_words, unsigned* __restrict__ counter,
                                                          const __grid_constant__ P2Consts leaf) {
  __shared__ unsigned long long s_first[kMaxManyTrees + 1];
  __shared__ unsigned long long s_start;
  for (int i = threadIdx.x; i <= count; i += blockDim.x)
    s_first[i] = i < count ? desc[i].leaf0 : desc[count - 1].leaf0 + (1ull << desc[count - 1].log_h);
  __syncthreads();
  const unsigned long long total = s_first[count];
  for (;;) {
    if (threadIdx.x == 0) s_start = (unsigned long long)atomicAdd(counter, 1u) * MANY_CTA;
    __syncthreads();
    const unsigned long long start = s_start;
    __syncthreads();
    if (start >= total) break;
    const unsigned long long g = start + threadIdx.x;
    if (g >= total) continue;
    const int tr = tree_of(s_first, count, g);
    const size_t i = (size_t)(g - s_first[tr]);
    uint32_t s[T];
#pragma unroll
    for (int k = 0; k < T; k++) s[k] = 0u;
    const uint32_t* row = desc[tr].rows + i * (size_t)row_words;
    for (int pos = 0; pos < row_words; pos += RATE) {
      const int take = row_words - pos < RATE ? row_words - pos : RATE;
#pragma unroll
      for (int k = 0; k < RATE; k++)
        if (k < take) s[k] = kb::from_mont(__ldg(row + pos + k));
      const bool first = pos == 0, last = pos + RATE >= row_words;
      if (first && last) p2::permute_sponge<T, RP, RATE, true, true, MAT>(s, leaf);
      else if (first) p2::permute_sponge<T, RP, RATE, true, false, MAT>(s, leaf);
      else if (last) p2::permute_sponge<T, RP, RATE, false, true, MAT>(s, leaf);
      else p2::permute_sponge<T, RP, RATE, false, false, MAT>(s, leaf);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) s[k] = kb::to_mont(s[k]);
    uint4* d = reinterpret_cast<uint4*>(desc[tr].digests + i * 8);
    d[0] = make_uint4(s[0], s[1], s[2], s[3]);
    d[1] = make_uint4(s[4], s[5], s[6], s[7]);
  }
}

// level `level` (>= 1) of every tree with log_h >= level; first[i] is tree
// i's first global node of this level (first[count] = all of them)
template <int MAT>
__global__ void __launch_bounds__(MANY_CTA) k_level_many(const TreeDesc* __restrict__ desc,
                                                         const unsigned long long* __restrict__ first, int count,
                                                         int level, const __grid_constant__ P2Consts comp) {
  __shared__ unsigned long long s_first[kMaxManyTrees + 1];
  for (int i = threadIdx.x; i <= count; i += blockDim.x) s_first[i] = first[i];
  __syncthreads();
  const unsigned long long total = s_first[count];
  for (unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (unsigned long long)gridDim.x * blockDim.x) {
    const int tr = tree_of(s_first, count, g);
    const size_t j = (size_t)(g - s_first[tr]);
    const int lh = desc[tr].log_h;
    // level l starts at node 2h - 2^(lh - l + 1)
    const size_t h2 = (size_t)2 << lh;
    const size_t in_off = h2 - ((size_t)1 << (lh - level + 2)), out_off = h2 - ((size_t)1 << (lh - level + 1));
    uint32_t* dg = desc[tr].digests;
    uint32_t x[16];
    const uint4* src = reinterpret_cast<const uint4*>(dg + (in_off + 2 * j) * 8);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint4 v = src[q];
      x[4 * q] = v.x;
      x[4 * q + 1] = v.y;
      x[4 * q + 2] = v.z;
      x[4 * q + 3] = v.w;
    }
    compress_mont<MAT>(x, comp);
    uint4* dst = reinterpret_cast<uint4*>(dg + (out_off + j) * 8);
    dst[0] = make_uint4(x[0], x[1], x[2], x[3]);
    dst[1] = make_uint4(x[4], x[5], x[6], x[7]);
  }
}

// the top of every tree in one launch, one CTA per tree: the levels above
// the tree's level of at most TOP_NODES nodes (level max(0, log_h - 8)), by
// four-lane cooperative permutations in shared memory (coop_levels)
template <int MAT>
__global__ void __launch_bounds__(TOP_CTA) k_tops_many(const TreeDesc* __restrict__ desc,
                                                       const __grid_constant__ P2Consts comp) {
  __shared__ uint32_t sh[TOP_NODES * 8];
  const int lh = desc[blockIdx.x].log_h;
  if (lh == 0) return;  // a one-leaf tree: its leaf is its root
  const int start = lh > kManyTopLevels ? lh - kManyTopLevels : 0;
  const int cnt = 1 << (lh - start);
  uint32_t* dg = desc[blockIdx.x].digests;
  size_t off = ((size_t)2 << lh) - ((size_t)1 << (lh - start + 1)), lsz = (size_t)cnt;
  for (int k = threadIdx.x; k < cnt * 8; k += blockDim.x) sh[k] = dg[off * 8 + k];
  __syncthreads();
  coop_levels<MAT>(sh, cnt, lh - start, 0, off, lsz, dg, comp);
}

// the roots (node 2h - 2 of every tree) gathered into roots[8 * i]
__global__ void k_roots_many(const TreeDesc* __restrict__ desc, int count, uint32_t* __restrict__ roots) {
  for (int k = threadIdx.x; k < count * 8; k += blockDim.x) {
    const int i = k >> 3;
    const size_t root = ((size_t)2 << desc[i].log_h) - 2;
    roots[k] = desc[i].digests[root * 8 + (k & 7)];
  }
}

}  // namespace

template <int MAT>
cudaError_t merkle_many_m(const TreeDesc* d_desc, const unsigned long long* d_level_first, int count, int max_log_h,
                          const unsigned long long* level_totals, int row_words, int leaf_hash, const P2Consts& p16,
                          const P2Consts& p24, unsigned* counter, uint32_t* d_roots, cudaStream_t st) {
  if (count < 1 || count > kMaxManyTrees || row_words < 1 || max_log_h < 0 || max_log_h > 30 ||
      (leaf_hash != 0 && leaf_hash != 1))
    return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  const unsigned long long leaves = level_totals[0];
  size_t blocks = (size_t)((leaves + MANY_CTA - 1) / MANY_CTA);
  const size_t cap = (size_t)sm_count() * 4;  // resident CTAs of the leaf sponge
  if (blocks > cap) blocks = cap;
  if (leaf_hash == 0)
    k_leaves_many<24, p2::RP24, 16, MAT><<<(unsigned)blocks, MANY_CTA, 0, st>>>(d_desc, count, row_words, counter, p24);
  else
    k_leaves_many<16, p2::RP16, 8, MAT><<<(unsigned)blocks, MANY_CTA, 0, st>>>(d_desc, count, row_words, counter, p16);
  count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // level launches up to each tree's top, then one CTA per tree for the tops
  for (int l = 1; l <= max_log_h - kManyTopLevels; l++) {
    size_t b = (size_t)((level_totals[l] + MANY_CTA - 1) / MANY_CTA);
    const size_t lcap = (size_t)sm_count() * 8;
    if (b > lcap) b = lcap;
    if (b < 1) b = 1;
    k_level_many<MAT><<<(unsigned)b, MANY_CTA, 0, st>>>(d_desc, d_level_first + (size_t)l * (count + 1), count, l,
                                                         p16);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (max_log_h > 0) {
    k_tops_many<MAT><<<count, TOP_CTA, 0, st>>>(d_desc, p16);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  k_roots_many<<<1, 256, 0, st>>>(d_desc, count, d_roots);
  LAUNCH_DONE();
}

}  // namespace wk
