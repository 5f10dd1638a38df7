// Kernels of the Keccak MMCS and of proof-of-work grinding on the Keccak
// challenger (the reference's Keccak WHIR configuration,
// src/whir/mod.rs:236-383). Digests are 8 words per node, laid out like the
// Poseidon2 trees (level 0 first, 2h - 1 nodes), so the opening kernel and the
// proof layout are shared.
#include "keccak.cuh"
#include "kernels.h"

namespace wk {
namespace {

// SerializingHasher<PaddingFreeSponge<KeccakF, 25, 17, 4>> of one row: the
// row's canonical values in pairs (v0 | v1 << 32), 17 lanes per permutation.
__global__ void __launch_bounds__(128) k_keccak_leaves(const uint32_t* __restrict__ rows, int row_words, size_t h,
                                                        uint32_t* __restrict__ digests) {
  const int lanes = (row_words + 1) >> 1;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < h; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t* row = rows + i * (size_t)row_words;
    uint64_t st[25];
#pragma unroll
    for (int k = 0; k < 25; k++) st[k] = 0;
    for (int pos = 0; pos < lanes; pos += 17) {
      const int take = lanes - pos < 17 ? lanes - pos : 17;
#pragma unroll
      for (int k = 0; k < 17; k++) {
        if (k < take) {
          const int j = 2 * (pos + k);
          const uint64_t lo = kb::from_mont(row[j]);
          const uint64_t hi = j + 1 < row_words ? kb::from_mont(row[j + 1]) : 0u;
          st[k] = lo | hi << 32;
        }
      }
      kk::keccak_f(st);
    }
    uint4* d = reinterpret_cast<uint4*>(digests + i * 8);
    d[0] = make_uint4((uint32_t)st[0], (uint32_t)(st[0] >> 32), (uint32_t)st[1], (uint32_t)(st[1] >> 32));
    d[1] = make_uint4((uint32_t)st[2], (uint32_t)(st[2] >> 32), (uint32_t)st[3], (uint32_t)(st[3] >> 32));
  }
}

// one tree level: node j of the next level compresses nodes 2j and 2j + 1
__global__ void __launch_bounds__(128) k_keccak_level(uint32_t* __restrict__ digests, size_t in_off, size_t in_count) {
  const size_t out_count = in_count >> 1, out_off = in_off + in_count;
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < out_count; j += (size_t)gridDim.x * blockDim.x) {
    uint32_t l[8], r[8], o[8];
    const uint4* src = reinterpret_cast<const uint4*>(digests + (in_off + 2 * j) * 8);
    const uint4 a = src[0], b = src[1], c = src[2], d = src[3];
    l[0] = a.x; l[1] = a.y; l[2] = a.z; l[3] = a.w; l[4] = b.x; l[5] = b.y; l[6] = b.z; l[7] = b.w;
    r[0] = c.x; r[1] = c.y; r[2] = c.z; r[3] = c.w; r[4] = d.x; r[5] = d.y; r[6] = d.z; r[7] = d.w;
    kk::compress(l, r, o);
    uint4* dst = reinterpret_cast<uint4*>(digests + (out_off + j) * 8);
    dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
    dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
  }
}

// the levels above `in_count` <= 2 * KECCAK_TOP nodes in one CTA, each level
// kept in shared memory for the next and written out; the root is posted to
// the mailbox when one is given
constexpr int KECCAK_TOP = 512;
__global__ void __launch_bounds__(KECCAK_TOP) k_keccak_top(uint32_t* __restrict__ digests, size_t in_off,
                                                           int in_count, uint32_t* mail, uint32_t seq) {
  __shared__ uint32_t sh[KECCAK_TOP * 8];
  const int t = threadIdx.x;
  size_t off = in_off;
  int cnt = in_count;
  for (int level = 0; cnt > 1; level++) {
    const int act = cnt >> 1;
    uint32_t o[8];
    if (t < act) {
      const uint32_t* l = level == 0 ? digests + (off + 2 * (size_t)t) * 8 : sh + 16 * t;
      uint32_t a[16];
#pragma unroll
      for (int k = 0; k < 16; k++) a[k] = l[k];
      kk::compress(a, a + 8, o);
    }
    __syncthreads();
    off += cnt;
    if (t < act) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        sh[8 * t + k] = o[k];
        digests[(off + t) * 8 + k] = o[k];
      }
    }
    __syncthreads();
    cnt = act;
  }
  if (t == 0 && mail) mail_post(mail, sh, 8, seq);
}

// Proof of work on SerializingChallenger32<F, HashChallenger<u8,
// Keccak256Hash, 32>>: candidate w is valid when Keccak-256 of the input
// buffer followed by w's 4 little-endian bytes, read from its last byte
// backwards as a little-endian word (the challenger pops bytes from the end
// of its output), has `bits` low zero bits. `in` is the input buffer absorbed
// so far (lanes and position in the current block). Claims of KECCAK_CLAIM
// candidates, CTA b's first claim chunk b, later claims from the counter;
// the smallest valid witness wins; the last CTA to stop posts the witness and
// the candidates the counter's claims cover and resets the search state.
constexpr int KECCAK_CLAIM = 128;
__global__ void __launch_bounds__(KECCAK_CLAIM) k_keccak_grind(const __grid_constant__ kk::K256 in, int bits,
                                                              uint64_t limit, uint32_t* result, uint32_t* counter,
                                                              uint32_t* done, uint32_t* mail, uint32_t seq) {
  __shared__ uint64_t s_start;
  __shared__ int s_go;
  const uint32_t mask = (uint32_t)((1ull << bits) - 1);
  for (bool first = true;; first = false) {
    if (threadIdx.x == 0) {
      const uint64_t chunk = first ? (uint64_t)blockIdx.x : (uint64_t)gridDim.x + atomicAdd(counter, 1u);
      const uint64_t start = chunk * KECCAK_CLAIM;
      s_start = start;
      s_go = start < limit && start < (uint64_t)*(volatile uint32_t*)result;
    }
    __syncthreads();
    const uint64_t start = s_start;
    const int go = s_go;
    __syncthreads();
    if (!go) {
      // with a mailbox the last CTA to stop posts and resets the search state
      // (without one the caller reads the result and resets it)
      if (threadIdx.x == 0 && mail) {
        __threadfence();
        if (atomicAdd(done, 1u) == gridDim.x - 1) {
          const uint32_t post[2] = {atomicAdd(result, 0u), atomicAdd(counter, 0u) * (uint32_t)KECCAK_CLAIM};
          if (mail) mail_post(mail, post, 2, seq);
          *result = kb::P;
          *counter = 0u;
          *done = 0u;
        }
      }
      return;
    }
    const uint64_t w = start + threadIdx.x;
    if (w < limit) {
      kk::K256 k = in;
      kk::k256_word(k, (uint32_t)w);
      uint8_t out[32];
      kk::k256_final(k, out);
      const uint32_t v = (uint32_t)out[31] | (uint32_t)out[30] << 8 | (uint32_t)out[29] << 16 | (uint32_t)out[28] << 24;
      if ((v & mask) == 0u) atomicMin(result, (uint32_t)w);
    }
  }
}

unsigned blocks_for(size_t work, int threads, int per_sm) {
  size_t b = (work + threads - 1) / threads;
  const size_t cap = (size_t)sm_count() * per_sm;
  if (b > cap) b = cap;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t keccak_leaves(const uint32_t* rows, int log_h, int row_words, uint32_t* digests, cudaStream_t st) {
  if (log_h < 0 || row_words < 1) return cudaErrorInvalidValue;
  const size_t h = (size_t)1 << log_h;
  k_keccak_leaves<<<blocks_for(h, 128, 16), 128, 0, st>>>(rows, row_words, h, digests);
  LAUNCH_DONE();
}

cudaError_t keccak_upper(int log_h, uint32_t* digests, uint32_t* mail, uint32_t seq, int* posted, cudaStream_t st) {
  if (posted) *posted = 0;
  size_t off = 0, cnt = (size_t)1 << log_h;
  if (cnt <= 1) return cudaSuccess;
  while (cnt > (size_t)2 * KECCAK_TOP) {
    k_keccak_level<<<blocks_for(cnt / 2, 128, 16), 128, 0, st>>>(digests, off, cnt);
    count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    off += cnt;
    cnt >>= 1;
  }
  k_keccak_top<<<1, KECCAK_TOP, 0, st>>>(digests, off, (int)cnt, mail, seq);
  count_launch();
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && posted && mail) *posted = 1;
  return e;
}

cudaError_t keccak_grind(const kk::K256& in, int bits, uint64_t limit, uint32_t* result, uint32_t* counter,
                         uint32_t* done, uint32_t* mail, uint32_t seq, cudaStream_t st, int window) {
  if (bits < 0 || bits > 30 || in.pos >= 136) return cudaErrorInvalidValue;
  if (limit > kb::P) limit = kb::P;
  if (!mail) {
    const cudaError_t e = grind_reset(result, counter, done, st);
    if (e != cudaSuccess) return e;
  }
  // about 2^(bits+3) candidates in flight, at most 8 CTAs per SM; window bit
  // kGrindLeanSmall: 2^(bits+1) for searches of up to kCoopGrindBits bits;
  // kGrindLeanLarge: at most one CTA per SM for larger ones
  const bool small = bits <= kCoopGrindBits;
  const size_t flight = (small && (window & kGrindLeanSmall) ? (size_t)2 : (size_t)8) << bits;
  const unsigned blocks = blocks_for(flight, KECCAK_CLAIM, !small && (window & kGrindLeanLarge) ? 1 : 8);
  k_keccak_grind<<<blocks, KECCAK_CLAIM, 0, st>>>(in, bits, limit, result, counter, done, mail, seq);
  LAUNCH_DONE();
}

}  // namespace wk
