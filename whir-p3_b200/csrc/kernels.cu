// Device kernels of the WHIR prover hot path for sm_100a.
//
// Every kernel here is a data-parallel replacement for an O(2^n) loop of the
// reference prover (tcoratger/whir-p3) or of the Plonky3 code it calls; the
// sequential Fiat-Shamir spine stays on the host (host.cu). Each kernel names
// the reference function whose result it reproduces bit for bit.
//
// Memory-bound kernels use coalesced 16-byte element accesses and grid-stride
// loops sized to the SM count; the Poseidon2 kernels keep the permutation state
// in registers with every round constant an immediate (kernel parameters live
// in the constant bank).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "devutil.cuh"

using kb::ef;
using p2::P2Consts;

namespace wk {

static std::atomic<unsigned long long> g_launches{0};
unsigned long long launches() { return g_launches.load(); }
void count_launch() { g_launches.fetch_add(1); }

// per-device SM counts, filled on first use; readers and the writer of an
// entry synchronise through its atomic
constexpr int kMaxDevices = 64;
static std::atomic<int> g_sms[kMaxDevices];
int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDevices) dev = 0;
  int v = g_sms[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    g_sms[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

static inline unsigned grid_for(size_t work, int threads, int per_sm = 8) {
  size_t b = (work + threads - 1) / threads;
  size_t cap = (size_t)sm_count() * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}


// ---------------------------------------------------------------------------
// Representation conversion
// ---------------------------------------------------------------------------

__global__ void k_encode(uint32_t* p, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = kb::to_mont(p[i]);
}
__global__ void k_decode(uint32_t* p, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = kb::from_mont(p[i]);
}
cudaError_t encode(uint32_t* p, size_t n, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_encode<<<grid_for(n, 256), 256, 0, st>>>(p, n);
  LAUNCH_DONE();
}
cudaError_t decode(uint32_t* p, size_t n, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_decode<<<grid_for(n, 256), 256, 0, st>>>(p, n);
  LAUNCH_DONE();
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------


__global__ void k_publish(const uint32_t* __restrict__ src, int words, volatile uint32_t* mail, uint32_t seq) {
  for (int i = threadIdx.x; i < words; i += blockDim.x) mail[i] = src[i];
  __threadfence_system();
  __syncthreads();
  if (threadIdx.x == 0) mail[kMailWords] = seq;
}

cudaError_t publish(const uint32_t* src, int words, uint32_t* mail, uint32_t seq, cudaStream_t st) {
  if (words < 0 || words > kMailWords) return cudaErrorInvalidValue;
  k_publish<<<1, 128, 0, st>>>(src, words, mail, seq);
  LAUNCH_DONE();
}

struct PutBlock {
  int words;
  uint32_t w[kPutWords];
};  // 4004 bytes: within the 4 KiB parameter block every launch supports
__global__ void k_put(const __grid_constant__ PutBlock b, uint32_t* __restrict__ dst) {
  for (int i = threadIdx.x; i < b.words; i += blockDim.x) dst[i] = b.w[i];
}

cudaError_t put_words(uint32_t* dst, const uint32_t* src, int words, cudaStream_t st) {
  if (words < 0 || words > kPutWords) return cudaErrorInvalidValue;
  PutBlock b;
  b.words = words;
  memcpy(b.w, src, (size_t)words * 4);
  k_put<<<1, 256, 0, st>>>(b, dst);
  LAUNCH_DONE();
}

// out[i] = sum_{b < nparts} partials[i * nparts + b]
__global__ void k_sum_partials(const ef* partials, int nparts, ef* out) {
  __shared__ ef sh[1][32];
  ef v[1] = {kb::ef_zero()};
  const ef* p = partials + (size_t)blockIdx.x * nparts;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) v[0] = kb::ef_add(v[0], p[b]);
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = v[0];
}

// ---------------------------------------------------------------------------
// DFT (TwoAdicSubgroupDft::dft_batch / dft_algebra_batch as called at
// src/whir/committer/writer.rs:86 and src/whir/prover/mod.rs:180, including
// the transpose & pad of writer.rs:70-82 and prover/mod.rs:166-176).
//
// Output row r, column j: sum_{i < L} x_j[i] * omega_H^(i*r). With H = H1*H2,
// i = i1*H2 + i2 and r = r1 + H1*r2:
//   pass 1 (columns): Y_j[r1][i2] = omega_H^(i2*r1) * DFT_H1(x_j[i1*H2 + i2])[r1]
//                     (only i1 < L/H2 are nonzero: the zero padding is free)
//   pass 2 (rows):    out[r1 + H1*r2][j] = DFT_H2(Y_j[r1][.])[r2]
// Both passes run radix-2 DFTs of <= 2^12 points in shared memory; pass 2
// writes whole output rows (all columns j of the CTA) contiguously.
// ---------------------------------------------------------------------------

__global__ void k_dft_tables(uint32_t* tw_stage, uint32_t* tw_lo, uint32_t* tw_hi, uint32_t w12, uint32_t wh,
                             uint32_t wh_hi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 2048) tw_stage[i] = kb::pow(w12, (uint64_t)i);
  if (i < 4096) {
    tw_lo[i] = kb::pow(wh, (uint64_t)i);
    tw_hi[i] = kb::pow(wh_hi, (uint64_t)i);
    const uint32_t c = kb::from_mont(kb::pow(w12, (uint64_t)i));
    reinterpret_cast<uint2*>(tw_stage + 2048)[i] = make_uint2(c, kb::shoup_const(c));
  }
}

cudaError_t build_dft_tables(uint32_t* tw_stage, uint32_t* tw_lo, uint32_t* tw_hi, int log_h, cudaStream_t st) {
  uint32_t w12 = kb::two_adic_generator(12);
  uint32_t wh = kb::two_adic_generator(log_h);
  uint32_t wh_hi = kb::pow(wh, 4096);
  k_dft_tables<<<16, 256, 0, st>>>(tw_stage, tw_lo, tw_hi, w12, wh, wh_hi);
  LAUNCH_DONE();
}

template <int LANES>
struct Elem;
template <>
struct Elem<1> {
  using T = uint32_t;
  __device__ static T zero() { return 0u; }
  __device__ static T add(T a, T b) { return kb::add(a, b); }
  __device__ static T sub(T a, T b) { return kb::sub(a, b); }
  __device__ static T mulb(T a, uint32_t w) { return kb::mul(a, w); }
};
template <>
struct Elem<4> {
  using T = uint4;
  __device__ static T zero() { return make_uint4(0, 0, 0, 0); }
  __device__ static T add(T a, T b) {
    return make_uint4(kb::add(a.x, b.x), kb::add(a.y, b.y), kb::add(a.z, b.z), kb::add(a.w, b.w));
  }
  __device__ static T sub(T a, T b) {
    return make_uint4(kb::sub(a.x, b.x), kb::sub(a.y, b.y), kb::sub(a.z, b.z), kb::sub(a.w, b.w));
  }
  __device__ static T mulb(T a, uint32_t w) {
    return make_uint4(kb::mul(a.x, w), kb::mul(a.y, w), kb::mul(a.z, w), kb::mul(a.w, w));
  }
};

__device__ __forceinline__ uint32_t bitrev(uint32_t x, int bits) { return bits ? (__brev(x) >> (32 - bits)) : 0u; }

// Shared-memory swizzle for the DFT tiles: XOR the bank bits with bits 5-9 and
// 10-14 of the index. It is a bijection (it only changes bits 0-4, as a
// function of higher bits), keeps any aligned run of 32 words conflict-free,
// and spreads the bit-reversed scatter (indices k * 2^(L-5), L <= 12) and the
// column-strided accesses of several vectors over all 32 banks.
__device__ __forceinline__ int swz(int i) { return i ^ (((i >> 5) ^ (i >> 10)) & 31); }

__device__ __forceinline__ uint32_t tw_pow(const uint32_t* tw_lo, const uint32_t* tw_hi, uint64_t e) {
  // omega_H^e for e < H <= 2^24
  return kb::mul(__ldg(tw_lo + (e & 4095)), __ldg(tw_hi + (e >> 12)));
}

// K consecutive radix-2 DIT stages (first stage `s`, 1-based) in registers:
// each thread owns 2^K elements of one vector spaced by h = 2^(s-1), which are
// closed under the butterflies of these K stages.
template <int LANES, int K>
__device__ __forceinline__ void dft_stages(typename Elem<LANES>::T* a, int nv, int log_s, int s,
                                           const uint32_t* tw) {
  using E = Elem<LANES>;
  constexpr int R = 1 << K;
  const int h = 1 << (s - 1);
  const int log_units = log_s - K;
  const int total = nv << log_units;
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    const int v = q >> log_units;
    const int u = q & ((1 << log_units) - 1);
    const int lowpos = u & (h - 1);
    const int base = (v << log_s) + ((u >> (s - 1)) << (s - 1 + K)) + lowpos;
    typename E::T x[R];
#pragma unroll
    for (int j = 0; j < R; j++) x[j] = a[swz(base + j * h)];
#pragma unroll
    for (int t = 0; t < K; t++) {
      const int tshift = 12 - (s + t);
#pragma unroll
      for (int j = 0; j < R; j++) {
        if ((j >> t) & 1) continue;
        const int pos = lowpos + (j & ((1 << t) - 1)) * h;
        const typename E::T w = E::mulb(x[j + (1 << t)], tw[pos << tshift]);
        const typename E::T u0 = x[j];
        x[j] = E::add(u0, w);
        x[j + (1 << t)] = E::sub(u0, w);
      }
    }
#pragma unroll
    for (int j = 0; j < R; j++) a[swz(base + j * h)] = x[j];
  }
}

// In-place radix-2 DIT over `nv` vectors of S = 2^log_s points stored
// contiguously (vector v at a[v*S], swizzled); inputs already in bit-reversed
// order. Stages run three at a time in registers.
template <int LANES>
__device__ __forceinline__ void smem_dft(typename Elem<LANES>::T* a, int nv, int log_s, const uint32_t* tw) {
  int s = 1;
  while (s <= log_s) {
    const int k = log_s - s + 1 >= 3 ? 3 : log_s - s + 1;
    if (k == 3)
      dft_stages<LANES, 3>(a, nv, log_s, s, tw);
    else if (k == 2)
      dft_stages<LANES, 2>(a, nv, log_s, s, tw);
    else
      dft_stages<LANES, 1>(a, nv, log_s, s, tw);
    __syncthreads();
    s += k;
  }
}

template <int LANES>
__global__ void k_dft_cols(const typename Elem<LANES>::T* __restrict__ x, typename Elem<LANES>::T* __restrict__ y,
                           int log_l, int log_h1, int log_h2, int log_h, int log_tile,
                           const uint32_t* __restrict__ tw_stage, const uint32_t* __restrict__ tw_lo,
                           const uint32_t* __restrict__ tw_hi) {
  using E = Elem<LANES>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* tw = reinterpret_cast<uint32_t*>(smem_raw);
  typename E::T* a = reinterpret_cast<typename E::T*>(smem_raw + 2048 * sizeof(uint32_t));
  const int H1 = 1 << log_h1, H2 = 1 << log_h2;
  const size_t L = (size_t)1 << log_l;
  const int L1 = (int)(L >> log_h2);  // nonzero rows of each column vector
  const int j = blockIdx.y;
  const int tile = 1 << log_tile;
  const int tmask = tile - 1;
  const int i2_0 = blockIdx.x * tile;
  const typename E::T* xj = x + (size_t)j * L;
  typename E::T* yj = y + ((size_t)j << log_h);
  for (int i = threadIdx.x; i < 2048; i += blockDim.x) tw[i] = __ldg(tw_stage + i);
  for (int idx = threadIdx.x; idx < tile * H1; idx += blockDim.x) {
    const int t = idx & tmask, i1 = idx >> log_tile;
    typename E::T v = E::zero();
    if (i1 < L1) v = xj[(size_t)i1 * H2 + i2_0 + t];
    a[swz(t * H1 + bitrev((uint32_t)i1, log_h1))] = v;
  }
  __syncthreads();
  smem_dft<LANES>(a, tile, log_h1, tw);
  for (int idx = threadIdx.x; idx < tile * H1; idx += blockDim.x) {
    const int t = idx & tmask, r1 = idx >> log_tile;
    const uint64_t e = (uint64_t)(i2_0 + t) * (uint64_t)r1;
    typename E::T v = a[swz(t * H1 + r1)];
    if (e) v = E::mulb(v, tw_pow(tw_lo, tw_hi, e));
    yj[((size_t)r1 << log_h2) + i2_0 + t] = v;
  }
}

// pass 2: out[r1 + H1*r2][j] = DFT_H2(Y_j[r1][.])[r2], jt columns per CTA
template <int LANES>
__global__ void k_dft_rows(const typename Elem<LANES>::T* __restrict__ y, typename Elem<LANES>::T* __restrict__ out,
                           int log_h1, int log_h2, int log_h, int log_w, int log_jt,
                           const uint32_t* __restrict__ tw_stage) {
  using E = Elem<LANES>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* tw = reinterpret_cast<uint32_t*>(smem_raw);
  typename E::T* a = reinterpret_cast<typename E::T*>(smem_raw + 2048 * sizeof(uint32_t));
  const int H2 = 1 << log_h2;
  const int r1 = blockIdx.x;
  const int jt = 1 << log_jt;
  const int j0 = blockIdx.y * jt;
  for (int i = threadIdx.x; i < 2048; i += blockDim.x) tw[i] = __ldg(tw_stage + i);
  for (int idx = threadIdx.x; idx < jt * H2; idx += blockDim.x) {
    const int jj = idx >> log_h2, i2 = idx & (H2 - 1);
    a[swz(jj * H2 + bitrev((uint32_t)i2, log_h2))] = y[((size_t)(j0 + jj) << log_h) + ((size_t)r1 << log_h2) + i2];
  }
  __syncthreads();
  smem_dft<LANES>(a, jt, log_h2, tw);
  for (int idx = threadIdx.x; idx < jt * H2; idx += blockDim.x) {
    const int jj = idx & (jt - 1), r2 = idx >> log_jt;
    const size_t row = (size_t)r1 + ((size_t)r2 << log_h1);
    out[(row << log_w) + j0 + jj] = a[swz(jj * H2 + r2)];
  }
}

// Small chunks (L <= 2^12): out[a*B + b][j] = DFT_L(x_j[i] * omega_H^(i*b))[a];
// one CTA per twist b and column group, H = L*B.
template <int LANES>
__global__ void k_dft_coset(const typename Elem<LANES>::T* __restrict__ x, typename Elem<LANES>::T* __restrict__ out,
                            int log_l, int log_b, int log_w, int log_jt, const uint32_t* __restrict__ tw_stage,
                            const uint32_t* __restrict__ tw_lo, const uint32_t* __restrict__ tw_hi) {
  using E = Elem<LANES>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* tw = reinterpret_cast<uint32_t*>(smem_raw);
  typename E::T* a = reinterpret_cast<typename E::T*>(smem_raw + 2048 * sizeof(uint32_t));
  const int L = 1 << log_l;
  const uint32_t b = blockIdx.x;
  const int jt = 1 << log_jt;
  const int j0 = blockIdx.y * jt;
  for (int i = threadIdx.x; i < 2048; i += blockDim.x) tw[i] = __ldg(tw_stage + i);
  for (int idx = threadIdx.x; idx < jt * L; idx += blockDim.x) {
    const int jj = idx >> log_l, i = idx & (L - 1);
    typename E::T v = x[(size_t)(j0 + jj) * L + i];
    const uint64_t e = (uint64_t)i * b;
    if (e) v = E::mulb(v, tw_pow(tw_lo, tw_hi, e));
    a[swz(jj * L + bitrev((uint32_t)i, log_l))] = v;
  }
  __syncthreads();
  smem_dft<LANES>(a, jt, log_l, tw);
  for (int idx = threadIdx.x; idx < jt * L; idx += blockDim.x) {
    const int jj = idx & (jt - 1), r = idx >> log_jt;
    const size_t row = ((size_t)r << log_b) + b;
    out[(row << log_w) + j0 + jj] = a[swz(jj * L + r)];
  }
}

// ---------------------------------------------------------------------------
// Register-resident DFT passes (base field). A length-N = E * G transform of
// one vector is split as in the four-step method but inside the CTA: with
// input index i = g + G*e and output index n = k + E*l,
//   X[k + E*l] = sum_g omega_G^(g*l) * omega_N^(g*k) * sum_e x[g + G*e] * omega_E^(e*k).
// G threads per vector each run the E-point inner DFT on registers (radix-2
// decimation in frequency, twiddles from the constant bank, products in Shoup
// form), multiply by omega_N^(g*k), and exchange through shared memory once;
// then each thread runs E/G of the G-point outer DFTs on registers. Every
// element is read and written once in shared memory per pass, against once
// per three stages in the radix-2 kernel, and no index arithmetic runs per
// butterfly.
// ---------------------------------------------------------------------------

namespace dftreg {

constexpr uint32_t cpow(uint64_t b, uint64_t e) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = r * b % kb::P;
    b = b * b % kb::P;
    e >>= 1;
  }
  return (uint32_t)r;
}
// omega_64^j (canonical) and its Shoup constant, j < 32
struct Tw64 {
  uint32_t w[32];
  uint32_t s[32];
};
constexpr Tw64 make_tw64() {
  Tw64 t{};
  const uint64_t g = cpow(3, (uint64_t)(kb::P - 1) / 64);
  uint64_t cur = 1;
  for (int j = 0; j < 32; j++) {
    t.w[j] = (uint32_t)cur;
    t.s[j] = (uint32_t)((cur << 32) / kb::P);
    cur = cur * g % kb::P;
  }
  return t;
}
__constant__ Tw64 c_tw64 = make_tw64();

__host__ __device__ constexpr int bitrev(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

// In-place DIF DFT of length 2^L <= 64 over registers: natural order in,
// a[r] = X[bitrev_L(r)] out. A difference that goes on to a twiddle product
// stays unreduced (u - v + p < 2p): the Shoup product takes any 32-bit input.
// ZERO_HIGH: the upper half of the input is zero, so the first stage is
// a[j + M/2] = a[j] * omega^j with a[j] unchanged.
template <int L, bool ZERO_HIGH = false>
__device__ __forceinline__ void dif(uint32_t (&a)[1 << L]) {
  constexpr int M = 1 << L;
#pragma unroll
  for (int half = M / 2; half >= 1; half >>= 1) {
#pragma unroll
    for (int start = 0; start < M; start += 2 * half) {
#pragma unroll
      for (int j = 0; j < half; j++) {
        const int tj = j * (32 / half);  // omega_{2*half}^j = omega_64^(j * 32 / half)
        const uint32_t u = a[start + j], v = a[start + j + half];
        if (ZERO_HIGH && half == M / 2) {
          a[start + j + half] = tj == 0 ? u : kb::mul_shoup(u, c_tw64.w[tj], c_tw64.s[tj]);
          continue;
        }
        a[start + j] = kb::add(u, v);
        a[start + j + half] = tj == 0 ? kb::sub(u, v) : kb::mul_shoup(u - v + kb::P, c_tw64.w[tj], c_tw64.s[tj]);
      }
    }
  }
}

// shared-memory layout of one vector: E rows (k) of G + 1 words (g); vectors
// `vs` words apart with vs = rest (mod 32), so lanes of a warp that differ in
// the vector or in k fall in different banks
template <int E, int G>
__host__ __device__ constexpr int vstride(int rest) {
  return E * (G + 1) + ((rest - (E * (G + 1)) % 32) % 32 + 32) % 32;
}

}  // namespace dftreg

// pass 1: T = 2^LT columns i2 per CTA, threads (t, g) with t fastest in both
// phases. Extension data (4 words per element) runs as 4 base columns per
// element: the caller passes word-level sizes (log_l, log_h2, log_h + 2) and
// ls = 2, and the twist exponent uses the element column i2 >> ls.
template <int LE, int LG, int LT>
__global__ void __launch_bounds__(1 << (LG + LT))
    k_dft_cols_reg(const uint32_t* __restrict__ x, uint32_t* __restrict__ y, int log_l, int log_h2, int log_h,
                   int ls, const uint2* __restrict__ tw_sh, const uint32_t* __restrict__ tw_lo,
                   const uint32_t* __restrict__ tw_hi) {
  constexpr int E = 1 << LE, G = 1 << LG, T = 1 << LT, N = E * G;
  constexpr int RS = G + 1;
  constexpr int VS = dftreg::vstride<E, G>(T >= 32 ? 1 : 32 / T);
  extern __shared__ uint32_t sm[];
  const int H2 = 1 << log_h2;
  const size_t L = (size_t)1 << log_l;
  const int L1 = (int)(L >> log_h2);  // nonzero entries of each column vector
  const int j = blockIdx.y;
  const int i2_0 = blockIdx.x * T;
  const int t = threadIdx.x & (T - 1), g = threadIdx.x >> LT;
  {
    uint32_t a[E];
    const uint32_t* xj = x + (size_t)j * L + i2_0 + t;
    if (2 * L1 <= N) {
      // a low-degree extension: the upper half of every column is padding
#pragma unroll
      for (int e = 0; e < E / 2; e++) {
        const int i1 = g + G * e;
        a[e] = i1 < L1 ? __ldg(xj + (size_t)i1 * H2) : 0u;
      }
#pragma unroll
      for (int e = E / 2; e < E; e++) a[e] = 0u;
      dftreg::dif<LE, true>(a);
    } else {
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int i1 = g + G * e;
        a[e] = i1 < L1 ? __ldg(xj + (size_t)i1 * H2) : 0u;
      }
      dftreg::dif<LE>(a);
    }
#pragma unroll
    for (int r = 0; r < E; r++) {
      constexpr int kshift = 12 - LE - LG;
      const int k = dftreg::bitrev(r, LE);
      uint32_t v = a[r];
      if (k != 0) {
        const uint2 w = __ldg(tw_sh + (((g * k) & (N - 1)) << kshift));
        v = kb::mul_shoup(v, w.x, w.y);
      }
      sm[t * VS + k * RS + g] = v;
    }
  }
  __syncthreads();
  const size_t i2 = (size_t)(i2_0 + t);
  // Four-step twist omega_H^(I r1) for the element column I = i2 >> ls and
  // r1 = k + E m: omega^(I k) times (omega^(I E))^m, as two running powers
  // (even and odd m, stepping by omega^(2 I E)) instead of a table lookup pair
  // per element. I k and I E stay below H.
  const uint32_t I = (uint32_t)(i2 >> ls);
  const auto twist = [&](uint32_t e) { return kb::mul(__ldg(tw_lo + (e & 4095u)), __ldg(tw_hi + (e >> 12))); };
  const uint32_t step = twist(I * (uint32_t)E);
  const uint32_t step2 = kb::mul(step, step);
#pragma unroll
  for (int q = 0; q < E / G; q++) {
    const int k = g + G * q;
    uint32_t b[G];
#pragma unroll
    for (int gg = 0; gg < G; gg++) b[gg] = sm[t * VS + k * RS + gg];
    dftreg::dif<LG>(b);
    uint32_t we = twist(I * (uint32_t)k);  // m even
    uint32_t wo = kb::mul(we, step);        // m odd
#pragma unroll
    for (int m = 0; m < G; m += 2) {
      const int r1 = k + E * m;
      y[((size_t)j << log_h) + ((size_t)r1 << log_h2) + i2] = kb::mul(b[dftreg::bitrev(m, LG)], we);
      y[((size_t)j << log_h) + ((size_t)(r1 + E) << log_h2) + i2] = kb::mul(b[dftreg::bitrev(m + 1, LG)], wo);
      if (m + 2 < G) {
        we = kb::mul(we, step2);
        wo = kb::mul(wo, step2);
      }
    }
  }
}

namespace dftreg {
// words of a register pass's exchange buffer, rounded up to 8 bytes, and the
// dynamic shared memory of the TMA-staged pass 2 (the buffer, then its mbarrier)
__host__ __device__ constexpr int xwords(int t, int vs) { return (t * vs + 1) & ~1; }

// One tensor copy of this CTA's input tile into `tile`; true when every thread
// may read it. Returns false (the caller then loads from global memory) when
// the tile is not 128-byte aligned or the wait gives up; the latter waits once
// more, bounded, for the copy in flight before the buffer is reused.
__device__ __forceinline__ bool stage_tile(uint32_t* tile, uint64_t* bar, const CUtensorMap* tm, int y, int z,
                                           uint32_t bytes, uint32_t* err) {
  if ((bulk::saddr(tile) & 127u) != 0u) {
    if (threadIdx.x == 0 && err) atomicOr(err, 2u);
    return false;
  }
  if (threadIdx.x == 0) {
    bulk::bar_init(bar);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    bulk::bar_expect(bar, bytes);
    bulk::tensor_load_3d(tile, tm, 0, y, z, bar);
  }
  __syncthreads();
  const bool ok = bulk::bar_wait(bar, 0);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      if (err) atomicOr(err, 1u);
      bulk::bar_wait(bar, 0);
    }
    __syncthreads();
    return false;
  }
  return true;
}
}  // namespace dftreg

// pass 2: T = 2^LT word columns per CTA (one r1); loads with g fastest (rows
// are contiguous in i2), outer DFTs and stores with t fastest (output rows are
// contiguous in j). Extension data (ls = 2) runs each element's 4 words as 4
// columns t = 4 * column + coefficient: loads take the coefficient fastest,
// then g, and log_w counts words.
// TMA: the CTA's input, T >> ls runs of N << ls contiguous words (one per
// element column), arrives as one box of the tensor map `tm` (dimensions 256
// words, (H << ls) / 256 rows of them, columns) in the exchange buffer, which
// the threads read before they overwrite it with the exchange.
template <int LE, int LG, int LT, bool TMA = false>
__global__ void __launch_bounds__(1 << (LG + LT))
    k_dft_rows_reg(const uint32_t* __restrict__ y, uint32_t* __restrict__ out, int log_h1, int log_h, int log_w,
                   int ls, const uint2* __restrict__ tw_sh, const __grid_constant__ CUtensorMap tm, uint32_t* err) {
  constexpr int E = 1 << LE, G = 1 << LG, T = 1 << LT, N = E * G;
  constexpr int RS = G + 1;
  constexpr int VS = dftreg::vstride<E, G>(T >= 32 ? 1 : 32 / T);
  extern __shared__ __align__(128) uint32_t sm[];
  const int r1 = blockIdx.x;
  const int j0 = blockIdx.y * T;
  {
    const int c = threadIdx.x & ((1 << ls) - 1);
    const int g = (threadIdx.x >> ls) & (G - 1);
    const int tq = threadIdx.x >> (ls + LG);
    const int t = (tq << ls) | c;
    uint32_t a[E];
    bool staged = false;
    if constexpr (TMA) {
      uint64_t* bar = reinterpret_cast<uint64_t*>(sm + dftreg::xwords(T, VS));
      staged = dftreg::stage_tile(sm, bar, &tm, (r1 * N << ls) >> 8, j0 >> ls, (uint32_t)(T * N * 4), err);
    }
    if (staged) {
      const uint32_t* tile = sm + ((tq * N) << ls) + c;
#pragma unroll
      for (int e = 0; e < E; e++) a[e] = tile[(g + G * e) << ls];
      __syncthreads();  // the exchange below overwrites the tile
    } else {
      const uint32_t* src = y + (((((size_t)((j0 >> ls) + tq)) << log_h) + (size_t)r1 * N + g) << ls) + c;
#pragma unroll
      for (int e = 0; e < E; e++) a[e] = __ldg(src + ((size_t)(G * e) << ls));
    }
    dftreg::dif<LE>(a);
#pragma unroll
    for (int r = 0; r < E; r++) {
      constexpr int kshift = 12 - LE - LG;
      const int k = dftreg::bitrev(r, LE);
      uint32_t v = a[r];
      if (k != 0) {
        const uint2 w = __ldg(tw_sh + (((g * k) & (N - 1)) << kshift));
        v = kb::mul_shoup(v, w.x, w.y);
      }
      sm[t * VS + k * RS + g] = v;
    }
  }
  __syncthreads();
  const int t = threadIdx.x & (T - 1), gq = threadIdx.x >> LT;
#pragma unroll
  for (int q = 0; q < E / G; q++) {
    const int k = gq + G * q;
    uint32_t b[G];
#pragma unroll
    for (int gg = 0; gg < G; gg++) b[gg] = sm[t * VS + k * RS + gg];
    dftreg::dif<LG>(b);
#pragma unroll
    for (int r = 0; r < G; r++) {
      const size_t n = (size_t)(k + E * dftreg::bitrev(r, LG));
      out[(((size_t)r1 + (n << log_h1)) << log_w) + j0 + t] = b[r];
    }
  }
}

// (LE, LG) of the register passes by length: E >= G, E * G = 2^m
static bool reg_split(int m, int* le, int* lg) {
  if (m < 8 || m > 12) return false;
  *lg = m / 2;
  *le = m - *lg;
  return true;
}
static size_t reg_smem(int m, int lt) {
  int le, lg;
  if (!reg_split(m, &le, &lg)) return 0;
  const int E = 1 << le, G = 1 << lg, T = 1 << lt;
  const int rest = T >= 32 ? 1 : 32 / T;
  const int vs = E * (G + 1) + ((rest - (E * (G + 1)) % 32) % 32 + 32) % 32;
  return (size_t)T * vs * 4;
}

// The dynamic shared-memory limit is raised once per kernel instantiation (the
// once-flag lives in each launcher instantiation; all instantiations share one
// function-pointer type) to the same value, so concurrent contexts never race.
constexpr int kDftRegSmemMax = 128 * 1024;  // plans keep register-pass tiles within this
template <typename K>
static void raise_smem(K kernel) {
  // the TMA-staged pass adds its mbarrier (and up to one padding word) past the tile
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kDftRegSmemMax + 16);
}

template <int LE, int LG, int LT>
static void launch_cols_reg(dim3 grid, size_t smem, cudaStream_t st, const uint32_t* x, uint32_t* y, int log_l,
                            int log_h2, int log_h, int ls, const DftTables& t) {
  static std::once_flag once;
  std::call_once(once, [] { raise_smem(k_dft_cols_reg<LE, LG, LT>); });
  k_dft_cols_reg<LE, LG, LT><<<grid, 1 << (LG + LT), smem, st>>>(x, y, log_l, log_h2, log_h, ls, t.tw_sh, t.tw_lo,
                                                                  t.tw_hi);
}
template <int LE, int LG, int LT>
static void launch_rows_reg(dim3 grid, size_t smem, cudaStream_t st, const uint32_t* y, uint32_t* out, int log_h1,
                            int log_h, int log_w, int ls, const DftTables& t, const CUtensorMap* tm) {
  if (tm) {
    static std::once_flag once;
    std::call_once(once, [] { raise_smem(k_dft_rows_reg<LE, LG, LT, true>); });
    constexpr int E = 1 << LE, G = 1 << LG, T = 1 << LT;
    const size_t bytes = (size_t)dftreg::xwords(T, dftreg::vstride<E, G>(T >= 32 ? 1 : 32 / T)) * 4 + 8;
    k_dft_rows_reg<LE, LG, LT, true>
        <<<grid, 1 << (LG + LT), bytes, st>>>(y, out, log_h1, log_h, log_w, ls, t.tw_sh, *tm, t.err);
    return;
  }
  static std::once_flag once;
  std::call_once(once, [] { raise_smem(k_dft_rows_reg<LE, LG, LT>); });
  k_dft_rows_reg<LE, LG, LT><<<grid, 1 << (LG + LT), smem, st>>>(y, out, log_h1, log_h, log_w, ls, t.tw_sh,
                                                                  CUtensorMap{}, nullptr);
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor map of pass 2's input for the TMA-staged kernel: the scratch array
// as `cols` element columns of H << ls words, viewed as (256 words, (H << ls)
// / 256 rows, cols), boxes of (256, (N << ls) / 256, T >> ls). False when the
// shape does not fit the copy engine's rules (the plain loads run instead).
// Encoding is a driver call that costs far more than a launch, so the maps of
// the last few (address, shape) keys are kept per host thread (a context's
// scratch array usually comes back at the same address from its pool).
static bool rows_tensor_map(CUtensorMap* tm, const uint32_t* y, int log_h, int ls, int log_cols, int log_n,
                            int log_t) {
  struct Entry {
    const uint32_t* y;
    int key;
    CUtensorMap map;
  };
  constexpr int kEntries = 8;
  thread_local Entry cache[kEntries] = {};
  thread_local int next = 0;
  const int key = 1 + (log_h | ls << 5 | log_cols << 7 | log_n << 12 | log_t << 16);
  for (const Entry& e : cache)
    if (e.key == key && e.y == y) {
      *tm = e.map;
      return true;
    }
  const auto enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)y & 15u) != 0u || log_h + ls < 8 || log_n + ls < 8 || log_t < ls) return false;
  const cuuint64_t dims[3] = {256u, (cuuint64_t)1 << (log_h + ls - 8), (cuuint64_t)1 << log_cols};
  const cuuint64_t strides[2] = {1024u, (cuuint64_t)4 << (log_h + ls)};
  const cuuint32_t box[3] = {256u, 1u << (log_n + ls - 8), 1u << (log_t - ls)};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  if (enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, const_cast<uint32_t*>(y), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  cache[next] = Entry{y, key, *tm};
  next = (next + 1) % kEntries;
  return true;
}

// supported (m, lt): pass 1 lt in {2, 3, 4}, pass 2 lt in {0, .., 4}
#define WK_REG_CASES(F, m, lt, ...)                                      \
  switch (m * 16 + lt) {                                                 \
    case 8 * 16 + 0: F<4, 4, 0>(__VA_ARGS__); break;                     \
    case 8 * 16 + 1: F<4, 4, 1>(__VA_ARGS__); break;                     \
    case 8 * 16 + 2: F<4, 4, 2>(__VA_ARGS__); break;                     \
    case 8 * 16 + 3: F<4, 4, 3>(__VA_ARGS__); break;                     \
    case 8 * 16 + 4: F<4, 4, 4>(__VA_ARGS__); break;                     \
    case 9 * 16 + 0: F<5, 4, 0>(__VA_ARGS__); break;                     \
    case 9 * 16 + 1: F<5, 4, 1>(__VA_ARGS__); break;                     \
    case 9 * 16 + 2: F<5, 4, 2>(__VA_ARGS__); break;                     \
    case 9 * 16 + 3: F<5, 4, 3>(__VA_ARGS__); break;                     \
    case 9 * 16 + 4: F<5, 4, 4>(__VA_ARGS__); break;                     \
    case 10 * 16 + 0: F<5, 5, 0>(__VA_ARGS__); break;                    \
    case 10 * 16 + 1: F<5, 5, 1>(__VA_ARGS__); break;                    \
    case 10 * 16 + 2: F<5, 5, 2>(__VA_ARGS__); break;                    \
    case 10 * 16 + 3: F<5, 5, 3>(__VA_ARGS__); break;                    \
    case 10 * 16 + 4: F<5, 5, 4>(__VA_ARGS__); break;                    \
    case 11 * 16 + 0: F<6, 5, 0>(__VA_ARGS__); break;                    \
    case 11 * 16 + 1: F<6, 5, 1>(__VA_ARGS__); break;                    \
    case 11 * 16 + 2: F<6, 5, 2>(__VA_ARGS__); break;                    \
    case 11 * 16 + 3: F<6, 5, 3>(__VA_ARGS__); break;                    \
    case 11 * 16 + 4: F<6, 5, 4>(__VA_ARGS__); break;                    \
    case 12 * 16 + 0: F<6, 6, 0>(__VA_ARGS__); break;                    \
    case 12 * 16 + 1: F<6, 6, 1>(__VA_ARGS__); break;                    \
    case 12 * 16 + 2: F<6, 6, 2>(__VA_ARGS__); break;                    \
    case 12 * 16 + 3: F<6, 6, 3>(__VA_ARGS__); break;                    \
    default: break;                                                      \
  }

// threads of a register pass of length 2^m with 2^lt vectors per CTA
static int reg_threads(int m, int lt) {
  int le, lg;
  if (!reg_split(m, &le, &lg)) return 0;
  return 1 << (lg + lt);
}

static int pow2_clamp(long v, int lo, int hi) {
  int r = lo;
  while ((long)r * 2 <= v && r * 2 <= hi) r *= 2;
  return r;
}
static int log2i(int v) {
  int r = 0;
  while ((1 << r) < v) r++;
  return r;
}

// Dynamic shared memory limits are per-kernel process-wide attributes: they
// are raised once to the largest size any launch uses and never lowered, so
// launches from concurrent contexts cannot race a smaller setting.
constexpr size_t kDftTwBytes = 2048 * 4;
constexpr size_t kDftTileMax = 128 * 1024;
constexpr size_t kDftSmemMax = kDftTwBytes + kDftTileMax;
constexpr size_t kSelectSmemMax = 160 * 1024;
template <int R>
__global__ void k_add_select(ef* __restrict__ w, size_t N, int lo_bits, const uint32_t* __restrict__ pow_lo,
                             const uint32_t* __restrict__ pow_hi, const ef* __restrict__ g, int m, int hi_bits);
static std::once_flag g_attr_once;
static void init_smem_attributes() {
  std::call_once(g_attr_once, [] {
    cudaFuncSetAttribute(k_dft_cols<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDftSmemMax);
    cudaFuncSetAttribute(k_dft_cols<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDftSmemMax);
    cudaFuncSetAttribute(k_dft_rows<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDftSmemMax);
    cudaFuncSetAttribute(k_dft_rows<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDftSmemMax);
    cudaFuncSetAttribute(k_dft_coset<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDftSmemMax);
    cudaFuncSetAttribute(k_dft_coset<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDftSmemMax);
    cudaFuncSetAttribute(k_add_select<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSelectSmemMax);
    cudaFuncSetAttribute(k_add_select<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSelectSmemMax);
  });
}

static bool dft_threads_ok(int t) { return t == 128 || t == 256 || t == 512; }

// Tile bytes of one pass: 2^log_t vectors of 2^log_len elements.
static size_t dft_tile_bytes(int log_t, int log_len, int lanes) { return ((size_t)4 * lanes << log_t) << log_len; }

bool dft_plan_ok(const DftPlan& p, int log_chunk, int log_w, int log_blowup, int lanes) {
  if (lanes != 1 && lanes != 4) return false;
  if (log_chunk < 0 || log_blowup < 0 || log_w < 0 || log_w > 15) return false;
  const int log_h = log_chunk + log_blowup;
  if (log_h > 24 || (!p.reg1 && !dft_threads_ok(p.threads1))) return false;
  if (p.log_h2 == 0) {  // one pass
    if (p.reg1 || p.reg2) return false;
    return log_chunk <= 12 && p.log_t1 >= 0 && p.log_t1 <= log_w &&
           dft_tile_bytes(p.log_t1, log_chunk, lanes) <= kDftTileMax;
  }
  const int log_h1 = log_h - p.log_h2;
  if (p.log_h2 < 1 || p.log_h2 > 12 || p.log_h2 > log_chunk || log_h1 < 0 || log_h1 > 12) return false;
  // register passes count their tiles in words (4 per extension element)
  const int ls = lanes == 4 ? 2 : 0;
  if (p.reg1) {  // register pass 1: 2^8..2^12 points, 4..16 word columns per CTA
    if (p.log_t1 < 2 || p.log_t1 > 4 || p.log_t1 > p.log_h2 + ls || p.threads1 != reg_threads(log_h1, p.log_t1) ||
        p.threads1 == 0 || reg_smem(log_h1, p.log_t1) > (size_t)kDftRegSmemMax)
      return false;
  } else if (p.log_t1 < 0 || p.log_t1 > p.log_h2 || dft_tile_bytes(p.log_t1, log_h1, lanes) > kDftTileMax) {
    return false;
  }
  if (p.reg2 < 0 || p.reg2 > 2 || p.reg1 < 0 || p.reg1 > 1) return false;
  if (p.reg2) {  // register pass 2: 2^8..2^12 points, 1..16 word columns per CTA (4..16 for extensions)
    if (p.log_t2 < ls || p.log_t2 > 4 || p.log_t2 > log_w + ls || p.threads2 != reg_threads(p.log_h2, p.log_t2) ||
        p.threads2 == 0 || reg_smem(p.log_h2, p.log_t2) > (size_t)kDftRegSmemMax)
      return false;
  } else if (p.log_t2 < 0 || p.log_t2 > log_w || !dft_threads_ok(p.threads2) ||
             dft_tile_bytes(p.log_t2, p.log_h2, lanes) > kDftTileMax) {
    return false;
  }
  return true;
}

DftPlan dft_default_plan(int log_chunk, int log_w, int log_blowup, int lanes) {
  const long budget = 64 * 1024;
  const long ebytes = 4 * lanes;
  const int W = 1 << log_w;
  const int log_h = log_chunk + log_blowup;
  DftPlan p{};
  p.threads1 = p.threads2 = 256;
  p.reg1 = p.reg2 = 0;
  const int max_single = lanes == 1 ? 12 : 11;
  if (log_chunk <= max_single) {
    p.log_h2 = 0;
    p.log_t1 = log2i(pow2_clamp(budget / ((long)ebytes << log_chunk), 1, W));
    return p;
  }
  int log_h2 = lanes == 1 ? 11 : 10;
  if (log_h - log_h2 > 12) log_h2 = log_h - 12;
  const int log_h1 = log_h - log_h2;
  p.log_h2 = log_h2;
  int tile = pow2_clamp(budget / ((long)ebytes << log_h1), 1, lanes == 1 ? 16 : 8);
  if (tile > (1 << log_h2)) tile = 1 << log_h2;
  p.log_t1 = log2i(tile);
  p.log_t2 = log2i(pow2_clamp(budget / ((long)ebytes << log_h2), 1, W));
  return p;
}

// Candidates: the one-pass kernel when the chunk fits, and every four-step
// split with both passes at least 2^4 long; per pass, tiles of 8 KiB to 128 KiB
// (at most 32 vectors in pass 1, whose global accesses are tile-wide) at 256
// and 512 threads. The default plan is always included.
void dft_candidates(int log_chunk, int log_w, int log_blowup, int lanes, DftPlan* out, int* count, int cap) {
  int n = 0;
  auto push = [&](const DftPlan& p) {
    if (n < cap && dft_plan_ok(p, log_chunk, log_w, log_blowup, lanes)) out[n++] = p;
  };
  push(dft_default_plan(log_chunk, log_w, log_blowup, lanes));
  const int log_h = log_chunk + log_blowup;
  const int threads[2] = {256, 512};
  auto tile_ok = [&](int log_t, int log_len) {
    const size_t b = dft_tile_bytes(log_t, log_len, lanes);
    return b >= 8 * 1024 || log_t == 0;
  };
  if (log_chunk <= 12) {
    for (int lt = 0; lt <= log_w; lt++)
      for (int th : threads)
        if (tile_ok(lt, log_chunk)) push(DftPlan{0, lt, th, 0, 256, 0, 0});
  }
  for (int h2 = 4; h2 <= 12; h2++) {
    const int h1 = log_h - h2;
    if (h1 < 4 || h1 > 12 || h2 > log_chunk) continue;
    for (int t1 = 0; t1 <= 5 && t1 <= h2; t1++)
      for (int th1 : threads)
        if (tile_ok(t1, h1)) push(DftPlan{h2, t1, th1, 0, 256, 0, 0});
    for (int t2 = 0; t2 <= log_w; t2++)
      for (int th2 : threads)
        if (tile_ok(t2, h2)) push(DftPlan{h2, 0, 256, t2, th2, 0, 0});
    for (int t1 = 2; t1 <= 4; t1++) push(DftPlan{h2, t1, reg_threads(h1, t1), 0, 256, 1, 0});
    for (int t2 = 0; t2 <= 4; t2++) push(DftPlan{h2, 0, 256, t2, reg_threads(h2, t2), 0, 1});
    for (int t2 = 0; t2 <= 4; t2++) push(DftPlan{h2, 0, 256, t2, reg_threads(h2, t2), 0, 2});
  }
  *count = n;
}

cudaError_t dft_batch(const uint32_t* in, uint32_t* out, uint32_t* scratch, int log_chunk, int log_w,
                      int log_blowup, int lanes, const DftTables& t, const DftPlan& plan, int passes,
                      cudaStream_t st, int col0, int ncols) {
  if (!dft_plan_ok(plan, log_chunk, log_w, log_blowup, lanes)) return cudaErrorInvalidValue;
  init_smem_attributes();
  const int log_h = log_chunk + log_blowup;
  int W = 1 << log_w;
  if (ncols > 0) {
    // a column range of pass 1 only: chunk j reads in + j * chunk and writes
    // scratch + j * height, so the range is a pointer offset and a grid height
    if (passes != 1 || plan.log_h2 == 0 || col0 < 0 || col0 + ncols > W) return cudaErrorInvalidValue;
    in += ((size_t)col0 * lanes) << log_chunk;
    scratch += ((size_t)col0 * lanes) << log_h;
    W = ncols;
  }
  if (plan.log_h2 == 0) {
    const int jt = 1 << plan.log_t1;
    const size_t smem = kDftTwBytes + dft_tile_bytes(plan.log_t1, log_chunk, lanes);
    dim3 grid(1u << log_blowup, W / jt);
    if (lanes == 1)
      k_dft_coset<1><<<grid, plan.threads1, smem, st>>>(in, out, log_chunk, log_blowup, log_w, plan.log_t1,
                                                        t.tw_stage, t.tw_lo, t.tw_hi);
    else
      k_dft_coset<4><<<grid, plan.threads1, smem, st>>>(reinterpret_cast<const uint4*>(in),
                                                        reinterpret_cast<uint4*>(out), log_chunk, log_blowup, log_w,
                                                        plan.log_t1, t.tw_stage, t.tw_lo, t.tw_hi);
    LAUNCH_DONE();
  }
  const int log_h2 = plan.log_h2, log_h1 = log_h - log_h2;
  const int H1 = 1 << log_h1, H2 = 1 << log_h2;
  const int ls = lanes == 4 ? 2 : 0;  // register passes run extension data as 4 base columns per element
  if ((passes & 1) && plan.reg1) {
    const int tile = 1 << plan.log_t1;
    dim3 grid((H2 << ls) / tile, W);
    WK_REG_CASES(launch_cols_reg, log_h1, plan.log_t1, grid, reg_smem(log_h1, plan.log_t1), st, in, scratch,
                 log_chunk + ls, log_h2 + ls, log_h + ls, ls, t)
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  } else if (passes & 1) {
    const int tile = 1 << plan.log_t1;
    const size_t smem = kDftTwBytes + dft_tile_bytes(plan.log_t1, log_h1, lanes);
    dim3 grid(H2 / tile, W);
    if (lanes == 1)
      k_dft_cols<1><<<grid, plan.threads1, smem, st>>>(in, scratch, log_chunk, log_h1, log_h2, log_h, plan.log_t1,
                                                       t.tw_stage, t.tw_lo, t.tw_hi);
    else
      k_dft_cols<4><<<grid, plan.threads1, smem, st>>>(reinterpret_cast<const uint4*>(in),
                                                       reinterpret_cast<uint4*>(scratch), log_chunk, log_h1, log_h2,
                                                       log_h, plan.log_t1, t.tw_stage, t.tw_lo, t.tw_hi);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if ((passes & 2) && plan.reg2) {
    const int jt = 1 << plan.log_t2;
    dim3 grid(H1, (W << ls) / jt);
    CUtensorMap tm;
    const bool tma = plan.reg2 == 2 && rows_tensor_map(&tm, scratch, log_h, ls, log_w, log_h2, plan.log_t2);
    WK_REG_CASES(launch_rows_reg, log_h2, plan.log_t2, grid, reg_smem(log_h2, plan.log_t2), st, scratch, out,
                 log_h1, log_h, log_w + ls, ls, t, tma ? &tm : nullptr)
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  } else if (passes & 2) {
    const int jt = 1 << plan.log_t2;
    const size_t smem = kDftTwBytes + dft_tile_bytes(plan.log_t2, log_h2, lanes);
    dim3 grid(H1, W / jt);
    if (lanes == 1)
      k_dft_rows<1><<<grid, plan.threads2, smem, st>>>(scratch, out, log_h1, log_h2, log_h, log_w, plan.log_t2,
                                                       t.tw_stage);
    else
      k_dft_rows<4><<<grid, plan.threads2, smem, st>>>(reinterpret_cast<const uint4*>(scratch),
                                                       reinterpret_cast<uint4*>(out), log_h1, log_h2, log_h, log_w,
                                                       plan.log_t2, t.tw_stage);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}


// ---------------------------------------------------------------------------
// Merkle tree and proof of work: the kernels live in merkle.cuh, built once per
// Poseidon2 external block (merkle_mds.cu, merkle_hl.cu); these pick the form
// that the constants carry. A context holds one form for both widths.
// ---------------------------------------------------------------------------

Shape merkle_leaf_default() { return Shape{256, 16, 0}; }
Shape merkle_node_default() { return Shape{256, 16, 0}; }

cudaError_t merkle_leaves(const uint32_t* rows, int log_h, int row_words, int leaf_hash, uint32_t* digests,
                          const P2Consts& p16, const P2Consts& p24, Shape leaf, cudaStream_t st) {
  if (p16.mat != p24.mat) return cudaErrorInvalidValue;
  if (p16.mat == (uint32_t)p2::kMatHl)
    return merkle_leaves_m<p2::kMatHl>(rows, log_h, row_words, leaf_hash, digests, p16, p24, leaf, st);
  return merkle_leaves_m<p2::kMatMds>(rows, log_h, row_words, leaf_hash, digests, p16, p24, leaf, st);
}

cudaError_t merkle_many(const TreeDesc* d_desc, const unsigned long long* d_level_first, int count, int max_log_h,
                        const unsigned long long* level_totals, int row_words, int leaf_hash, const P2Consts& p16,
                        const P2Consts& p24, unsigned* counter, uint32_t* d_roots, cudaStream_t st) {
  if (p16.mat != p24.mat) return cudaErrorInvalidValue;
  if (p16.mat == (uint32_t)p2::kMatHl)
    return merkle_many_m<p2::kMatHl>(d_desc, d_level_first, count, max_log_h, level_totals, row_words, leaf_hash,
                                     p16, p24, counter, d_roots, st);
  return merkle_many_m<p2::kMatMds>(d_desc, d_level_first, count, max_log_h, level_totals, row_words, leaf_hash, p16,
                                    p24, counter, d_roots, st);
}

cudaError_t merkle_upper(int log_h, uint32_t* digests, const P2Consts& p16, Shape node, unsigned* counter,
                         uint32_t* mail, uint32_t seq, int* posted, cudaStream_t st) {
  if (p16.mat == (uint32_t)p2::kMatHl)
    return merkle_upper_m<p2::kMatHl>(log_h, digests, p16, node, counter, mail, seq, posted, st);
  return merkle_upper_m<p2::kMatMds>(log_h, digests, p16, node, counter, mail, seq, posted, st);
}

__global__ void k_grind_init(uint32_t* result, uint32_t* counter, uint32_t* done) {
  *result = kb::P;
  *counter = 0u;
  *done = 0u;
}

cudaError_t grind_reset(uint32_t* result, uint32_t* counter, uint32_t* done, cudaStream_t st) {
  k_grind_init<<<1, 1, 0, st>>>(result, counter, done);
  LAUNCH_DONE();
}

cudaError_t grind(const uint32_t* state, const uint32_t* in, int in_len, int bits, uint64_t limit,
                  uint32_t* result, uint32_t* counter, uint32_t* done, uint32_t* mail, uint32_t seq,
                  const P2Consts& p16, cudaStream_t st, const uint32_t* cp_dev, uint32_t* res_out, DevChal* ch,
                  ef* r_out, uint32_t* err, int window) {
  if (p16.mat == (uint32_t)p2::kMatHl)
    return grind_m<p2::kMatHl>(state, in, in_len, bits, limit, result, counter, done, mail, seq, p16, st, cp_dev,
                               res_out, ch, r_out, err, window);
  return grind_m<p2::kMatMds>(state, in, in_len, bits, limit, result, counter, done, mail, seq, p16, st, cp_dev,
                              res_out, ch, r_out, err, window);
}

cudaError_t sumcheck_round_tr(ef* f, ef* w, size_t q, int fold, ef r, ef* partials, unsigned* counter, ef* out,
                              const ef* r_dev, DevChal* ch, const DevChal* init, uint32_t* err, int grind_next,
                              uint32_t* cp_out, ef* r_out, const P2Consts& p16, cudaStream_t st) {
  if (p16.mat == (uint32_t)p2::kMatHl)
    return sumcheck_round_tr_m<p2::kMatHl>(f, w, q, fold, r, partials, counter, out, r_dev, ch, init, err, grind_next,
                                           cp_out, r_out, p16, st);
  return sumcheck_round_tr_m<p2::kMatMds>(f, w, q, fold, r, partials, counter, out, r_dev, ch, init, err, grind_next,
                                          cp_out, r_out, p16, st);
}

cudaError_t merkle_build(const uint32_t* rows, int log_h, int row_words, int leaf_hash, uint32_t* digests,
                         const P2Consts& p16, const P2Consts& p24, unsigned* counter, cudaStream_t st) {
  cudaError_t e = merkle_leaves(rows, log_h, row_words, leaf_hash, digests, p16, p24, merkle_leaf_default(), st);
  if (e != cudaSuccess) return e;
  return merkle_upper(log_h, digests, p16, merkle_node_default(), counter, nullptr, 0u, nullptr, st);
}

// Mmcs::open_batch gather (src/whir/prover/mod.rs:248-300, 378-401)
__device__ __forceinline__ void open_one(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ digests,
                                         int log_h, int row_words, int q, uint64_t i, uint32_t* __restrict__ rows_out,
                                         uint32_t* __restrict__ paths_out) {
  for (int w = threadIdx.x; w < row_words; w += blockDim.x)
    rows_out[(size_t)q * row_words + w] = rows[i * row_words + w];
  for (int k = threadIdx.x; k < log_h * 8; k += blockDim.x) {
    const int l = k >> 3, c = k & 7;
    size_t off = 0, n = (size_t)1 << log_h;
    for (int m = 0; m < l; m++) {
      off += n;
      n >>= 1;
    }
    const size_t sib = (size_t)((i >> l) ^ 1u);
    paths_out[((size_t)q * log_h + l) * 8 + c] = digests[(off + sib) * 8 + c];
  }
}

__global__ void k_merkle_open(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ digests, int log_h,
                              int row_words, const uint64_t* __restrict__ idx, uint32_t* __restrict__ rows_out,
                              uint32_t* __restrict__ paths_out) {
  open_one(rows, digests, log_h, row_words, blockIdx.x, idx[blockIdx.x], rows_out, paths_out);
}

// the indices in the launch's parameter block
struct OpenIdx {
  uint64_t i[kOpenParamIdx];
};
__global__ void k_merkle_open_p(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ digests, int log_h,
                                int row_words, const __grid_constant__ OpenIdx idx, uint32_t* __restrict__ rows_out,
                                uint32_t* __restrict__ paths_out) {
  open_one(rows, digests, log_h, row_words, blockIdx.x, idx.i[blockIdx.x], rows_out, paths_out);
}

cudaError_t merkle_open(const uint32_t* rows, const uint32_t* digests, int log_h, int row_words,
                        const uint64_t* d_idx, int count, uint32_t* d_rows_out, uint32_t* d_paths_out,
                        cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  k_merkle_open<<<count, 128, 0, st>>>(rows, digests, log_h, row_words, d_idx, d_rows_out, d_paths_out);
  LAUNCH_DONE();
}

cudaError_t merkle_open_host_idx(const uint32_t* rows, const uint32_t* digests, int log_h, int row_words,
                                 const uint64_t* h_idx, int count, uint32_t* d_rows_out, uint32_t* d_paths_out,
                                 cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  if (count > kOpenParamIdx) return cudaErrorInvalidValue;
  OpenIdx ix;
  memcpy(ix.i, h_idx, (size_t)count * 8);
  k_merkle_open_p<<<count, 128, 0, st>>>(rows, digests, log_h, row_words, ix, d_rows_out, d_paths_out);
  LAUNCH_DONE();
}

// ---------------------------------------------------------------------------
// eq tables (EvaluationsList::new_from_point, src/poly/evals.rs:312-320, and
// the split tables of evals.rs:254-295 / svo.rs:387-403)
// ---------------------------------------------------------------------------

__global__ void k_eq_small(const __grid_constant__ EqPoint pt, ef* out) {
  const size_t n = (size_t)1 << pt.h;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n; x += (size_t)gridDim.x * blockDim.x) {
    ef acc = pt.scale;
    for (int j = 0; j < pt.h; j++) {
      const ef& z = pt.z[j];
      const bool bit = (x >> (pt.h - 1 - j)) & 1;
      acc = kb::ef_mul(acc, bit ? z : kb::ef_sub(kb::ef_one(), z));
    }
    st_ef(out + x, acc);
  }
}

// two eq tables in one launch (the hi and lo tables of a split point)
__global__ void k_eq_pair(const __grid_constant__ EqPoint p1, ef* out1, const __grid_constant__ EqPoint p2, ef* out2) {
  const size_t n1 = (size_t)1 << p1.h, n2 = (size_t)1 << p2.h;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n1 + n2; i += (size_t)gridDim.x * blockDim.x) {
    const EqPoint& pt = i < n1 ? p1 : p2;
    const size_t x = i < n1 ? i : i - n1;
    ef acc = pt.scale;
    for (int j = 0; j < pt.h; j++) {
      const ef& z = pt.z[j];
      const bool bit = (x >> (pt.h - 1 - j)) & 1;
      acc = kb::ef_mul(acc, bit ? z : kb::ef_sub(kb::ef_one(), z));
    }
    st_ef((i < n1 ? out1 : out2) + x, acc);
  }
}

cudaError_t eq_table_pair(const EqPoint& p1, ef* out1, const EqPoint& p2, ef* out2, cudaStream_t st) {
  if (p1.h < 0 || p1.h > 20 || p2.h < 0 || p2.h > 20) return cudaErrorInvalidValue;
  const size_t n = ((size_t)1 << p1.h) + ((size_t)1 << p2.h);
  k_eq_pair<<<grid_for(n, 256), 256, 0, st>>>(p1, out1, p2, out2);
  LAUNCH_DONE();
}

// several eq tables in one launch (the split tables of several points)
__global__ void k_eq_multi(const __grid_constant__ EqMulti m) {
  size_t total = 0;
  for (int t = 0; t < m.count; t++) total += (size_t)1 << m.h[t];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    int t = 0;
    size_t x = i;
    while (x >= ((size_t)1 << m.h[t])) {
      x -= (size_t)1 << m.h[t];
      t++;
    }
    const int h = m.h[t];
    const ef* z = m.z + m.zoff[t];
    ef acc = m.scale[t];
    for (int j = 0; j < h; j++) {
      const bool bit = (x >> (h - 1 - j)) & 1;
      acc = kb::ef_mul(acc, bit ? z[j] : kb::ef_sub(kb::ef_one(), z[j]));
    }
    st_ef(m.out[t] + x, acc);
  }
}

cudaError_t eq_tables_multi(const EqMulti& m, cudaStream_t st) {
  if (m.count < 1 || m.count > kEqMultiTables) return cudaErrorInvalidValue;
  size_t n = 0;
  for (int t = 0; t < m.count; t++) {
    if (m.h[t] < 0 || m.h[t] > kEqMultiCoords || m.zoff[t] < 0 ||
        m.zoff[t] + m.h[t] > kEqMultiTables * kEqMultiCoords || !m.out[t])
      return cudaErrorInvalidValue;
    n += (size_t)1 << m.h[t];
  }
  k_eq_multi<<<grid_for(n, 256), 256, 0, st>>>(m);
  LAUNCH_DONE();
}

cudaError_t eq_table_small(const EqPoint& pt, ef* out, cudaStream_t st) {
  if (pt.h < 0 || pt.h > 20) return cudaErrorInvalidValue;
  const size_t n = (size_t)1 << pt.h;
  k_eq_small<<<grid_for(n, 256), 256, 0, st>>>(pt, out);
  LAUNCH_DONE();
}

__global__ void k_eq_outer(const ef* __restrict__ hi, const ef* __restrict__ lo, int lo_bits, size_t n,
                           ef* __restrict__ out) {
  const size_t mask = ((size_t)1 << lo_bits) - 1;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n; x += (size_t)gridDim.x * blockDim.x)
    st_ef(out + x, kb::ef_mul(ld_ef(hi + (x >> lo_bits)), ld_ef(lo + (x & mask))));
}

cudaError_t eq_outer(const ef* hi, const ef* lo, int lo_bits, size_t n, ef* out, cudaStream_t st) {
  k_eq_outer<<<grid_for(n, 256), 256, 0, st>>>(hi, lo, lo_bits, n, out);
  LAUNCH_DONE();
}

// ---------------------------------------------------------------------------
// Split-eq dot products: multilinear evaluation (evaluate_hypercube_base/_ext,
// src/poly/evals.rs:334-366, 648-738) and the SVO partial evaluations
// (SplitEqInner::partial_evals, src/sumcheck/svo.rs:465-502). Each thread
// keeps one low index xl and accumulates f * hi[xh] over its xh, multiplying
// by lo[xl] once at the end.
// ---------------------------------------------------------------------------

constexpr int DOT_CTA = 256;

// Block sum of each thread's `total`; the last CTA to finish (atomic counter,
// no waiting) adds up every segment's partial sums into out[segment] and, with
// `mail`, posts them to the mailbox. If *poison is set (a device wait in the
// caller gave up), the results are 0xffffffff, which no field element is.
__device__ __forceinline__ void dot_finish(ef total, ef* __restrict__ partials, unsigned* __restrict__ counter,
                                           ef* __restrict__ out, uint32_t* mail, uint32_t seq,
                                           const uint32_t* poison) {
  __shared__ ef sh[1][32];
  __shared__ bool s_last;
  ef v[1] = {total};
  block_sum<1>(v, sh);
  // the last CTA to finish adds up every segment's partial sums
  const unsigned nblocks = gridDim.x * gridDim.y;
  if (threadIdx.x == 0) {
    partials[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = v[0];
    __threadfence();
    s_last = atomicAdd(counter, 1u) == nblocks - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const bool bad = poison && *reinterpret_cast<volatile const uint32_t*>(poison) != 0u;
  const unsigned segs = gridDim.y, nb = gridDim.x;
  if (segs >= 8 && DOT_CTA % segs == 0 && DOT_CTA / segs <= 32) {
    // one group of DOT_CTA / segs lanes per segment, all segments at once
    const unsigned gsz = DOT_CTA / segs, lane = threadIdx.x % gsz, sg = threadIdx.x / gsz;
    ef a = kb::ef_zero();
    for (unsigned b = lane; b < nb; b += gsz) {
      const uint4 x = __ldcg(reinterpret_cast<const uint4*>(partials + (size_t)sg * nb + b));
      a = kb::ef_add(a, ef{{x.x, x.y, x.z, x.w}});
    }
    for (unsigned o = gsz / 2; o >= 1; o >>= 1)
#pragma unroll
      for (int c = 0; c < 4; c++) a.c[c] = kb::add(a.c[c], __shfl_xor_sync(0xffffffffu, a.c[c], o));
    if (bad) a = ef{{0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu}};
    if (lane == 0) {
      out[sg] = a;
      if (mail) {
        for (int c = 0; c < 4; c++) reinterpret_cast<volatile uint32_t*>(mail)[4 * sg + c] = a.c[c];
        __threadfence_system();
      }
    }
    __syncthreads();
  } else {
    for (unsigned s2 = 0; s2 < segs; s2++) {
      ef a[1] = {kb::ef_zero()};
      for (unsigned b = threadIdx.x; b < nb; b += blockDim.x) {
        const uint4 x = __ldcg(reinterpret_cast<const uint4*>(partials + (size_t)s2 * nb + b));
        a[0] = kb::ef_add(a[0], ef{{x.x, x.y, x.z, x.w}});
      }
      block_sum<1>(a, sh);
      if (bad) a[0] = ef{{0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu}};
      if (threadIdx.x == 0) {
        out[s2] = a[0];
        if (mail)
          for (int c = 0; c < 4; c++) reinterpret_cast<volatile uint32_t*>(mail)[4 * s2 + c] = a[0].c[c];
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    *counter = 0u;
    if (mail) {
      __threadfence_system();
      reinterpret_cast<volatile uint32_t*>(mail)[kMailWords] = seq;
    }
  }
}

template <int EXT>
__global__ void __launch_bounds__(DOT_CTA) k_dot_split(const uint32_t* __restrict__ f, int m_bits,
                                                        const ef* __restrict__ hi, const ef* __restrict__ lo,
                                                        int lo_bits, int wide, ef* __restrict__ partials,
                                                        unsigned* __restrict__ counter, ef* __restrict__ out,
                                                        uint32_t* mail, uint32_t seq) {
  const size_t M = (size_t)1 << m_bits;
  const int seg = blockIdx.y;
  const uint32_t lomask = (1u << lo_bits) - 1;
  ef total = kb::ef_zero();
  if (!EXT && wide) {
    // four consecutive base entries per thread and step (one 16-byte load):
    // they share their high index (lo_bits >= 2), and the stride is a multiple
    // of 2^lo_bits, so each of the four keeps its low index across steps. Four
    // steps' loads are issued together; each accumulator then takes four
    // products (< 4p^2 < 2^64) and is reduced once.
    const uint32_t x0 = 4u * threadIdx.x;
    ef acc[4];
    uint64_t t[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++) acc[j] = kb::ef_zero();
    const uint4* f4 = reinterpret_cast<const uint4*>(f + (size_t)seg * M);
    const size_t S = (size_t)gridDim.x * DOT_CTA * 4;
    size_t x = (size_t)blockIdx.x * DOT_CTA * 4 + x0;
    for (; x + 3 * S < M; x += 4 * S) {
      uint4 v[4];
      ef h[4];
#pragma unroll
      for (int u = 0; u < 4; u++) v[u] = __ldg(f4 + ((x + u * S) >> 2));
#pragma unroll
      for (int u = 0; u < 4; u++) h[u] = ld_ef(hi + ((x + u * S) >> lo_bits));
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int c = 0; c < 4; c++) t[j][c] = 0;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint32_t e[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
          for (int c = 0; c < 4; c++) t[j][c] += (uint64_t)h[u].c[c] * e[j];
      }
#pragma unroll
      for (int j = 0; j < 4; j++)
        acc[j] = kb::ef_add(acc[j], ef{{kb::reduce_wide(t[j][0]), kb::reduce_wide(t[j][1]),
                                        kb::reduce_wide(t[j][2]), kb::reduce_wide(t[j][3])}});
    }
    for (; x < M; x += S) {
      const uint4 v = __ldg(f4 + (x >> 2));
      const ef h = ld_ef(hi + (x >> lo_bits));
      acc[0] = kb::ef_add(acc[0], kb::ef_mul_base(h, v.x));
      acc[1] = kb::ef_add(acc[1], kb::ef_mul_base(h, v.y));
      acc[2] = kb::ef_add(acc[2], kb::ef_mul_base(h, v.z));
      acc[3] = kb::ef_add(acc[3], kb::ef_mul_base(h, v.w));
    }
#pragma unroll
    for (int j = 0; j < 4; j++) total = kb::ef_add(total, kb::ef_mul(acc[j], ld_ef(lo + ((x0 + j) & lomask))));
  } else if ((size_t)threadIdx.x < M || M >= DOT_CTA) {
    const uint32_t xl = threadIdx.x & lomask;
    ef acc = kb::ef_zero();
    kb::ef_acc lazy;
    lazy.clear();
#pragma unroll 4
    for (size_t x = (size_t)blockIdx.x * DOT_CTA + threadIdx.x; x < M; x += (size_t)gridDim.x * DOT_CTA) {
      const ef h = ld_ef(hi + (x >> lo_bits));
      if (EXT) {
        const ef v = ld_ef(reinterpret_cast<const ef*>(f) + (size_t)seg * M + x);
        acc = kb::ef_add(acc, kb::ef_mul(v, h));
      } else {
        lazy.mac(h, __ldg(f + (size_t)seg * M + x), acc);
      }
    }
    if (!EXT) lazy.fold(acc);
    total = kb::ef_mul(acc, ld_ef(lo + xl));
  }
  dot_finish(total, partials, counter, out, mail, seq, nullptr);
}

// Base-field dot product streamed through shared memory: each CTA takes a
// contiguous run of its segment in 16 KiB chunks, which one thread loads with
// bulk copies (cp.async.bulk, completion counted on an mbarrier per stage) four
// stages ahead, together with the chunk's 16 high-index eq entries, so the
// copy engine keeps the bytes in flight while every thread computes from
// shared memory. With lo_bits = 8, thread t takes the 16-byte words t + 256u
// (u < 4) of a chunk: elements 4t + 1024u + j, whose high index is entry
// (t >> 6) + 4u of the chunk's slice and whose low index (4t + j) is the same
// in every chunk.
namespace dstream {
constexpr int kCta = 256, kStages = 4, kChunk = kCta * 16;  // elements per stage
constexpr uint32_t kBytes = kChunk * 4;
constexpr int kHi = kChunk >> 8;                    // high-index entries per chunk
constexpr uint32_t kHiBytes = kHi * 16;
constexpr int kStageWords = kCta * 4 + kHi;         // 16-byte words per stage
using bulk::bar_expect;
using bulk::bar_init;
using bulk::bar_wait;
using bulk::bulk_load;
// chunk c of the segment and its high-index slice into stage buffer `buf`
__device__ __forceinline__ void load_chunk(uint4* buf, const uint32_t* src, const kb::ef* hi, unsigned c, uint64_t* b) {
  bar_expect(b, kBytes + kHiBytes);
  bulk_load(buf, src + (size_t)c * kChunk, kBytes, b);
  bulk_load(buf + kCta * 4, hi + (size_t)c * kHi, kHiBytes, b);
}
}  // namespace dstream

__global__ void __launch_bounds__(dstream::kCta) k_dot_stream(const uint32_t* __restrict__ f, int m_bits,
                                                               const ef* __restrict__ hi, const ef* __restrict__ lo,
                                                               ef* __restrict__ partials,
                                                               unsigned* __restrict__ counter, ef* __restrict__ out,
                                                               uint32_t* mail, uint32_t seq, uint32_t* err) {
  using namespace dstream;
  extern __shared__ __align__(128) uint4 stage_buf[];  // kStages * kStageWords words of 16 bytes
  __shared__ __align__(8) uint64_t full[kStages];
  const size_t M = (size_t)1 << m_bits;
  const int seg = blockIdx.y, t = threadIdx.x;
  const unsigned nch = (unsigned)(M / kChunk);
  const unsigned c0 = (unsigned)((uint64_t)nch * blockIdx.x / gridDim.x);
  const unsigned n = (unsigned)((uint64_t)nch * (blockIdx.x + 1) / gridDim.x) - c0;
  const uint32_t* src = f + (size_t)seg * M;
  if (t == 0) {
    for (int st = 0; st < kStages; st++) bar_init(&full[st]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (unsigned i = 0; i < n && i < (unsigned)kStages; i++)
      load_chunk(stage_buf + (size_t)i * kStageWords, src, hi, c0 + i, &full[i]);
  }
  __syncthreads();
  ef acc[4];
#pragma unroll
  for (int j = 0; j < 4; j++) acc[j] = kb::ef_zero();
  unsigned i = 0;
  bool bad = false;
  for (; i < n; i++) {
    const int st = (int)(i % kStages);
    const bool ok = bar_wait(&full[st], (i / kStages) & 1u);
    if (ok) {
      const uint4* b = stage_buf + (size_t)st * kStageWords;
      uint64_t acc64[4][4];
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc64[j][c] = 0;
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint4 v = b[t + kCta * u];
        const uint4 hw = b[kCta * 4 + (t >> 6) + 4 * u];
        const ef h{{hw.x, hw.y, hw.z, hw.w}};
        const uint32_t e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
          for (int c = 0; c < 4; c++) acc64[j][c] += (uint64_t)h.c[c] * e[j];  // four products < 2^64
      }
#pragma unroll
      for (int j = 0; j < 4; j++)
        acc[j] = kb::ef_add(acc[j], ef{{kb::reduce_wide(acc64[j][0]), kb::reduce_wide(acc64[j][1]),
                                        kb::reduce_wide(acc64[j][2]), kb::reduce_wide(acc64[j][3])}});
    }
    // every thread has read stage st (or the CTA gives up together)
    if (__syncthreads_or(!ok)) {
      bad = true;
      break;
    }
    if (t == 0 && i + kStages < n) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      load_chunk(stage_buf + (size_t)st * kStageWords, src, hi, c0 + i + kStages, &full[st]);
    }
  }
  if (bad && t == 0) {
    // a wait gave up: flag it, then wait (bounded again) for the copies this
    // CTA still has in flight before its shared memory is released
    atomicOr(err, 1u);
    for (unsigned k = i; k < n && k < i + kStages; k++) bar_wait(&full[k % kStages], (k / kStages) & 1u);
  }
  ef total = kb::ef_zero();
#pragma unroll
  for (int j = 0; j < 4; j++) total = kb::ef_add(total, kb::ef_mul(acc[j], ld_ef(lo + ((4u * t + j) & 255u))));
  dot_finish(total, partials, counter, out, mail, seq, err);
}

cudaError_t dot_split(const uint32_t* f, int ext, int seg_bits, int m_bits, const ef* hi, const ef* lo, int lo_bits,
                      ef* partials, unsigned* counter, ef* out, uint32_t* mail, uint32_t seq, uint32_t* err,
                      cudaStream_t st) {
  if (mail && (4 << seg_bits) > kMailWords) return cudaErrorInvalidValue;
  if (lo_bits > 8 || lo_bits > m_bits || seg_bits < 0 || seg_bits > 8) return cudaErrorInvalidValue;
  const size_t M = (size_t)1 << m_bits;
  const int segs = 1 << seg_bits;
  if (!ext && err && lo_bits == 8 && M >= (size_t)dstream::kChunk && ((uintptr_t)f & 15) == 0 &&
      ((uintptr_t)hi & 15) == 0) {
    constexpr int smem = dstream::kStages * dstream::kStageWords * 16;
    static std::once_flag once;
    static int per_sm = 1;
    std::call_once(once, [] {
      cudaFuncSetAttribute(k_dot_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      int n = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_dot_stream, dstream::kCta, smem);
      per_sm = n > 0 ? n : 1;
    });
    const size_t nch = M / dstream::kChunk;
    size_t bx = ((size_t)sm_count() * per_sm + segs - 1) / segs;
    if (bx > nch) bx = nch;
    if (bx < 1) bx = 1;
    k_dot_stream<<<dim3((unsigned)bx, segs), dstream::kCta, smem, st>>>(f, m_bits, hi, lo, partials, counter, out,
                                                                         mail, seq, err);
    LAUNCH_DONE();
  }
  const int wide = !ext && lo_bits >= 2 && M >= 4 * (size_t)DOT_CTA && ((uintptr_t)f & 15) == 0;
  // one wave of resident CTAs (the wide path holds many registers): more CTAs
  // than fit would only queue behind the first wave
  static std::once_flag resident_once;
  static int resident[2] = {1, 1};
  std::call_once(resident_once, [] {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_dot_split<0>, DOT_CTA, 0);
    resident[0] = n > 0 ? n : 1;
    n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_dot_split<1>, DOT_CTA, 0);
    resident[1] = n > 0 ? n : 1;
  });
  const int per_sm = resident[ext ? 1 : 0];
  unsigned bx = grid_for(wide ? M / 4 : M, DOT_CTA, per_sm);
  unsigned cap = (unsigned)((sm_count() * per_sm + segs - 1) / segs);
  if (bx > cap) bx = cap;
  if (bx < 1) bx = 1;
  dim3 grid(bx, segs);
  if (ext)
    k_dot_split<1><<<grid, DOT_CTA, 0, st>>>(f, m_bits, hi, lo, lo_bits, 0, partials, counter, out, mail, seq);
  else
    k_dot_split<0><<<grid, DOT_CTA, 0, st>>>(f, m_bits, hi, lo, lo_bits, wide, partials, counter, out, mail, seq);
  LAUNCH_DONE();
}

// ---------------------------------------------------------------------------
// Folding (EvaluationsList::compress / compress_ext / compress_multi_into_packed,
// src/poly/evals.rs:127-148, 382-400, 422-447)
// ---------------------------------------------------------------------------

template <int CTA>
__global__ void __launch_bounds__(CTA) k_fold_ext(ef* __restrict__ a, ef* __restrict__ b, size_t half, ef r) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < half; i += (size_t)gridDim.x * blockDim.x) {
    ef lo = ld_ef(a + i), hi = ld_ef(a + i + half);
    st_ef(a + i, kb::ef_add(lo, kb::ef_mul(kb::ef_sub(hi, lo), r)));
    if (b) {
      ef lo2 = ld_ef(b + i), hi2 = ld_ef(b + i + half);
      st_ef(b + i, kb::ef_add(lo2, kb::ef_mul(kb::ef_sub(hi2, lo2), r)));
    }
  }
}

Shape fold_default() { return Shape{256, 8, 0}; }

cudaError_t fold_ext(ef* a, ef* b, size_t half, ef r, Shape shape, cudaStream_t st) {
  if (shape.per_sm < 0 || (shape.threads != 128 && shape.threads != 256 && shape.threads != 512))
    return cudaErrorInvalidValue;
  const unsigned blocks = grid_shape(half, shape);
  if (shape.threads == 128)
    k_fold_ext<128><<<blocks, 128, 0, st>>>(a, b, half, r);
  else if (shape.threads == 256)
    k_fold_ext<256><<<blocks, 256, 0, st>>>(a, b, half, r);
  else
    k_fold_ext<512><<<blocks, 512, 0, st>>>(a, b, half, r);
  LAUNCH_DONE();
}

__global__ void k_fold_base(const uint32_t* __restrict__ f, size_t half, ef r, ef* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < half; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t lo = __ldg(f + i), hi = __ldg(f + i + half);
    ef v = kb::ef_mul_base(r, kb::sub(hi, lo));
    v.c[0] = kb::add(v.c[0], lo);
    st_ef(out + i, v);
  }
}

cudaError_t fold_base(const uint32_t* f, size_t half, ef r, ef* out, cudaStream_t st) {
  k_fold_base<<<grid_for(half, 256), 256, 0, st>>>(f, half, r, out);
  LAUNCH_DONE();
}

// Loads of four strided inputs are issued together, then their four products
// (< 4p^2 < 2^64 per coefficient) are summed and reduced once.
__global__ void k_fold_multi_base(const uint32_t* __restrict__ f, int k, size_t m,
                                  const __grid_constant__ EqSmall eqrs, ef* __restrict__ out) {
  const int K = 1 << k;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < m; x += (size_t)gridDim.x * blockDim.x) {
    ef acc = kb::ef_zero();
    int y = 0;
    for (; y + 4 <= K; y += 4) {
      uint32_t v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) v[u] = __ldg(f + (size_t)(y + u) * m + x);
      uint64_t t[4] = {0, 0, 0, 0};
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int c = 0; c < 4; c++) t[c] += (uint64_t)eqrs.v[y + u].c[c] * v[u];
      acc = kb::ef_add(acc, ef{{kb::reduce_wide(t[0]), kb::reduce_wide(t[1]), kb::reduce_wide(t[2]),
                                kb::reduce_wide(t[3])}});
    }
    for (; y < K; y++) acc = kb::ef_add(acc, kb::ef_mul_base(eqrs.v[y], __ldg(f + (size_t)y * m + x)));
    st_ef(out + x, acc);
  }
}

cudaError_t fold_multi_base(const uint32_t* f, int k, size_t m, const EqSmall& eqrs, ef* out, cudaStream_t st) {
  if (k < 0 || k > 6) return cudaErrorInvalidValue;
  k_fold_multi_base<<<grid_for(m, 256), 256, 0, st>>>(f, k, m, eqrs, out);
  LAUNCH_DONE();
}

// ---------------------------------------------------------------------------
// Sumcheck round coefficients (EvaluationsList::sumcheck_coefficients,
// src/poly/evals.rs:493-526): c0 = sum e_lo*w_lo, c2 = sum (2e_hi-e_lo)(2w_hi-w_lo)
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_sumcheck_coeffs(const ef* __restrict__ f, const ef* __restrict__ w,
                                                          size_t half, ef* __restrict__ partials) {
  __shared__ ef sh[2][32];
  ef v[2] = {kb::ef_zero(), kb::ef_zero()};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < half; i += (size_t)gridDim.x * blockDim.x) {
    const ef el = ld_ef(f + i), eh = ld_ef(f + i + half);
    const ef wl = ld_ef(w + i), wh = ld_ef(w + i + half);
    v[0] = kb::ef_add(v[0], kb::ef_mul(el, wl));
    v[1] = kb::ef_add(v[1], kb::ef_mul(kb::ef_sub(kb::ef_dbl(eh), el), kb::ef_sub(kb::ef_dbl(wh), wl)));
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v[0];
    partials[gridDim.x + blockIdx.x] = v[1];
  }
}

cudaError_t sumcheck_coeffs(const ef* f, const ef* w, size_t half, ef* partials, ef* out, cudaStream_t st) {
  const unsigned b = grid_for(half, 256, 8);
  k_sumcheck_coeffs<<<b, 256, 0, st>>>(f, w, half, partials);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sum_partials<<<2, 256, 0, st>>>(partials, (int)b, out);
  LAUNCH_DONE();
}

// One launch per sumcheck round in the prover (sumcheck_round_body); the last
// CTA also posts (c0, c2) to the mailbox when one is given, so no second
// launch is needed.
template <bool FOLD>
__global__ void __launch_bounds__(256) k_sumcheck_round(ef* __restrict__ f, ef* __restrict__ w, size_t q, ef r,
                                                         ef* __restrict__ partials, unsigned* __restrict__ counter,
                                                         ef* __restrict__ out, uint32_t* mail, uint32_t seq,
                                                         const ef* __restrict__ r_dev) {
  __shared__ ef sh[2][32];
  __shared__ bool s_last;
  ef res[2];
  if (!sumcheck_round_body<FOLD>(f, w, q, r, partials, counter, out, r_dev, res, sh, s_last)) return;
  if (threadIdx.x == 0 && mail) mail_post(mail, res[0].c, 8, seq);
}

unsigned sumcheck_round_blocks(size_t q) { return grid_for(q, 256, 8); }

cudaError_t sumcheck_round(ef* f, ef* w, size_t q, int fold, ef r, ef* partials, unsigned* counter, ef* out,
                           uint32_t* mail, uint32_t seq, cudaStream_t st, const ef* r_dev) {
  if (q == 0) return cudaErrorInvalidValue;
  const unsigned b = sumcheck_round_blocks(q);
  if (fold)
    k_sumcheck_round<true><<<b, 256, 0, st>>>(f, w, q, r, partials, counter, out, mail, seq, r_dev);
  else
    k_sumcheck_round<false><<<b, 256, 0, st>>>(f, w, q, r, partials, counter, out, mail, seq, r_dev);
  LAUNCH_DONE();
}

cudaError_t sumcheck_coeffs_capped(const ef* f, const ef* w, size_t half, ef* partials, unsigned max_blocks, ef* out,
                                   cudaStream_t st) {
  unsigned b = grid_for(half, 256, 8);
  if (b > max_blocks) b = max_blocks;
  k_sumcheck_coeffs<<<b, 256, 0, st>>>(f, w, half, partials);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sum_partials<<<2, 256, 0, st>>>(partials, (int)b, out);
  LAUNCH_DONE();
}

// ---------------------------------------------------------------------------
// Constraint weights (Constraint::combine, src/whir/constraints/mod.rs:197-248)
//   eq part:     EqStatement::combine_hypercube(_packed), statement/eq.rs:182-312
//   select part: SelectStatement::combine(_packed), statement/select.rs:296-496
// ---------------------------------------------------------------------------

__global__ void k_add_eq_batch(ef* __restrict__ w, size_t N, int hi_count_bits, const ef* __restrict__ hi,
                               const ef* __restrict__ lo, int lo_bits, int m, int accumulate) {
  const size_t lomask = ((size_t)1 << lo_bits) - 1;
  const size_t H = (size_t)1 << hi_count_bits, Lc = (size_t)1 << lo_bits;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < N; x += (size_t)gridDim.x * blockDim.x) {
    ef acc = accumulate ? ld_ef(w + x) : kb::ef_zero();
    for (int c = 0; c < m; c++)
      acc = kb::ef_add(acc, kb::ef_mul(ld_ef(hi + c * H + (x >> lo_bits)), ld_ef(lo + c * Lc + (x & lomask))));
    st_ef(w + x, acc);
  }
}

cudaError_t add_eq_batch(ef* w, int n, const ef* hi, const ef* lo, int lo_bits, int m, int accumulate,
                         cudaStream_t st) {
  const size_t N = (size_t)1 << n;
  k_add_eq_batch<<<grid_for(N, 256), 256, 0, st>>>(w, N, n - lo_bits, hi, lo, lo_bits, m, accumulate);
  LAUNCH_DONE();
}

__global__ void k_select_tables(const uint32_t* __restrict__ vars, int m, int n, int lo_bits,
                                uint32_t* __restrict__ pow_lo, uint32_t* __restrict__ pow_hi) {
  const size_t Lc = (size_t)1 << lo_bits, Hc = (size_t)1 << (n - lo_bits);
  const size_t per = Lc + Hc;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)m * per;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t s = t / per, r = t % per;
    const uint32_t v = vars[s];
    if (r < Lc)
      pow_lo[s * Lc + r] = kb::pow(v, r);
    else
      pow_hi[s * Hc + (r - Lc)] = kb::pow(v, (r - Lc) << lo_bits);
  }
}

cudaError_t select_tables(const uint32_t* vars, int m, int n, int lo_bits, uint32_t* pow_lo, uint32_t* pow_hi,
                          cudaStream_t st) {
  if (m <= 0) return cudaSuccess;
  const size_t work = (size_t)m * (((size_t)1 << lo_bits) + ((size_t)1 << (n - lo_bits)));
  k_select_tables<<<grid_for(work, 256), 256, 0, st>>>(vars, m, n, lo_bits, pow_lo, pow_hi);
  LAUNCH_DONE();
}

// W[x] += sum_s g[s] * v_s^x with x = xh * 2^lo_bits + xl and
// v_s^x = v_s^(xh * 2^lo_bits) * v_s^xl. A tile is R consecutive xh by blockDim
// consecutive xl: the CTA forms the R x m factors g[s] * pow_hi[s][xh] once in
// shared memory, and each thread loads the low power pow_lo[s][xl] once per
// constraint for its R outputs (R-fold fewer table loads than one output per
// thread).
template <int R>
__global__ void k_add_select(ef* __restrict__ w, size_t N, int lo_bits, const uint32_t* __restrict__ pow_lo,
                             const uint32_t* __restrict__ pow_hi, const ef* __restrict__ g, int m, int hi_bits) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ef* cs = reinterpret_cast<ef*>(smem_raw);  // [R][m]
  const size_t Lc = (size_t)1 << lo_bits, Hc = (size_t)1 << hi_bits;
  const size_t col_tiles = Lc / blockDim.x, tiles = (Hc / R) * col_tiles;
  for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const size_t xh0 = (tile / col_tiles) * R, xl = (tile % col_tiles) * blockDim.x + threadIdx.x;
    __syncthreads();
    for (int i = threadIdx.x; i < R * m; i += blockDim.x) {
      const int r = i / m, s = i - r * m;
      cs[i] = kb::ef_mul_base(ld_ef(g + s), __ldg(pow_hi + s * Hc + xh0 + r));
    }
    __syncthreads();
    ef acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = ld_ef(w + (xh0 + r) * Lc + xl);
    // four constraints per step: the products of a coefficient (< 4p^2 < 2^64)
    // are summed and reduced once
    int s = 0;
    const uint32_t* pp = pow_lo + xl;  // row s of the power table at pp
    for (; s + 4 <= m; s += 4, pp += 4 * Lc) {
      uint32_t pv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) pv[u] = __ldg(pp + u * Lc);
#pragma unroll
      for (int r = 0; r < R; r++) {
        uint64_t tq[4] = {0, 0, 0, 0};
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const ef c = cs[r * m + s + u];
#pragma unroll
          for (int q = 0; q < 4; q++) tq[q] += (uint64_t)c.c[q] * pv[u];
        }
        acc[r] = kb::ef_add(acc[r], ef{{kb::reduce_wide(tq[0]), kb::reduce_wide(tq[1]), kb::reduce_wide(tq[2]),
                                        kb::reduce_wide(tq[3])}});
      }
    }
    for (; s < m; s++) {
      const uint32_t pv = __ldg(pow_lo + (size_t)s * Lc + xl);
#pragma unroll
      for (int r = 0; r < R; r++) acc[r] = kb::ef_add(acc[r], kb::ef_mul_base(cs[r * m + s], pv));
    }
#pragma unroll
    for (int r = 0; r < R; r++) st_ef(w + (xh0 + r) * Lc + xl, acc[r]);
  }
}

cudaError_t add_select(ef* w, int n, const uint32_t* pow_lo, const uint32_t* pow_hi, int lo_bits, const ef* g, int m,
                       cudaStream_t st) {
  if (m <= 0) return cudaSuccess;
  const size_t N = (size_t)1 << n;
  const int threads = (int)(N < 256 ? N : 256);
  if (((size_t)1 << lo_bits) < (size_t)threads || lo_bits > n) return cudaErrorInvalidValue;
  const size_t Hc = (size_t)1 << (n - lo_bits);
  init_smem_attributes();
  if (Hc >= 4) {
    const size_t smem = (size_t)4 * m * sizeof(ef);
    if (smem > kSelectSmemMax) return cudaErrorInvalidValue;
    k_add_select<4><<<grid_for(N / 4, threads), threads, smem, st>>>(w, N, lo_bits, pow_lo, pow_hi, g, m,
                                                                       n - lo_bits);
  } else {
    const size_t smem = (size_t)m * sizeof(ef);
    if (smem > kSelectSmemMax) return cudaErrorInvalidValue;
    k_add_select<1><<<grid_for(N, threads), threads, smem, st>>>(w, N, lo_bits, pow_lo, pow_hi, g, m, n - lo_bits);
  }
  LAUNCH_DONE();
}

}  // namespace wk
