// Device helpers shared by the kernel translation units: 16-byte extension
// element loads and stores, warp and block sums of extension values, and the
// body of one prover sumcheck round (fold by the previous challenge, then the
// round's coefficients), which both the plain round kernel (kernels.cu) and the
// round kernel that also runs the transcript step (merkle.cuh) use.
#pragma once
#include "kernels.h"

namespace wk {

// mbarrier and bulk-copy helpers: one elected thread arms the barrier with the
// byte count and issues the copies; the threads wait on the barrier's phase
// with a bounded number of polls.
namespace bulk {
constexpr uint32_t kPolls = 1u << 22;  // bound on the polls of one wait
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(b)) : "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_test(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0u;
}
// Waits for the phase of `parity` to complete; false after kPolls polls.
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity) {
  for (uint32_t i = 0; i < kPolls; i++) {
    if (bar_test(b, parity)) return true;
    if (i >= 64) __nanosleep(128);
  }
  return false;
}
// contiguous bytes (16-byte aligned addresses, a multiple of 16 bytes)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   saddr(dst)),
               "l"(src), "r"(bytes), "r"(saddr(b))
               : "memory");
}
// one box of a three-dimensional tensor map (tile mode, no multicast) at
// element coordinates (x, y, z); x counts elements of the innermost dimension
__device__ __forceinline__ void tensor_load_3d(void* dst, const void* tmap, int x, int y, int z, uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(saddr(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(saddr(b))
      : "memory");
}
}  // namespace bulk

__device__ __forceinline__ kb::ef ld_ef(const kb::ef* p) {
  uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
  return kb::ef{{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ void st_ef(kb::ef* p, const kb::ef& v) {
  *reinterpret_cast<uint4*>(p) = make_uint4(v.c[0], v.c[1], v.c[2], v.c[3]);
}

__device__ __forceinline__ kb::ef warp_sum(kb::ef v) {
#pragma unroll
  for (int off = 16; off; off >>= 1) {
#pragma unroll
    for (int c = 0; c < 4; c++) v.c[c] = kb::add(v.c[c], __shfl_down_sync(0xffffffffu, v.c[c], off));
  }
  return v;
}

// Block-wide sum of K extension values; thread 0 gets the result.
template <int K>
__device__ __forceinline__ void block_sum(kb::ef (&v)[K], kb::ef (&sh)[K][32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; k++) sh[k][warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      v[k] = lane < nw ? sh[k][lane] : kb::ef_zero();
      v[k] = warp_sum(v[k]);
    }
  }
}

// One prover sumcheck round (ProductPolynomial::round with the fold of
// Sumcheck::compute_sumcheck_polynomials, src/sumcheck/product_polynomial.rs):
// optionally the previous round's fold (FOLD: f, w hold 4q entries;
// f'(i) = f(i) + r (f(i + 2q) - f(i)) for i < 2q, in place, each thread owning
// i, i + q, i + 2q, i + 3q; r from r_dev when it is set), then the round's
// coefficients over the pairs (i, i + q) of the (folded) arrays. Each CTA
// writes its two partial sums; the last CTA to finish (atomic counter, no
// waiting) adds them up, writes out[0] = c0 and out[1] = c2, re-arms the
// counter and returns true with thread 0 holding (c0, c2) in res. Every other
// CTA returns false. All threads of the CTA must call it.
template <bool FOLD>
__device__ __forceinline__ bool sumcheck_round_body(kb::ef* __restrict__ f, kb::ef* __restrict__ w, size_t q,
                                                    kb::ef r, kb::ef* __restrict__ partials,
                                                    unsigned* __restrict__ counter, kb::ef* __restrict__ out,
                                                    const kb::ef* __restrict__ r_dev, kb::ef (&res)[2],
                                                    kb::ef (&sh)[2][32], bool& s_last) {
  using kb::ef;
  if (FOLD && r_dev) r = ld_ef(r_dev);
  ef v[2] = {kb::ef_zero(), kb::ef_zero()};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < q; i += (size_t)gridDim.x * blockDim.x) {
    ef el, eh, wl, wh;
    if (FOLD) {
      const ef fa = ld_ef(f + i), fb = ld_ef(f + i + 2 * q), fc = ld_ef(f + i + q), fd = ld_ef(f + i + 3 * q);
      const ef wa = ld_ef(w + i), wb = ld_ef(w + i + 2 * q), wc = ld_ef(w + i + q), wd = ld_ef(w + i + 3 * q);
      el = kb::ef_add(fa, kb::ef_mul(kb::ef_sub(fb, fa), r));
      eh = kb::ef_add(fc, kb::ef_mul(kb::ef_sub(fd, fc), r));
      wl = kb::ef_add(wa, kb::ef_mul(kb::ef_sub(wb, wa), r));
      wh = kb::ef_add(wc, kb::ef_mul(kb::ef_sub(wd, wc), r));
      st_ef(f + i, el);
      st_ef(f + i + q, eh);
      st_ef(w + i, wl);
      st_ef(w + i + q, wh);
    } else {
      el = ld_ef(f + i);
      eh = ld_ef(f + i + q);
      wl = ld_ef(w + i);
      wh = ld_ef(w + i + q);
    }
    v[0] = kb::ef_add(v[0], kb::ef_mul(el, wl));
    v[1] = kb::ef_add(v[1], kb::ef_mul(kb::ef_sub(kb::ef_dbl(eh), el), kb::ef_sub(kb::ef_dbl(wh), wl)));
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v[0];
    partials[gridDim.x + blockIdx.x] = v[1];
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  res[0] = res[1] = kb::ef_zero();
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    const uint4 x0 = __ldcg(reinterpret_cast<const uint4*>(partials + b));
    const uint4 x1 = __ldcg(reinterpret_cast<const uint4*>(partials + gridDim.x + b));
    res[0] = kb::ef_add(res[0], ef{{x0.x, x0.y, x0.z, x0.w}});
    res[1] = kb::ef_add(res[1], ef{{x1.x, x1.y, x1.z, x1.w}});
  }
  block_sum<2>(res, sh);
  if (threadIdx.x == 0) {
    out[0] = res[0];
    out[1] = res[1];
    *counter = 0u;
  }
  return true;
}

}  // namespace wk
