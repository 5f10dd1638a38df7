// Allocation-free sumcheck coefficients.
//
// Some callers cannot allocate device memory at the point where they need a
// sumcheck round: a prover embedded in a host application whose device memory
// is handed out by its own pool (or pre-partitioned per tenant) must not call
// cudaMalloc behind that pool's back, and code running under a driver or
// runtime that forbids allocation on its hot path (a latency-critical loop)
// cannot pay for it. Those callers already own the inputs and the output; the
// only other memory this reduction needs is its per-block partial sums, which
// live here in a fixed array inside the library instead of a context arena.
#include <mutex>

#include "host.h"

namespace {

// Partial sums of c0 and c2 for at most kMaxBlocks CTAs: 2 * 2048 extension
// elements = 64 KiB on every device that loads the library, held until exit.
constexpr unsigned kMaxBlocks = 2048;
static __device__ __align__(256) kb::ef g_sumcheck_scratch[2 * kMaxBlocks];

// In host code g_sumcheck_scratch names a host-side stand-in, not the device
// array, so kernels receive the device address looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
kb::ef* g_scratch_addr[kMaxDevices] = {};

int scratch_for_current_device(kb::ef** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    wh::set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return WHIR_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    wh::set_error("device index beyond the scratch table");
    return WHIR_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sumcheck_scratch);
    if (e != cudaSuccess || !p) {
      wh::set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return WHIR_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<kb::ef*>(p);
  }
  *out = g_scratch_addr[dev];
  return WHIR_OK;
}

}  // namespace

extern "C" int whir_sumcheck_coeffs_noalloc(const uint32_t* d_f, const uint32_t* d_w, int32_t n, uint32_t* d_out,
                                            void* cuda_stream) {
  if (!d_f || !d_w || !d_out) {
    wh::set_error("null device pointer");
    return WHIR_ERR_INVALID;
  }
  if (n < 1 || n > 30) {
    wh::set_error("n must be in [1, 30] (2^n extension elements per array)");
    return WHIR_ERR_INVALID;
  }
  kb::ef* scratch = nullptr;
  int s = scratch_for_current_device(&scratch);
  if (s != WHIR_OK) return s;
  cudaError_t e = wk::sumcheck_coeffs_capped(reinterpret_cast<const kb::ef*>(d_f), reinterpret_cast<const kb::ef*>(d_w),
                                             (size_t)1 << (n - 1), scratch, kMaxBlocks,
                                             reinterpret_cast<kb::ef*>(d_out), (cudaStream_t)cuda_stream);
  if (e != cudaSuccess) {
    wh::set_error(std::string("launch: ") + cudaGetErrorString(e));
    return WHIR_ERR_CUDA;
  }
  return WHIR_OK;
}
