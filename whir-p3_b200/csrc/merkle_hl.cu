// Merkle and proof-of-work kernels with the Poseidon2 paper's external block
// M4 (Plonky3's HLMDSMat4, the Horizen Labs form), selectable per context.
#include "merkle.cuh"

namespace wk {
template cudaError_t merkle_leaves_m<p2::kMatHl>(const uint32_t*, int, int, int, uint32_t*, const p2::P2Consts&,
                                                 const p2::P2Consts&, Shape, cudaStream_t);
template cudaError_t merkle_upper_m<p2::kMatHl>(int, uint32_t*, const p2::P2Consts&, Shape, unsigned*, uint32_t*,
                                                uint32_t, int*, cudaStream_t);
template cudaError_t grind_m<p2::kMatHl>(const uint32_t*, const uint32_t*, int, int, uint64_t, uint32_t*, uint32_t*,
                                          uint32_t*, uint32_t*, uint32_t, const p2::P2Consts&, cudaStream_t,
                                          const uint32_t*, uint32_t*);
template cudaError_t chal_coeffs_m<p2::kMatHl>(DevChal*, const kb::ef*, int, uint32_t*, kb::ef*, const p2::P2Consts&,
                                          cudaStream_t);
template cudaError_t chal_witness_m<p2::kMatHl>(DevChal*, const uint32_t*, int, kb::ef*, uint32_t*, const p2::P2Consts&,
                                           cudaStream_t);
}  // namespace wk
