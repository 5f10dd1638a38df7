// Merkle and proof-of-work kernels with the Poseidon2 paper's external block
// M4 (Plonky3's HLMDSMat4, the Horizen Labs form), selectable per context.
#include "merkle.cuh"

namespace wk {
template cudaError_t merkle_leaves_m<p2::kMatHl>(const uint32_t*, int, int, int, uint32_t*, const p2::P2Consts&,
                                                 const p2::P2Consts&, Shape, cudaStream_t);
template cudaError_t merkle_upper_m<p2::kMatHl>(int, uint32_t*, const p2::P2Consts&, Shape, unsigned*, uint32_t*,
                                                uint32_t, int*, cudaStream_t);
template cudaError_t merkle_many_m<p2::kMatHl>(const TreeDesc*, const unsigned long long*, int, int,
                                               const unsigned long long*, int, int, const p2::P2Consts&,
                                               const p2::P2Consts&, unsigned*, uint32_t*, cudaStream_t);
template cudaError_t grind_m<p2::kMatHl>(const uint32_t*, const uint32_t*, int, int, uint64_t, uint32_t*, uint32_t*,
                                          uint32_t*, uint32_t*, uint32_t, const p2::P2Consts&, cudaStream_t,
                                          const uint32_t*, uint32_t*, DevChal*, kb::ef*, uint32_t*, int);
template cudaError_t sumcheck_round_tr_m<p2::kMatHl>(kb::ef*, kb::ef*, size_t, int, kb::ef, kb::ef*, unsigned*, kb::ef*,
                                                 const kb::ef*, DevChal*, const DevChal*, uint32_t*, int, uint32_t*,
                                                 kb::ef*, const p2::P2Consts&, cudaStream_t);
}  // namespace wk
