// Merkle and proof-of-work kernels with Plonky3's Monty-31 external block
// (MDSMat4, the circulant [2, 3, 1, 1]): the permutation of p3-koala-bear's
// Poseidon2KoalaBear, and the library's default.
#include "merkle.cuh"

namespace wk {
template cudaError_t merkle_leaves_m<p2::kMatMds>(const uint32_t*, int, int, int, uint32_t*, const p2::P2Consts&,
                                                  const p2::P2Consts&, Shape, cudaStream_t);
template cudaError_t merkle_upper_m<p2::kMatMds>(int, uint32_t*, const p2::P2Consts&, Shape, unsigned*, uint32_t*,
                                                 uint32_t, int*, cudaStream_t);
template cudaError_t merkle_many_m<p2::kMatMds>(const TreeDesc*, const unsigned long long*, int, int,
                                               const unsigned long long*, int, int, const p2::P2Consts&,
                                               const p2::P2Consts&, unsigned*, uint32_t*, cudaStream_t);
template cudaError_t grind_m<p2::kMatMds>(const uint32_t*, const uint32_t*, int, int, uint64_t, uint32_t*, uint32_t*,
                                          uint32_t*, uint32_t*, uint32_t, const p2::P2Consts&, cudaStream_t,
                                          const uint32_t*, uint32_t*, DevChal*, kb::ef*, uint32_t*, int);
template cudaError_t sumcheck_round_tr_m<p2::kMatMds>(kb::ef*, kb::ef*, size_t, int, kb::ef, kb::ef*, unsigned*, kb::ef*,
                                                 const kb::ef*, DevChal*, const DevChal*, uint32_t*, int, uint32_t*,
                                                 kb::ef*, const p2::P2Consts&, cudaStream_t);
}  // namespace wk
