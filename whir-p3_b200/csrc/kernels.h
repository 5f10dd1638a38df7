// Launchers for the device kernels of the WHIR prover hot path. All device
// arrays hold field elements in Montgomery form (see kb.cuh); an extension
// element is 4 consecutive words. Every launcher enqueues on `st` and returns
// the launch status; none of them synchronizes.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "kb.cuh"
#include "keccak.cuh"
#include "poseidon2.cuh"

namespace wk {

// Kernel launch counter (the number of kernels this library enqueued).
unsigned long long launches();
void count_launch();

// SM count of the current device (read once per device, thread-safe)
int sm_count();

#define LAUNCH_DONE()              \
  do {                             \
    count_launch();                \
    return cudaGetLastError();     \
  } while (0)

// small device-side tables owned by the caller
struct DftTables {
  const uint32_t* tw_stage;  // omega_{2^12}^k, k < 2^11 (Montgomery)
  const uint2* tw_sh;        // omega_{2^12}^k, k < 2^12: (canonical, Shoup constant)
  const uint32_t* tw_lo;     // omega_H^e, e < 2^12
  const uint32_t* tw_hi;     // omega_H^(e * 2^12), e < 2^12
  uint32_t* err = nullptr;   // flags of the staged passes (bit 0: a tile wait gave up, bit 1: unaligned tile)
};
// words of the per-context stage table: 2^11 Montgomery twiddles, then 2^12 Shoup pairs
constexpr int kDftStageTableWords = 2048 + 2 * 4096;

// Mailbox of small results in mapped host memory: kMailWords payload words,
// then the sequence flag at word kMailWords.
constexpr int kMailWords = 512;
// copy `words` (<= kMailWords) device words into the mailbox, then (after a
// system-wide fence) write `seq` to the flag
cudaError_t publish(const uint32_t* src, int words, uint32_t* mail, uint32_t seq, cudaStream_t st);
// Small host data to device memory in stream order without a host-side
// synchronisation: the words travel in the launch's parameter block and one
// CTA stores them to `dst` (at most kPutWords words).
constexpr int kPutWords = 1000;
cudaError_t put_words(uint32_t* dst, const uint32_t* src, int words, cudaStream_t st);

#ifdef __CUDACC__
// Mailbox write by one thread: payload, a system-wide fence, then the flag.
__device__ __forceinline__ void mail_post(volatile uint32_t* mail, const uint32_t* src, int words, uint32_t seq) {
  for (int i = 0; i < words; i++) mail[i] = src[i];
  __threadfence_system();
  mail[kMailWords] = seq;
}
#endif

cudaError_t encode(uint32_t* p, size_t n, cudaStream_t st);
cudaError_t decode(uint32_t* p, size_t n, cudaStream_t st);

// tables: tw_stage needs kDftStageTableWords words, tw_lo/tw_hi 2^12 words each
cudaError_t build_dft_tables(uint32_t* tw_stage, uint32_t* tw_lo, uint32_t* tw_hi, int log_h, cudaStream_t st);

// Launch plan of dft_batch. log_h2 = 0 selects the one-pass twisted kernel
// (chunks of at most 2^12 points, 2^log_t1 columns per CTA); otherwise the
// four-step split H = H1 * H2 with H2 = 2^log_h2, pass 1 transforming
// 2^log_t1 length-H1 columns per CTA and pass 2 2^log_t2 length-H2 rows.
// A pass runs either the shared-memory radix-2 kernel (threads1/threads2 per
// CTA) or, with reg1/reg2 set, the register-resident kernel, whose CTA size
// is fixed by the pass length and tile. reg2 = 2 runs the register pass 2 with
// its input tile staged in shared memory by one tensor copy (TMA).
struct DftPlan {
  int log_h2;
  int log_t1, threads1;
  int log_t2, threads2;
  int reg1, reg2;  // pass uses the register-resident kernel (2^8..2^12 points); reg2 2: TMA-staged tile
};
// the fixed plan used when tuning is off (64 KiB tiles, 256 threads)
DftPlan dft_default_plan(int log_chunk, int log_w, int log_blowup, int lanes);
// every candidate plan the tuner may time for this shape (all pass dft_plan_ok)
void dft_candidates(int log_chunk, int log_w, int log_blowup, int lanes, DftPlan* out, int* count, int cap);
bool dft_plan_ok(const DftPlan& p, int log_chunk, int log_w, int log_blowup, int lanes);

// transpose & pad & DFT: 2^log_w chunks of 2^log_chunk elements -> row-major
// (2^(log_chunk+log_blowup)) x 2^log_w; `scratch` needs out-size elements.
// `passes` selects the four-step passes to run (bit 0: pass 1, bit 1: pass 2;
// 3 for the whole transform). Pass 1 works column by column: with passes == 1
// and ncols > 0 it runs only chunks [col0, col0 + ncols) (a four-step plan;
// the tuner and the pipelined upload of a polynomial run single passes).
cudaError_t dft_batch(const uint32_t* in, uint32_t* out, uint32_t* scratch, int log_chunk, int log_w,
                      int log_blowup, int lanes, const DftTables& t, const DftPlan& plan, int passes,
                      cudaStream_t st, int col0 = 0, int ncols = 0);

// Grid shape of a streaming kernel: threads per CTA, a cap on CTAs per SM
// (0: one CTA per `threads` work items, no cap) and a kernel variant where a
// launcher has several.
struct Shape {
  int threads;
  int per_sm;
  int variant;
};

// CTAs for `work` items at sh.threads per CTA, capped at sh.per_sm CTAs per SM
// (per_sm 0: no cap)
inline unsigned grid_shape(size_t work, Shape sh) {
  size_t b = (work + sh.threads - 1) / sh.threads;
  if (sh.per_sm > 0) {
    const size_t cap = (size_t)sm_count() * sh.per_sm;
    if (b > cap) b = cap;
  }
  if (b < 1) b = 1;
  return (unsigned)b;
}

// Merkle tree: digests has (2h-1)*8 words, leaves first. leaf_hash 0: sponge
// over Poseidon2-24 rate 16; 1: Poseidon2-16 rate 8. Compression: Poseidon2-16.
// `counter` (device, one word, 0 before the first launch, left at 0) joins the
// CTAs of the top kernel
cudaError_t merkle_build(const uint32_t* rows, int log_h, int row_words, int leaf_hash, uint32_t* digests,
                         const p2::P2Consts& p16, const p2::P2Consts& p24, unsigned* counter, cudaStream_t st);
// the two halves of merkle_build: leaf hashing with the CTA subtrees, then the
// upper levels. `leaf` shapes the leaf-digest kernel of trees with at least
// kMerkleLevelPairMin leaves (threads 128, 256 or 512), `node` the two-level
// compression kernel (threads 128 or 256) and picks the top kernel (variant
// bit 0 clear: cooperative four-lane permutations in many CTAs; set: one CTA,
// one permutation per thread) and the two-level kernel's form (bit 1 set: its
// two permutations one after the other, fewer registers; bit 2 set: the last,
// narrow two-level step with four-lane cooperative permutations).
constexpr int kMerkleLevelPairMin = 1 << 12;
Shape merkle_leaf_default();
Shape merkle_node_default();
cudaError_t merkle_leaves(const uint32_t* rows, int log_h, int row_words, int leaf_hash, uint32_t* digests,
                          const p2::P2Consts& p16, const p2::P2Consts& p24, Shape leaf, cudaStream_t st);
// With `mail` set the top kernel posts the root (8 words) to that mailbox with
// flag `seq` and *posted becomes 1 (trees of one leaf post nothing).
cudaError_t merkle_upper(int log_h, uint32_t* digests, const p2::P2Consts& p16, Shape node, unsigned* counter,
                         uint32_t* mail, uint32_t seq, int* posted, cudaStream_t st);
// gather opened rows and sibling paths for `count` indices
cudaError_t merkle_open(const uint32_t* rows, const uint32_t* digests, int log_h, int row_words,
                        const uint64_t* d_idx, int count, uint32_t* d_rows_out, uint32_t* d_paths_out,
                        cudaStream_t st);
// the same with up to kOpenParamIdx indices read from host memory into the
// launch's parameter block (no upload of the indices)
constexpr int kOpenParamIdx = 480;
cudaError_t merkle_open_host_idx(const uint32_t* rows, const uint32_t* digests, int log_h, int row_words,
                                 const uint64_t* h_idx, int count, uint32_t* d_rows_out, uint32_t* d_paths_out,
                                 cudaStream_t st);

// PoW search: smallest w in [0, limit) such that the duplex challenger whose
// sponge state is `state` (16 words) with pending inputs in[0..in_len) samples
// `bits` zero low bits after observing w. `result` (device, 1 word) receives
// the witness or p if none; `counter` and `done` (device, 1 word each) are
// scratch. With `mail` set, the result is also posted to that mailbox with
// flag `seq` by the last CTA to stop.
// Search state (result = p, counters 0) before the first search with a
// mailbox on these words; each such search leaves it reset for the next.
cudaError_t grind_reset(uint32_t* result, uint32_t* counter, uint32_t* done, cudaStream_t st);
// With `cp_dev` set, the folded initial state (16 canonical words, see
// p2::grind_fold) is read from device memory instead of being formed from
// `state` and `in` on the host (in_len still selects the witness position);
// with `res_out` set, the last CTA to stop writes the witness and the number of
// evaluated candidates there (2 words) and resets the search state, and no
// initialising launch precedes the search. Searches of up to kCoopGrindBits bits run the four-lane
// permutation (lower latency per pass, more instructions per candidate).
// With `ch` set (res_out, r_out and err too), the search's last CTA also runs
// the transcript step after it on the device challenger: observe the witness,
// check that sample_bits(bits) is 0, sample the round's challenge into r_out
// (a failed check sets bit 0, no witness, or bit 1, check failed, of *err).
// `window` sizes the candidates in flight: kGrindLatency (0) for the shortest
// search on an otherwise idle GPU; bits kGrindLeanSmall (four-lane searches
// with 2^(bits+1) in flight instead of 2^(bits+3)) and kGrindLeanLarge (larger
// searches with one CTA per SM) for fewer evaluated candidates when other
// work shares the GPU. The witness is the same.
constexpr int kCoopGrindBits = 11;
constexpr int kGrindLatency = 0, kGrindLeanSmall = 1, kGrindLeanLarge = 2;
struct DevChal;
cudaError_t grind(const uint32_t* state, const uint32_t* in, int in_len, int bits, uint64_t limit,
                  uint32_t* result, uint32_t* counter, uint32_t* done, uint32_t* mail, uint32_t seq,
                  const p2::P2Consts& p16, cudaStream_t st, const uint32_t* cp_dev = nullptr,
                  uint32_t* res_out = nullptr, DevChal* ch = nullptr, kb::ef* r_out = nullptr,
                  uint32_t* err = nullptr, int window = kGrindLatency);

// Keccak family (keccak.cu): the Keccak MMCS's leaf digests (rows in
// Montgomery form, hashed as canonical values) and tree levels, digests laid
// out as for Poseidon2 (8 words per node, 2^log_h leaves first); and the
// proof-of-work search on the Keccak challenger whose input buffer is `in`
// (same result, counter and done words and mailbox convention as `grind`,
// without a mailbox the search state is reset first by its own launch).
cudaError_t keccak_leaves(const uint32_t* rows, int log_h, int row_words, uint32_t* digests, cudaStream_t st);
cudaError_t keccak_upper(int log_h, uint32_t* digests, uint32_t* mail, uint32_t seq, int* posted, cudaStream_t st);
cudaError_t keccak_grind(const kk::K256& in, int bits, uint64_t limit, uint32_t* result, uint32_t* counter,
                         uint32_t* done, uint32_t* mail, uint32_t seq, cudaStream_t st, int window = kGrindLatency);

// Duplex challenger on the device (DuplexChallenger<F, Poseidon2-16, 16, 8>),
// Montgomery words, laid out like the host's challenger: sponge state, pending
// inputs, buffered outputs. Its steps run in one warp with the four-lane
// permutation, in the tails of the kernels whose results they observe, so a
// chain of sumcheck rounds, searches and challenges can be queued without the
// host in between.
struct DevChal {
  uint32_t st[16];
  uint32_t in[8];
  int32_t in_len;
  uint32_t out[8];
  int32_t out_len;
};
// sumcheck_round followed, in its last CTA, by the round's transcript step on
// the device challenger `ch` (set from *init first and *err cleared when init
// is not null): observe c0, c2; then with grind_next write the folded initial
// state of the next proof-of-work search (16 canonical words, see
// p2::grind_fold) to cp_out, otherwise sample the round's challenge into r_out.
cudaError_t sumcheck_round_tr(kb::ef* f, kb::ef* w, size_t q, int fold, kb::ef r, kb::ef* partials,
                              unsigned* counter, kb::ef* out, const kb::ef* r_dev, DevChal* ch, const DevChal* init,
                              uint32_t* err, int grind_next, uint32_t* cp_out, kb::ef* r_out,
                              const p2::P2Consts& p16, cudaStream_t st);

// Many independent Poseidon2 trees (the same row width and leaf hash, tree i
// of 2^log_h leaves with its own digest array laid out as merkle_build's) in
// one leaf launch, one launch per tree level and one root gather: the leaf
// kernel's CTAs claim chunks of leaves from `counter` over all trees' leaves.
// d_desc: the trees (leaf0 = the tree's first global leaf, increasing from
// 0); d_level_first: for every level l in 0..max_log_h, count + 1 entries
// (tree i's first global node of level l among the trees whose level l is
// below their top, then the level's total); level_totals (host): those
// totals. The roots land in d_roots[8 * i].
struct TreeDesc {
  const uint32_t* rows;
  uint32_t* digests;
  unsigned long long leaf0;
  int log_h;
  int pad;
};
constexpr int kMaxManyTrees = 256;
// the levels of a tree's top done in one CTA: the top starts at the level of
// 2^kManyTopLevels nodes (level log_h - kManyTopLevels), or at the leaves; the
// level launches (d_level_first) cover levels 1 .. log_h - kManyTopLevels only
constexpr int kManyTopLevels = 8;
cudaError_t merkle_many(const TreeDesc* d_desc, const unsigned long long* d_level_first, int count, int max_log_h,
                        const unsigned long long* level_totals, int row_words, int leaf_hash, const p2::P2Consts& p16,
                        const p2::P2Consts& p24, unsigned* counter, uint32_t* d_roots, cudaStream_t st);

// The Poseidon2 launchers above for one external block MAT (p2::kMatMds or
// p2::kMatHl), each form built in its own translation unit; merkle_leaves,
// merkle_upper and grind pick the form of their constants (P2Consts::mat).
template <int MAT>
cudaError_t merkle_leaves_m(const uint32_t* rows, int log_h, int row_words, int leaf_hash, uint32_t* digests,
                            const p2::P2Consts& p16, const p2::P2Consts& p24, Shape leaf, cudaStream_t st);
template <int MAT>
cudaError_t merkle_upper_m(int log_h, uint32_t* digests, const p2::P2Consts& p16, Shape node, unsigned* counter,
                           uint32_t* mail, uint32_t seq, int* posted, cudaStream_t st);
template <int MAT>
cudaError_t merkle_many_m(const TreeDesc* d_desc, const unsigned long long* d_level_first, int count, int max_log_h,
                          const unsigned long long* level_totals, int row_words, int leaf_hash,
                          const p2::P2Consts& p16, const p2::P2Consts& p24, unsigned* counter, uint32_t* d_roots,
                          cudaStream_t st);
template <int MAT>
cudaError_t grind_m(const uint32_t* state, const uint32_t* in, int in_len, int bits, uint64_t limit,
                    uint32_t* result, uint32_t* counter, uint32_t* done, uint32_t* mail, uint32_t seq,
                    const p2::P2Consts& p16, cudaStream_t st, const uint32_t* cp_dev, uint32_t* res_out,
                    DevChal* ch, kb::ef* r_out, uint32_t* err, int window);
template <int MAT>
cudaError_t sumcheck_round_tr_m(kb::ef* f, kb::ef* w, size_t q, int fold, kb::ef r, kb::ef* partials,
                                unsigned* counter, kb::ef* out, const kb::ef* r_dev, DevChal* ch, const DevChal* init,
                                uint32_t* err, int grind_next, uint32_t* cp_out, kb::ef* r_out,
                                const p2::P2Consts& p16, cudaStream_t st);

// eq table of `h` coordinates scaled by `scale`: out[x] = scale * prod eq(z_j, bit_j(x)), MSB <-> z[0].
struct EqPoint {
  kb::ef z[32];
  int h;
  kb::ef scale;
};
cudaError_t eq_table_small(const EqPoint& pt, kb::ef* out, cudaStream_t st);
// out[x] = hi[x >> lo_bits] * lo[x & (2^lo_bits - 1)]
cudaError_t eq_outer(const kb::ef* hi, const kb::ef* lo, int lo_bits, size_t n, kb::ef* out, cudaStream_t st);

// both tables of a split point in one launch
cudaError_t eq_table_pair(const EqPoint& p1, kb::ef* out1, const EqPoint& p2, kb::ef* out2, cudaStream_t st);
// up to kEqMultiTables tables of at most kEqMultiCoords coordinates each in one
// launch: table t is scale[t] * eq(z[zoff[t] ..], .) over 2^h[t] entries into out[t]
constexpr int kEqMultiTables = 8, kEqMultiCoords = 16;
struct EqMulti {
  int count;
  int h[kEqMultiTables];
  int zoff[kEqMultiTables];
  kb::ef* out[kEqMultiTables];
  kb::ef scale[kEqMultiTables];
  kb::ef z[kEqMultiTables * kEqMultiCoords];
};
cudaError_t eq_tables_multi(const EqMulti& m, cudaStream_t st);

// segmented split-eq dot products:
//   out[s] = sum_{x < M} f[s*M + x] * hi[x >> lo_bits] * lo[x & mask],  M = 2^m_bits, s < 2^seg_bits
// f is base (ext=0) or extension (ext=1). partials needs blocks*2^seg_bits ef
// (at most 8 * SMs); the last CTA to finish reduces them into out, using
// `counter` (device, one word, 0 before the first launch, left at 0), and with
// `mail` set also posts them to that mailbox with flag `seq` (needs
// 4 * 2^seg_bits <= kMailWords). Base-field inputs (16-byte aligned, at least
// 4096 per segment) stream through shared memory by bulk copies; `err`
// (device, one word) is set if one of that kernel's bounded waits gives up,
// and then every result is 0xffffffff.
cudaError_t dot_split(const uint32_t* f, int ext, int seg_bits, int m_bits, const kb::ef* hi, const kb::ef* lo,
                      int lo_bits, kb::ef* partials, unsigned* counter, kb::ef* out, uint32_t* mail, uint32_t seq,
                      uint32_t* err, cudaStream_t st);

// compress (fold the first variable) on one or two extension arrays in place;
// `shape` threads 128, 256 or 512
Shape fold_default();
cudaError_t fold_ext(kb::ef* a, kb::ef* b, size_t half, kb::ef r, Shape shape, cudaStream_t st);
// compress_ext: base evals of 2*half entries -> extension evals of half entries
cudaError_t fold_base(const uint32_t* f, size_t half, kb::ef r, kb::ef* out, cudaStream_t st);
// compress_multi: out[x] = sum_{y < 2^k} eqrs[y] * f[y*M + x]
struct EqSmall {
  kb::ef v[64];
};
cudaError_t fold_multi_base(const uint32_t* f, int k, size_t m, const EqSmall& eqrs, kb::ef* out,
                            cudaStream_t st);
// sumcheck coefficients over extension f, w of 2*half entries: out[0] = c0, out[1] = c2
cudaError_t sumcheck_coeffs(const kb::ef* f, const kb::ef* w, size_t half, kb::ef* partials, kb::ef* out,
                            cudaStream_t st);

// One prover sumcheck round in one launch: with `fold`, first fold f and w
// (4q entries each) in place by r into 2q entries; then out[0] = c0, out[1] =
// c2 over the pairs (i, i + q). `partials` needs 2 * grid_for(q) entries and
// `counter` (device, one word) must hold 0 before the first launch; the
// kernel leaves it at 0. With `mail` set, (c0, c2) are also posted to that
// mailbox with flag `seq`.
// With r_dev set, the fold's challenge is read from device memory (r_dev[0])
// instead of `r`.
// grid size of sumcheck_round (and of sumcheck_round_tr): partial sums of
// this many CTAs
unsigned sumcheck_round_blocks(size_t q);
cudaError_t sumcheck_round(kb::ef* f, kb::ef* w, size_t q, int fold, kb::ef r, kb::ef* partials, unsigned* counter,
                           kb::ef* out, uint32_t* mail, uint32_t seq, cudaStream_t st, const kb::ef* r_dev = nullptr);

// The same reduction with the block count capped at max_blocks, so that the
// partials fit a fixed-size buffer (2 * max_blocks entries).
cudaError_t sumcheck_coeffs_capped(const kb::ef* f, const kb::ef* w, size_t half, kb::ef* partials,
                                   unsigned max_blocks, kb::ef* out, cudaStream_t st);

// W[x] (+)= sum_c hi_c[x >> lo_bits] * lo_c[x & mask] for c < m constraints (the
// scale of each constraint is folded into its hi table); tables are laid out
// constraint-major (hi: m * 2^(n-lo_bits), lo: m * 2^lo_bits).
cudaError_t add_eq_batch(kb::ef* w, int n, const kb::ef* hi, const kb::ef* lo, int lo_bits, int m, int accumulate,
                         cudaStream_t st);

// select weights: W[x] += sum_s g[s] * v_s^x. Tables: pow_lo[s*2^lo + xl] = v_s^xl,
// pow_hi[s*2^(n-lo) + xh] = v_s^(xh * 2^lo); built by select_tables.
cudaError_t select_tables(const uint32_t* vars, int m, int n, int lo_bits, uint32_t* pow_lo, uint32_t* pow_hi,
                          cudaStream_t st);
cudaError_t add_select(kb::ef* w, int n, const uint32_t* pow_lo, const uint32_t* pow_hi, int lo_bits,
                       const kb::ef* g, int m, cudaStream_t st);

}  // namespace wk
