// Host-side pieces of the WHIR prover: context, parameter derivation, the
// duplex-sponge challenger and the proof writer. Internal to the library.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <string>
#include <vector>

#include "../../include/whir_b200.h"
#include "kb.cuh"
#include "kernels.h"
#include "poseidon2.cuh"

namespace wh {

void set_error(const std::string& msg);

// status helpers
#define WH_TRY_CUDA(expr)                                                   \
  do {                                                                      \
    cudaError_t _e = (expr);                                                \
    if (_e != cudaSuccess) {                                                \
      ::wh::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
      return _e == cudaErrorMemoryAllocation ? WHIR_ERR_NOMEM : WHIR_ERR_CUDA; \
    }                                                                       \
  } while (0)
#define WH_TRY(expr)        \
  do {                      \
    int _s = (expr);        \
    if (_s != WHIR_OK) return _s; \
  } while (0)
#define WH_CHECK(cond, msg)                 \
  do {                                      \
    if (!(cond)) {                          \
      ::wh::set_error(msg);                 \
      return WHIR_ERR_INVALID;              \
    }                                       \
  } while (0)

p2::P2Consts to_consts(const whir_poseidon2_params& p);  // canonical -> Montgomery
void default_params(whir_poseidon2_params* p16, whir_poseidon2_params* p24);
void params_from_rng(uint64_t seed, uint32_t mat, whir_poseidon2_params* p16, whir_poseidon2_params* p24);

// rand::rngs::SmallRng (xoshiro256++ seeded through SplitMix64) and
// KoalaBear's StandardUniform sampler on it; field() returns canonical values.
struct SmallRng {
  uint64_t s[4];
  explicit SmallRng(uint64_t seed);
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next_u64();
  uint32_t next_u32() { return (uint32_t)(next_u64() >> 32); }
  uint32_t field();
};
int validate_params(const whir_poseidon2_params& p, uint32_t width);

// WhirConfig::new restated (src/whir/parameters.rs:81-234); returns WHIR_OK or an error
int config_new(const whir_protocol_params& prm, int n, whir_config* out);
whir_round_config final_round_config(const whir_config& c);
int ff_at(const whir_config& c, int round);
int rsr_at(const whir_config& c, int round);
std::vector<uint32_t> domain_separator(const whir_config& c, int digest_elems);  // canonical

// Host-side width-16 Poseidon2 for the transcript, in canonical form with
// 64-bit lazy reduction: the linear layers accumulate unreduced (all sums stay
// below 2^40) and every output is reduced once, about three times fewer
// operations than reducing after each addition. Same permutation as
// p2::permute<16, 20>.
struct HostP16 {
  uint32_t ext_rc[8 * 16];
  uint32_t int_rc[20];
  uint32_t diag[16];
  uint32_t mat;  // WHIR_P2_MDS_MAT4 or WHIR_P2_HL_MAT4
};
HostP16 host_consts16(const whir_poseidon2_params& p);
void host_permute16(uint32_t* state_canonical, const HostP16& k);

// DuplexChallenger with Montgomery-form state
// The transcript's challenger. Family 0: DuplexChallenger<F, Poseidon2-16,
// 16, 8> (st / in / out). Family 1: SerializingChallenger32<F,
// HashChallenger<u8, Keccak256Hash, 32>> of the Keccak configuration, its
// input buffer held as an absorbing Keccak-256 state (kin; a flush hashes it,
// and the 32 output bytes both fill kout and start the next input buffer).
// Values in and out are Montgomery words either way.
constexpr int kChalDuplex = 0, kChalKeccak = 1;
struct Chal {
  uint32_t st[16];
  uint32_t in[8];
  int in_len;
  uint32_t out[8];
  int out_len;
  int family;
  kk::K256 kin;
  uint8_t kout[32];
  int kout_len;
  void init();
  void init_keccak();
  void duplex(const HostP16& k);
  void observe(const HostP16& k, uint32_t v);  // Montgomery value
  uint32_t sample(const HostP16& k);           // Montgomery value
  uint64_t sample_bits(const HostP16& k, int bits);
  kb::ef sample_ef(const HostP16& k);
  void observe_ef(const HostP16& k, const kb::ef& v);
  // a Merkle root: Poseidon2 digests as 8 canonical field elements, Keccak
  // digests as their 32 little-endian bytes
  void observe_digest(const HostP16& k, const uint32_t* words8);
  void load(const whir_challenger& c);   // canonical -> internal
  void store(whir_challenger& c) const;  // internal -> canonical
};

// A digest word as the API returns it: Poseidon2 digests are held in
// Montgomery form and returned canonical; Keccak digest words are raw bytes.
inline uint32_t digest_word_out(int leaf_hash, uint32_t w) {
  return leaf_hash == WHIR_LEAF_KECCAK ? w : kb::from_mont(w);
}

// Per-stage device timing (CUDA events on the context's stream), on when
// profiling is enabled for the context.
enum Stage { kStDft = 0, kStLeaves, kStNodes, kStGrind, kStSumcheck, kStEval, kStWeights, kStOpen, kStCount };

// twiddle tables of one subgroup height: omega_H^e and omega_H^(e * 2^12), e < 2^12
constexpr int kDftLogHeights = 25;  // heights 2^0 .. 2^24
constexpr size_t kDftTableWords = 2 * 4096;
constexpr int kUploadGroups = 8;  // chunk groups of a pipelined polynomial upload
// device transcript area: DevChal at word 0, the search's folded state at
// kTrCp, the error word at kTrErr, then per sumcheck round (kTrRound words):
// c0 and c2 (8 words), the witness and its evaluated-candidate count (2), the
// sampled challenge (4 words, at offset 12)
constexpr int kDevTrWords = 1024;
constexpr int kTrCp = 40, kTrErr = 64, kTrLog = 68, kTrRound = 16;
constexpr int kTrMaxRounds = (kDevTrWords - kTrLog) / kTrRound;

}  // namespace wh

struct whir_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  whir_poseidon2_params p16_params, p24_params;
  p2::P2Consts p16, p24;  // canonical round constants for the kernels
  wh::HostP16 hp16;       // canonical, for the host transcript
  uint32_t* tw_stage = nullptr;
  // twiddle tables of every height, built at creation so that proving never
  // allocates them (a device allocation mid-run would stall other contexts)
  uint32_t* tw_heights = nullptr;  // kDftLogHeights * kDftTableWords words
  // scratch
  kb::ef* d_partials = nullptr;  // 8192 ef
  kb::ef* d_small = nullptr;     // 256 ef
  uint32_t* d_words = nullptr;   // 16 words: grind result, claim and done counters (0-2), sumcheck round (8),
                                 // dot product (9) and tree-top (10) counters, streamed-dot wait flag (11),
                                 // staged DFT pass flags (12), batched-tree work counter (13)
  void* d_arena = nullptr;       // general scratch (tables, gathers)
  // device transcript area (kDevTrWords words): the device challenger, the
  // folded state of the next search, an error word and per-round logs of a
  // sumcheck stage run with the transcript on the device
  uint32_t* d_tr = nullptr;
  // device bytes the context holds outside its memory pool (tables, scratch,
  // arena), each allocation rounded up to the driver's 2 MiB granularity
  size_t fixed_device_bytes = 0;
  size_t arena_bytes = 0;
  void* h_pinned = nullptr;      // staging for small transfers (the first pinned_bytes)
  size_t pinned_bytes = 0;
  // the rest of the same pinned block: query openings copied back while the
  // prover queues the next work (open_ev marks the copy's completion)
  void* h_open = nullptr;
  size_t open_bytes = 0;
  cudaEvent_t open_ev = nullptr;
  // mailbox for small results: mapped host memory the GPU writes directly
  // (payload, then a sequence flag), polled by the host instead of a copy and
  // a stream synchronisation
  uint32_t* h_mail = nullptr;
  uint32_t* d_mail = nullptr;  // device alias of h_mail
  uint32_t mail_seq = 0;
  // this context's stream-ordered memory pool: a pool per context keeps the
  // allocator from reusing one stream's freed blocks on another stream (which
  // would make concurrent contexts wait on each other's queued work)
  cudaMemPool_t pool = nullptr;
  // upload of a host polynomial in chunk groups on a stream of its own, each
  // group's DFT first pass queued on `stream` behind the group's copy
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t up_ev[wh::kUploadGroups + 1] = {};
  // stage timing
  bool profiling = false;
  // run a sumcheck stage's transcript steps on the device (see
  // whir_ctx_set_device_transcript); off: each step round-trips to the host.
  // Atomic: a batch may switch it while its worker proves.
  std::atomic<bool> device_transcript{false};
  // how long a wait for a device result spins before it polls with yields
  // (whir_ctx_set_wait_spin)
  std::atomic<int> wait_spin_us{30};
  // candidates in flight of proof-of-work searches (wk::kGrindLatency or
  // wk::kGrindLean* bits; whir_ctx_set_grind_window)
  std::atomic<int> grind_window{0};
  // the challenger after the domain separator, per (parameters, size): where a
  // whir_commit_and_prove starts (observing the pattern is a few dozen host
  // permutations, ahead of the first launch); a handful of entries, the
  // oldest replaced
  struct DsEntry {
    whir_protocol_params params;
    int32_t n;
    wh::Chal ch;
  };
  std::vector<DsEntry> ds_cache;
  std::vector<cudaEvent_t> event_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> stage_events;
  double stage_ms[wh::kStCount] = {};
  uint64_t stage_launches[wh::kStCount] = {};
  uint64_t stage_work[wh::kStCount] = {};
};

namespace wh {
// Dot-product results are field elements (< p); 0xffffffff in every word marks a
// bounded device wait that gave up.
inline int check_dot(const void* v, size_t bytes) {
  const uint32_t* w = static_cast<const uint32_t*>(v);
  for (size_t i = 0; i < bytes / 4; i++)
    if (w[i] >= kb::P) return set_error("a device wait of the dot product timed out"), WHIR_ERR_CUDA;
  return WHIR_OK;
}
// Stream-ordered allocation from the context's pool.
inline cudaError_t ctx_malloc(whir_ctx* ctx, void* p, size_t bytes) {
  return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, ctx->pool, ctx->stream);
}
// Records a CUDA event pair around a scope when the context is profiling.
// Records CUDA events around a stage when profiling is on, and adds `work`
// units to the stage's work count (DFT: algorithmic bytes; Merkle leaves and
// upper levels: permutations; grinding adds its evaluated candidates after the
// search, see add_stage_work).
struct StageTimer {
  whir_ctx* ctx;
  int stage;
  cudaEvent_t a = nullptr, b = nullptr;
  StageTimer(whir_ctx* c, int s, uint64_t work = 0);
  ~StageTimer();
};
void add_stage_work(whir_ctx* ctx, int stage, uint64_t work);

int ensure_dft_tables(whir_ctx* ctx, int log_h, wk::DftTables* t);
int fetch(whir_ctx* ctx, void* host, const void* dev, size_t bytes);
// mailbox: the next sequence number, a wait for a posted result, and a fetch
// that waits for `seq` when it is nonzero (else copies `dev`)
uint32_t mail_next(whir_ctx* ctx);
int mail_wait(whir_ctx* ctx, uint32_t seq, void* host, size_t bytes);
int fetch_posted(whir_ctx* ctx, uint32_t seq, void* host, const void* dev, size_t bytes);
int dot_eq(whir_ctx* ctx, const uint32_t* d_f, int ext, int seg_bits, const kb::ef* z, int m_bits, uint32_t* posted);

// Tuned launches (launch shapes chosen per shape on first use, process-wide)
// The DFT plan run_dft would use for this shape, if it needs no tuning run
// first (false: the tuner has not timed it yet).
bool dft_plan_known(const whir_ctx* ctx, int log_chunk, int log_w, int log_blowup, int lanes, wk::DftPlan* plan);
int run_dft(whir_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t* scratch, int log_chunk, int log_w,
            int log_blowup, int lanes, const wk::DftTables& t);
int run_merkle_leaves(whir_ctx* ctx, const uint32_t* rows, int log_h, int row_words, int leaf_hash,
                      uint32_t* digests);
// with posted_seq set, the root goes to the mailbox: *posted_seq receives the
// sequence to wait for (0 when nothing was posted)
int run_merkle_upper(whir_ctx* ctx, int log_h, int leaf_hash, uint32_t* digests, uint32_t* posted_seq);
int run_fold(whir_ctx* ctx, kb::ef* a, kb::ef* b, size_t half, const kb::ef& r);
}  // namespace wh
