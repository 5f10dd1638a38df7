/*
 * whir_b200 — C ABI of the B200 (sm_100a) implementation of the WHIR prover
 * hot path of tcoratger/whir-p3 (KoalaBear base field, degree-4 binomial
 * extension, Poseidon2 Merkle commitments, duplex-sponge Fiat-Shamir).
 *
 * Conventions
 *   - Every function returns an int status: WHIR_OK (0) or a negative
 *     WHIR_ERR_* code; whir_last_error() describes the last failure of the
 *     calling thread. No C++ exception crosses this boundary.
 *   - Field elements passed through HOST pointers are canonical uint32 values
 *     in [0, p), p = 2^31 - 2^24 + 1. An extension element is 4 consecutive
 *     words (coefficients of 1, X, X^2, X^3 with X^4 = 3).
 *   - Field elements in DEVICE buffers are in Montgomery form (x * 2^32 mod p).
 *     whir_monty_encode / whir_monty_decode convert device buffers in place.
 *   - A whir_ctx owns one CUDA stream on one device; calls on a context are
 *     ordered on its stream and must come from one host thread at a time.
 *     Functions that return values to the host return once every earlier
 *     operation on that stream has completed (small values arrive through
 *     mapped host memory; a one-CTA copy kernel of the context may still be
 *     retiring, and it touches only context-owned memory).
 *
 * Each entry point cites the reference interface it replaces (paths are
 * inside the reference project; Plonky3 items are at git rev c38eb05).
 */
#ifndef WHIR_B200_H
#define WHIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  WHIR_OK = 0,
  WHIR_ERR_INVALID = -1,     /* bad argument or unsupported shape */
  WHIR_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  WHIR_ERR_NOMEM = -3,       /* device or host allocation failed */
  WHIR_ERR_NOT_FOUND = -4,   /* proof-of-work search exhausted its limit */
  WHIR_ERR_BUFFER = -5,      /* caller buffer too small; required size reported */
  WHIR_ERR_NO_DEVICE = -6    /* no CUDA device available */
};

typedef struct whir_ctx whir_ctx;
typedef struct whir_witness whir_witness;

/* Poseidon2 permutation data (canonical values). Supported shapes: width 16
 * with 8 full + 20 partial rounds, width 24 with 8 full + 23 partial rounds.
 * Replaces p3-koala-bear Poseidon2KoalaBear<16>/<24> (src/bin/main.rs:31-32). */
enum {
  WHIR_P2_MDS_MAT4 = 0,  /* external 4x4 block circ(2,3,1,1): Plonky3's Monty-31 MDSMat4 (KoalaBear) */
  WHIR_P2_HL_MAT4 = 1    /* the Poseidon2 paper's M4 [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] (HLMDSMat4) */
};
typedef struct {
  uint32_t width;
  uint32_t rounds_f;
  uint32_t rounds_p;
  uint32_t external_matrix; /* WHIR_P2_MDS_MAT4 or WHIR_P2_HL_MAT4; both widths of a context use the same */
  uint32_t ext_rc[8 * 24]; /* rounds_f rows of `width`: first half before, second half after the partial rounds */
  uint32_t int_rc[32];     /* one per partial round, added to lane 0 */
  uint32_t diag[24];       /* internal matrix = all-ones + diag(diag); fixed, as p3-koala-bear's internal
                            * layer takes no diagonal: must equal whir_poseidon2_default_params' diag
                            * (small integers and signed powers of two), else WHIR_ERR_INVALID */
} whir_poseidon2_params;

/* Hash family of the Merkle commitments and the transcript:
 *   WHIR_LEAF_P24: leaves PaddingFreeSponge<P24, 24, 16, 8>, nodes
 *     TruncatedPermutation<P16, 2, 8, 16>, DuplexChallenger<F, P16, 16, 8>
 *     (src/bin/main.rs:34-39, benches/whir.rs);
 *   WHIR_LEAF_P16: leaves PaddingFreeSponge<P16, 16, 8, 8>, otherwise the same
 *     (src/whir/mod.rs:39 tests);
 *   WHIR_LEAF_KECCAK: MerkleTreeMmcs<F, u64, SerializingHasher<
 *     PaddingFreeSponge<KeccakF, 25, 17, 4>>, CompressionFunctionFromHasher<
 *     .., 2, 4>, 4> with SerializingChallenger32<F, HashChallenger<u8,
 *     Keccak256Hash, 32>> (src/whir/mod.rs:236-383). Digests are [u64; 4],
 *     held and returned as 8 words (little-endian halves of each u64), never
 *     converted; field elements enter the hash and the challenger as their
 *     canonical values (Plonky3's serialisation, assumed). Runs through
 *     whir_commit_and_prove (the split commit / prove API carries the duplex
 *     challenger's state). */
#define WHIR_LEAF_P24 0
#define WHIR_LEAF_P16 1
#define WHIR_LEAF_KECCAK 2

/* ProtocolParameters (src/parameters/mod.rs:147-166) plus the hash and
 * domain-separator choices of the caller's set-up (src/bin/main.rs:34-39,178-180). */
typedef struct {
  int32_t security_level;
  int32_t pow_bits;
  int32_t folding_factor_0;      /* FoldingFactor::ConstantFromSecondRound(f0, f); Constant(f) has f0 == f */
  int32_t folding_factor;
  int32_t soundness;             /* 0 UniqueDecoding, 1 JohnsonBound, 2 CapacityBound */
  int32_t starting_log_inv_rate;
  int32_t rs_reduction;          /* rs_domain_initial_reduction_factor */
  int32_t leaf_hash;             /* WHIR_LEAF_P24, WHIR_LEAF_P16 or WHIR_LEAF_KECCAK */
  int32_t ds_digest_elems;       /* DIGEST_ELEMS constant given to DomainSeparator::commit_statement */
} whir_protocol_params;

#define WHIR_MAX_ROUNDS 32
/* RoundConfig (src/whir/parameters.rs:31-40); folded_domain_gen canonical */
typedef struct {
  int32_t pow_bits, folding_pow_bits, num_queries, ood_samples, num_variables, folding_factor;
  uint64_t domain_size;
  uint32_t folded_domain_gen;
} whir_round_config;

/* WhirConfig (src/whir/parameters.rs:43-68) */
typedef struct {
  int32_t num_variables, security_level, max_pow_bits, commitment_ood_samples;
  int32_t starting_log_inv_rate, starting_folding_pow_bits;
  int32_t folding_factor_0, folding_factor, rs_reduction, soundness;
  int32_t n_rounds;
  whir_round_config rounds[WHIR_MAX_ROUNDS];
  int32_t final_queries, final_pow_bits, final_sumcheck_rounds, final_folding_pow_bits;
} whir_config;

/* DuplexChallenger<KoalaBear, Poseidon2-16, 16, 8> state (canonical values):
 * sponge_state, input_buffer and output_buffer of p3-challenger. */
typedef struct {
  uint32_t state[16];
  uint32_t input[8];
  int32_t input_len;
  uint32_t output[8];
  int32_t output_len;
} whir_challenger;

/* ---- library / context ---------------------------------------------------- */
const char* whir_last_error(void);
/* Number of CUDA kernels this library has enqueued in this process. */
uint64_t whir_kernel_launches(void);
/* The library's default Poseidon2 data: whir_poseidon2_params_from_rng(1,
 * WHIR_P2_MDS_MAT4), the set-up of src/bin/main.rs:100-102 and
 * benches/whir.rs:66-68 (Poseidon16 then Poseidon24 from one SmallRng seeded 1). */
int whir_poseidon2_default_params(whir_poseidon2_params* p16, whir_poseidon2_params* p24);
/* Poseidon2KoalaBear<16>::new_from_rng_128 followed by <24>::new_from_rng_128
 * on one rand::rngs::SmallRng::seed_from_u64(seed) stream (p3-poseidon2
 * new_from_rng: initial external rows, terminal external rows, then the
 * internal constants), with the given external block. */
int whir_poseidon2_params_from_rng(uint64_t seed, uint32_t external_matrix, whir_poseidon2_params* p16,
                                   whir_poseidon2_params* p24);
/* The first `count` KoalaBear elements (canonical) that `rng.random::<F>()`
 * draws from rand::rngs::SmallRng::seed_from_u64(seed): the polynomial and
 * constraint point of benches/whir.rs:92-100 (seed 0: 2^n base elements, then
 * 4 per extension coordinate). Host only. */
int whir_rng_koalabear(uint64_t seed, uint32_t* out, size_t count);
int whir_ctx_create(int32_t device, const whir_poseidon2_params* p16, const whir_poseidon2_params* p24,
                    whir_ctx** out);
int whir_ctx_destroy(whir_ctx* ctx);
/* Enqueue on a caller-owned cudaStream_t instead of the context's own stream. */
int whir_ctx_set_stream(whir_ctx* ctx, void* cuda_stream);
int whir_ctx_synchronize(whir_ctx* ctx);
/* Per-stage device timing with CUDA events recorded on the context's stream
 * (tracing; off by default). Stages: 0 DFT, 1 Merkle leaf hashing, 2 Merkle
 * upper levels, 3 grinding, 4 sumcheck (coefficients, folds), 5 evaluations
 * (OOD / constraint points), 6 constraint weights, 7 openings.
 * whir_ctx_stage_times synchronizes, accumulates the recorded pairs and writes
 * min(8, cap) entries (milliseconds and scope counts); returns the stage count. */
int whir_ctx_set_profiling(whir_ctx* ctx, int32_t enable);
int whir_ctx_stage_times(whir_ctx* ctx, double* ms, uint64_t* counts, int32_t cap, int32_t reset);
/* Work done per stage while profiling was on, in the stage's own unit: DFT
 * algorithmic bytes (chunks read once, LDE written once), Merkle leaf
 * permutations, Merkle compressions, grinding candidates evaluated (one
 * Poseidon2-16 permutation each); other stages 0. Writes min(8, cap) entries;
 * returns the stage count. */
int whir_ctx_stage_work(whir_ctx* ctx, uint64_t* work, int32_t cap, int32_t reset);
/* Where the transcript steps of a sumcheck stage run (the folding rounds of
 * Prover::round, src/whir/prover/mod.rs:305-325, and the final sumcheck):
 * enable = 1 queues each stage's coefficient kernels, challenger steps
 * (DuplexChallenger observe / sample / grind on the device) and folds without
 * the host in between, then replays the stage's log on the host challenger;
 * enable = 0 (default) makes one host round trip per step. Proofs are the
 * same either way. */
int whir_ctx_set_device_transcript(whir_ctx* ctx, int32_t enable);
/* A wait for a small device result (a root, coefficients, a witness) polls a
 * flag in mapped host memory: it spins for `microseconds` (default 30), then
 * polls with a yield between checks. 0 yields from the start (less host CPU
 * per waiting context, e.g. many batch workers on few cores). */
int whir_ctx_set_wait_spin(whir_ctx* ctx, int32_t microseconds);
/* Candidates in flight of the proof-of-work searches (GrindingChallenger::grind
 * replacement): 0 (default) sizes each search for its own latency on an
 * otherwise idle GPU (8x the expected candidates in flight for searches of up
 * to 11 bits, an expected-cost model above). Bit 0 keeps 2x in flight in the
 * small searches, bit 1 runs the larger ones with one CTA per SM: fewer
 * evaluated candidates for a GPU shared with other work, at some latency.
 * The witness (the smallest valid one) is the same in every mode. */
int whir_ctx_set_grind_window(whir_ctx* ctx, int32_t mode);
/* Host permutation with the context's data (width taken from the state length 16 or 24). */
int whir_poseidon2_permute(const whir_ctx* ctx, uint32_t* state, int32_t width);

/* ---- launch-shape tuning ---------------------------------------------------
 * The DFT plan (four-step split, tile and CTA size of each pass), the Merkle
 * leaf and node batch widths (threads per CTA, CTAs per SM) and the fold tile
 * are chosen per shape: the first time a shape runs, every candidate is timed
 * with CUDA events on the calling context's stream and the fastest is cached
 * for the process (keyed by device ordinal). All candidates compute identical
 * values. Mode 1 (default): tune on first use; mode 0: fixed default shapes
 * (entries already cached stay in use until whir_tune_clear). No counterpart
 * in the reference, whose CPU code has no launch shapes. */
enum {
  WHIR_TUNE_DFT = 1,
  WHIR_TUNE_MERKLE_LEAVES = 2,
  WHIR_TUNE_MERKLE_NODES = 3,
  WHIR_TUNE_FOLD = 4
};
typedef struct {
  int32_t kind;      /* WHIR_TUNE_* */
  int32_t device;
  int32_t key[4];    /* DFT: log_chunk, log_width, log_blowup, lanes (1 or 4); Merkle leaves: log_height,
                        row_words, leaf_hash; nodes: log_height; fold: log2(pairs), arrays (1 or 2) */
  int32_t choice[7]; /* DFT: log_h2 (0 = one pass), log_t1, threads1, log_t2, threads2, reg1, reg2 (pass runs
                        the register-resident kernel); others: threads, per_sm, variant (Merkle nodes:
                        0 = cooperative top subtrees, 1 = one-CTA top) */
  int32_t candidates;
  float ms_default;  /* device time of the default shape */
  float ms_best;     /* device time of the chosen shape */
} whir_tune_entry;
int whir_tune_set_mode(int32_t mode);
int whir_tune_get_mode(void);
/* Returns the number of cached entries and writes min(count, cap). */
int whir_tune_entries(whir_tune_entry* out, int32_t cap);
int whir_tune_clear(void);
/* Candidate DFT plans of a shape, 7 words each (the whir_tune_entry choice
 * layout); returns the count and writes min(count, cap) plans. */
int whir_dft_plans(int32_t log_chunk, int32_t log_width, int32_t log_blowup, int32_t ext, int32_t* plans,
                   int32_t cap);
/* whir_dft_batch / whir_merkle_commit / whir_fold_ext with an explicit launch
 * shape instead of the tuned one: plan = 7 words as above; Merkle shape =
 * {leaf threads, leaf CTAs per SM, node threads, node CTAs per SM, node variant (bit 0:
 * one-CTA top kernel, bit 1: sequential two-level kernel, bit 2: cooperative last
 * two-level step)}; fold
 * shape = {threads, CTAs per SM} (CTAs per SM 0: no cap). */
int whir_dft_batch_plan(whir_ctx* ctx, const uint32_t* d_chunks, int32_t log_chunk, int32_t log_width,
                        int32_t log_blowup, int32_t ext, const int32_t* plan, uint32_t* d_out);
int whir_merkle_commit_shaped(whir_ctx* ctx, const uint32_t* d_rows, int32_t log_height, int32_t row_words,
                              int32_t leaf_hash, const int32_t* shape, uint32_t* d_digests, uint32_t* root);
int whir_fold_ext_shaped(whir_ctx* ctx, uint32_t* d_evals, int32_t n, const uint32_t* r, const int32_t* shape);
/* whir_sumcheck_coeffs with its reduction's block count capped at max_blocks
 * (1 .. 4096): the launch shape whir_sumcheck_coeffs_noalloc uses at its cap of
 * 2048, reachable at any cap for shape tests. */
int whir_sumcheck_coeffs_shaped(whir_ctx* ctx, const uint32_t* d_f, const uint32_t* d_w, int32_t n,
                                int32_t max_blocks, uint32_t* c0, uint32_t* c2);

/* ---- parameters (WhirConfig::new, src/whir/parameters.rs:81-234) ----------- */
int whir_config_new(const whir_protocol_params* params, int32_t num_variables, whir_config* out);
/* DomainSeparator::commit_statement + add_whir_proof pattern
 * (src/fiat_shamir/domain_separator.rs:95-213); returns the pattern length
 * (>= 0) and writes min(length, cap) words. */
int whir_domain_separator(const whir_config* cfg, int32_t digest_elems, uint32_t* out, int32_t cap);

/* ---- challenger (p3-challenger DuplexChallenger + GrindingChallenger) ------- */
void whir_challenger_init(whir_challenger* ch);
int whir_challenger_observe(const whir_ctx* ctx, whir_challenger* ch, const uint32_t* values, size_t n);
int whir_challenger_sample(const whir_ctx* ctx, whir_challenger* ch, uint32_t* out, size_t n);
int whir_challenger_sample_bits(const whir_ctx* ctx, whir_challenger* ch, int32_t bits, uint64_t* out);
/* GrindingChallenger::grind (called at src/whir/proof.rs:188,
 * src/whir/prover/mod.rs:224,363): searches on the GPU and returns the
 * smallest witness; absorbs it into `ch` like the reference. */
int whir_challenger_grind(whir_ctx* ctx, whir_challenger* ch, int32_t bits, uint32_t* witness);
/* GrindingChallenger::check_witness: 1 valid, 0 invalid, < 0 error */
int whir_challenger_check_witness(const whir_ctx* ctx, whir_challenger* ch, int32_t bits, uint32_t witness);

/* ---- device buffers ------------------------------------------------------- */
int whir_device_alloc(whir_ctx* ctx, size_t bytes, void** d_ptr);
int whir_device_free(whir_ctx* ctx, void* d_ptr);
int whir_memcpy_h2d(whir_ctx* ctx, void* d_dst, const void* h_src, size_t bytes);
int whir_memcpy_d2h(whir_ctx* ctx, void* h_dst, const void* d_src, size_t bytes);
int whir_monty_encode(whir_ctx* ctx, uint32_t* d_words, size_t n);
int whir_monty_decode(whir_ctx* ctx, uint32_t* d_words, size_t n);

/* ---- Plonky3 trait kernels (device buffers, Montgomery form) -------------- */
/* transpose & pad & TwoAdicSubgroupDft::dft_batch / dft_algebra_batch
 * (src/whir/committer/writer.rs:70-86, src/whir/prover/mod.rs:166-180):
 * 2^log_width contiguous chunks of 2^log_chunk elements (ext: 4 words each) ->
 * row-major matrix of 2^(log_chunk+log_blowup) rows x 2^log_width elements. */
int whir_dft_batch(whir_ctx* ctx, const uint32_t* d_chunks, int32_t log_chunk, int32_t log_width,
                   int32_t log_blowup, int32_t ext, uint32_t* d_out);
/* Mmcs::commit_matrix (MerkleTreeMmcs, writer.rs:89, prover/mod.rs:182-184).
 * d_digests: (2 * 2^log_height - 1) * 8 words, leaf digests first; root (host)
 * canonical (Poseidon2 families) or the raw words of the Keccak digest. */
int whir_merkle_commit(whir_ctx* ctx, const uint32_t* d_rows, int32_t log_height, int32_t row_words,
                       int32_t leaf_hash, uint32_t* d_digests, uint32_t* root);
/* `count` (1..256) independent trees of one Poseidon2 hash family (leaf_hash
 * WHIR_LEAF_P24 or WHIR_LEAF_P16) and row width, tree i of 2^log_heights[i]
 * rows at d_rows[i] with its digests at d_digests[i] (laid out as for
 * whir_merkle_commit), committed together by multi-instance kernels: one leaf
 * launch whose CTAs claim chunks of leaves from one work queue over all trees,
 * one launch per tree level across the trees, one root gather. roots: count x
 * 8 words (host, canonical). Each tree equals whir_merkle_commit's. A batching
 * entry point with no reference counterpart (the reference commits one matrix
 * per MerkleTreeMmcs::commit_matrix call). */
int whir_merkle_commit_many(whir_ctx* ctx, int32_t count, const uint32_t* const* d_rows, const int32_t* log_heights,
                            int32_t row_words, int32_t leaf_hash, uint32_t* const* d_digests, uint32_t* roots);
/* Mmcs::open_batch (prover/mod.rs:248-300): row (row_words) and sibling path
 * (log_height digests, leaf level first) for `index`, canonical, to host. */
/* the same for a tree of hash family leaf_hash (Keccak path words are raw) */
int whir_merkle_open_ex(whir_ctx* ctx, const uint32_t* d_rows, const uint32_t* d_digests, int32_t log_height,
                        int32_t row_words, int32_t leaf_hash, uint64_t index, uint32_t* row_out,
                        uint32_t* path_out);
/* Keccak256Hash (p3-keccak; Keccak-256 with the original padding) of n bytes,
 * on the host */
int whir_keccak256(const uint8_t* data, size_t n, uint8_t* out32);
int whir_merkle_open(whir_ctx* ctx, const uint32_t* d_rows, const uint32_t* d_digests, int32_t log_height,
                     int32_t row_words, uint64_t index, uint32_t* row_out, uint32_t* path_out);

/* ---- multilinear kernels (src/poly/evals.rs); points/challenges on host ---- */
/* EvaluationsList::new_from_point (evals.rs:312-320): d_out[x] = scale*eq(point, x) */
int whir_eq_table(whir_ctx* ctx, const uint32_t* point, int32_t n, const uint32_t* scale, uint32_t* d_out);
/* evaluate_hypercube_base / evaluate_hypercube_ext (evals.rs:334-366) */
int whir_eval_base(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* point, uint32_t* out);
int whir_eval_ext(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* point, uint32_t* out);
/* compress (evals.rs:127-148), in place: keeps the first 2^(n-1) entries */
int whir_fold_ext(whir_ctx* ctx, uint32_t* d_evals, int32_t n, const uint32_t* r);
/* compress_ext (evals.rs:382-400): base -> extension */
int whir_fold_base(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* r, uint32_t* d_out);
/* compress_multi_into_packed (evals.rs:422-447), k <= 6 */
int whir_fold_multi_base(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* rs, int32_t k,
                         uint32_t* d_out);
/* sumcheck_coefficients (evals.rs:493-526) on extension f, w */
int whir_sumcheck_coeffs(whir_ctx* ctx, const uint32_t* d_f, const uint32_t* d_w, int32_t n, uint32_t* c0,
                         uint32_t* c2);
/* Allocation-free variant of whir_sumcheck_coeffs. It has no counterpart in
 * the reference: it exists for callers that cannot allocate device memory on
 * this path (a host application that owns all device memory through its own
 * pool, or a latency-critical loop where allocation is not allowed). It takes
 * no context: inputs d_f, d_w (2^n extension elements each, Montgomery form),
 * output d_out (8 words: c0 then c2, Montgomery form), all device pointers
 * owned by the caller, and an optional cudaStream_t (NULL = default stream).
 * The per-block partial sums live in a fixed 64 KiB array inside the library
 * (2048 blocks at most), present on every device that loads the library until
 * the process exits. The first call on a device looks up that array's device
 * address; make that first call before any stream capture. Calls that overlap
 * on the GPU share the array and race: run them on one stream at a time.
 * n must be in [1, 30]. Nothing is allocated or freed. Asynchronous: results
 * are ready when the stream reaches this point. */
int whir_sumcheck_coeffs_noalloc(const uint32_t* d_f, const uint32_t* d_w, int32_t n, uint32_t* d_out,
                                 void* cuda_stream);
/* EqStatement::combine_hypercube with INITIALIZED (statement/eq.rs:182-246):
 * d_w[x] += sum_i gamma_pows[i] * eq(points_i, x); m <= 16 */
int whir_combine_eq(whir_ctx* ctx, uint32_t* d_w, int32_t n, const uint32_t* points, int32_t m,
                    const uint32_t* gamma_pows);
/* SelectStatement::combine (statement/select.rs:296-380): d_w[x] += sum_j gamma_pows[j] * vars_j^x */
int whir_combine_select(whir_ctx* ctx, uint32_t* d_w, int32_t n, const uint32_t* vars, int32_t m,
                        const uint32_t* gamma_pows);
/* SplitEqInner::partial_evals (src/sumcheck/svo.rs:465-502): out[y] =
 * sum_x poly[y*2^(n-l) + x] * eq(point[l..], x) for y < 2^l, and the full
 * evaluation poly(point) in eval_out (may be NULL). */
int whir_svo_partial_evals(whir_ctx* ctx, const uint32_t* d_poly, int32_t n, int32_t l, const uint32_t* point,
                           uint32_t* out, uint32_t* eval_out);

/* ---- protocol entry points -------------------------------------------------
 * Proof encoding (uint32 words, canonical values):
 *   0x50524857 'WHRP', 1,
 *   root[8], n_ood, ood[4*n_ood],                                  (commit)
 *   sumcheck, n_rounds,
 *   per round: root[8], n_ood, ood[4*n_ood], pow_witness, n_queries,
 *              queries, sumcheck,
 *   n_final, final_poly[4*n_final], final_pow_witness, n_final_queries,
 *   queries, has_final_sumcheck, [sumcheck]
 * sumcheck = n_polys, (c0[4], c2[4]) * n_polys, n_pow, pow[n_pow]
 * query    = kind (0 base, 1 ext), n_values, values, path_len, path[8*path_len]
 * This mirrors WhirProof (src/whir/proof.rs:17-121) field by field.
 */
/* The bytes bincode::serialize gives for WhirProof (src/whir/proof.rs:11-141,
 * src/bin/main.rs:221): bincode 1.3 default options (little-endian, fixed-width
 * integers, u64 sequence lengths, one-byte Option tags), field elements as
 * their Montgomery u32 words, extension elements / digests / Merkle path
 * nodes as fixed arrays, Merkle proofs as Vec<[F; 8]>, and QueryOpening
 * internally tagged ("type": "base" | "extension"). The Plonky3 serde forms
 * are assumed, not checked against the reference. out may be NULL to get the
 * length; WHIR_ERR_BUFFER if cap is too small (out_len holds the length). */
int whir_proof_to_bincode(const uint32_t* words, size_t n_words, uint8_t* out, size_t cap, size_t* out_len);
/* The inverse: bincode bytes to the flat stream; rejects malformed input and
 * field words >= p. words may be NULL to get the length. */
int whir_proof_from_bincode(const uint8_t* bytes, size_t len, uint32_t* words, size_t cap, size_t* n_words);
/* InitialStatement::evaluate for each user point (src/whir/constraints/statement/initial.rs:143-152)
 * followed by CommitmentWriter::commit (src/whir/committer/writer.rs:56-109).
 * poly: 2^n values, host canonical (poly_on_device = 0) or device Montgomery
 * (poly_on_device = 1, borrowed until whir_witness_free). user_points: num_points
 * * n extension elements; user_evals_out receives num_points evaluations (may
 * be NULL). The challenger must already have observed the domain separator. */
int whir_commit(whir_ctx* ctx, const whir_protocol_params* params, int32_t n, const uint32_t* poly,
                int32_t poly_on_device, const uint32_t* user_points, int32_t num_points, uint32_t* user_evals_out,
                whir_challenger* ch, whir_witness** out);
/* Prover::prove (src/whir/prover/mod.rs:97-128); writes the whole proof
 * (commit part included). proof_words receives the length; WHIR_ERR_BUFFER if
 * cap_words is too small (the witness stays usable for a retry only before proving). */
int whir_prove(whir_ctx* ctx, whir_witness* w, whir_challenger* ch, uint32_t* proof_out, size_t cap_words,
               size_t* proof_words);
int whir_witness_free(whir_witness* w);

/* Convenience: domain separator + commit + prove + one checkpoint sample
 * (the sequence of src/whir/mod.rs:103-141). checkpoint may be NULL. */
int whir_commit_and_prove(whir_ctx* ctx, const whir_protocol_params* params, int32_t n, const uint32_t* poly,
                          int32_t poly_on_device, const uint32_t* user_points, int32_t num_points,
                          uint32_t* user_evals_out, uint32_t* proof_out, size_t cap_words, size_t* proof_words,
                          uint32_t* checkpoint);

/* ---- batching and serving -------------------------------------------------
 * A pool of worker threads on one device, each with its own context and CUDA
 * stream, proves submitted jobs concurrently (batching and serving; no
 * counterpart in the reference, which proves one polynomial per call). A job is admitted when the device memory the pool
 * would then hold fits the HBM budget: every worker context's fixed
 * allocations, plus per worker the larger of its stream-ordered pool's
 * reservation and its running job's charge (footprint plus one 32 MiB pool
 * chunk, the granule in which the pool reserves memory). When nothing fits, idle
 * workers' pools are trimmed first; the first queued job that fits starts (a
 * job passed over more than twice the worker count is waited for), and with
 * nothing running the oldest job runs alone even beyond the budget. The first
 * proof of a new shape also tunes its launch shapes (whir_tune_set_mode) on
 * scratch arrays outside the footprint; a server that must stay within its
 * budget proves each shape once before taking traffic. Each job
 * runs whir_commit_and_prove on its worker's context, so its proof is
 * identical to the one-at-a-time result. */
typedef struct whir_batch whir_batch;
typedef struct {
  whir_protocol_params params;
  int32_t n;
  const uint32_t* poly;      /* 2^n values: host canonical, or device Montgomery if poly_on_device */
  int32_t poly_on_device;
  const uint32_t* points;    /* num_points * n extension elements (may be NULL if num_points == 0) */
  int32_t num_points;
  uint32_t* evals_out;       /* num_points * 4 words, may be NULL */
  uint32_t* proof_out;       /* proof_cap words */
  size_t proof_cap;
  size_t proof_words;        /* out */
  uint32_t checkpoint[4];    /* out: challenger sample after the proof */
  int32_t status;            /* out: WHIR_OK or an error code */
  int32_t done;              /* out: set under the batch lock; read it through whir_batch_wait */
  uint64_t footprint_bytes;  /* out: admitted device footprint */
  double t_submit_ms, t_start_ms, t_done_ms; /* out: steady-clock timestamps */
  char error[160];           /* out: message of a failed job (the worker thread's whir_last_error) */
} whir_job;

/* Device bytes one job holds at its peak (polynomial, trees, codewords, sumcheck arrays). */
int whir_job_footprint(const whir_protocol_params* params, int32_t n, int32_t poly_on_device, uint64_t* bytes);
int whir_batch_create(int32_t device, int32_t workers, const whir_poseidon2_params* p16,
                      const whir_poseidon2_params* p24, uint64_t hbm_budget_bytes, whir_batch** out);
int whir_batch_destroy(whir_batch* b);
/* The admission accounting now: fixed device bytes of all worker contexts and
 * the bytes their memory pools reserve. */
int whir_batch_memory(whir_batch* b, uint64_t* fixed_bytes, uint64_t* pool_reserved_bytes);
/* whir_ctx_set_device_transcript on every worker context; jobs that start
 * afterwards use the setting (jobs already running keep theirs). */
int whir_batch_set_device_transcript(whir_batch* b, int32_t enable);
/* whir_ctx_set_wait_spin on every worker context */
int whir_batch_set_wait_spin(whir_batch* b, int32_t microseconds);
/* whir_ctx_set_grind_window on every worker context */
int whir_batch_set_grind_window(whir_batch* b, int32_t mode);
/* Enqueue (non-blocking). The job and its buffers must stay valid until it is done. */
int whir_batch_submit(whir_batch* b, whir_job* job);
/* Wait for one job (timeout_ms < 0: no limit); returns the job's status. */
int whir_batch_wait(whir_batch* b, whir_job* job, int32_t timeout_ms);
int whir_batch_wait_all(whir_batch* b);
/* Submit `count` jobs and wait for all of them. */
int whir_batch_run(whir_batch* b, whir_job* jobs, int32_t count);

#ifdef __cplusplus
}
#endif
#endif
