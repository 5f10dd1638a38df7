/*
 * Oracle (test infrastructure only): CPU restatement of the WHIR prover hot
 * path of tcoratger/whir-p3 and of the Plonky3 primitives it calls.
 *
 * Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
 * load this library, and only as the checker or the timed CPU baseline. The
 * product library (whir-p3_b200) never includes, links or calls it.
 *
 * Parity status: the whir-p3 protocol logic (src/) is restated line by line.
 * The Plonky3 primitives (rev c38eb05, not vendored in the reference) and the
 * rand 0.10 generator behind `new_from_rng_128(SmallRng::seed_from_u64(1))`
 * and the RNG-drawn inputs are restated from their published algorithms and
 * documented behaviour. No output of the reference (roots, transcripts,
 * proofs) exists to check them against, so those values are "parity
 * unpinned" against the reference.
 *
 * All field elements at this interface are canonical uint32 values; an
 * extension element is 4 consecutive words (coefficients of 1, X, X^2, X^3).
 */
#ifndef WHIR_ORACLE_H
#define WHIR_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Poseidon2 ---------------------------------------------------------- */
typedef struct {
  uint32_t width;            /* 16 or 24 */
  uint32_t rounds_f;         /* full rounds (half before, half after the partial rounds) */
  uint32_t rounds_p;         /* partial rounds */
  uint32_t mat;              /* external block: 0 circ(2,3,1,1) (Plonky3 MDSMat4), 1 the paper's M4 */
  uint32_t ext_rc[8 * 24];   /* rounds_f rows of `width` constants */
  uint32_t int_rc[32];       /* rounds_p constants, added to lane 0 */
  uint32_t diag[24];         /* internal matrix = all-ones + diag(diag) */
} or_p2_params;

void or_p2_default(or_p2_params* p16, or_p2_params* p24);
/* new_from_rng_128 for width 16, then 24, on one SmallRng::seed_from_u64(seed) */
void or_p2_from_rng(uint64_t seed, uint32_t mat, or_p2_params* p16, or_p2_params* p24);
/* the permutations or_whir_prove / or_whir_verify use (NULL: or_p2_default) */
void or_p2_select(const or_p2_params* p16, const or_p2_params* p24);
/* the first `count` KoalaBear elements rng.random::<F>() draws from
 * SmallRng::seed_from_u64(seed), canonical */
void or_rng_fields(uint64_t seed, uint32_t* out, size_t count);
/* the generator's state after seed_from_u64(seed), and raw next_u64 outputs
 * from a given state (known-answer checks of xoshiro256++ and SplitMix64) */
void or_rng_seed_state(uint64_t seed, uint64_t* state4);
void or_rng_u64_from_state(const uint64_t* state4, uint64_t* out, size_t count);
void or_p2_permute(const or_p2_params* prm, uint32_t* state);

/* ---- Protocol parameters (ProtocolParameters, src/parameters/mod.rs:147-166) */
typedef struct {
  int32_t security_level;
  int32_t pow_bits;
  int32_t folding_factor_0;      /* FoldingFactor::ConstantFromSecondRound(f0, f) or Constant(f0 == f) */
  int32_t folding_factor;
  int32_t soundness;             /* 0 UniqueDecoding, 1 JohnsonBound, 2 CapacityBound */
  int32_t starting_log_inv_rate;
  int32_t rs_reduction;          /* rs_domain_initial_reduction_factor */
  int32_t leaf_hash;             /* 0: PaddingFreeSponge<P24,24,16,8>; 1: PaddingFreeSponge<P16,16,8,8>;
                                  * 2: the Keccak MMCS and SerializingChallenger32 (or_keccak.c) */
  int32_t ds_digest_elems;       /* DIGEST_ELEMS const used in DomainSeparator (32 in main/bench, 8 in tests) */
} or_params;

#define OR_MAX_ROUNDS 32
typedef struct {
  int32_t pow_bits, folding_pow_bits, num_queries, ood_samples, num_variables, folding_factor;
  uint64_t domain_size;
  uint32_t folded_domain_gen;
} or_round_cfg;

typedef struct {
  int32_t num_variables, security_level, max_pow_bits, commitment_ood_samples;
  int32_t starting_log_inv_rate, starting_folding_pow_bits;
  int32_t folding_factor_0, folding_factor, rs_reduction, soundness;
  int32_t n_rounds;
  or_round_cfg rounds[OR_MAX_ROUNDS];
  int32_t final_queries, final_pow_bits, final_sumcheck_rounds, final_folding_pow_bits;
} or_config;

int or_config_new(const or_params* prm, int num_variables, or_config* out);

/* ---- Challenger (DuplexChallenger<F, Poseidon2-16, 16, 8>) ------------- */
typedef struct {
  uint32_t state[16];
  uint32_t in[8];
  int32_t in_len;
  uint32_t out[8];
  int32_t out_len;
} or_chal;

void or_chal_init(or_chal* c);
void or_chal_observe(or_chal* c, const or_p2_params* p16, uint32_t v);
uint32_t or_chal_sample(or_chal* c, const or_p2_params* p16);
uint64_t or_chal_sample_bits(or_chal* c, const or_p2_params* p16, int bits);
uint32_t or_chal_grind(or_chal* c, const or_p2_params* p16, int bits);
int or_chal_check_witness(or_chal* c, const or_p2_params* p16, int bits, uint32_t w);
/* ---- Keccak family (or_keccak.c) --------------------------------------- */
void or_keccak_f1600(uint64_t* lanes25);
typedef struct {
  uint64_t st[25];
  uint32_t pos; /* bytes absorbed into the current 136-byte block */
} or_k256;
void or_k256_init(or_k256* k);
void or_k256_update(or_k256* k, const uint8_t* in, size_t len);
void or_k256_final(const or_k256* k, uint8_t out[32]);
void or_keccak256(const uint8_t* in, size_t len, uint8_t out[32]);
/* leaf digest of a row (canonical values) and 2-to-1 compression, digests as
 * 8 words (little-endian halves of [u64; 4]) */
void or_keccak_leaf(const uint32_t* row, int words, uint32_t out8[8]);
void or_keccak_compress(const uint32_t* l8, const uint32_t* r8, uint32_t out8[8]);
/* SerializingChallenger32<F, HashChallenger<u8, Keccak256Hash, 32>>; the
 * input buffer is held as an absorbing Keccak-256 state */
typedef struct {
  or_k256 in;
  uint8_t out[32];
  int32_t out_len;
} or_kchal;
void or_kchal_init(or_kchal* c);
void or_kchal_observe(or_kchal* c, uint32_t v); /* a canonical value, or a raw digest word */
void or_kchal_observe_bytes(or_kchal* c, const uint8_t* b, size_t n);
uint32_t or_kchal_sample(or_kchal* c);
uint64_t or_kchal_sample_bits(or_kchal* c, int bits);
int or_kchal_check_witness(or_kchal* c, int bits, uint32_t w);
uint32_t or_kchal_grind(or_kchal* c, int bits);

/* domain separator pattern of DomainSeparator::commit_statement + add_whir_proof */
int or_domain_separator(const or_config* cfg, int digest_elems, uint32_t* out, int cap);

/* ---- Kernels' CPU counterparts ---------------------------------------- */
void or_dft_batch(const uint32_t* chunks, int log_chunk, int log_width, int log_blowup, int ext,
                  uint32_t* out);
/* digests: (2*height - 1) * 8 words, level 0 (leaves) first; returns root in root[8] */
void or_merkle_build(const or_p2_params* p16, const or_p2_params* p24, int leaf_hash,
                     const uint32_t* rows, int log_height, int row_words, uint32_t* digests,
                     uint32_t* root);
void or_eq_table(const uint32_t* point, int n, const uint32_t* scale, uint32_t* out);
void or_eval_base(const uint32_t* evals, int n, const uint32_t* point, uint32_t* out);
void or_eval_ext(const uint32_t* evals, int n, const uint32_t* point, uint32_t* out);
void or_fold_ext(uint32_t* evals, int n, const uint32_t* r);
void or_fold_base(const uint32_t* evals, int n, const uint32_t* r, uint32_t* out);
void or_fold_multi_base(const uint32_t* evals, int n, const uint32_t* rs, int k, uint32_t* out);
void or_sumcheck_coeffs(const uint32_t* f, const uint32_t* w, int n, uint32_t* c0, uint32_t* c2);
void or_extrapolate_012(const uint32_t* e0, const uint32_t* e1, const uint32_t* e2, const uint32_t* r,
                        uint32_t* out);
void or_combine_select(uint32_t* weights, int n, const uint32_t* vars, int n_vars,
                       const uint32_t* gamma_pows);

/* ---- End-to-end commit + prove and verify ------------------------------ */
/* user_points: num_points * n extension elements. Produces the flat proof
 * encoding (uint32 words) in a buffer allocated with malloc (free with
 * or_free). checkpoint: 4 words sampled after the proof (as whir/mod.rs:141). */
int or_whir_prove(const or_params* prm, int n, const uint32_t* poly, const uint32_t* user_points,
                  int num_points, uint32_t** proof, size_t* proof_words, uint32_t* checkpoint);
int or_whir_verify(const or_params* prm, int n, const uint32_t* user_points,
                   const uint32_t* user_evals, int num_points, const uint32_t* proof,
                   size_t proof_words, uint32_t* checkpoint);
void or_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
