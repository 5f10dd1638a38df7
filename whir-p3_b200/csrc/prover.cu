// WHIR commit and prove on one GPU (CommitmentWriter::commit,
// src/whir/committer/writer.rs:56-109, and Prover::prove/round/final_round,
// src/whir/prover/mod.rs:97-417).
//
// The polynomial, codewords, Merkle trees and sumcheck arrays stay in HBM for
// the whole proof; the host runs the Fiat-Shamir transcript and reads back
// only transcript values (digests, OOD answers, sumcheck coefficients, opened
// rows). The initial sumcheck uses split-eq partial evaluations (the
// reference's SVO strategy, src/sumcheck/svo.rs): one pass over the base
// polynomial per constraint yields 2^k values from which all k first-round
// sumcheck polynomials follow exactly, so no 2^n extension weight table is
// materialised. Classic and SVO give identical transcripts in the reference
// (src/sumcheck/tests.rs:459-490), and so does this path.
#include <string.h>

#include <algorithm>

#include "host.h"

using kb::ef;

namespace wh {
int ensure_dft_tables(whir_ctx* ctx, int log_h, wk::DftTables* t);
int fetch(whir_ctx* ctx, void* host, const void* dev, size_t bytes);
int upload(whir_ctx* ctx, void* dev, const void* host, size_t bytes);
int grind(whir_ctx* ctx, Chal& ch, int bits, uint32_t* witness);
wk::EqSmall eq_small_host(const ef* rs, int k);
int add_eq_points(whir_ctx* ctx, ef* d_w, int n, const std::vector<std::vector<ef>>& pts, const std::vector<ef>& scales,
                  int accumulate);
int add_select_vars(whir_ctx* ctx, ef* d_w, int n, const std::vector<uint32_t>& vars, const std::vector<ef>& g);
}  // namespace wh

namespace {

struct Tree {
  uint32_t* rows = nullptr;     // codeword, row-major (Montgomery)
  uint32_t* digests = nullptr;  // (2h - 1) * 8 words
  int log_h = 0;
  int row_words = 0;
  int ext = 0;
  int leaf_hash = 0;  // hash family (WHIR_LEAF_*)
};

struct Constraint {
  std::vector<ef> point;  // n coordinates (Montgomery)
  ef eval;
  std::vector<ef> partial;  // 2^k0 split partial evaluations
};

void put_ef(std::vector<uint32_t>& out, const ef& v) {
  for (int i = 0; i < 4; i++) out.push_back(kb::from_mont(v.c[i]));
}

std::vector<ef> expand_from_univariate(const ef& z, int n) {
  std::vector<ef> r(n);
  ef cur = z;
  for (int i = n - 1; i >= 0; i--) {
    r[i] = cur;
    cur = kb::ef_sqr(cur);
  }
  return r;
}

// extrapolate_012 (src/sumcheck/lagrange.rs:141-147)
ef extrapolate_012(const ef& e0, const ef& e1, const ef& e2, const ef& r) {
  const uint32_t inv2 = kb::to_mont((kb::P + 1) / 2);
  const ef one = kb::ef_one(), two = kb::ef_dbl(kb::ef_one());
  const ef l0 = kb::ef_mul_base(kb::ef_mul(kb::ef_sub(r, one), kb::ef_sub(r, two)), inv2);
  const ef l1 = kb::ef_mul(r, kb::ef_sub(two, r));
  const ef l2 = kb::ef_mul_base(kb::ef_mul(r, kb::ef_sub(r, one)), inv2);
  return kb::ef_add(kb::ef_add(kb::ef_mul(e0, l0), kb::ef_mul(e1, l1)), kb::ef_mul(e2, l2));
}

// in-place first-variable fold of a host table
void host_fold(std::vector<ef>& t, const ef& r) {
  const size_t half = t.size() / 2;
  for (size_t i = 0; i < half; i++) t[i] = kb::ef_add(t[i], kb::ef_mul(kb::ef_sub(t[i + half], t[i]), r));
  t.resize(half);
}

// multilinear evaluation of 2^k host values at k coordinates (MSB first)
ef host_eval(std::vector<ef> t, const ef* pt, int k) {
  for (int i = 0; i < k; i++) host_fold(t, pt[i]);
  return t[0];
}

struct Sumcheck {
  std::vector<uint32_t> words;  // sumcheck section of the proof
  int npolys = 0;
  std::vector<ef> polys;
  std::vector<uint32_t> pows;
  void emit(std::vector<uint32_t>& out) const {
    out.push_back((uint32_t)npolys);
    for (const ef& v : polys) put_ef(out, v);
    out.push_back((uint32_t)pows.size());
    for (uint32_t w : pows) out.push_back(w);
  }
};

// SumcheckData::observe_and_sample (src/whir/proof.rs:163-193)
int observe_and_sample(whir_ctx* ctx, wh::Chal& ch, Sumcheck& sd, const ef& c0, const ef& c2, int pow_bits, ef* r) {
  sd.polys.push_back(c0);
  sd.polys.push_back(c2);
  sd.npolys++;
  ch.observe_ef(ctx->hp16, c0);
  ch.observe_ef(ctx->hp16, c2);
  if (pow_bits > 0) {
    uint32_t w;
    WH_TRY(wh::grind(ctx, ch, pow_bits, &w));
    sd.pows.push_back(w);
  }
  *r = ch.sample_ef(ctx->hp16);
  return WHIR_OK;
}

int ilog2u(uint64_t v) {
  int r = -1;
  while (v) {
    r++;
    v >>= 1;
  }
  return r;
}

// get_challenge_stir_queries (src/whir/utils.rs:24-145)
std::vector<uint64_t> stir_queries(whir_ctx* ctx, wh::Chal& ch, uint64_t domain_size, int ff, int nq) {
  const uint64_t folded = domain_size >> ff;
  const int bits = ilog2u(folded);
  const int max_bits = 20;  // min(F::bits() - 1, 20)
  const int total = nq * bits;
  std::vector<uint64_t> q;
  q.reserve(nq);
  if (total <= max_bits) {
    uint64_t all = ch.sample_bits(ctx->hp16, total);
    const uint64_t mask = (1ull << bits) - 1;
    for (int i = 0; i < nq; i++) {
      q.push_back((all & mask) % folded);
      all >>= bits;
    }
  } else {
    const int per = max_bits / bits;
    if (per >= 2) {
      const uint64_t mask = (1ull << bits) - 1;
      int rem = nq;
      while (rem > 0) {
        const int b = std::min(rem, per);
        uint64_t all = ch.sample_bits(ctx->hp16, b * bits);
        for (int i = 0; i < b; i++) {
          q.push_back((all & mask) % folded);
          all >>= bits;
        }
        rem -= b;
      }
    } else {
      for (int i = 0; i < nq; i++) q.push_back(ch.sample_bits(ctx->hp16, bits));
    }
  }
  std::sort(q.begin(), q.end());
  q.erase(std::unique(q.begin(), q.end()), q.end());
  return q;
}

}  // namespace

struct whir_witness {
  whir_ctx* ctx = nullptr;
  whir_protocol_params params;
  whir_config cfg;
  int n = 0;
  uint32_t* d_poly = nullptr;
  bool own_poly = false;
  Tree commit_tree;
  // set when the upload already ran the commitment DFT's first pass (the
  // tree's rows and digests are then allocated too)
  uint32_t* pre_scratch = nullptr;
  wk::DftPlan pre_plan;
  std::vector<Constraint> cons;
  std::vector<uint32_t> proof;
  bool proved = false;
};

namespace {

void free_tree(whir_ctx* ctx, Tree& t) {
  if (t.rows) cudaFreeAsync(t.rows, ctx->stream);
  if (t.digests) cudaFreeAsync(t.digests, ctx->stream);
  t.rows = nullptr;
  t.digests = nullptr;
}

// DFT + Merkle commitment of 2^log_w contiguous chunks of 2^log_chunk elements.
// With `pass1` set, t->rows and t->digests are allocated and the DFT's first
// pass already wrote *pre_scratch with that plan; this call frees the scratch
// and clears *pre_scratch.
int commit_matrix(whir_ctx* ctx, const uint32_t* d_src, int log_chunk, int log_w, int log_blowup, int ext,
                  int leaf_hash, Tree* t, uint32_t* root_canon, const wk::DftPlan* pass1 = nullptr,
                  uint32_t** pre_scratch = nullptr) {
  const int lanes = ext ? 4 : 1;
  t->log_h = log_chunk + log_blowup;
  t->row_words = lanes << log_w;
  t->ext = ext;
  t->leaf_hash = leaf_hash;
  const size_t h = (size_t)1 << t->log_h;
  const size_t words = h * (size_t)t->row_words;
  if (!pass1) {
    WH_TRY_CUDA(wh::ctx_malloc(ctx, &t->rows, words * 4));
    WH_TRY_CUDA(wh::ctx_malloc(ctx, &t->digests, (2 * h - 1) * 8 * 4));
  }
  wk::DftTables tab;
  WH_TRY(wh::ensure_dft_tables(ctx, t->log_h, &tab));
  uint32_t* scratch = pass1 ? *pre_scratch : nullptr;
  if (!pass1) WH_TRY_CUDA(wh::ctx_malloc(ctx, &scratch, words * 4));
  int s = WHIR_OK;
  {
    // algorithmic bytes: the 2^log_w chunks read once, the LDE written once
    wh::StageTimer timer(ctx, wh::kStDft, ((uint64_t)lanes << (log_chunk + log_w)) * 4 + (uint64_t)words * 4);
    if (pass1) {
      const cudaError_t ce =
          wk::dft_batch(d_src, t->rows, scratch, log_chunk, log_w, log_blowup, lanes, tab, *pass1, 2, ctx->stream);
      if (ce != cudaSuccess) {
        wh::set_error(std::string("DFT second pass: ") + cudaGetErrorString(ce));
        s = WHIR_ERR_CUDA;
      }
    } else {
      s = wh::run_dft(ctx, d_src, t->rows, scratch, log_chunk, log_w, log_blowup, lanes, tab);
    }
  }
  cudaFreeAsync(scratch, ctx->stream);
  if (pass1) *pre_scratch = nullptr;
  WH_TRY(s);
  {
    // one permutation per rate-sized chunk of each row (rate 16 for Poseidon2-24, 8 for Poseidon2-16,
    // 34 words for the Keccak sponge's 17 lanes)
    const uint64_t rate = leaf_hash == WHIR_LEAF_P24 ? 16 : leaf_hash == WHIR_LEAF_P16 ? 8 : 34;
    wh::StageTimer timer(ctx, wh::kStLeaves, (uint64_t)h * (((uint64_t)t->row_words + rate - 1) / rate));
    WH_TRY(wh::run_merkle_leaves(ctx, t->rows, t->log_h, t->row_words, leaf_hash, t->digests));
  }
  uint32_t posted = 0;
  {
    wh::StageTimer timer(ctx, wh::kStNodes, (uint64_t)h - 1);  // one compression per inner node
    WH_TRY(wh::run_merkle_upper(ctx, t->log_h, leaf_hash, t->digests, &posted));
  }
  uint32_t r[8];
  WH_TRY(wh::fetch_posted(ctx, posted, r, t->digests + (2 * h - 2) * 8, 32));
  for (int i = 0; i < 8; i++) root_canon[i] = wh::digest_word_out(leaf_hash, r[i]);
  return WHIR_OK;
}

// Opening of `idx` on tree t in two steps. open_start queues the gather of
// the rows and authentication paths and their copy to host memory, so the
// prover can queue the next work (constraint weights, a sumcheck stage) before
// it needs them: the opened values enter no challenger, only the proof and the
// claimed sum. open_finish waits for the copy, appends the query records to
// the proof and returns the opened rows (Montgomery) in `rows`. The gathered
// data live in the scratch arena, which the next work overwrites; the copy is
// ordered before it on the stream (or, when it does not fit the staging
// block, done at once).
struct OpenPending {
  int q = 0;
  size_t per = 0;
  bool staged = false;
  std::vector<uint32_t> tmp;
};

int open_start(whir_ctx* ctx, const Tree& t, const std::vector<uint64_t>& idx, OpenPending& op) {
  const int q = (int)idx.size();
  const size_t per = (size_t)t.row_words + (size_t)t.log_h * 8;
  op.q = q;
  op.per = per;
  op.staged = false;
  WH_CHECK((size_t)q * 8 + (size_t)q * per * 4 + 64 <= ctx->arena_bytes, "too many queries for the scratch arena");
  uint64_t* d_idx = reinterpret_cast<uint64_t*>(ctx->d_arena);
  uint32_t* d_rows = reinterpret_cast<uint32_t*>(d_idx + q + 1);
  uint32_t* d_paths = d_rows + (size_t)q * t.row_words;
  if (q == 0) return WHIR_OK;
  if (q <= wk::kOpenParamIdx) {
    // the indices travel in the gather kernel's parameters
    wh::StageTimer timer(ctx, wh::kStOpen);
    WH_TRY_CUDA(wk::merkle_open_host_idx(t.rows, t.digests, t.log_h, t.row_words, idx.data(), q, d_rows, d_paths,
                                         ctx->stream));
  } else {
    WH_TRY(wh::upload(ctx, d_idx, idx.data(), (size_t)q * 8));
    wh::StageTimer timer(ctx, wh::kStOpen);
    WH_TRY_CUDA(wk::merkle_open(t.rows, t.digests, t.log_h, t.row_words, d_idx, q, d_rows, d_paths, ctx->stream));
  }
  const size_t bytes = (size_t)q * per * 4;
  if (ctx->h_open && bytes <= ctx->open_bytes) {
    WH_TRY_CUDA(cudaMemcpyAsync(ctx->h_open, d_rows, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    WH_TRY_CUDA(cudaEventRecord(ctx->open_ev, ctx->stream));
    op.staged = true;
  } else {
    op.tmp.resize((size_t)q * per);
    WH_TRY(wh::fetch(ctx, op.tmp.data(), d_rows, bytes));
  }
  return WHIR_OK;
}

int open_finish(whir_ctx* ctx, const Tree& t, OpenPending& op, std::vector<uint32_t>& proof,
                std::vector<uint32_t>& rows) {
  const int q = op.q;
  const size_t per = op.per;
  if (q == 0) return WHIR_OK;
  if (op.staged) {
    WH_TRY_CUDA(cudaEventSynchronize(ctx->open_ev));
    op.tmp.resize((size_t)q * per);
    memcpy(op.tmp.data(), ctx->h_open, (size_t)q * per * 4);
    op.staged = false;
  }
  const std::vector<uint32_t>& tmp = op.tmp;
  rows.assign(tmp.begin(), tmp.begin() + (size_t)q * t.row_words);
  const uint32_t* paths = tmp.data() + (size_t)q * t.row_words;
  const int nvals = t.ext ? t.row_words / 4 : t.row_words;
  for (int k = 0; k < q; k++) {
    proof.push_back((uint32_t)t.ext);
    proof.push_back((uint32_t)nvals);
    for (int i = 0; i < t.row_words; i++) proof.push_back(kb::from_mont(rows[(size_t)k * t.row_words + i]));
    proof.push_back((uint32_t)t.log_h);
    for (int i = 0; i < t.log_h * 8; i++)
      proof.push_back(wh::digest_word_out(t.leaf_hash, paths[(size_t)k * t.log_h * 8 + i]));
  }
  return WHIR_OK;
}

// A fold by the last sampled challenge that has not been applied yet. The
// next sumcheck round applies it in the same launch as its coefficients;
// flush_fold applies it before anything else reads f or w.
struct PendingFold {
  bool on = false;
  ef r;
  size_t half = 0;  // pairs folded: the arrays hold 2 * half entries before the fold
};

int flush_fold(whir_ctx* ctx, ef* d_f, ef* d_w, PendingFold& pend) {
  if (!pend.on) return WHIR_OK;
  {
    wh::StageTimer timer(ctx, wh::kStSumcheck);
    WH_TRY(wh::run_fold(ctx, d_f, d_w, pend.half, pend.r));
  }
  pend.on = false;
  return WHIR_OK;
}

unsigned* round_counter(whir_ctx* ctx) { return reinterpret_cast<unsigned*>(ctx->d_words) + 8; }

// One ProductPolynomial::round on the device arrays f, w of 2^m entries (of
// 2^(m+1) entries still to be folded by pend.r when a fold is pending); leaves
// this round's fold pending.
int sumcheck_round(whir_ctx* ctx, wh::Chal& ch, Sumcheck& sd, ef* d_f, ef* d_w, int m, ef* sum, int pow_bits,
                   ef* r_out, PendingFold& pend) {
  const size_t half = (size_t)1 << (m - 1);
  WH_CHECK(!pend.on || pend.half == 2 * half, "pending fold does not match the round size");
  const uint32_t seq = ctx->h_mail ? wh::mail_next(ctx) : 0u;
  {
    wh::StageTimer timer(ctx, wh::kStSumcheck);
    WH_TRY_CUDA(wk::sumcheck_round(d_f, d_w, half, pend.on ? 1 : 0, pend.on ? pend.r : kb::ef_zero(),
                                   ctx->d_partials, round_counter(ctx), ctx->d_small,
                                   ctx->h_mail ? ctx->d_mail : nullptr, seq, ctx->stream));
  }
  pend.on = false;
  ef c[2];
  WH_TRY(wh::fetch_posted(ctx, seq, c, ctx->d_small, sizeof(c)));
  ef r;
  WH_TRY(observe_and_sample(ctx, ch, sd, c[0], c[1], pow_bits, &r));
  pend.on = true;
  pend.r = r;
  pend.half = half;
  *sum = extrapolate_012(c[0], kb::ef_sub(*sum, c[0]), c[1], r);
  *r_out = r;
  return WHIR_OK;
}

// The rounds of one sumcheck stage (k rounds over arrays of 2^m0 entries,
// pending fold included) with every transcript step on the device: the last
// CTA of each round's kernel observes (c0, c2) on the device challenger and
// either samples the folding challenge or prepares the proof-of-work search,
// whose last CTA observes the witness, checks it and samples the challenge;
// the next round's kernel folds by that challenge from device memory. The host
// queues the whole stage without waiting, tracking only the challenger's
// buffer lengths (they do not depend on values, and they select the search's
// witness position), then fetches the stage's log once and replays it on its
// own challenger, which must sample the same challenges.
int sumcheck_stage_device(whir_ctx* ctx, wh::Chal& ch, Sumcheck& sd, ef* d_f, ef* d_w, int m0, int k, ef* sum,
                          int pow_bits, std::vector<ef>* rs, PendingFold& pend) {
  wk::DevChal* dch = reinterpret_cast<wk::DevChal*>(ctx->d_tr);
  uint32_t* cp = ctx->d_tr + wh::kTrCp;
  uint32_t* err = ctx->d_tr + wh::kTrErr;
  auto log_c = [&](int j) { return reinterpret_cast<ef*>(ctx->d_tr + wh::kTrLog + wh::kTrRound * j); };
  auto log_w = [&](int j) { return ctx->d_tr + wh::kTrLog + wh::kTrRound * j + 8; };
  auto log_r = [&](int j) { return reinterpret_cast<ef*>(ctx->d_tr + wh::kTrLog + wh::kTrRound * j + 12); };
  static_assert(sizeof(wk::DevChal) == sizeof(uint32_t) * 34 && sizeof(wk::DevChal) <= 4 * wh::kTrCp, "layout");
  wk::DevChal init;
  memcpy(init.st, ch.st, sizeof(init.st));
  memcpy(init.in, ch.in, sizeof(init.in));
  init.in_len = ch.in_len;
  memcpy(init.out, ch.out, sizeof(init.out));
  init.out_len = ch.out_len;
  int in_len = ch.in_len, out_len = ch.out_len;  // the challenger's buffer lengths as the device runs
  auto observed = [&] {
    out_len = 0;
    if (++in_len == 8) {
      in_len = 0;
      out_len = 8;
    }
  };
  auto sampled = [&] {
    if (in_len > 0 || out_len == 0) {
      in_len = 0;
      out_len = 8;
    }
    out_len--;
  };
  for (int j = 0; j < k; j++) {
    const size_t half = (size_t)1 << (m0 - j - 1);
    const bool fold = j > 0 || pend.on;
    WH_CHECK(j > 0 || !pend.on || pend.half == 2 * half, "pending fold does not match the round size");
    {
      // the round, then its coefficients observed on the device challenger
      // (set from the host's at the stage's first round)
      wh::StageTimer timer(ctx, wh::kStSumcheck);
      WH_TRY_CUDA(wk::sumcheck_round_tr(d_f, d_w, half, fold ? 1 : 0, j == 0 && pend.on ? pend.r : kb::ef_zero(),
                                        ctx->d_partials, round_counter(ctx), log_c(j), j > 0 ? log_r(j - 1) : nullptr,
                                        dch, j == 0 ? &init : nullptr, err, pow_bits > 0 ? 1 : 0, cp, log_r(j),
                                        ctx->p16, ctx->stream));
    }
    for (int i = 0; i < 8; i++) observed();
    if (pow_bits > 0) {
      // the search, then the witness observed, checked and the challenge
      // sampled in its last CTA
      wh::StageTimer timer(ctx, wh::kStGrind);
      WH_TRY_CUDA(wk::grind(nullptr, nullptr, in_len, pow_bits, kb::P, ctx->d_words, ctx->d_words + 1,
                            ctx->d_words + 2, nullptr, 0u, ctx->p16, ctx->stream, cp, log_w(j), dch, log_r(j), err,
                            ctx->grind_window.load()));
      observed();
      sampled();
    }
    for (int i = 0; i < 4; i++) sampled();
  }
  std::vector<uint32_t> lg((size_t)(wh::kTrLog - wh::kTrErr) + (size_t)wh::kTrRound * k);
  WH_TRY(wh::fetch(ctx, lg.data(), err, lg.size() * 4));
  if (lg[0] != 0u) {
    wh::set_error(lg[0] & 1u ? "proof-of-work search found no witness" : "device grinding returned an invalid witness");
    return (lg[0] & 1u) ? WHIR_ERR_NOT_FOUND : WHIR_ERR_CUDA;
  }
  for (int j = 0; j < k; j++) {
    const uint32_t* rec = lg.data() + (wh::kTrLog - wh::kTrErr) + wh::kTrRound * j;
    const ef c0{{rec[0], rec[1], rec[2], rec[3]}}, c2{{rec[4], rec[5], rec[6], rec[7]}};
    const ef rd{{rec[12], rec[13], rec[14], rec[15]}};
    sd.polys.push_back(c0);
    sd.polys.push_back(c2);
    sd.npolys++;
    ch.observe_ef(ctx->hp16, c0);
    ch.observe_ef(ctx->hp16, c2);
    if (pow_bits > 0) {
      const uint32_t w = rec[8];
      wh::add_stage_work(ctx, wh::kStGrind, (uint64_t)rec[9]);
      ch.observe(ctx->hp16, kb::to_mont(w));
      if (ch.sample_bits(ctx->hp16, pow_bits) != 0) return wh::set_error("device grinding returned an invalid witness"), WHIR_ERR_CUDA;
      sd.pows.push_back(w);
    }
    const ef r = ch.sample_ef(ctx->hp16);
    if (!kb::ef_eq(r, rd)) return wh::set_error("device transcript diverged from the host's"), WHIR_ERR_CUDA;
    *sum = extrapolate_012(c0, kb::ef_sub(*sum, c0), c2, r);
    if (rs) rs->push_back(r);
    pend.on = true;
    pend.r = r;
    pend.half = (size_t)1 << (m0 - j - 1);
  }
  return WHIR_OK;
}

// The rounds of one sumcheck stage: on the device when the context allows it,
// else one host round trip per transcript step (sumcheck_round).
int sumcheck_stage(whir_ctx* ctx, wh::Chal& ch, Sumcheck& sd, ef* d_f, ef* d_w, int m0, int k, ef* sum, int pow_bits,
                   std::vector<ef>* rs, PendingFold& pend) {
  if (ctx->device_transcript && ctx->d_tr && ch.family == wh::kChalDuplex && k >= 1 && k <= wh::kTrMaxRounds)
    return sumcheck_stage_device(ctx, ch, sd, d_f, d_w, m0, k, sum, pow_bits, rs, pend);
  for (int j = 0; j < k; j++) {
    ef r;
    WH_TRY(sumcheck_round(ctx, ch, sd, d_f, d_w, m0 - j, sum, pow_bits, &r, pend));
    if (rs) rs->push_back(r);
  }
  return WHIR_OK;
}

// InitialStatement::evaluate for the split strategy: partial evaluations over
// the first k0 variables, then the full evaluation.
int evaluate_constraint(whir_ctx* ctx, whir_witness* w, const std::vector<ef>& point, Constraint* out) {
  const int n = w->n, k0 = w->cfg.folding_factor_0;
  uint32_t posted = 0;
  WH_TRY(wh::dot_eq(ctx, w->d_poly, 0, k0, point.data() + k0, n - k0, &posted));
  out->point = point;
  out->partial.resize((size_t)1 << k0);
  WH_TRY(wh::fetch_posted(ctx, posted, out->partial.data(), ctx->d_small, out->partial.size() * sizeof(ef)));
  WH_TRY(wh::check_dot(out->partial.data(), out->partial.size() * sizeof(ef)));
  wk::EqSmall e = wh::eq_small_host(point.data(), k0);
  ef eval = kb::ef_zero();
  for (size_t y = 0; y < out->partial.size(); y++) eval = kb::ef_add(eval, kb::ef_mul(e.v[y], out->partial[y]));
  out->eval = eval;
  return WHIR_OK;
}

int do_commit(whir_ctx* ctx, whir_witness* w, wh::Chal& ch, const uint32_t* user_points, int num_points,
              uint32_t* user_evals_out) {
  const whir_config& c = w->cfg;
  const int n = w->n, k0 = c.folding_factor_0;
  for (int i = 0; i < num_points; i++) {
    std::vector<ef> pt(n);
    for (int j = 0; j < n; j++)
      for (int l = 0; l < 4; l++) {
        const uint32_t v = user_points[4 * ((size_t)i * n + j) + l];
        WH_CHECK(v < kb::P, "point value out of range");
        pt[j].c[l] = kb::to_mont(v);
      }
    Constraint con;
    WH_TRY(evaluate_constraint(ctx, w, pt, &con));
    if (user_evals_out)
      for (int l = 0; l < 4; l++) user_evals_out[4 * i + l] = kb::from_mont(con.eval.c[l]);
    w->cons.push_back(std::move(con));
  }
  std::vector<uint32_t>& pf = w->proof;
  pf.push_back(0x50524857u);
  pf.push_back(1u);
  uint32_t root[8];
  WH_TRY(commit_matrix(ctx, w->d_poly, n - k0, k0, c.starting_log_inv_rate, 0, w->params.leaf_hash, &w->commit_tree,
                       root, w->pre_scratch ? &w->pre_plan : nullptr, &w->pre_scratch));
  for (int i = 0; i < 8; i++) pf.push_back(root[i]);
  ch.observe_digest(ctx->hp16, root);
  pf.push_back((uint32_t)c.commitment_ood_samples);
  for (int i = 0; i < c.commitment_ood_samples; i++) {
    const ef z = ch.sample_ef(ctx->hp16);
    Constraint con;
    WH_TRY(evaluate_constraint(ctx, w, expand_from_univariate(z, n), &con));
    put_ef(pf, con.eval);
    ch.observe_ef(ctx->hp16, con.eval);
    w->cons.push_back(std::move(con));
  }
  return WHIR_OK;
}

int do_prove(whir_ctx* ctx, whir_witness* wit, wh::Chal& ch) {
  const whir_config& c = wit->cfg;
  const int n = wit->n, k0 = c.folding_factor_0;
  std::vector<uint32_t>& pf = wit->proof;
  const int m = (int)wit->cons.size();

  // ---- initial sumcheck (Sumcheck::from_base_evals, sumcheck_prover.rs:237-292)
  const ef alpha = ch.sample_ef(ctx->hp16);
  std::vector<ef> apow(m > 0 ? m : 1);
  ef sum = kb::ef_zero();
  {
    ef a = kb::ef_one();
    for (int i = 0; i < m; i++) {
      apow[i] = a;
      sum = kb::ef_add(sum, kb::ef_mul(a, wit->cons[i].eval));
      a = kb::ef_mul(a, alpha);
    }
  }
  std::vector<std::vector<ef>> G(m), E(m);
  for (int i = 0; i < m; i++) {
    G[i] = wit->cons[i].partial;
    wk::EqSmall e = wh::eq_small_host(wit->cons[i].point.data(), k0);
    E[i].assign(e.v, e.v + ((size_t)1 << (k0 & 7)));
  }
  Sumcheck sd0;
  std::vector<ef> rs;
  for (int j = 0; j < k0; j++) {
    ef c0 = kb::ef_zero(), c2 = kb::ef_zero();
    for (int i = 0; i < m; i++) {
      const size_t half = G[i].size() / 2;
      ef a0 = kb::ef_zero(), a2 = kb::ef_zero();
      for (size_t y = 0; y < half; y++) {
        a0 = kb::ef_add(a0, kb::ef_mul(G[i][y], E[i][y]));
        a2 = kb::ef_add(a2, kb::ef_mul(kb::ef_sub(kb::ef_dbl(G[i][y + half]), G[i][y]),
                                       kb::ef_sub(kb::ef_dbl(E[i][y + half]), E[i][y])));
      }
      c0 = kb::ef_add(c0, kb::ef_mul(apow[i], a0));
      c2 = kb::ef_add(c2, kb::ef_mul(apow[i], a2));
    }
    ef r;
    WH_TRY(observe_and_sample(ctx, ch, sd0, c0, c2, c.starting_folding_pow_bits, &r));
    sum = extrapolate_012(c0, kb::ef_sub(sum, c0), c2, r);
    for (int i = 0; i < m; i++) {
      host_fold(G[i], r);
      host_fold(E[i], r);
    }
    rs.push_back(r);
  }
  sd0.emit(pf);

  // fold the polynomial by the k0 challenges and build the weights
  int nv = n - k0;
  const size_t N = (size_t)1 << nv;
  ef *d_f = nullptr, *d_w = nullptr;
  WH_TRY_CUDA(wh::ctx_malloc(ctx, &d_f, N * sizeof(ef)));
  WH_TRY_CUDA(wh::ctx_malloc(ctx, &d_w, N * sizeof(ef)));
  struct Guard {
    whir_ctx* ctx;
    ef** a;
    ef** b;
    ~Guard() {
      cudaFreeAsync(*a, ctx->stream);
      cudaFreeAsync(*b, ctx->stream);
    }
  } guard{ctx, &d_f, &d_w};
  {
    wk::EqSmall e = wh::eq_small_host(rs.data(), k0);
    {
      wh::StageTimer timer(ctx, wh::kStSumcheck);
      WH_TRY_CUDA(wk::fold_multi_base(wit->d_poly, k0, N, e, d_f, ctx->stream));
    }
    std::vector<std::vector<ef>> tails(m);
    std::vector<ef> scales(m);
    for (int i = 0; i < m; i++) {
      tails[i].assign(wit->cons[i].point.begin() + k0, wit->cons[i].point.end());
      scales[i] = kb::ef_mul(apow[i], E[i][0]);  // alpha^i * eq(z_i[0:k0], rs)
    }
    WH_TRY(wh::add_eq_points(ctx, d_w, nv, tails, scales, 0));
  }

  pf.push_back((uint32_t)c.n_rounds);
  PendingFold pend;
  WH_TRY_CUDA(cudaMemsetAsync(round_counter(ctx), 0, sizeof(unsigned), ctx->stream));
  Tree prev = wit->commit_tree;
  bool prev_owned = false;  // the commit tree belongs to the witness
  std::vector<ef> fold_rs = rs;
  std::vector<uint32_t> rows;
  for (int round = 0; round < c.n_rounds; round++) {
    const whir_round_config& rc = c.rounds[round];
    const int ffn = wh::ff_at(c, round + 1);
    const uint64_t new_dom = rc.domain_size >> wh::rsr_at(c, round);
    const int log_blowup = ilog2u(new_dom) - nv;
    Tree nt;
    uint32_t root[8];
    WH_TRY(flush_fold(ctx, d_f, d_w, pend));
    WH_TRY(commit_matrix(ctx, reinterpret_cast<const uint32_t*>(d_f), nv - ffn, ffn, log_blowup, 1,
                         wit->params.leaf_hash, &nt, root));
    ch.observe_digest(ctx->hp16, root);
    for (int i = 0; i < 8; i++) pf.push_back(root[i]);
    // OOD samples
    std::vector<std::vector<ef>> opts;
    std::vector<ef> oevs;
    pf.push_back((uint32_t)rc.ood_samples);
    for (int i = 0; i < rc.ood_samples; i++) {
      const ef z = ch.sample_ef(ctx->hp16);
      std::vector<ef> pt = expand_from_univariate(z, nv);
      uint32_t posted = 0;
      WH_TRY(wh::dot_eq(ctx, reinterpret_cast<const uint32_t*>(d_f), 1, 0, pt.data(), nv, &posted));
      ef ev;
      WH_TRY(wh::fetch_posted(ctx, posted, &ev, ctx->d_small, sizeof(ef)));
      ch.observe_ef(ctx->hp16, ev);
      put_ef(pf, ev);
      opts.push_back(std::move(pt));
      oevs.push_back(ev);
    }
    uint32_t pw = 0;
    if (rc.pow_bits > 0) WH_TRY(wh::grind(ctx, ch, rc.pow_bits, &pw));
    pf.push_back(pw);
    (void)ch.sample(ctx->hp16);
    const std::vector<uint64_t> idx = stir_queries(ctx, ch, rc.domain_size, wh::ff_at(c, round), rc.num_queries);
    pf.push_back((uint32_t)idx.size());
    // the openings are gathered and copied back while the constraint weights
    // are queued; their values are needed for the claimed sum only
    OpenPending op;
    WH_TRY(open_start(ctx, prev, idx, op));
    const int kprev = wh::ff_at(c, round);
    const ef* frs = fold_rs.data() + fold_rs.size() - kprev;
    std::vector<uint32_t> svars(idx.size());
    std::vector<ef> sevs(idx.size());
    const uint32_t gen = kb::to_mont(rc.folded_domain_gen);
    for (size_t q = 0; q < idx.size(); q++) svars[q] = kb::pow(gen, idx[q]);
    // Constraint::combine (constraints/mod.rs:234-248) then the sumcheck rounds
    const ef gamma = ch.sample_ef(ctx->hp16);
    std::vector<ef> gpow(opts.size());
    ef g = kb::ef_one();
    for (size_t i = 0; i < opts.size(); i++) {
      gpow[i] = g;
      sum = kb::ef_add(sum, kb::ef_mul(g, oevs[i]));
      g = kb::ef_mul(g, gamma);
    }
    WH_TRY(wh::add_eq_points(ctx, d_w, nv, opts, gpow, 1));
    std::vector<ef> spow(idx.size());
    for (size_t q = 0; q < idx.size(); q++) {
      spow[q] = g;
      g = kb::ef_mul(g, gamma);
    }
    WH_TRY(wh::add_select_vars(ctx, d_w, nv, svars, spow));
    WH_TRY(open_finish(ctx, prev, op, pf, rows));
    for (size_t q = 0; q < idx.size(); q++) {
      std::vector<ef> vals((size_t)1 << kprev);
      for (size_t v = 0; v < vals.size(); v++) {
        if (prev.ext)
          for (int l = 0; l < 4; l++) vals[v].c[l] = rows[q * prev.row_words + 4 * v + l];
        else
          vals[v] = kb::ef_from_base(rows[q * prev.row_words + v]);
      }
      sevs[q] = host_eval(vals, frs, kprev);
      sum = kb::ef_add(sum, kb::ef_mul(spow[q], sevs[q]));
    }
    Sumcheck sd;
    fold_rs.clear();
    WH_TRY(sumcheck_stage(ctx, ch, sd, d_f, d_w, nv, ffn, &sum, rc.folding_pow_bits, &fold_rs, pend));
    sd.emit(pf);
    nv -= ffn;
    if (prev_owned) free_tree(ctx, prev);
    prev = nt;
    prev_owned = true;
  }

  // ---- final round (prover/mod.rs:330-417)
  {
    const size_t fn = (size_t)1 << nv;
    std::vector<ef> fin(fn);
    WH_TRY(flush_fold(ctx, d_f, d_w, pend));
    WH_TRY(wh::fetch(ctx, fin.data(), d_f, fn * sizeof(ef)));
    pf.push_back((uint32_t)fn);
    for (size_t i = 0; i < fn; i++) {
      ch.observe_ef(ctx->hp16, fin[i]);
      put_ef(pf, fin[i]);
    }
    uint32_t pw = 0;
    if (c.final_pow_bits > 0) WH_TRY(wh::grind(ctx, ch, c.final_pow_bits, &pw));
    pf.push_back(pw);
    const whir_round_config fc = wh::final_round_config(c);
    const std::vector<uint64_t> idx = stir_queries(ctx, ch, fc.domain_size, wh::ff_at(c, c.n_rounds), c.final_queries);
    pf.push_back((uint32_t)idx.size());
    // the final openings go into the proof only: their copy overlaps the final
    // sumcheck rounds, whose records follow them in the proof
    OpenPending op;
    WH_TRY(open_start(ctx, prev, idx, op));
    if (c.final_sumcheck_rounds > 0) {
      Sumcheck sd;
      WH_TRY(sumcheck_stage(ctx, ch, sd, d_f, d_w, nv, c.final_sumcheck_rounds, &sum, c.final_folding_pow_bits,
                            nullptr, pend));
      WH_TRY(open_finish(ctx, prev, op, pf, rows));
      pf.push_back(1u);
      sd.emit(pf);
    } else {
      WH_TRY(open_finish(ctx, prev, op, pf, rows));
      pf.push_back(0u);
    }
  }
  if (prev_owned) free_tree(ctx, prev);
  return WHIR_OK;
}

// Upload of a host polynomial overlapped with the commitment DFT's first pass.
// Each of the 2^k0 columns of the committed matrix is one contiguous chunk of
// the polynomial, and pass 1 transforms a column from its own chunk only; so
// the chunks go up in kUploadGroups groups on the context's copy stream, and
// each group's Montgomery encoding and pass 1 queue on the context's stream
// behind that group's copy. Sets *done = false and queues nothing when the
// shape does not allow it: fewer columns than groups, a one-pass plan, or a
// shape the tuner has not timed yet (its first run tunes on the whole input).
int upload_with_dft(whir_ctx* ctx, whir_witness* w, const uint32_t* poly, bool* done) {
  *done = false;
  const whir_config& c = w->cfg;
  const int k0 = c.folding_factor_0, log_chunk = w->n - k0, log_blowup = c.starting_log_inv_rate;
  const int W = 1 << k0, G = wh::kUploadGroups;
  if (W < G || log_chunk < 12) return WHIR_OK;
  wk::DftPlan plan;
  if (!wh::dft_plan_known(ctx, log_chunk, k0, log_blowup, 1, &plan) || plan.log_h2 == 0) return WHIR_OK;
  Tree& t = w->commit_tree;
  const int log_h = log_chunk + log_blowup;
  const size_t h = (size_t)1 << log_h, words = h << k0;
  wk::DftTables tab;
  WH_TRY(wh::ensure_dft_tables(ctx, log_h, &tab));
  WH_TRY_CUDA(wh::ctx_malloc(ctx, &t.rows, words * 4));
  WH_TRY_CUDA(wh::ctx_malloc(ctx, &t.digests, (2 * h - 1) * 8 * 4));
  WH_TRY_CUDA(wh::ctx_malloc(ctx, &w->pre_scratch, words * 4));
  // the copies start once the allocations are ordered on the context's stream
  WH_TRY_CUDA(cudaEventRecord(ctx->up_ev[G], ctx->stream));
  WH_TRY_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->up_ev[G], 0));
  const int per = W / G;
  const size_t group = (size_t)per << log_chunk;  // words per group
  for (int g = 0; g < G; g++) {
    WH_TRY_CUDA(cudaMemcpyAsync(w->d_poly + (size_t)g * group, poly + (size_t)g * group, group * 4,
                                cudaMemcpyHostToDevice, ctx->copy_stream));
    WH_TRY_CUDA(cudaEventRecord(ctx->up_ev[g], ctx->copy_stream));
  }
  for (int g = 0; g < G; g++) {
    WH_TRY_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->up_ev[g], 0));
    WH_TRY_CUDA(wk::encode(w->d_poly + (size_t)g * group, group, ctx->stream));
    WH_TRY_CUDA(wk::dft_batch(w->d_poly, t.rows, w->pre_scratch, log_chunk, k0, log_blowup, 1, tab, plan, 1,
                              ctx->stream, g * per, per));
  }
  w->pre_plan = plan;
  *done = true;
  return WHIR_OK;
}

}  // namespace

namespace {

// whir_commit on the transcript's challenger `ch` (either family)
int commit_with(whir_ctx* ctx, const whir_protocol_params* params, int32_t n, const uint32_t* poly,
                int32_t poly_on_device, const uint32_t* user_points, int32_t num_points, uint32_t* user_evals_out,
                wh::Chal& ch, whir_witness** out) {
  WH_CHECK(ctx && params && poly && out && num_points >= 0 && (num_points == 0 || user_points), "null argument");
  *out = nullptr;
  whir_witness* w = new whir_witness();
  w->ctx = ctx;
  w->params = *params;
  w->n = n;
  int s = wh::config_new(*params, n, &w->cfg);
  if (s != WHIR_OK) {
    delete w;
    return s;
  }
  if (ctx->device < 0) {
    delete w;
    wh::set_error("host-only context (device -1) cannot run device work");
    return WHIR_ERR_NO_DEVICE;
  }
  if (w->cfg.folding_factor_0 > 6) {
    delete w;
    wh::set_error("folding factor above 6 is not supported");
    return WHIR_ERR_INVALID;
  }
  cudaSetDevice(ctx->device);
  const size_t N = (size_t)1 << n;
  if (poly_on_device) {
    w->d_poly = const_cast<uint32_t*>(poly);
  } else {
    // values are KoalaBear elements, canonical by type as in the reference
    if (wh::ctx_malloc(ctx, &w->d_poly, N * 4) != cudaSuccess) {
      delete w;
      wh::set_error("polynomial allocation failed");
      return WHIR_ERR_NOMEM;
    }
    w->own_poly = true;
    bool piped = false;
    s = upload_with_dft(ctx, w, poly, &piped);
    if (s != WHIR_OK) {
      whir_witness_free(w);
      return s;
    }
    if (!piped && (cudaMemcpyAsync(w->d_poly, poly, N * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
                   wk::encode(w->d_poly, N, ctx->stream) != cudaSuccess)) {
      whir_witness_free(w);
      wh::set_error("polynomial upload failed");
      return WHIR_ERR_CUDA;
    }
  }
  s = do_commit(ctx, w, ch, user_points, num_points, user_evals_out);
  if (s != WHIR_OK) {
    whir_witness_free(w);
    return s;
  }
  *out = w;
  return WHIR_OK;
}

// whir_prove on the transcript's challenger `ch`
int prove_with(whir_ctx* ctx, whir_witness* w, wh::Chal& ch, uint32_t* proof_out, size_t cap_words,
               size_t* proof_words) {
  WH_CHECK(ctx && w && proof_words && w->ctx == ctx, "bad argument");
  WH_CHECK(!w->proved, "witness already proved");
  cudaSetDevice(ctx->device);
  WH_TRY(do_prove(ctx, w, ch));
  w->proved = true;
  *proof_words = w->proof.size();
  if (!proof_out || cap_words < w->proof.size()) {
    wh::set_error("proof buffer too small");
    return WHIR_ERR_BUFFER;
  }
  memcpy(proof_out, w->proof.data(), w->proof.size() * 4);
  return WHIR_OK;
}

}  // namespace

extern "C" {

// The split API carries the duplex challenger's state (whir_challenger); the
// Keccak configuration, whose challenger state is a hash input buffer, runs
// through whir_commit_and_prove.
int whir_commit(whir_ctx* ctx, const whir_protocol_params* params, int32_t n, const uint32_t* poly,
                int32_t poly_on_device, const uint32_t* user_points, int32_t num_points, uint32_t* user_evals_out,
                whir_challenger* chs, whir_witness** out) {
  WH_CHECK(params && chs, "null argument");
  WH_CHECK(params->leaf_hash != WHIR_LEAF_KECCAK, "the Keccak configuration runs through whir_commit_and_prove");
  wh::Chal ch;
  ch.load(*chs);
  WH_TRY(commit_with(ctx, params, n, poly, poly_on_device, user_points, num_points, user_evals_out, ch, out));
  ch.store(*chs);
  return WHIR_OK;
}

int whir_prove(whir_ctx* ctx, whir_witness* w, whir_challenger* chs, uint32_t* proof_out, size_t cap_words,
               size_t* proof_words) {
  WH_CHECK(w && chs, "bad argument");
  wh::Chal ch;
  ch.load(*chs);
  const int s = prove_with(ctx, w, ch, proof_out, cap_words, proof_words);
  if (s == WHIR_OK || s == WHIR_ERR_BUFFER) ch.store(*chs);
  return s;
}

int whir_witness_free(whir_witness* w) {
  if (!w) return WHIR_OK;
  whir_ctx* ctx = w->ctx;
  // copies of a pipelined upload end before their buffers go back to the pool
  // (and before the caller may reuse the host polynomial)
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  free_tree(ctx, w->commit_tree);
  if (w->pre_scratch) cudaFreeAsync(w->pre_scratch, ctx->stream);
  if (w->own_poly && w->d_poly) cudaFreeAsync(w->d_poly, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  delete w;
  return WHIR_OK;
}

int whir_commit_and_prove(whir_ctx* ctx, const whir_protocol_params* params, int32_t n, const uint32_t* poly,
                          int32_t poly_on_device, const uint32_t* user_points, int32_t num_points,
                          uint32_t* user_evals_out, uint32_t* proof_out, size_t cap_words, size_t* proof_words,
                          uint32_t* checkpoint) {
  WH_CHECK(ctx && params && proof_words, "null argument");
  whir_config cfg;
  WH_TRY(wh::config_new(*params, n, &cfg));
  WH_CHECK(ctx->device >= 0, "host-only context (device -1) cannot run device work");
  wh::Chal ch;
  bool cached = false;
  for (const whir_ctx::DsEntry& e : ctx->ds_cache)
    if (e.n == n && memcmp(&e.params, params, sizeof(*params)) == 0) {
      ch = e.ch;
      cached = true;
      break;
    }
  if (!cached) {
    if (params->leaf_hash == WHIR_LEAF_KECCAK) ch.init_keccak();
    else ch.init();
    for (uint32_t v : wh::domain_separator(cfg, params->ds_digest_elems)) ch.observe(ctx->hp16, kb::to_mont(v));
    if (ctx->ds_cache.size() >= 8) ctx->ds_cache.erase(ctx->ds_cache.begin());
    ctx->ds_cache.push_back(whir_ctx::DsEntry{*params, n, ch});
  }
  whir_witness* w = nullptr;
  WH_TRY(commit_with(ctx, params, n, poly, poly_on_device, user_points, num_points, user_evals_out, ch, &w));
  int s = prove_with(ctx, w, ch, proof_out, cap_words, proof_words);
  whir_witness_free(w);
  if (s != WHIR_OK) return s;
  if (checkpoint)
    for (int i = 0; i < 4; i++) checkpoint[i] = kb::from_mont(ch.sample(ctx->hp16));
  return WHIR_OK;
}

}  // extern "C"
