/*
 * Oracle (test infrastructure only): the WHIR protocol of tcoratger/whir-p3
 * restated on the CPU — parameter derivation, domain separator, STIR query
 * sampling, commit, prove (Classic sumcheck strategy) and verify.
 *
 * Followed line by line (paths inside the reference project):
 *   WhirConfig::new ................. src/whir/parameters.rs:81-234
 *   final_round_config / inv_rate ... src/whir/parameters.rs:372-416
 *   SecurityAssumption .............. src/parameters/errors.rs:25-187
 *   compute_number_of_rounds ........ src/parameters/mod.rs:91-125
 *   DomainSeparator ................. src/fiat_shamir/domain_separator.rs:57-213
 *   get_challenge_stir_queries ...... src/whir/utils.rs:24-145
 *   CommitmentWriter::commit ........ src/whir/committer/writer.rs:56-109
 *   Prover::prove/round/final_round . src/whir/prover/mod.rs:97-417
 *   Sumcheck (Classic path) ......... src/sumcheck/sumcheck_prover.rs:65-161,331-357
 *   ProductPolynomial::round ........ src/sumcheck/product_polynomial.rs:307-364
 *   SumcheckData::observe_and_sample  src/whir/proof.rs:163-193
 *   EqStatement / SelectStatement ... src/whir/constraints/statement/{eq,select}.rs
 *   Verifier::verify ................ src/whir/verifier/mod.rs:58-400, sumcheck.rs:31-101
 *   ParsedCommitment ................ src/whir/committer/reader.rs:55-120
 *   ConstraintPolyEvaluator ......... src/whir/constraints/evaluator.rs:8-62
 *
 * The proof is emitted in a flat little-endian uint32 encoding (documented in
 * the product's include/whir_b200.h) that the GPU path must reproduce word
 * for word.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "or_field.h"

#define EF_BITS 124 /* EF::bits() for the quartic KoalaBear extension */
static const double LOG2_10_ = 3.321928094887362347870319429489390175864831393;

/* ------------------------------------------------------------------------ */
/* Parameters                                                                */
/* ------------------------------------------------------------------------ */

static int ff_at(const or_params* p, int round) {
  return round == 0 ? p->folding_factor_0 : p->folding_factor;
}

static double log_eta(int s, int lir) {
  switch (s) {
    case 0: return 0.;
    case 1: return -(0.5 * (double)lir + LOG2_10_ + 1.);
    default: return -((double)lir + LOG2_10_ + 1.);
  }
}
static double list_size_bits(int s, int d, int lir) {
  double le = log_eta(s, lir);
  switch (s) {
    case 0: return 0.;
    case 1: return (double)lir / 2. - (1. + le);
    default: return (double)(d + lir) - le;
  }
}
static double prox_gaps_error(int s, int d, int lir, int fbits, int nf) {
  double le = log_eta(s, lir), e;
  switch (s) {
    case 0: e = (double)(d + lir); break;
    case 1: {
      double num = (double)(2 * d);
      double sr = 1. + LOG2_10_ + 0.5 * (double)lir;
      e = num + 7. * (fmin(sr, -le) - 1.);
      break;
    }
    default: e = (double)(d + 2 * lir) - le;
  }
  return (double)fbits - (e + log2((double)nf - 1.));
}
static double log_1_delta(int s, int lir) {
  double le = log_eta(s, lir);
  double eta = pow(2., le);
  double rate = 1. / (double)(1 << lir);
  double delta;
  switch (s) {
    case 0: delta = 0.5 * (1. - rate); break;
    case 1: delta = 1. - sqrt(rate) - eta; break;
    default: delta = 1. - rate - eta;
  }
  return log2(1. - delta);
}
static int queries_for(int s, int psl, int lir) {
  double q = -(double)psl / log_1_delta(s, lir);
  return (int)ceil(q);
}
static double queries_error(int s, int lir, int q) { return -(double)q * log_1_delta(s, lir); }
static double ood_error(int s, int d, int lir, int fbits, int o) {
  if (s == 0) return 0.;
  double lsb = list_size_bits(s, d, lir);
  double err = 2. * lsb + (double)(d * o);
  return (double)(o * fbits) + 1. - err;
}
static int ood_samples_for(int s, int sec, int d, int lir, int fbits) {
  if (s == 0) return 0;
  for (int o = 1; o < 64; o++)
    if (ood_error(s, d, lir, fbits, o) >= (double)sec) return o;
  return -1;
}
static double fold_sumcheck_err(int s, int fbits, int nv, int lir) {
  return (double)fbits - (list_size_bits(s, nv, lir) + 1.);
}
static double folding_pow_bits(int sec, int s, int fbits, int nv, int lir) {
  double pg = prox_gaps_error(s, nv, lir, fbits, 2);
  double sc = fold_sumcheck_err(s, fbits, nv, lir);
  return fmax(0., (double)sec - fmin(pg, sc));
}
static double combination_err(int s, int fbits, int nv, int lir, int ood, int q) {
  double ls = list_size_bits(s, nv, lir);
  return (double)fbits - (log2((double)(ood + q)) + ls + 1.);
}
static size_t as_usize(double v) { return v <= 0. ? 0 : (size_t)v; }

static void rounds_of(const or_params* p, int n, int* nr, int* fin) {
  if (p->folding_factor_0 == p->folding_factor) {
    int f = p->folding_factor;
    if (n <= 6) { *nr = 0; *fin = n - f; return; }
    int r = (n - 6 + f - 1) / f;
    *nr = r - 1;
    *fin = n - r * f;
  } else {
    int nv1 = n - p->folding_factor_0, f = p->folding_factor;
    if (nv1 < 6) { *nr = 0; *fin = nv1; return; }
    int r = (nv1 - 6 + f - 1) / f;
    *nr = r;
    *fin = nv1 - r * f;
  }
}

static int ilog2_u64(uint64_t v) { int r = -1; while (v) { r++; v >>= 1; } return r; }

int or_config_new(const or_params* p, int n, or_config* c) {
  memset(c, 0, sizeof(*c));
  if (p->folding_factor_0 <= 0 || p->folding_factor <= 0) return -1;
  if (p->folding_factor_0 > n || p->folding_factor > n) return -1;
  if (p->rs_reduction > p->folding_factor_0) return -2;
  const int s = p->soundness, sec = p->security_level, fb = EF_BITS;
  const int psl = sec > p->pow_bits ? sec - p->pow_bits : 0;
  int lir = p->starting_log_inv_rate, nv = n;
  int log_domain = n + lir;
  uint64_t domain = 1ull << log_domain;
  if (log_domain - p->folding_factor_0 > OR_TWO_ADICITY) return -3;
  int nr, fin;
  rounds_of(p, n, &nr, &fin);
  if (nr > OR_MAX_ROUNDS) return -4;
  c->num_variables = n;
  c->security_level = sec;
  c->max_pow_bits = p->pow_bits;
  c->soundness = s;
  c->starting_log_inv_rate = lir;
  c->folding_factor_0 = p->folding_factor_0;
  c->folding_factor = p->folding_factor;
  c->rs_reduction = p->rs_reduction;
  c->commitment_ood_samples = ood_samples_for(s, sec, n, lir, fb);
  c->starting_folding_pow_bits = (int)as_usize(folding_pow_bits(sec, s, fb, n, lir));
  nv -= p->folding_factor_0;
  for (int r = 0; r < nr; r++) {
    int rsr = r == 0 ? p->rs_reduction : 1;
    int next_rate = lir + (ff_at(p, r) - rsr);
    int q = queries_for(s, psl, lir);
    int ood = ood_samples_for(s, sec, nv, next_rate, fb);
    double qe = queries_error(s, lir, q);
    double ce = combination_err(s, fb, nv, next_rate, ood, q);
    double pw = fmax(0., (double)sec - fmin(qe, ce));
    double fpw = folding_pow_bits(sec, s, fb, nv, next_rate);
    or_round_cfg* rc = &c->rounds[r];
    rc->pow_bits = (int)as_usize(pw);
    rc->folding_pow_bits = (int)as_usize(fpw);
    rc->num_queries = q;
    rc->ood_samples = ood;
    rc->num_variables = nv;
    rc->folding_factor = ff_at(p, r);
    rc->domain_size = domain;
    rc->folded_domain_gen = or_two_adic_generator(ilog2_u64(domain) - ff_at(p, r));
    nv -= ff_at(p, r + 1);
    lir = next_rate;
    domain >>= rsr;
  }
  c->n_rounds = nr;
  c->final_sumcheck_rounds = fin;
  c->final_queries = queries_for(s, psl, lir);
  c->final_pow_bits = (int)as_usize(fmax(0., (double)sec - queries_error(s, lir, c->final_queries)));
  c->final_folding_pow_bits = (int)as_usize(fmax(0., (double)sec - (double)(fb - 1)));
  return 0;
}

static int cfg_ff(const or_config* c, int round) {
  return round == 0 ? c->folding_factor_0 : c->folding_factor;
}
static int cfg_rsr(const or_config* c, int round) { return round == 0 ? c->rs_reduction : 1; }

static or_round_cfg final_round_config(const or_config* c) {
  or_round_cfg r;
  memset(&r, 0, sizeof(r));
  if (c->n_rounds == 0) {
    uint64_t d = 1ull << (c->num_variables + c->starting_log_inv_rate);
    r.num_variables = c->num_variables - c->folding_factor_0;
    r.folding_factor = cfg_ff(c, 0);
    r.num_queries = c->final_queries;
    r.pow_bits = c->final_pow_bits;
    r.domain_size = d;
    r.folded_domain_gen = or_two_adic_generator(ilog2_u64(d) - c->folding_factor_0);
    r.ood_samples = 0;
    r.folding_pow_bits = c->final_folding_pow_bits;
  } else {
    const or_round_cfg* last = &c->rounds[c->n_rounds - 1];
    int ff = cfg_ff(c, c->n_rounds);
    uint64_t d = last->domain_size >> cfg_rsr(c, c->n_rounds - 1);
    r.num_variables = last->num_variables - ff;
    r.folding_factor = ff;
    r.num_queries = c->final_queries;
    r.pow_bits = c->final_pow_bits;
    r.domain_size = d;
    r.folded_domain_gen = or_two_adic_generator(ilog2_u64(d) - ff);
    r.ood_samples = last->ood_samples;
    r.folding_pow_bits = c->final_folding_pow_bits;
  }
  return r;
}

/* ------------------------------------------------------------------------ */
/* Domain separator                                                          */
/* ------------------------------------------------------------------------ */

typedef struct { uint32_t* v; int len, cap; } u32vec;
static void push(u32vec* a, uint32_t x) { if (a->len < a->cap) a->v[a->len] = x; a->len++; }
enum { PAT_SAMPLE = 0, PAT_OBSERVE = 1, PAT_HINT = 2 };
enum { S_INIT_COMB = 0, S_FOLD_SKIP = 1, S_FOLD = 2, S_COMB = 3, S_STIR = 4, S_FINAL_Q = 5, S_POW = 6, S_OOD = 7 };
enum { O_DIGEST = 0, O_OOD_ANS = 1, O_SC_POLY = 2, O_SC_SKIP = 3, O_STIR_ANS = 4, O_FINAL = 5, O_POW_NONCE = 6 };
enum { H_STIR_Q = 0, H_STIR_A = 1, H_MERKLE = 2, H_DEFERRED = 3 };
static void ds_obs(u32vec* a, uint64_t cnt, int tag) { push(a, or_add(or_add(tag, (uint32_t)(cnt % OR_P)), PAT_OBSERVE)); }
static void ds_smp(u32vec* a, uint64_t cnt, int tag) { push(a, or_add(or_add(tag, (uint32_t)(cnt % OR_P)), PAT_SAMPLE)); }
static void ds_hint(u32vec* a, int tag) { push(a, or_add(tag, PAT_HINT)); }
static void ds_pow(u32vec* a, int bits) { if (bits > 0) { ds_smp(a, 32, S_POW); ds_obs(a, 8, O_POW_NONCE); } }
static void ds_sumcheck(u32vec* a, int rounds, int pow_bits) {
  for (int i = 0; i < rounds; i++) { ds_obs(a, 3, O_SC_POLY); ds_smp(a, 1, S_FOLD); ds_pow(a, pow_bits); }
}
static void ds_ood(u32vec* a, int n) { if (n > 0) { ds_smp(a, n, S_OOD); ds_obs(a, n, O_OOD_ANS); } }
static int ceil_div(int a, int b) { return (a + b - 1) / b; }

int or_domain_separator(const or_config* c, int digest_elems, uint32_t* out, int cap) {
  u32vec a = {out, 0, cap};
  ds_obs(&a, digest_elems, O_DIGEST);
  if (c->commitment_ood_samples > 0) ds_ood(&a, c->commitment_ood_samples);
  ds_smp(&a, 1, S_INIT_COMB);
  ds_sumcheck(&a, cfg_ff(c, 0), c->starting_folding_pow_bits);
  uint64_t domain = 1ull << (c->num_variables + c->starting_log_inv_rate);
  for (int r = 0; r < c->n_rounds; r++) {
    const or_round_cfg* rc = &c->rounds[r];
    uint64_t folded = domain >> cfg_ff(c, r);
    int bytes = ceil_div(ilog2_u64(folded * 2 - 1), 8);
    ds_obs(&a, digest_elems, O_DIGEST);
    ds_ood(&a, rc->ood_samples);
    ds_smp(&a, (uint64_t)rc->num_queries * bytes, S_STIR);
    ds_hint(&a, H_STIR_Q);
    ds_hint(&a, H_MERKLE);
    ds_pow(&a, rc->pow_bits);
    ds_smp(&a, 1, S_COMB);
    ds_sumcheck(&a, cfg_ff(c, r + 1), rc->folding_pow_bits);
    domain >>= cfg_rsr(c, r);
  }
  uint64_t folded = domain >> cfg_ff(c, c->n_rounds);
  int bytes = ceil_div(ilog2_u64(folded * 2 - 1), 8);
  ds_obs(&a, 1ull << c->final_sumcheck_rounds, O_FINAL);
  ds_smp(&a, (uint64_t)bytes * c->final_queries, S_FINAL_Q);
  ds_hint(&a, H_STIR_A);
  ds_hint(&a, H_MERKLE);
  ds_pow(&a, c->final_pow_bits);
  ds_sumcheck(&a, c->final_sumcheck_rounds, c->final_folding_pow_bits);
  ds_hint(&a, H_DEFERRED);
  return a.len;
}

/* ------------------------------------------------------------------------ */
/* Transcript helpers                                                        */
/* ------------------------------------------------------------------------ */

typedef struct {
  or_chal ch;
  or_p2_params p16, p24;
  int keccak;   /* leaf_hash 2: Keccak MMCS with SerializingChallenger32 */
  or_kchal kc;
} tr_t;

/* the transcript's challenger: DuplexChallenger over Poseidon2-16, or the
 * Keccak SerializingChallenger32 of the Keccak configuration */
static void t_obs(tr_t* t, uint32_t v) {
  if (t->keccak) or_kchal_observe(&t->kc, v);
  else or_chal_observe(&t->ch, &t->p16, v);
}
static uint32_t t_smp(tr_t* t) { return t->keccak ? or_kchal_sample(&t->kc) : or_chal_sample(&t->ch, &t->p16); }
static uint64_t t_bits(tr_t* t, int bits) {
  return t->keccak ? or_kchal_sample_bits(&t->kc, bits) : or_chal_sample_bits(&t->ch, &t->p16, bits);
}
static uint32_t t_grind(tr_t* t, int bits) {
  return t->keccak ? or_kchal_grind(&t->kc, bits) : or_chal_grind(&t->ch, &t->p16, bits);
}
static int t_check(tr_t* t, int bits, uint32_t w) {
  return t->keccak ? or_kchal_check_witness(&t->kc, bits, w) : or_chal_check_witness(&t->ch, &t->p16, bits, w);
}

static int g_p2_set = 0;
static or_p2_params g_p16, g_p24;

void or_p2_select(const or_p2_params* p16, const or_p2_params* p24) {
  if (p16 && p24) {
    g_p16 = *p16;
    g_p24 = *p24;
    g_p2_set = 1;
  } else {
    g_p2_set = 0;
  }
}

static void p2_selected(or_p2_params* p16, or_p2_params* p24) {
  if (g_p2_set) {
    *p16 = g_p16;
    *p24 = g_p24;
  } else {
    or_p2_default(p16, p24);
  }
}

static or_ef sample_ef(tr_t* t) {
  or_ef r;
  for (int i = 0; i < 4; i++) r.c[i] = t_smp(t);
  return r;
}
static void observe_ef(tr_t* t, or_ef v) {
  for (int i = 0; i < 4; i++) t_obs(t, v.c[i]);
}
static void observe_digest(tr_t* t, const uint32_t* d) {
  for (int i = 0; i < 8; i++) t_obs(t, d[i]);
}

/* get_challenge_stir_queries (src/whir/utils.rs:24-145); returns count after sort+dedup */
static int stir_queries(tr_t* t, uint64_t domain_size, int ff, int nq, uint64_t* out) {
  uint64_t folded = domain_size >> ff;
  int bits = ilog2_u64(folded);
  const int max_bits = 20; /* min(F::bits() - 1, 20) with F::bits() = 31 */
  int total = nq * bits;
  int cnt = 0;
  if (total <= max_bits) {
    uint64_t all = t_bits(t, total);
    uint64_t mask = (1ull << bits) - 1;
    for (int i = 0; i < nq; i++) { out[cnt++] = (all & mask) % folded; all >>= bits; }
  } else {
    int per = max_bits / bits;
    if (per >= 2) {
      int rem = nq;
      uint64_t mask = (1ull << bits) - 1;
      while (rem > 0) {
        int b = rem < per ? rem : per;
        uint64_t all = t_bits(t, b * bits);
        for (int i = 0; i < b; i++) { out[cnt++] = (all & mask) % folded; all >>= bits; }
        rem -= b;
      }
    } else {
      for (int i = 0; i < nq; i++) out[cnt++] = t_bits(t, bits);
    }
  }
  /* sort_unstable + dedup */
  for (int i = 1; i < cnt; i++) {
    uint64_t v = out[i];
    int j = i - 1;
    while (j >= 0 && out[j] > v) { out[j + 1] = out[j]; j--; }
    out[j + 1] = v;
  }
  int m = 0;
  for (int i = 0; i < cnt; i++)
    if (m == 0 || out[m - 1] != out[i]) out[m++] = out[i];
  return m;
}

/* ------------------------------------------------------------------------ */
/* Proof writer                                                              */
/* ------------------------------------------------------------------------ */

typedef struct { uint32_t* w; size_t len, cap; } buf_t;
static void bw(buf_t* b, uint32_t x) {
  if (b->len == b->cap) { b->cap = b->cap ? 2 * b->cap : 1024; b->w = (uint32_t*)realloc(b->w, b->cap * 4); }
  b->w[b->len++] = x;
}
static void bw_ef(buf_t* b, or_ef v) { for (int i = 0; i < 4; i++) bw(b, v.c[i]); }

/* sumcheck section: n_polys, (c0,c2) pairs, n_pow, witnesses */
typedef struct {
  or_ef* polys;
  uint32_t* pows;
  int n, npow;
} sc_data;
static void sc_push(sc_data* d, or_ef c0, or_ef c2) {
  d->polys = (or_ef*)realloc(d->polys, (size_t)(d->n + 1) * 2 * sizeof(or_ef));
  d->polys[2 * d->n] = c0;
  d->polys[2 * d->n + 1] = c2;
  d->n++;
}
static void sc_pow(sc_data* d, uint32_t w) {
  d->pows = (uint32_t*)realloc(d->pows, (size_t)(d->npow + 1) * 4);
  d->pows[d->npow++] = w;
}
static void bw_sc(buf_t* b, const sc_data* d) {
  bw(b, (uint32_t)d->n);
  for (int i = 0; i < 2 * d->n; i++) bw_ef(b, d->polys[i]);
  bw(b, (uint32_t)d->npow);
  for (int i = 0; i < d->npow; i++) bw(b, d->pows[i]);
}
static void sc_free(sc_data* d) { free(d->polys); free(d->pows); memset(d, 0, sizeof(*d)); }

/* ------------------------------------------------------------------------ */
/* Prover state                                                              */
/* ------------------------------------------------------------------------ */

typedef struct {
  int log_h, row_words, ext;
  uint32_t* rows;    /* codeword matrix, row-major */
  uint32_t* digests; /* (2h-1)*8 */
} tree_t;

static void tree_build(tr_t* t, const or_params* p, tree_t* tr, uint32_t* root) {
  size_t h = (size_t)1 << tr->log_h;
  tr->digests = (uint32_t*)malloc((2 * h - 1) * 8 * 4);
  or_merkle_build(&t->p16, &t->p24, p->leaf_hash, tr->rows, tr->log_h, tr->row_words, tr->digests, root);
}
static void tree_free(tree_t* tr) { free(tr->rows); free(tr->digests); memset(tr, 0, sizeof(*tr)); }

/* query opening: kind, n_values, values, path_len, path */
static void tree_open(const tree_t* tr, uint64_t idx, buf_t* b, uint32_t* row_out) {
  bw(b, (uint32_t)tr->ext);
  int nvals = tr->ext ? tr->row_words / 4 : tr->row_words;
  bw(b, (uint32_t)nvals);
  for (int i = 0; i < tr->row_words; i++) {
    uint32_t v = tr->rows[idx * tr->row_words + i];
    bw(b, v);
    if (row_out) row_out[i] = v;
  }
  bw(b, (uint32_t)tr->log_h);
  size_t off = 0, n = (size_t)1 << tr->log_h;
  for (int l = 0; l < tr->log_h; l++) {
    size_t sib = (idx >> l) ^ 1;
    for (int i = 0; i < 8; i++) bw(b, tr->digests[(off + sib) * 8 + i]);
    off += n;
    n >>= 1;
  }
}

static or_ef ldv(const uint32_t* p) { or_ef r; memcpy(r.c, p, 16); return r; }

/* extrapolate_012 (src/sumcheck/lagrange.rs:141-147) */
static or_ef extrapolate_012(or_ef e0, or_ef e1, or_ef e2, or_ef r) {
  const uint32_t inv2 = (OR_P + 1) / 2;
  or_ef one = or_ef_from(1), two = or_ef_from(2);
  or_ef l0 = or_ef_mul_base(or_ef_mul(or_ef_sub(r, one), or_ef_sub(r, two)), inv2);
  or_ef l1 = or_ef_mul(r, or_ef_sub(two, r));
  or_ef l2 = or_ef_mul_base(or_ef_mul(r, or_ef_sub(r, one)), inv2);
  return or_ef_add(or_ef_add(or_ef_mul(e0, l0), or_ef_mul(e1, l1)), or_ef_mul(e2, l2));
}

void or_extrapolate_012(const uint32_t* e0, const uint32_t* e1, const uint32_t* e2, const uint32_t* r,
                        uint32_t* out) {
  or_ef v = extrapolate_012(ldv(e0), ldv(e1), ldv(e2), ldv(r));
  memcpy(out, v.c, 16);
}

/* SumcheckData::observe_and_sample */
static or_ef observe_and_sample(tr_t* t, sc_data* d, or_ef c0, or_ef c2, int pow_bits) {
  sc_push(d, c0, c2);
  observe_ef(t, c0);
  observe_ef(t, c2);
  if (pow_bits > 0) sc_pow(d, t_grind(t, pow_bits));
  return sample_ef(t);
}

static void expand_from_univariate(or_ef z, int n, uint32_t* out) {
  or_ef cur = z;
  for (int i = n - 1; i >= 0; i--) {
    memcpy(out + 4 * i, cur.c, 16);
    cur = or_ef_square(cur);
  }
}


/* W += sum_i gamma^i eq(z_i, .) over 2^n entries; returns sum_i gamma^i s_i */
static or_ef combine_eq(uint32_t* w, int n, const uint32_t* pts, const or_ef* evals, int m, or_ef gamma) {
  size_t N = (size_t)1 << n;
  uint32_t* tmp = (uint32_t*)malloc(N * 16);
  or_ef g = or_ef_from(1), s = or_ef_zero();
  for (int i = 0; i < m; i++) {
    or_eq_table(pts + (size_t)i * n * 4, n, g.c, tmp);
#pragma omp parallel for schedule(static) if (N > 4096)
    for (size_t x = 0; x < N; x++) {
      or_ef a = ldv(w + 4 * x), b = ldv(tmp + 4 * x);
      a = or_ef_add(a, b);
      memcpy(w + 4 * x, a.c, 16);
    }
    s = or_ef_add(s, or_ef_mul(evals[i], g));
    g = or_ef_mul(g, gamma);
  }
  free(tmp);
  return s;
}

/* one ProductPolynomial::round on extension f, w of 2^n entries (n >= 1) */
static or_ef sc_round(tr_t* t, sc_data* d, uint32_t* f, uint32_t* w, int n, or_ef* sum, int pow_bits) {
  uint32_t c0[4], c2[4];
  or_sumcheck_coeffs(f, w, n, c0, c2);
  or_ef e0 = ldv(c0), e2 = ldv(c2);
  or_ef r = observe_and_sample(t, d, e0, e2, pow_bits);
  or_fold_ext(f, n, r.c);
  or_fold_ext(w, n, r.c);
  *sum = extrapolate_012(e0, or_ef_sub(*sum, e0), e2, r);
  return r;
}

int or_whir_prove(const or_params* prm, int n, const uint32_t* poly, const uint32_t* user_points,
                  int num_points, uint32_t** proof_out, size_t* proof_words, uint32_t* checkpoint) {
  or_config cfg;
  int rc = or_config_new(prm, n, &cfg);
  if (rc) return rc;
  tr_t t;
  p2_selected(&t.p16, &t.p24);
  or_chal_init(&t.ch);
  t.keccak = prm->leaf_hash == 2;
  or_kchal_init(&t.kc);
  {
    int len = or_domain_separator(&cfg, prm->ds_digest_elems, NULL, 0);
    uint32_t* pat = (uint32_t*)malloc((size_t)len * 4);
    or_domain_separator(&cfg, prm->ds_digest_elems, pat, len);
    for (int i = 0; i < len; i++) t_obs(&t, pat[i]);
    free(pat);
  }
  const size_t N = (size_t)1 << n;
  buf_t b = {0, 0, 0};
  bw(&b, 0x50524857u); /* "WHRP" */
  bw(&b, 1u);

  /* statement: user constraints evaluated before commit, OOD appended in commit */
  int max_c = num_points + cfg.commitment_ood_samples;
  uint32_t* pts = (uint32_t*)malloc((size_t)(max_c > 0 ? max_c : 1) * n * 16 + 16);
  or_ef* evs = (or_ef*)malloc((size_t)(max_c > 0 ? max_c : 1) * sizeof(or_ef));
  int nc = 0;
  for (int i = 0; i < num_points; i++) {
    memcpy(pts + (size_t)nc * n * 4, user_points + (size_t)i * n * 4, (size_t)n * 16);
    uint32_t e[4];
    or_eval_base(poly, n, user_points + (size_t)i * n * 4, e);
    evs[nc++] = ldv(e);
  }

  /* ---- commit (writer.rs:56-109) ---- */
  tree_t cur_tree;
  memset(&cur_tree, 0, sizeof(cur_tree));
  {
    int ff0 = cfg.folding_factor_0;
    int log_chunk = n - ff0;
    cur_tree.log_h = n + cfg.starting_log_inv_rate - ff0;
    cur_tree.row_words = 1 << ff0;
    cur_tree.ext = 0;
    cur_tree.rows = (uint32_t*)malloc(((size_t)1 << cur_tree.log_h) * cur_tree.row_words * 4);
    or_dft_batch(poly, log_chunk, ff0, cfg.starting_log_inv_rate, 0, cur_tree.rows);
    uint32_t root[8];
    tree_build(&t, prm, &cur_tree, root);
    for (int i = 0; i < 8; i++) bw(&b, root[i]);
    observe_digest(&t, root);
    bw(&b, (uint32_t)cfg.commitment_ood_samples);
    for (int i = 0; i < cfg.commitment_ood_samples; i++) {
      or_ef z = sample_ef(&t);
      expand_from_univariate(z, n, pts + (size_t)nc * n * 4);
      uint32_t e[4];
      or_eval_base(poly, n, pts + (size_t)nc * n * 4, e);
      evs[nc] = ldv(e);
      bw_ef(&b, evs[nc]);
      observe_ef(&t, evs[nc]);
      nc++;
    }
  }

  /* ---- initial sumcheck, Classic strategy (sumcheck_prover.rs:65-161) ---- */
  sc_data scd;
  memset(&scd, 0, sizeof(scd));
  int ff0 = cfg.folding_factor_0;
  uint32_t* f = (uint32_t*)malloc((N / 2) * 16);
  uint32_t* w = (uint32_t*)calloc(N, 16);
  or_ef sum;
  or_ef* rs = (or_ef*)malloc(sizeof(or_ef) * 64);
  int nrs = 0;
  {
    or_ef alpha = sample_ef(&t);
    sum = combine_eq(w, n, pts, evs, nc, alpha);
    /* first round on base evals */
    size_t mid = N / 2;
    or_ef a0 = or_ef_zero(), a2 = or_ef_zero();
    for (size_t i = 0; i < mid; i++) {
      or_ef el = or_ef_from(poly[i]), eh = or_ef_from(poly[i + mid]);
      or_ef wl = ldv(w + 4 * i), wh = ldv(w + 4 * (i + mid));
      a0 = or_ef_add(a0, or_ef_mul(wl, el));
      a2 = or_ef_add(a2, or_ef_mul(or_ef_sub(or_ef_double(wh), wl), or_ef_sub(or_ef_double(eh), el)));
    }
    or_ef r = observe_and_sample(&t, &scd, a0, a2, cfg.starting_folding_pow_bits);
    or_fold_ext(w, n, r.c);
    or_fold_base(poly, n, r.c, f);
    sum = extrapolate_012(a0, or_ef_sub(sum, a0), a2, r);
    rs[nrs++] = r;
    for (int j = 1; j < ff0; j++) rs[nrs++] = sc_round(&t, &scd, f, w, n - j, &sum, cfg.starting_folding_pow_bits);
  }
  bw_sc(&b, &scd);
  sc_free(&scd);
  int nv = n - ff0;

  bw(&b, (uint32_t)cfg.n_rounds);
  uint32_t* row = (uint32_t*)malloc(4096 * 4);
  uint64_t* idx = (uint64_t*)malloc(sizeof(uint64_t) * 4096);
  for (int round = 0; round < cfg.n_rounds; round++) {
    const or_round_cfg* rp = &cfg.rounds[round];
    int ffn = cfg_ff(&cfg, round + 1);
    uint64_t new_dom = rp->domain_size >> cfg_rsr(&cfg, round);
    int log_blowup = ilog2_u64(new_dom) - nv;
    tree_t nt;
    memset(&nt, 0, sizeof(nt));
    nt.log_h = nv - ffn + log_blowup;
    nt.ext = 1;
    nt.row_words = 4 << ffn;
    nt.rows = (uint32_t*)malloc(((size_t)1 << nt.log_h) * nt.row_words * 4);
    or_dft_batch(f, nv - ffn, ffn, log_blowup, 1, nt.rows);
    uint32_t root[8];
    tree_build(&t, prm, &nt, root);
    observe_digest(&t, root);
    for (int i = 0; i < 8; i++) bw(&b, root[i]);
    /* OOD */
    int no = rp->ood_samples;
    uint32_t* opts = (uint32_t*)malloc((size_t)(no > 0 ? no : 1) * nv * 16 + 16);
    or_ef* oevs = (or_ef*)malloc(sizeof(or_ef) * (no > 0 ? no : 1));
    bw(&b, (uint32_t)no);
    for (int i = 0; i < no; i++) {
      or_ef z = sample_ef(&t);
      expand_from_univariate(z, nv, opts + (size_t)i * nv * 4);
      uint32_t e[4];
      or_eval_ext(f, nv, opts + (size_t)i * nv * 4, e);
      oevs[i] = ldv(e);
      observe_ef(&t, oevs[i]);
      bw_ef(&b, oevs[i]);
    }
    uint32_t pw = 0;
    if (rp->pow_bits > 0) pw = t_grind(&t, rp->pow_bits);
    bw(&b, pw);
    (void)t_smp(&t);
    int nq = stir_queries(&t, rp->domain_size, cfg_ff(&cfg, round), rp->num_queries, idx);
    uint32_t* svars = (uint32_t*)malloc(sizeof(uint32_t) * (nq + 1));
    or_ef* sevs = (or_ef*)malloc(sizeof(or_ef) * (nq + 1));
    bw(&b, (uint32_t)nq);
    int kprev = cfg_ff(&cfg, round);
    for (int q = 0; q < nq; q++) {
      tree_open(&cur_tree, idx[q], &b, row);
      /* evaluate_hypercube_base / _ext of the opened row at the folding randomness */
      uint32_t e[4], pt[4 * 32];
      for (int j = 0; j < kprev; j++) memcpy(pt + 4 * j, rs[nrs - kprev + j].c, 16);
      if (cur_tree.ext) or_eval_ext(row, kprev, pt, e);
      else or_eval_base(row, kprev, pt, e);
      svars[q] = or_pow(rp->folded_domain_gen, idx[q]);
      sevs[q] = ldv(e);
    }
    /* constraint + sumcheck (compute_sumcheck_polynomials with Some(constraint)) */
    or_ef gamma = sample_ef(&t);
    sum = or_ef_add(sum, combine_eq(w, nv, opts, oevs, no, gamma));
    {
      or_ef g = or_ef_pow(gamma, (uint64_t)no);
      uint32_t* gp = (uint32_t*)malloc(16 * (size_t)(nq + 1));
      for (int q = 0; q < nq; q++) {
        memcpy(gp + 4 * q, g.c, 16);
        sum = or_ef_add(sum, or_ef_mul(g, sevs[q]));
        g = or_ef_mul(g, gamma);
      }
      or_combine_select(w, nv, svars, nq, gp);
      free(gp);
    }
    sc_data sd;
    memset(&sd, 0, sizeof(sd));
    for (int j = 0; j < ffn; j++) rs[nrs++] = sc_round(&t, &sd, f, w, nv - j, &sum, rp->folding_pow_bits);
    bw_sc(&b, &sd);
    sc_free(&sd);
    nv -= ffn;
    tree_free(&cur_tree);
    cur_tree = nt;
    free(opts); free(oevs); free(svars); free(sevs);
  }

  /* ---- final round (prover/mod.rs:330-417) ---- */
  {
    size_t fn = (size_t)1 << nv;
    bw(&b, (uint32_t)fn);
    for (size_t i = 0; i < fn; i++) {
      or_ef v = ldv(f + 4 * i);
      observe_ef(&t, v);
      bw_ef(&b, v);
    }
    uint32_t pw = 0;
    if (cfg.final_pow_bits > 0) pw = t_grind(&t, cfg.final_pow_bits);
    bw(&b, pw);
    or_round_cfg fc = final_round_config(&cfg);
    int nq = stir_queries(&t, fc.domain_size, cfg_ff(&cfg, cfg.n_rounds), cfg.final_queries, idx);
    bw(&b, (uint32_t)nq);
    for (int q = 0; q < nq; q++) tree_open(&cur_tree, idx[q], &b, NULL);
    if (cfg.final_sumcheck_rounds > 0) {
      sc_data sd;
      memset(&sd, 0, sizeof(sd));
      for (int j = 0; j < cfg.final_sumcheck_rounds; j++)
        rs[nrs++] = sc_round(&t, &sd, f, w, nv - j, &sum, cfg.final_folding_pow_bits);
      bw(&b, 1u);
      bw_sc(&b, &sd);
      sc_free(&sd);
    } else {
      bw(&b, 0u);
    }
  }
  if (checkpoint) {
    or_ef cp = sample_ef(&t);
    memcpy(checkpoint, cp.c, 16);
  }
  tree_free(&cur_tree);
  free(f); free(w); free(rs); free(pts); free(evs); free(row); free(idx);
  *proof_out = b.w;
  *proof_words = b.len;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Verifier                                                                  */
/* ------------------------------------------------------------------------ */

typedef struct { const uint32_t* w; size_t len, pos; int err; } rd_t;
static uint32_t rd(rd_t* r) { if (r->pos >= r->len) { r->err = 1; return 0; } return r->w[r->pos++]; }
static or_ef rd_ef(rd_t* r) { or_ef v; for (int i = 0; i < 4; i++) v.c[i] = rd(r); return v; }

/* one constraint for the final weight evaluation */
typedef struct {
  int nv, neq, nsel;
  uint32_t* eq_pts; /* neq * nv EF */
  uint32_t* sel_vars;
  or_ef gamma;
} cons_t;

static or_ef eq_poly(const uint32_t* a, const or_ef* b, int n) {
  or_ef acc = or_ef_from(1), one = or_ef_from(1);
  for (int i = 0; i < n; i++) {
    or_ef l = ldv(a + 4 * i), r = b[i];
    /* 1 + l*2r - l - r */
    or_ef t = or_ef_sub(or_ef_sub(or_ef_add(one, or_ef_mul(l, or_ef_double(r))), l), r);
    acc = or_ef_mul(acc, t);
  }
  return acc;
}

static int verify_sc(tr_t* t, rd_t* r, or_ef* claimed, int pow_bits, or_ef* rs_out, int* nrs, int expect) {
  int np = (int)rd(r);
  if (expect >= 0 && np != expect) return -10;
  or_ef* polys = (or_ef*)malloc(sizeof(or_ef) * 2 * (np + 1));
  for (int i = 0; i < 2 * np; i++) polys[i] = rd_ef(r);
  int npow = (int)rd(r);
  uint32_t* pows = (uint32_t*)malloc(4 * (npow + 1));
  for (int i = 0; i < npow; i++) pows[i] = rd(r);
  if (r->err) { free(polys); free(pows); return -11; }
  for (int i = 0; i < np; i++) {
    observe_ef(t, polys[2 * i]);
    observe_ef(t, polys[2 * i + 1]);
    if (pow_bits > 0) {
      if (i >= npow || !t_check(t, pow_bits, pows[i])) {
        free(polys); free(pows); return -12;
      }
    }
    or_ef rr = sample_ef(t);
    *claimed = extrapolate_012(polys[2 * i], or_ef_sub(*claimed, polys[2 * i]), polys[2 * i + 1], rr);
    rs_out[(*nrs)++] = rr;
  }
  free(polys); free(pows);
  return 0;
}

/* Merkle path verification for one opened row */
static int verify_path(tr_t* t, int leaf_hash, const uint32_t* root, uint64_t idx, const uint32_t* row,
                       int row_words, const uint32_t* path, int path_len) {
  uint32_t cur[8], tmp[16];
  uint32_t st[24];
  memset(st, 0, sizeof(st));
  if (leaf_hash == 2) {
    /* Keccak MMCS: leaf hash and compression of or_keccak.c */
    or_keccak_leaf(row, row_words, cur);
    for (int l = 0; l < path_len; l++) {
      const uint32_t* sib = path + 8 * l;
      if ((idx >> l) & 1) or_keccak_compress(sib, cur, cur);
      else or_keccak_compress(cur, sib, cur);
    }
    return memcmp(cur, root, 32) == 0;
  }
  /* leaf digest via the same sponge as the builder */
  {
    const or_p2_params* p = leaf_hash == 0 ? &t->p24 : &t->p16;
    int rate = leaf_hash == 0 ? 16 : 8;
    int pos = 0;
    while (pos < row_words) {
      int take = row_words - pos < rate ? row_words - pos : rate;
      for (int i = 0; i < take; i++) st[i] = row[pos + i];
      pos += take;
      or_p2_permute(p, st);
    }
    memcpy(cur, st, 32);
  }
  for (int l = 0; l < path_len; l++) {
    const uint32_t* sib = path + 8 * l;
    if ((idx >> l) & 1) { memcpy(tmp, sib, 32); memcpy(tmp + 8, cur, 32); }
    else { memcpy(tmp, cur, 32); memcpy(tmp + 8, sib, 32); }
    or_p2_permute(&t->p16, tmp);
    memcpy(cur, tmp, 32);
  }
  return memcmp(cur, root, 32) == 0;
}

static int verify_stir(tr_t* t, rd_t* r, const or_params* prm, const or_round_cfg* rp, const uint32_t* root,
                       const or_ef* fr, int kfr, int is_final_round, uint32_t pow_w, uint32_t** vars_out,
                       or_ef** folds_out, int* nq_out) {
  /* the opened tree has domain_size >> folding_factor leaves */
  const int expect_height_log = ilog2_u64(rp->domain_size) - rp->folding_factor;
  if (rp->pow_bits > 0 && !t_check(t, rp->pow_bits, pow_w)) return -20;
  if (!is_final_round) (void)t_smp(t);
  uint64_t idx[4096];
  int nq = stir_queries(t, rp->domain_size, rp->folding_factor, rp->num_queries, idx);
  int got = (int)rd(r);
  if (got != nq) return -21;
  uint32_t* vars = (uint32_t*)malloc(4 * (nq + 1));
  or_ef* folds = (or_ef*)malloc(sizeof(or_ef) * (nq + 1));
  for (int q = 0; q < nq; q++) {
    int kind = (int)rd(r), nvals = (int)rd(r);
    int words = kind ? 4 * nvals : nvals;
    if (nvals != (1 << rp->folding_factor) || words > 4096) { free(vars); free(folds); return -22; }
    uint32_t row[4096];
    for (int i = 0; i < words; i++) row[i] = rd(r);
    int plen = (int)rd(r);
    if (plen != expect_height_log || plen > 64) { free(vars); free(folds); return -23; }
    uint32_t path[64 * 8];
    for (int i = 0; i < 8 * plen; i++) path[i] = rd(r);
    if (r->err) { free(vars); free(folds); return -24; }
    if (!verify_path(t, prm->leaf_hash, root, idx[q], row, words, path, plen)) { free(vars); free(folds); return -25; }
    uint32_t pt[4 * 64], e[4];
    for (int j = 0; j < kfr; j++) memcpy(pt + 4 * j, fr[j].c, 16);
    if (kind) or_eval_ext(row, rp->folding_factor, pt, e);
    else or_eval_base(row, rp->folding_factor, pt, e);
    folds[q] = ldv(e);
    vars[q] = or_pow(rp->folded_domain_gen, idx[q]);
  }
  *vars_out = vars;
  *folds_out = folds;
  *nq_out = nq;
  return 0;
}

int or_whir_verify(const or_params* prm, int n, const uint32_t* user_points, const uint32_t* user_evals,
                   int num_points, const uint32_t* proof, size_t proof_words, uint32_t* checkpoint) {
  or_config cfg;
  int rc = or_config_new(prm, n, &cfg);
  if (rc) return rc;
  tr_t t;
  p2_selected(&t.p16, &t.p24);
  or_chal_init(&t.ch);
  t.keccak = prm->leaf_hash == 2;
  or_kchal_init(&t.kc);
  {
    int len = or_domain_separator(&cfg, prm->ds_digest_elems, NULL, 0);
    uint32_t* pat = (uint32_t*)malloc((size_t)len * 4);
    or_domain_separator(&cfg, prm->ds_digest_elems, pat, len);
    for (int i = 0; i < len; i++) t_obs(&t, pat[i]);
    free(pat);
  }
  rd_t r = {proof, proof_words, 0, 0};
  if (rd(&r) != 0x50524857u || rd(&r) != 1u) return -1;
  int ret = 0;
  cons_t cons[OR_MAX_ROUNDS + 2];
  memset(cons, 0, sizeof(cons));
  int ncons = 0;
  or_ef rs[256];
  int nrs = 0;
  int rs_start[OR_MAX_ROUNDS + 3];
  or_ef claimed = or_ef_zero();

  /* parse_commitment */
  uint32_t root[8];
  for (int i = 0; i < 8; i++) root[i] = rd(&r);
  observe_digest(&t, root);
  int nood = (int)rd(&r);
  if (nood != cfg.commitment_ood_samples) return -2;
  int neq = num_points + nood;
  cons_t* c0 = &cons[ncons++];
  c0->nv = n; c0->neq = neq; c0->nsel = 0; c0->sel_vars = NULL;
  c0->eq_pts = (uint32_t*)malloc((size_t)(neq + 1) * n * 16);
  or_ef* evs = (or_ef*)malloc(sizeof(or_ef) * (neq + 1));
  for (int i = 0; i < num_points; i++) {
    memcpy(c0->eq_pts + (size_t)i * n * 4, user_points + (size_t)i * n * 4, (size_t)n * 16);
    evs[i] = ldv(user_evals + 4 * i);
  }
  for (int i = 0; i < nood; i++) {
    or_ef z = sample_ef(&t);
    expand_from_univariate(z, n, c0->eq_pts + (size_t)(num_points + i) * n * 4);
    evs[num_points + i] = rd_ef(&r);
    observe_ef(&t, evs[num_points + i]);
  }
  c0->gamma = sample_ef(&t);
  {
    or_ef g = or_ef_from(1);
    for (int i = 0; i < neq; i++) { claimed = or_ef_add(claimed, or_ef_mul(evs[i], g)); g = or_ef_mul(g, c0->gamma); }
  }
  free(evs);
  rs_start[0] = nrs;
  ret = verify_sc(&t, &r, &claimed, cfg.starting_folding_pow_bits, rs, &nrs, -1);
  if (ret) goto done;
  if ((int)rd(&r) != cfg.n_rounds) { ret = -3; goto done; }
  uint32_t prev_root[8];
  memcpy(prev_root, root, 32);
  for (int round = 0; round < cfg.n_rounds; round++) {
    const or_round_cfg* rp = &cfg.rounds[round];
    uint32_t nroot[8];
    for (int i = 0; i < 8; i++) nroot[i] = rd(&r);
    observe_digest(&t, nroot);
    int no = (int)rd(&r);
    if (no != rp->ood_samples) { ret = -4; goto done; }
    cons_t* c = &cons[ncons++];
    c->nv = rp->num_variables; c->neq = no;
    c->eq_pts = (uint32_t*)malloc((size_t)(no + 1) * rp->num_variables * 16);
    or_ef* oev = (or_ef*)malloc(sizeof(or_ef) * (no + 1));
    for (int i = 0; i < no; i++) {
      or_ef z = sample_ef(&t);
      expand_from_univariate(z, rp->num_variables, c->eq_pts + (size_t)i * rp->num_variables * 4);
      oev[i] = rd_ef(&r);
      observe_ef(&t, oev[i]);
    }
    uint32_t pw = rd(&r);
    int kfr = nrs - rs_start[round];
    or_ef* folds;
    int nq;
    ret = verify_stir(&t, &r, prm, rp, prev_root, rs + rs_start[round], kfr, 0, pw, &c->sel_vars, &folds, &nq);
    if (ret) { free(oev); goto done; }
    c->nsel = nq;
    c->gamma = sample_ef(&t);
    or_ef g = or_ef_from(1);
    for (int i = 0; i < no; i++) { claimed = or_ef_add(claimed, or_ef_mul(oev[i], g)); g = or_ef_mul(g, c->gamma); }
    for (int q = 0; q < nq; q++) { claimed = or_ef_add(claimed, or_ef_mul(folds[q], g)); g = or_ef_mul(g, c->gamma); }
    free(oev); free(folds);
    rs_start[round + 1] = nrs;
    ret = verify_sc(&t, &r, &claimed, rp->folding_pow_bits, rs, &nrs, -1);
    if (ret) goto done;
    memcpy(prev_root, nroot, 32);
  }
  {
    /* final round */
    int nfin = (int)rd(&r);
    if (nfin != (1 << cfg.final_sumcheck_rounds)) { ret = -5; goto done; }
    or_ef* fin = (or_ef*)malloc(sizeof(or_ef) * nfin);
    for (int i = 0; i < nfin; i++) { fin[i] = rd_ef(&r); observe_ef(&t, fin[i]); }
    uint32_t pw = rd(&r);
    or_round_cfg fc = final_round_config(&cfg);
    int kfr = nrs - rs_start[cfg.n_rounds];
    uint32_t* vars;
    or_ef* folds;
    int nq;
    ret = verify_stir(&t, &r, prm, &fc, prev_root, rs + rs_start[cfg.n_rounds], kfr, 1, pw, &vars, &folds, &nq);
    if (ret) { free(fin); goto done; }
    for (int q = 0; q < nq; q++) {
      /* SelectStatement::verify: sum_x fin[x] var^x via reverse Horner */
      or_ef acc = or_ef_zero();
      for (int x = nfin - 1; x >= 0; x--) acc = or_ef_add(or_ef_mul_base(acc, vars[q]), fin[x]);
      if (!or_ef_eq(acc, folds[q])) { ret = -30; break; }
    }
    free(vars); free(folds);
    if (ret) { free(fin); goto done; }
    int has = (int)rd(&r);
    int fstart = nrs;
    if (cfg.final_sumcheck_rounds > 0) {
      if (!has) { free(fin); ret = -31; goto done; }
      ret = verify_sc(&t, &r, &claimed, cfg.final_folding_pow_bits, rs, &nrs, cfg.final_sumcheck_rounds);
      if (ret) { free(fin); goto done; }
    }
    /* weights evaluation at the reversed folding randomness */
    or_ef* rev = (or_ef*)malloc(sizeof(or_ef) * (nrs + 1));
    for (int i = 0; i < nrs; i++) rev[i] = rs[nrs - 1 - i];
    or_ef weval = or_ef_zero();
    for (int ci = 0; ci < ncons; ci++) {
      cons_t* c = &cons[ci];
      or_ef* pt = (or_ef*)malloc(sizeof(or_ef) * (c->nv + 1));
      for (int i = 0; i < c->nv; i++) pt[i] = rev[c->nv - 1 - i];
      or_ef g = or_ef_from(1);
      for (int i = 0; i < c->neq; i++) {
        weval = or_ef_add(weval, or_ef_mul(g, eq_poly(c->eq_pts + (size_t)i * c->nv * 4, pt, c->nv)));
        g = or_ef_mul(g, c->gamma);
      }
      for (int q = 0; q < c->nsel; q++) {
        /* select_poly(expand(var), pt) = prod_j (pt_j * (var^(2^(nv-1-j)) - 1) + 1) */
        or_ef acc = or_ef_from(1);
        uint32_t cur = c->sel_vars[q];
        for (int j = c->nv - 1; j >= 0; j--) {
          or_ef term = or_ef_add(or_ef_mul_base(pt[j], or_sub(cur, 1)), or_ef_from(1));
          acc = or_ef_mul(acc, term);
          cur = or_mul(cur, cur);
        }
        weval = or_ef_add(weval, or_ef_mul(g, acc));
        g = or_ef_mul(g, c->gamma);
      }
      free(pt);
    }
    /* final_value = final poly at the final sumcheck randomness */
    uint32_t fpt[4 * 64], fv[4];
    for (int i = fstart; i < nrs; i++) memcpy(fpt + 4 * (i - fstart), rs[i].c, 16);
    uint32_t* fw = (uint32_t*)malloc(16 * nfin);
    for (int i = 0; i < nfin; i++) memcpy(fw + 4 * i, fin[i].c, 16);
    or_eval_ext(fw, cfg.final_sumcheck_rounds, fpt, fv);
    free(fw); free(rev); free(fin);
    if (!or_ef_eq(claimed, or_ef_mul(weval, ldv(fv)))) { ret = -32; goto done; }
  }
  if (r.pos != r.len) { ret = -33; goto done; }
  if (checkpoint) {
    or_ef cp = sample_ef(&t);
    memcpy(checkpoint, cp.c, 16);
  }
done:
  for (int i = 0; i < ncons; i++) { free(cons[i].eq_pts); free(cons[i].sel_vars); }
  return ret;
}
