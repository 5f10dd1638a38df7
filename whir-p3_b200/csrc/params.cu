// Host-side protocol pieces: Poseidon2 data, WhirConfig derivation, the
// domain separator and the duplex-sponge challenger.
#include <math.h>
#include <string.h>

#include "host.h"

namespace wh {

static thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }
const char* last_error() { return g_error.c_str(); }

// ---------------------------------------------------------------------------
// Poseidon2 data
// ---------------------------------------------------------------------------

p2::P2Consts to_consts(const whir_poseidon2_params& p) {
  p2::P2Consts k;
  memset(&k, 0, sizeof(k));
  k.width = p.width;
  k.rounds_f = p.rounds_f;
  k.rounds_p = p.rounds_p;
  k.mat = p.external_matrix;
  memcpy(k.ext_rc, p.ext_rc, sizeof(k.ext_rc));
  memcpy(k.int_rc, p.int_rc, sizeof(k.int_rc));
  for (int i = 0; i < 24; i++) {
    k.diag_c[i] = p.diag[i];
    k.diag_s[i] = kb::shoup_const(p.diag[i]);
  }
  for (int i = 0; i < 8 * 24; i++) k.ext_rc_m[i] = kb::to_mont(p.ext_rc[i]);
  for (int i = 0; i < 32; i++) k.int_rc_m[i] = kb::to_mont(p.int_rc[i]);
  return k;
}

int validate_params(const whir_poseidon2_params& p, uint32_t width) {
  const uint32_t rp = width == 16 ? p2::RP16 : p2::RP24;
  if (p.width != width || p.rounds_f != (uint32_t)p2::RF || p.rounds_p != rp) {
    set_error("unsupported Poseidon2 shape: width " + std::to_string(p.width) + ", rounds " +
              std::to_string(p.rounds_f) + "+" + std::to_string(p.rounds_p) + " (supported: 16 with 8+20, 24 with 8+23)");
    return WHIR_ERR_INVALID;
  }
  if (p.external_matrix != WHIR_P2_MDS_MAT4 && p.external_matrix != WHIR_P2_HL_MAT4)
    return set_error("unknown Poseidon2 external matrix " + std::to_string(p.external_matrix)), WHIR_ERR_INVALID;
  for (int i = 0; i < 8 * 24; i++)
    if (p.ext_rc[i] >= kb::P) return set_error("Poseidon2 constant out of range"), WHIR_ERR_INVALID;
  for (int i = 0; i < 32; i++)
    if (p.int_rc[i] >= kb::P) return set_error("Poseidon2 constant out of range"), WHIR_ERR_INVALID;
  // the internal diagonal is fixed (p3-koala-bear's internal layer takes only
  // round constants); the field is kept so the struct carries the whole
  // permutation, and must hold that diagonal
  for (uint32_t i = 0; i < width; i++) {
    if (p.diag[i] != p2::diag_value(p2::diag_code((int)width, (int)i)))
      return set_error("Poseidon2 internal diagonal differs from the fixed KoalaBear diagonal at entry " +
                       std::to_string(i)),
             WHIR_ERR_INVALID;
  }
  return WHIR_OK;
}

// rand::rngs::SmallRng on 64-bit targets: xoshiro256++ (Blackman and Vigna,
// "Scrambled linear pseudorandom number generators", 2021) whose
// seed_from_u64 fills the four state words with SplitMix64 (Steele, Lea,
// Flood, OOPSLA 2014) outputs; next_u32 is the high half of next_u64.
// KoalaBear's StandardUniform draws next_u32() >> 1 and rejects values >= p;
// the accepted value is the element's Montgomery representation (x * 2^32 mod
// p), so its canonical value is that word reduced once.
SmallRng::SmallRng(uint64_t seed) {
  for (int i = 0; i < 4; i++) {
    seed += 0x9e3779b97f4a7c15ull;
    uint64_t z = seed;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    s[i] = z ^ (z >> 31);
  }
}
uint64_t SmallRng::next_u64() {
  const uint64_t r = rotl(s[0] + s[3], 23) + s[0];
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return r;
}
uint32_t SmallRng::field() {
  for (;;) {
    const uint32_t v = next_u32() >> 1;
    if (v < kb::P) return kb::from_mont(v);
  }
}

namespace {
// Poseidon2::new_from_rng: ExternalLayerConstants::new_from_rng (rounds_f / 2
// initial rows, then rounds_f / 2 terminal rows, each row `width` elements in
// order), then rounds_p internal constants.
void fill(whir_poseidon2_params* p, uint32_t width, uint32_t rp, uint32_t mat, SmallRng& g) {
  memset(p, 0, sizeof(*p));
  p->width = width;
  p->rounds_f = p2::RF;
  p->rounds_p = rp;
  p->external_matrix = mat;
  for (uint32_t r = 0; r < (uint32_t)p2::RF; r++)
    for (uint32_t i = 0; i < width; i++) p->ext_rc[r * width + i] = g.field();
  for (uint32_t r = 0; r < rp; r++) p->int_rc[r] = g.field();
  for (uint32_t i = 0; i < width; i++) p->diag[i] = p2::diag_value(p2::diag_code((int)width, (int)i));
}
}  // namespace

void params_from_rng(uint64_t seed, uint32_t mat, whir_poseidon2_params* p16, whir_poseidon2_params* p24) {
  SmallRng g(seed);
  whir_poseidon2_params a, b;
  fill(&a, 16, p2::RP16, mat, g);
  fill(&b, 24, p2::RP24, mat, g);
  if (p16) *p16 = a;
  if (p24) *p24 = b;
}

void default_params(whir_poseidon2_params* p16, whir_poseidon2_params* p24) {
  params_from_rng(1, WHIR_P2_MDS_MAT4, p16, p24);
}

// ---------------------------------------------------------------------------
// WhirConfig::new (src/whir/parameters.rs:81-234) with SecurityAssumption
// (src/parameters/errors.rs:25-187) and FoldingFactor
// (src/parameters/mod.rs:31-125). All real arithmetic is IEEE double, as in
// the reference; EF::bits() = 124 for the quartic extension.
// ---------------------------------------------------------------------------

namespace {
constexpr int kFieldBits = 124;
constexpr int kMaxSendCoeffs = 6;  // MAX_NUM_VARIABLES_TO_SEND_COEFFS
const double kLog2_10 = 3.321928094887362347870319429489390175864831393;

struct Sec {
  int s;  // 0 UD, 1 JB, 2 CB
  double log_eta(int lir) const {
    if (s == 0) return 0.;
    if (s == 1) return -(0.5 * (double)lir + kLog2_10 + 1.);
    return -((double)lir + kLog2_10 + 1.);
  }
  double list_size_bits(int d, int lir) const {
    const double le = log_eta(lir);
    if (s == 0) return 0.;
    if (s == 1) return (double)lir / 2. - (1. + le);
    return (double)(d + lir) - le;
  }
  double prox_gaps_error(int d, int lir, int fb, int nf) const {
    const double le = log_eta(lir);
    double e;
    if (s == 0)
      e = (double)(d + lir);
    else if (s == 1)
      e = (double)(2 * d) + 7. * (fmin(1. + kLog2_10 + 0.5 * (double)lir, -le) - 1.);
    else
      e = (double)(d + 2 * lir) - le;
    return (double)fb - (e + log2((double)nf - 1.));
  }
  double log_1_delta(int lir) const {
    const double eta = pow(2., log_eta(lir));
    const double rate = 1. / (double)(1 << lir);
    double delta;
    if (s == 0)
      delta = 0.5 * (1. - rate);
    else if (s == 1)
      delta = 1. - sqrt(rate) - eta;
    else
      delta = 1. - rate - eta;
    return log2(1. - delta);
  }
  int queries(int psl, int lir) const { return (int)ceil(-(double)psl / log_1_delta(lir)); }
  double queries_error(int lir, int q) const { return -(double)q * log_1_delta(lir); }
  double ood_error(int d, int lir, int fb, int o) const {
    if (s == 0) return 0.;
    return (double)(o * fb) + 1. - (2. * list_size_bits(d, lir) + (double)(d * o));
  }
  int ood_samples(int sec, int d, int lir, int fb) const {
    if (s == 0) return 0;
    for (int o = 1; o < 64; o++)
      if (ood_error(d, lir, fb, o) >= (double)sec) return o;
    return -1;
  }
  double folding_pow_bits(int sec, int fb, int nv, int lir) const {
    const double pg = prox_gaps_error(nv, lir, fb, 2);
    const double sc = (double)fb - (list_size_bits(nv, lir) + 1.);
    return fmax(0., (double)sec - fmin(pg, sc));
  }
  double combination_error(int fb, int nv, int lir, int ood, int q) const {
    return (double)fb - (log2((double)(ood + q)) + list_size_bits(nv, lir) + 1.);
  }
};

int as_int(double v) { return v <= 0. ? 0 : (int)(uint64_t)v; }
int ilog2u(uint64_t v) {
  int r = -1;
  while (v) {
    r++;
    v >>= 1;
  }
  return r;
}
}  // namespace

int ff_at(const whir_config& c, int round) { return round == 0 ? c.folding_factor_0 : c.folding_factor; }
int rsr_at(const whir_config& c, int round) { return round == 0 ? c.rs_reduction : 1; }

int config_new(const whir_protocol_params& p, int n, whir_config* out) {
  whir_config c;
  memset(&c, 0, sizeof(c));
  WH_CHECK(p.soundness >= 0 && p.soundness <= 2, "soundness must be 0 (UD), 1 (JB) or 2 (CB)");
  WH_CHECK(p.folding_factor_0 > 0 && p.folding_factor > 0, "folding factor must be non-zero");
  WH_CHECK(p.folding_factor_0 <= n && p.folding_factor <= n, "folding factor larger than the number of variables");
  WH_CHECK(p.rs_reduction <= p.folding_factor_0, "rs_domain_initial_reduction_factor exceeds folding factor");
  WH_CHECK(n >= 1 && n <= 30, "num_variables out of range");
  WH_CHECK(p.starting_log_inv_rate >= 0 && p.starting_log_inv_rate <= 16, "starting_log_inv_rate out of range");
  WH_CHECK(p.security_level >= 0 && p.pow_bits >= 0, "negative security parameter");
  WH_CHECK(p.leaf_hash == WHIR_LEAF_P24 || p.leaf_hash == WHIR_LEAF_P16 || p.leaf_hash == WHIR_LEAF_KECCAK,
           "leaf_hash must be WHIR_LEAF_P24, WHIR_LEAF_P16 or WHIR_LEAF_KECCAK");
  const Sec S{p.soundness};
  const int sec = p.security_level, fb = kFieldBits;
  const int psl = sec > p.pow_bits ? sec - p.pow_bits : 0;
  int lir = p.starting_log_inv_rate, nv = n;
  const int log_domain = n + lir;
  uint64_t domain = 1ull << log_domain;
  WH_CHECK(log_domain - p.folding_factor_0 <= kb::TWO_ADICITY, "Increase folding_factor_0");
  // FoldingFactor::compute_number_of_rounds
  int nr, fin;
  if (p.folding_factor_0 == p.folding_factor) {
    const int f = p.folding_factor;
    if (n <= kMaxSendCoeffs) {
      nr = 0;
      fin = n - f;
    } else {
      const int r = (n - kMaxSendCoeffs + f - 1) / f;
      nr = r - 1;
      fin = n - r * f;
    }
  } else {
    const int nv1 = n - p.folding_factor_0, f = p.folding_factor;
    if (nv1 < kMaxSendCoeffs) {
      nr = 0;
      fin = nv1;
    } else {
      const int r = (nv1 - kMaxSendCoeffs + f - 1) / f;
      nr = r;
      fin = nv1 - r * f;
    }
  }
  WH_CHECK(nr <= WHIR_MAX_ROUNDS, "too many rounds");
  c.num_variables = n;
  c.security_level = sec;
  c.max_pow_bits = p.pow_bits;
  c.soundness = p.soundness;
  c.starting_log_inv_rate = lir;
  c.folding_factor_0 = p.folding_factor_0;
  c.folding_factor = p.folding_factor;
  c.rs_reduction = p.rs_reduction;
  c.commitment_ood_samples = S.ood_samples(sec, n, lir, fb);
  WH_CHECK(c.commitment_ood_samples >= 0, "Could not find an appropriate number of OOD samples");
  c.starting_folding_pow_bits = as_int(S.folding_pow_bits(sec, fb, n, lir));
  nv -= p.folding_factor_0;
  for (int r = 0; r < nr; r++) {
    const int rsr = r == 0 ? p.rs_reduction : 1;
    const int ff = r == 0 ? p.folding_factor_0 : p.folding_factor;
    const int next_rate = lir + (ff - rsr);
    const int q = S.queries(psl, lir);
    const int ood = S.ood_samples(sec, nv, next_rate, fb);
    WH_CHECK(ood >= 0, "Could not find an appropriate number of OOD samples");
    const double qe = S.queries_error(lir, q);
    const double ce = S.combination_error(fb, nv, next_rate, ood, q);
    whir_round_config& rc = c.rounds[r];
    rc.pow_bits = as_int(fmax(0., (double)sec - fmin(qe, ce)));
    rc.folding_pow_bits = as_int(S.folding_pow_bits(sec, fb, nv, next_rate));
    rc.num_queries = q;
    rc.ood_samples = ood;
    rc.num_variables = nv;
    rc.folding_factor = ff;
    rc.domain_size = domain;
    rc.folded_domain_gen = kb::from_mont(kb::two_adic_generator(ilog2u(domain) - ff));
    nv -= p.folding_factor;  // folding factor of round r + 1
    lir = next_rate;
    domain >>= rsr;
  }
  c.n_rounds = nr;
  c.final_sumcheck_rounds = fin;
  c.final_queries = S.queries(psl, lir);
  c.final_pow_bits = as_int(fmax(0., (double)sec - S.queries_error(lir, c.final_queries)));
  c.final_folding_pow_bits = as_int(fmax(0., (double)sec - (double)(fb - 1)));
  *out = c;
  return WHIR_OK;
}

whir_round_config final_round_config(const whir_config& c) {
  whir_round_config r;
  memset(&r, 0, sizeof(r));
  if (c.n_rounds == 0) {
    const uint64_t d = 1ull << (c.num_variables + c.starting_log_inv_rate);
    r.num_variables = c.num_variables - c.folding_factor_0;
    r.folding_factor = ff_at(c, 0);
    r.domain_size = d;
    r.folded_domain_gen = kb::from_mont(kb::two_adic_generator(ilog2u(d) - c.folding_factor_0));
    r.ood_samples = 0;
  } else {
    const whir_round_config& last = c.rounds[c.n_rounds - 1];
    const int ff = ff_at(c, c.n_rounds);
    const uint64_t d = last.domain_size >> rsr_at(c, c.n_rounds - 1);
    r.num_variables = last.num_variables - ff;
    r.folding_factor = ff;
    r.domain_size = d;
    r.folded_domain_gen = kb::from_mont(kb::two_adic_generator(ilog2u(d) - ff));
    r.ood_samples = last.ood_samples;
  }
  r.num_queries = c.final_queries;
  r.pow_bits = c.final_pow_bits;
  r.folding_pow_bits = c.final_folding_pow_bits;
  return r;
}

// ---------------------------------------------------------------------------
// DomainSeparator (src/fiat_shamir/domain_separator.rs:57-213, pattern.rs)
// ---------------------------------------------------------------------------

namespace {
enum Pat { kSample = 0, kObserve = 1, kHint = 2 };
enum SampleTag { kInitComb = 0, kFoldSkip = 1, kFold = 2, kComb = 3, kStirQ = 4, kFinalQ = 5, kPowQ = 6, kOod = 7 };
enum ObserveTag { kDigest = 0, kOodAns = 1, kScPoly = 2, kScSkip = 3, kStirAns = 4, kFinalCoeffs = 5, kPowNonce = 6 };
enum HintTag { kHStirQ = 0, kHStirA = 1, kHMerkle = 2, kHDeferred = 3 };

struct Ds {
  std::vector<uint32_t> v;
  static uint32_t canon_add(uint64_t a, uint64_t b) { return (uint32_t)((a + b) % kb::P); }
  void observe(uint64_t count, int tag) { v.push_back(canon_add(canon_add(tag, count % kb::P), kObserve)); }
  void sample(uint64_t count, int tag) { v.push_back(canon_add(canon_add(tag, count % kb::P), kSample)); }
  void hint(int tag) { v.push_back(canon_add(tag, kHint)); }
  void pow(int bits) {
    if (bits > 0) {
      sample(32, kPowQ);
      observe(8, kPowNonce);
    }
  }
  void sumcheck(int rounds, int pow_bits) {
    for (int i = 0; i < rounds; i++) {
      observe(3, kScPoly);
      sample(1, kFold);
      pow(pow_bits);
    }
  }
  void ood(int n) {
    if (n > 0) {
      sample(n, kOod);
      observe(n, kOodAns);
    }
  }
};
}  // namespace

std::vector<uint32_t> domain_separator(const whir_config& c, int digest_elems) {
  Ds d;
  d.observe(digest_elems, kDigest);
  if (c.commitment_ood_samples > 0) d.ood(c.commitment_ood_samples);
  d.sample(1, kInitComb);
  d.sumcheck(ff_at(c, 0), c.starting_folding_pow_bits);
  uint64_t domain = 1ull << (c.num_variables + c.starting_log_inv_rate);
  for (int r = 0; r < c.n_rounds; r++) {
    const whir_round_config& rc = c.rounds[r];
    const uint64_t folded = domain >> ff_at(c, r);
    const int bytes = (ilog2u(folded * 2 - 1) + 7) / 8;
    d.observe(digest_elems, kDigest);
    d.ood(rc.ood_samples);
    d.sample((uint64_t)rc.num_queries * bytes, kStirQ);
    d.hint(kHStirQ);
    d.hint(kHMerkle);
    d.pow(rc.pow_bits);
    d.sample(1, kComb);
    d.sumcheck(ff_at(c, r + 1), rc.folding_pow_bits);
    domain >>= rsr_at(c, r);
  }
  const uint64_t folded = domain >> ff_at(c, c.n_rounds);
  const int bytes = (ilog2u(folded * 2 - 1) + 7) / 8;
  d.observe(1ull << c.final_sumcheck_rounds, kFinalCoeffs);
  d.sample((uint64_t)bytes * c.final_queries, kFinalQ);
  d.hint(kHStirA);
  d.hint(kHMerkle);
  d.pow(c.final_pow_bits);
  d.sumcheck(c.final_sumcheck_rounds, c.final_folding_pow_bits);
  d.hint(kHDeferred);
  return d.v;
}

// ---------------------------------------------------------------------------
// DuplexChallenger<F, Poseidon2-16, WIDTH = 16, RATE = 8> (p3-challenger):
// observe clears the output buffer and absorbs into the input buffer,
// duplexing when RATE inputs are pending; sample duplexes when inputs are
// pending or no output is left, then pops the last output.
// ---------------------------------------------------------------------------

HostP16 host_consts16(const whir_poseidon2_params& p) {
  HostP16 k;
  memcpy(k.ext_rc, p.ext_rc, sizeof(k.ext_rc));
  memcpy(k.int_rc, p.int_rc, sizeof(k.int_rc));
  memcpy(k.diag, p.diag, sizeof(k.diag));
  k.mat = p.external_matrix;
  return k;
}

namespace {
constexpr uint64_t P64 = kb::P;
inline uint64_t cube64(uint64_t v) {  // v < 2p: v^2 < 2^64, (v^2 mod p) * v < 2^63
  const uint64_t sq = (v * v) % P64;
  return (sq * v) % P64;
}
// external layer on canonical inputs: block outputs < 16p, chunk sums < 64p,
// results < 80p < 2^38, reduced once
inline void ext_layer64(uint64_t* x, uint32_t mat) {
  for (int c = 0; c < 16; c += 4) {
    const uint64_t a = x[c], b = x[c + 1], cc = x[c + 2], d = x[c + 3];
    if (mat == WHIR_P2_HL_MAT4) {
      const uint64_t t0 = a + b, t1 = cc + d, t2 = 2 * b + t1, t3 = 2 * d + t0;
      const uint64_t t4 = 4 * t1 + t3, t5 = 4 * t0 + t2;
      x[c] = t3 + t5;
      x[c + 1] = t5;
      x[c + 2] = t2 + t4;
      x[c + 3] = t4;
    } else {  // circ(2, 3, 1, 1)
      const uint64_t s = a + b + cc + d;
      x[c] = s + a + 2 * b;
      x[c + 1] = s + b + 2 * cc;
      x[c + 2] = s + cc + 2 * d;
      x[c + 3] = s + d + 2 * a;
    }
  }
  for (int j = 0; j < 4; j++) {
    const uint64_t s = x[j] + x[4 + j] + x[8 + j] + x[12 + j];
    for (int c = 0; c < 16; c += 4) x[c + j] = (x[c + j] + s) % P64;
  }
}
}  // namespace

void host_permute16(uint32_t* st, const HostP16& k) {
  uint64_t x[16];
  for (int i = 0; i < 16; i++) x[i] = st[i];
  ext_layer64(x, k.mat);
  for (int r = 0; r < 4; r++) {
    for (int i = 0; i < 16; i++) x[i] = cube64(x[i] + k.ext_rc[r * 16 + i]);
    ext_layer64(x, k.mat);
  }
  for (int r = 0; r < p2::RP16; r++) {
    x[0] = cube64(x[0] + k.int_rc[r]);
    uint64_t s = 0;
    for (int i = 0; i < 16; i++) s += x[i];  // < 16p
    for (int i = 0; i < 16; i++) x[i] = (s + k.diag[i] * x[i]) % P64;  // < 16p + p^2 < 2^63
  }
  for (int r = 4; r < 8; r++) {
    for (int i = 0; i < 16; i++) x[i] = cube64(x[i] + k.ext_rc[r * 16 + i]);
    ext_layer64(x, k.mat);
  }
  for (int i = 0; i < 16; i++) st[i] = (uint32_t)x[i];
}

void Chal::init() { memset(this, 0, sizeof(*this)); }
void Chal::init_keccak() {
  init();
  family = kChalKeccak;
  kk::k256_init(kin);
}
void Chal::duplex(const HostP16& k) {
  for (int i = 0; i < in_len; i++) st[i] = in[i];
  in_len = 0;
  uint32_t c[16];
  for (int i = 0; i < 16; i++) c[i] = kb::from_mont(st[i]);
  host_permute16(c, k);
  for (int i = 0; i < 16; i++) st[i] = kb::to_mont(c[i]);
  for (int i = 0; i < 8; i++) out[i] = st[i];
  out_len = 8;
}
void Chal::observe(const HostP16& k, uint32_t v) {
  if (family == kChalKeccak) {
    // the 4 little-endian bytes of the canonical value
    kout_len = 0;
    kk::k256_word(kin, kb::from_mont(v));
    return;
  }
  out_len = 0;
  in[in_len++] = v;
  if (in_len == 8) duplex(k);
}
namespace {
// HashChallenger::sample on the Keccak challenger: pop a byte from the end of
// the output, hashing the input buffer first when the output is empty
uint8_t keccak_byte(Chal& c) {
  if (c.kout_len == 0) {
    kk::k256_final(c.kin, c.kout);
    c.kout_len = 32;
    kk::k256_init(c.kin);
    kk::k256_update(c.kin, c.kout, 32);
  }
  return c.kout[--c.kout_len];
}
uint32_t keccak_u32(Chal& c) {
  uint32_t v = 0;
  for (int i = 0; i < 4; i++) v |= (uint32_t)keccak_byte(c) << (8 * i);
  return v;
}
}  // namespace
uint32_t Chal::sample(const HostP16& k) {
  if (family == kChalKeccak) {
    // 4 bytes little-endian, masked to 31 bits, rejected while >= p
    for (;;) {
      const uint32_t v = keccak_u32(*this) & 0x7fffffffu;
      if (v < kb::P) return kb::to_mont(v);
    }
  }
  if (in_len > 0 || out_len == 0) duplex(k);
  return out[--out_len];
}
uint64_t Chal::sample_bits(const HostP16& k, int bits) {
  if (family == kChalKeccak) return (uint64_t)keccak_u32(*this) & ((1ull << bits) - 1);
  const uint32_t v = kb::from_mont(sample(k));
  return (uint64_t)v & ((1ull << bits) - 1);
}
void Chal::observe_digest(const HostP16& k, const uint32_t* words8) {
  if (family == kChalKeccak) {
    kout_len = 0;
    for (int i = 0; i < 8; i++) kk::k256_word(kin, words8[i]);
    return;
  }
  for (int i = 0; i < 8; i++) observe(k, kb::to_mont(words8[i]));
}
kb::ef Chal::sample_ef(const HostP16& k) {
  kb::ef r;
  for (int i = 0; i < 4; i++) r.c[i] = sample(k);
  return r;
}
void Chal::observe_ef(const HostP16& k, const kb::ef& v) {
  for (int i = 0; i < 4; i++) observe(k, v.c[i]);
}
void Chal::load(const whir_challenger& c) {
  init();
  for (int i = 0; i < 16; i++) st[i] = kb::to_mont(c.state[i]);
  for (int i = 0; i < 8; i++) in[i] = kb::to_mont(c.input[i]);
  for (int i = 0; i < 8; i++) out[i] = kb::to_mont(c.output[i]);
  in_len = c.input_len;
  out_len = c.output_len;
}
void Chal::store(whir_challenger& c) const {
  for (int i = 0; i < 16; i++) c.state[i] = kb::from_mont(st[i]);
  for (int i = 0; i < 8; i++) c.input[i] = kb::from_mont(in[i]);
  for (int i = 0; i < 8; i++) c.output[i] = kb::from_mont(out[i]);
  c.input_len = in_len;
  c.output_len = out_len;
}

}  // namespace wh
