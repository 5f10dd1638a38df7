// Proof wire format: the library's flat proof stream (uint32 words, canonical
// values; layout in include/whir_b200.h) to and from the bytes that
// `bincode::serialize(&proof)` gives for the reference's
// WhirProof<KoalaBear, BinomialExtensionField<KoalaBear, 4>, MerkleTreeMmcs<..., 8>>
// (src/whir/proof.rs:11-141; serialised at src/bin/main.rs:221).
//
// bincode 1.3 with its default options writes integers little-endian at fixed
// width, a sequence as a u64 length then its elements, an Option as one byte
// (0 None, 1 Some) then the value, a struct as its fields in order, and a
// fixed-size array or tuple as its elements with no length. The serde forms
// assumed for the Plonky3 types (rev c38eb05, not available here to check):
//   - KoalaBear (MontyField31) serialises its Montgomery word as a u32;
//   - the extension element, the Merkle root (`Hash<F, F, 8>`) and a Merkle
//     path node (`[F; 8]`) are fixed arrays of field elements;
//   - the Merkle opening proof of MerkleTreeMmcs is a Vec of [F; 8] nodes;
//   - EvaluationsList<EF> is a newtype over Vec<EF>.
// QueryOpening is internally tagged (`#[serde(tag = "type")]`), so each
// opening starts with the tag as a string ("base" or "extension"), followed by
// its fields.
#include <string.h>

#include <string>
#include <vector>

#include "host.h"

namespace {

struct Writer {
  uint8_t* out;
  size_t cap;
  size_t len = 0;
  void bytes(const void* p, size_t n) {
    if (out && len + n <= cap) memcpy(out + len, p, n);
    len += n;
  }
  void u8(uint8_t v) { bytes(&v, 1); }
  void u32(uint32_t v) {
    uint8_t b[4] = {(uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24)};
    bytes(b, 4);
  }
  void u64(uint64_t v) {
    for (int i = 0; i < 8; i++) u8((uint8_t)(v >> (8 * i)));
  }
  void field(uint32_t canonical) { u32(kb::to_mont(canonical)); }
  void str(const char* s) {
    const size_t n = strlen(s);
    u64(n);
    bytes(s, n);
  }
};

// reads the flat stream
struct Words {
  const uint32_t* w;
  size_t n;
  size_t pos = 0;
  bool ok = true;
  uint32_t next() {
    if (pos >= n) {
      ok = false;
      return 0;
    }
    return w[pos++];
  }
  // a count that must fit in what is left, at `per` words per item
  uint32_t count(size_t per) {
    const uint32_t c = next();
    if (!ok || (per && (size_t)c > (n - pos) / per)) ok = false;
    return ok ? c : 0;
  }
};

void put_fields(Words& in, Writer& o, size_t count) {
  for (size_t i = 0; i < count; i++) o.field(in.next());
}

void put_sumcheck(Words& in, Writer& o) {
  const uint32_t np = in.count(8);
  o.u64(np);
  put_fields(in, o, (size_t)np * 8);  // [EF; 2] per round: c0 then c2
  const uint32_t nw = in.count(1);
  o.u64(nw);
  put_fields(in, o, nw);
}

void put_queries(Words& in, Writer& o) {
  const uint32_t nq = in.count(3);
  o.u64(nq);
  for (uint32_t q = 0; q < nq && in.ok; q++) {
    const uint32_t kind = in.next();
    if (kind > 1) in.ok = false;
    o.str(kind ? "extension" : "base");
    const uint32_t nv = in.count(kind ? 4 : 1);
    o.u64(nv);
    put_fields(in, o, (size_t)nv * (kind ? 4 : 1));
    const uint32_t path = in.count(8);
    o.u64(path);
    put_fields(in, o, (size_t)path * 8);
  }
}

// reads the bincode bytes
struct Reader {
  const uint8_t* b;
  size_t n;
  size_t pos = 0;
  bool ok = true;
  bool take(void* dst, size_t k) {
    if (!ok || k > n - pos) return ok = false;
    memcpy(dst, b + pos, k);
    pos += k;
    return true;
  }
  uint8_t u8() {
    uint8_t v = 0;
    take(&v, 1);
    return v;
  }
  uint32_t u32() {
    uint8_t t[4] = {0, 0, 0, 0};
    take(t, 4);
    return (uint32_t)t[0] | ((uint32_t)t[1] << 8) | ((uint32_t)t[2] << 16) | ((uint32_t)t[3] << 24);
  }
  uint64_t u64() {
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v |= (uint64_t)u8() << (8 * i);
    return v;
  }
  uint32_t field() {
    const uint32_t m = u32();
    if (m >= kb::P) ok = false;
    return ok ? kb::from_mont(m) : 0u;
  }
  // a length whose items need at least `per` bytes each
  uint32_t len(size_t per) {
    const uint64_t v = u64();
    if (!ok || v > 0xffffffffull || (per && v > (n - pos) / per)) ok = false;
    return ok ? (uint32_t)v : 0u;
  }
  bool option() {
    const uint8_t t = u8();
    if (t > 1) ok = false;
    return t == 1;
  }
};

void get_fields(Reader& r, std::vector<uint32_t>& w, size_t count) {
  for (size_t i = 0; i < count && r.ok; i++) w.push_back(r.field());
}

void get_sumcheck(Reader& r, std::vector<uint32_t>& w) {
  const uint32_t np = r.len(32);
  w.push_back(np);
  get_fields(r, w, (size_t)np * 8);
  const uint32_t nw = r.len(4);
  w.push_back(nw);
  get_fields(r, w, nw);
}

void get_queries(Reader& r, std::vector<uint32_t>& w) {
  const uint32_t nq = r.len(8 + 4 + 8 + 8);
  w.push_back(nq);
  for (uint32_t q = 0; q < nq && r.ok; q++) {
    const uint32_t tl = r.len(1);
    std::string tag(tl, '\0');
    if (tl) r.take(&tag[0], tl);
    const int kind = tag == "base" ? 0 : tag == "extension" ? 1 : -1;
    if (kind < 0) {
      r.ok = false;
      return;
    }
    w.push_back((uint32_t)kind);
    const uint32_t nv = r.len(kind ? 16 : 4);
    w.push_back(nv);
    get_fields(r, w, (size_t)nv * (kind ? 4 : 1));
    const uint32_t path = r.len(32);
    w.push_back(path);
    get_fields(r, w, (size_t)path * 8);
  }
}

}  // namespace

extern "C" {

int whir_proof_to_bincode(const uint32_t* words, size_t n_words, uint8_t* out, size_t cap, size_t* out_len) {
  WH_CHECK(words && out_len, "null argument");
  Words in{words, n_words};
  Writer o{out, out ? cap : 0};
  if (in.next() != 0x50524857u || in.next() != 1u) return wh::set_error("not a proof stream"), WHIR_ERR_INVALID;
  // initial_commitment: Option<Hash>, initial_ood_answers, initial_sumcheck
  o.u8(1);
  put_fields(in, o, 8);
  const uint32_t nood = in.count(4);
  o.u64(nood);
  put_fields(in, o, (size_t)nood * 4);
  put_sumcheck(in, o);
  // rounds
  const uint32_t nr = in.count(8);
  o.u64(nr);
  for (uint32_t r = 0; r < nr && in.ok; r++) {
    o.u8(1);  // commitment: Some(root)
    put_fields(in, o, 8);
    const uint32_t no = in.count(4);
    o.u64(no);
    put_fields(in, o, (size_t)no * 4);
    o.field(in.next());  // pow_witness
    put_queries(in, o);
    put_sumcheck(in, o);
  }
  // final_poly: Option<EvaluationsList<EF>>, final_pow_witness, final_queries
  const uint32_t nf = in.count(4);
  o.u8(1);
  o.u64(nf);
  put_fields(in, o, (size_t)nf * 4);
  o.field(in.next());
  put_queries(in, o);
  // final_sumcheck: Option<SumcheckData>
  const uint32_t has = in.next();
  if (has > 1) in.ok = false;
  o.u8((uint8_t)has);
  if (has == 1) put_sumcheck(in, o);
  if (!in.ok || in.pos != n_words) return wh::set_error("malformed proof stream"), WHIR_ERR_INVALID;
  *out_len = o.len;
  if (!out || o.len > cap) return wh::set_error("output buffer too small"), WHIR_ERR_BUFFER;
  return WHIR_OK;
}

int whir_proof_from_bincode(const uint8_t* bytes, size_t len, uint32_t* words, size_t cap, size_t* n_words) {
  WH_CHECK(bytes && n_words, "null argument");
  Reader r{bytes, len};
  std::vector<uint32_t> w = {0x50524857u, 1u};
  if (!r.option()) r.ok = false;  // the initial commitment is always present
  get_fields(r, w, 8);
  const uint32_t nood = r.len(16);
  w.push_back(nood);
  get_fields(r, w, (size_t)nood * 4);
  get_sumcheck(r, w);
  const uint32_t nr = r.len(1 + 32 + 8 + 4 + 8 + 16);
  w.push_back(nr);
  for (uint32_t k = 0; k < nr && r.ok; k++) {
    if (!r.option()) r.ok = false;
    get_fields(r, w, 8);
    const uint32_t no = r.len(16);
    w.push_back(no);
    get_fields(r, w, (size_t)no * 4);
    w.push_back(r.field());
    get_queries(r, w);
    get_sumcheck(r, w);
  }
  if (!r.option()) r.ok = false;  // the final polynomial is always present
  const uint32_t nf = r.len(16);
  w.push_back(nf);
  get_fields(r, w, (size_t)nf * 4);
  w.push_back(r.field());
  get_queries(r, w);
  const bool has = r.option();
  w.push_back(has ? 1u : 0u);
  if (has) get_sumcheck(r, w);
  if (!r.ok || r.pos != len) return wh::set_error("malformed bincode proof"), WHIR_ERR_INVALID;
  *n_words = w.size();
  if (!words || w.size() > cap) return wh::set_error("output buffer too small"), WHIR_ERR_BUFFER;
  memcpy(words, w.data(), w.size() * 4);
  return WHIR_OK;
}

}  // extern "C"
