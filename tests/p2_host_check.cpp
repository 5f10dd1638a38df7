// Host build of the device Poseidon2 header (poseidon2.cuh) checking the
// specialised forms the kernels use against the plain permutation, on the
// same templates the GPU compiles (only the S-box's product method differs
// between host and device), for both external blocks (MAT 0: the circulant
// (2, 3, 1, 1); MAT 1: the paper's M4):
//   - m4<MAT> and m4_row3<MAT> against the block's matrix entries;
//   - grind_word7<slot> (folded initial layer, output word 7 only) for every
//     witness position 0..7;
//   - permute_sponge (zero-capacity first layer, digest-only last layer) for
//     width 24 / rate 16 and width 16 / rate 8;
//   - diag_axpy for every diagonal code, against s + mu * x mod p;
//   - sum_mod against a plain sum.
// Prints "ok <checks>" or the first mismatch, and exits non-zero on one.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <initializer_list>

#include "poseidon2.cuh"

namespace {
uint64_t g_state = 0x9e3779b97f4a7c15ull;
uint32_t next_field() {
  for (;;) {
    g_state ^= g_state << 13;
    g_state ^= g_state >> 7;
    g_state ^= g_state << 17;
    const uint32_t v = (uint32_t)(g_state >> 33);
    if (v < kb::P) return v;
  }
}
uint32_t pick(int i) {  // edge values first, then random
  const uint32_t edge[6] = {0u, 1u, 2u, kb::P - 1, kb::P - 2, (kb::P - 1) / 2};
  return i < 6 ? edge[i] : next_field();
}

p2::P2Consts consts(int width) {
  p2::P2Consts k;
  memset(&k, 0, sizeof(k));
  k.width = width;
  k.rounds_f = p2::RF;
  k.rounds_p = width == 16 ? p2::RP16 : p2::RP24;
  for (int i = 0; i < 8 * 24; i++) k.ext_rc[i] = next_field();
  for (int i = 0; i < 32; i++) k.int_rc[i] = next_field();
  for (int i = 0; i < width; i++) {
    k.diag_c[i] = p2::diag_value(p2::diag_code(width, i));
    k.diag_s[i] = kb::shoup_const(k.diag_c[i]);
  }
  return k;
}

long g_checks = 0;
bool fail(const char* what, int a, int b) {
  printf("mismatch %s %d %d\n", what, a, b);
  return false;
}

template <int MAT>
bool check_m4() {
  for (int t = 0; t < 400; t++) {
    uint32_t x[4];
    for (int i = 0; i < 4; i++) x[i] = pick(t < 6 ? t : (t < 30 ? (t + i) % 6 : 6));
    uint32_t y[4] = {x[0], x[1], x[2], x[3]};
    p2::m4<MAT>(y[0], y[1], y[2], y[3]);
    for (int i = 0; i < 4; i++) {
      uint64_t want = 0;
      for (int j = 0; j < 4; j++) want += (uint64_t)p2::m4_entry<MAT>(i, j) * x[j];
      if (y[i] != want % kb::P) return fail("m4", MAT, i);
    }
    if (p2::m4_row3<MAT>(x[0], x[1], x[2], x[3]) != y[3]) return fail("m4_row3", MAT, t);
    g_checks++;
  }
  return true;
}

template <int SLOT, int MAT>
bool check_grind(const p2::P2Consts& k) {
  for (int t = 0; t < 40; t++) {
    uint32_t st[16];
    for (int i = 0; i < 16; i++) st[i] = pick(t == 0 ? i % 6 : 6);
    const uint32_t w = t < 6 ? pick(t) : next_field();
    uint32_t full[16];
    memcpy(full, st, sizeof(full));
    full[SLOT] = w;
    p2::permute_canonical<16, p2::RP16, MAT>(full, k);
    uint32_t cp[16];
    memcpy(cp, st, sizeof(cp));
    cp[SLOT] = 0u;
    p2::grind_fold<MAT>(cp, k);
    if (p2::grind_word7<SLOT, MAT>(w, cp, k) != full[7]) return fail("grind_word7", SLOT + 8 * MAT, t);
    g_checks++;
  }
  return true;
}

template <int T, int RP, int RATE, bool FIRST, bool LAST, int MAT>
bool check_sponge(const p2::P2Consts& k) {
  for (int t = 0; t < 40; t++) {
    uint32_t a[T], b[T];
    for (int i = 0; i < T; i++) a[i] = (FIRST && i >= RATE) ? 0u : pick(t == 0 ? i % 6 : 6);
    memcpy(b, a, sizeof(a));
    p2::permute_canonical<T, RP, MAT>(a, k);
    p2::permute_sponge<T, RP, RATE, FIRST, LAST, MAT>(b, k);
    const int n = LAST ? 8 : T;
    for (int i = 0; i < n; i++)
      if (a[i] != b[i]) return fail("permute_sponge", T * 10 + (FIRST ? 1 : 0) + (LAST ? 2 : 0), i);
    g_checks++;
  }
  return true;
}

bool check_diag() {
  for (int width : {16, 24})
    for (int i = 0; i < width; i++) {
      const uint64_t mu = p2::diag_value(p2::diag_code(width, i));
      for (int t = 0; t < 200; t++) {
        const uint32_t s = pick(t % 7 == 0 ? t % 6 : 6), x = pick(t < 6 ? t : 6);
        const uint32_t want = (uint32_t)((s + mu * x) % kb::P);
        if (p2::diag_axpy(p2::diag_code(width, i), s, x) != want) return fail("diag_axpy", width, i);
        g_checks++;
      }
    }
  return true;
}

bool check_sum() {
  for (int t = 0; t < 2000; t++) {
    uint32_t x[24];
    uint64_t ref = 0;
    for (int i = 0; i < 24; i++) {
      x[i] = t % 3 == 0 ? kb::P - 1 : pick(t < 6 ? t : 6);
      ref += x[i];
    }
    uint32_t y[16];
    uint64_t ref16 = 0;
    for (int i = 0; i < 16; i++) {
      y[i] = x[i];
      ref16 += y[i];
    }
    // sum_rest leaves out word 0
    if (p2::sum_rest<24>(x) != (ref - x[0]) % kb::P || p2::sum_rest<16>(y) != (ref16 - y[0]) % kb::P)
      return fail("sum_rest", t, 0);
    g_checks++;
  }
  return true;
}
}  // namespace

template <int MAT>
bool check_forms(const p2::P2Consts& k16, const p2::P2Consts& k24) {
  bool ok = check_m4<MAT>();
  ok = ok && check_grind<0, MAT>(k16) && check_grind<1, MAT>(k16) && check_grind<2, MAT>(k16) &&
       check_grind<3, MAT>(k16) && check_grind<4, MAT>(k16) && check_grind<5, MAT>(k16) &&
       check_grind<6, MAT>(k16) && check_grind<7, MAT>(k16);
  ok = ok && check_sponge<24, p2::RP24, 16, true, true, MAT>(k24) &&
       check_sponge<24, p2::RP24, 16, true, false, MAT>(k24) &&
       check_sponge<24, p2::RP24, 16, false, true, MAT>(k24) &&
       check_sponge<24, p2::RP24, 16, false, false, MAT>(k24);
  ok = ok && check_sponge<16, p2::RP16, 8, true, true, MAT>(k16) &&
       check_sponge<16, p2::RP16, 8, false, true, MAT>(k16);
  return ok;
}

int main() {
  const p2::P2Consts k16 = consts(16), k24 = consts(24);
  bool ok = check_forms<p2::kMatMds>(k16, k24) && check_forms<p2::kMatHl>(k16, k24);
  ok = ok && check_diag() && check_sum();
  if (!ok) return 1;
  printf("ok %ld\n", g_checks);
  return 0;
}
