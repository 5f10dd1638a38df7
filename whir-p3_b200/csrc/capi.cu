// extern "C" entry points: context, parameters, challenger and the
// Plonky3-trait / multilinear kernels on caller-owned device buffers.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>

#include "host.h"

namespace wh {
const char* last_error();
}

using kb::ef;

namespace {

constexpr size_t kArenaBytes = 64ull << 20;
constexpr size_t kPinnedBytes = 8ull << 20;

int check_ctx(const whir_ctx* ctx) {
  if (!ctx) {
    wh::set_error("null context");
    return WHIR_ERR_INVALID;
  }
  return WHIR_OK;
}

// device work needs a context created on a device (not a host-only one)
int check_gpu(const whir_ctx* ctx) {
  WH_TRY(check_ctx(ctx));
  if (ctx->device < 0) {
    wh::set_error("host-only context (device -1) cannot run device work");
    return WHIR_ERR_NO_DEVICE;
  }
  cudaSetDevice(ctx->device);
  return WHIR_OK;
}

ef load_ef_canon(const uint32_t* p) {
  return ef{{kb::to_mont(p[0]), kb::to_mont(p[1]), kb::to_mont(p[2]), kb::to_mont(p[3])}};
}
void store_ef_canon(uint32_t* p, const ef& v) {
  for (int i = 0; i < 4; i++) p[i] = kb::from_mont(v.c[i]);
}
bool canon_ok(const uint32_t* p, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (p[i] >= kb::P) return false;
  return true;
}

int sync(whir_ctx* ctx) {
  WH_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
  return WHIR_OK;
}

}  // namespace

// shared with prover.cu
namespace wh {

void add_stage_work(whir_ctx* ctx, int stage, uint64_t work) {
  if (ctx && ctx->profiling && stage >= 0 && stage < kStCount) ctx->stage_work[stage] += work;
}

StageTimer::StageTimer(whir_ctx* c, int s, uint64_t work) : ctx(c), stage(s) {
  if (!ctx || !ctx->profiling) return;
  ctx->stage_work[s] += work;
  for (cudaEvent_t* e : {&a, &b}) {
    if (!ctx->event_pool.empty()) {
      *e = ctx->event_pool.back();
      ctx->event_pool.pop_back();
    } else if (cudaEventCreate(e) != cudaSuccess) {
      *e = nullptr;
    }
  }
  if (a) cudaEventRecord(a, ctx->stream);
}

StageTimer::~StageTimer() {
  if (!ctx || !ctx->profiling || !a || !b) return;
  cudaEventRecord(b, ctx->stream);
  ctx->stage_events.push_back({stage, {a, b}});
}

int ensure_dft_tables(whir_ctx* ctx, int log_h, wk::DftTables* t) {
  WH_CHECK(log_h >= 0 && log_h < kDftLogHeights && ctx->tw_heights, "DFT height out of range");
  t->tw_stage = ctx->tw_stage;
  t->tw_sh = reinterpret_cast<const uint2*>(ctx->tw_stage + 2048);
  t->tw_lo = ctx->tw_heights + (size_t)log_h * kDftTableWords;
  t->tw_hi = t->tw_lo + 4096;
  t->err = ctx->d_words + 12;
  return WHIR_OK;
}

// Split-eq tables of a point with `n` coordinates into the arena at `at`:
// hi (2^(n-lo)) scaled by `scale`, then lo (2^lo); returns the lo bit count.
int split_eq_tables(whir_ctx* ctx, const ef* z, int n, const ef& scale, int lo_bits, ef* hi, ef* lo) {
  wk::EqPoint a;
  memset(&a, 0, sizeof(a));
  a.h = n - lo_bits;
  for (int i = 0; i < a.h; i++) a.z[i] = z[i];
  a.scale = scale;
  wk::EqPoint b;
  memset(&b, 0, sizeof(b));
  b.h = lo_bits;
  for (int i = 0; i < lo_bits; i++) b.z[i] = z[n - lo_bits + i];
  b.scale = kb::ef_one();
  WH_TRY_CUDA(wk::eq_table_pair(a, hi, b, lo, ctx->stream));
  return WHIR_OK;
}

// sum_x f[x] eq(z, x) for extension (ext=1) or base f of 2^n entries, split
// into 2^seg_bits segments of 2^(n - seg_bits) (the point covers one segment).
// Results (Montgomery) land in ctx->d_small[0 .. 2^seg_bits).
// The results also go to the mailbox when they fit: *posted receives the
// sequence to wait for (0 when not posted).
int dot_eq(whir_ctx* ctx, const uint32_t* d_f, int ext, int seg_bits, const ef* z, int m_bits, uint32_t* posted) {
  if (m_bits > 40) return set_error("dot_eq: size"), WHIR_ERR_INVALID;
  StageTimer timer(ctx, kStEval);
  const int lo_bits = std::min(m_bits, 8);
  ef* hi = reinterpret_cast<ef*>(ctx->d_arena);
  ef* lo = hi + ((size_t)1 << (m_bits - lo_bits));
  WH_TRY(split_eq_tables(ctx, z, m_bits, kb::ef_one(), lo_bits, hi, lo));
  const bool post = posted && ctx->h_mail && (4 << seg_bits) <= wk::kMailWords;
  const uint32_t seq = post ? mail_next(ctx) : 0u;
  if (posted) *posted = seq;
  WH_TRY_CUDA(wk::dot_split(d_f, ext, seg_bits, m_bits, hi, lo, lo_bits, ctx->d_partials,
                            reinterpret_cast<unsigned*>(ctx->d_words) + 9, ctx->d_small, post ? ctx->d_mail : nullptr,
                            seq, ctx->d_words + 11, ctx->stream));
  return WHIR_OK;
}

int mail_wait(whir_ctx* ctx, uint32_t seq, void* host, size_t bytes);

// spin-loop hint: lets a sibling hardware thread run and lowers the cost of
// polling
inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#elif defined(__aarch64__)
  asm volatile("yield");
#endif
}

// Small results come back through the mailbox: the producing kernel (or a
// one-CTA copy kernel queued after it) writes them into mapped host memory and
// then bumps a sequence flag, which this thread polls (about 9 us per round
// trip on B200 against 16 us for a copy plus a stream synchronisation).
uint32_t mail_next(whir_ctx* ctx) {
  uint32_t seq = ++ctx->mail_seq;
  if (seq == 0) seq = ++ctx->mail_seq;
  return seq;
}

int fetch_mail(whir_ctx* ctx, void* host, const void* dev, size_t bytes) {
  const uint32_t seq = mail_next(ctx);
  WH_TRY_CUDA(wk::publish(static_cast<const uint32_t*>(dev), (int)((bytes + 3) / 4), ctx->d_mail, seq, ctx->stream));
  return mail_wait(ctx, seq, host, bytes);
}

// Waits until the mailbox flag reaches `seq` and copies `bytes` of payload.
int mail_wait(whir_ctx* ctx, uint32_t seq, void* host, size_t bytes) {
  volatile uint32_t* flag = ctx->h_mail + wk::kMailWords;
  // Spin for a short while (typical results arrive within tens of
  // microseconds); past that, poll with a yield between checks, so that many
  // waiting contexts (batch workers) leave the host's cores to each other,
  // and ask the stream every ~100 us whether it failed or finished without
  // posting (the result is posted before the stream completes). Polling
  // rather than a stream synchronisation also returns as soon as the result
  // is posted, not when the work queued behind its producer is done.
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  const auto spin = std::chrono::microseconds(ctx->wait_spin_us.load(std::memory_order_relaxed));
  bool spinning = spin.count() > 0;
  auto next_query = t0;
  for (uint64_t n = 1; *flag != seq; n++) {
    if (spinning) {
      cpu_relax();
      if ((n & 255) == 0 && clk::now() - t0 > spin) spinning = false;
      continue;
    }
    std::this_thread::yield();
    const auto now = clk::now();
    if (now < next_query) continue;
    next_query = now + std::chrono::microseconds(100);
    const cudaError_t q = cudaStreamQuery(ctx->stream);
    std::atomic_thread_fence(std::memory_order_acquire);
    if (q == cudaSuccess && *flag != seq) {
      set_error("device result missing after the stream completed");
      return WHIR_ERR_CUDA;
    }
    if (q != cudaSuccess && q != cudaErrorNotReady) {
      set_error(std::string("stream failed while waiting for a result: ") + cudaGetErrorString(q));
      return WHIR_ERR_CUDA;
    }
    if (now - t0 > std::chrono::seconds(120)) {
      set_error("timed out waiting for a device result");
      return WHIR_ERR_CUDA;
    }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  memcpy(host, const_cast<const uint32_t*>(ctx->h_mail), bytes);
  return WHIR_OK;
}

int fetch_posted(whir_ctx* ctx, uint32_t seq, void* host, const void* dev, size_t bytes) {
  return seq ? mail_wait(ctx, seq, host, bytes) : fetch(ctx, host, dev, bytes);
}

int fetch(whir_ctx* ctx, void* host, const void* dev, size_t bytes) {
  if (ctx->h_mail && bytes % 4 == 0 && bytes <= (size_t)wk::kMailWords * 4) return fetch_mail(ctx, host, dev, bytes);
  if (bytes <= ctx->pinned_bytes) {
    WH_TRY_CUDA(cudaMemcpyAsync(ctx->h_pinned, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    WH_TRY(sync(ctx));
    memcpy(host, ctx->h_pinned, bytes);
  } else {
    WH_TRY_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    WH_TRY(sync(ctx));
  }
  return WHIR_OK;
}

int upload(whir_ctx* ctx, void* dev, const void* host, size_t bytes) {
  if (bytes % 4 == 0 && bytes <= (size_t)wk::kPutWords * 4 && ((uintptr_t)dev & 3) == 0) {
    // small data (query indices, select weights): in a launch's parameters,
    // ordered on the stream, without waiting for the work queued before it
    WH_TRY_CUDA(wk::put_words(static_cast<uint32_t*>(dev), static_cast<const uint32_t*>(host), (int)(bytes / 4),
                              ctx->stream));
    return WHIR_OK;
  }
  if (bytes <= ctx->pinned_bytes) {
    // the staging buffer may still feed an earlier copy: wait for the stream first
    WH_TRY(sync(ctx));
    memcpy(ctx->h_pinned, host, bytes);
    WH_TRY_CUDA(cudaMemcpyAsync(dev, ctx->h_pinned, bytes, cudaMemcpyHostToDevice, ctx->stream));
  } else {
    WH_TRY_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    WH_TRY(sync(ctx));
  }
  return WHIR_OK;
}

// GrindingChallenger::grind on the device, then check_witness on the host
// state (absorbing the witness exactly as the reference does).
int grind(whir_ctx* ctx, Chal& ch, int bits, uint32_t* witness) {
  if (bits <= 0) {
    *witness = 0;
    return WHIR_OK;
  }
  WH_CHECK(bits <= 30, "grinding bits above 30");
  // inputs pending beyond 7 never occur (8 inputs trigger a duplexing)
  const uint32_t seq = ctx->h_mail ? mail_next(ctx) : 0u;
  {
    StageTimer t(ctx, kStGrind);
    if (ch.family == kChalKeccak)
      WH_TRY_CUDA(wk::keccak_grind(ch.kin, bits, kb::P, ctx->d_words, ctx->d_words + 1, ctx->d_words + 2,
                                   ctx->h_mail ? ctx->d_mail : nullptr, seq, ctx->stream, ctx->grind_window.load()));
    else
      WH_TRY_CUDA(wk::grind(ch.st, ch.in, ch.in_len, bits, kb::P, ctx->d_words, ctx->d_words + 1, ctx->d_words + 2,
                            ctx->h_mail ? ctx->d_mail : nullptr, seq, ctx->p16, ctx->stream, nullptr, nullptr,
                            nullptr, nullptr, nullptr, ctx->grind_window.load()));
  }
  // with a mailbox the search posts its witness and the number of candidates
  // it evaluated
  uint32_t got[2] = {0u, 0u};
  WH_TRY(fetch_posted(ctx, ctx->h_mail ? seq : 0u, got, ctx->d_words, ctx->h_mail ? 8 : 4));
  const uint32_t w = got[0];
  if (ctx->h_mail) add_stage_work(ctx, kStGrind, (uint64_t)got[1]);
  if (w >= kb::P) {
    set_error("proof-of-work search found no witness");
    return WHIR_ERR_NOT_FOUND;
  }
  ch.observe(ctx->hp16, kb::to_mont(w));
  if (ch.sample_bits(ctx->hp16, bits) != 0) {
    set_error("device grinding returned an invalid witness");
    return WHIR_ERR_CUDA;
  }
  *witness = w;
  return WHIR_OK;
}

}  // namespace wh

namespace wh {
// eq table of k challenge coordinates on the host (Montgomery), 2^k entries
std::vector<ef> eq_host(const ef* rs, int k) {
  std::vector<ef> v((size_t)1 << k, kb::ef_zero());
  v[0] = kb::ef_one();
  for (int i = 0; i < k; i++) {
    // bit i (from the bottom) of y <-> rs[k-1-i]
    const ef z = rs[k - 1 - i];
    const size_t half = (size_t)1 << i;
    for (size_t y = 0; y < half; y++) {
      const ef lo = v[y];
      const ef hi = kb::ef_mul(lo, z);
      v[y + half] = hi;
      v[y] = kb::ef_sub(lo, hi);
    }
  }
  return v;
}
// the same for k <= 6 (the kernels' fixed-size table; callers check k)
wk::EqSmall eq_small_host(const ef* rs, int k) {
  wk::EqSmall e;
  memset(&e, 0, sizeof(e));
  const std::vector<ef> v = eq_host(rs, k < 6 ? k : 6);
  for (size_t y = 0; y < v.size(); y++) e.v[y] = v[y];
  return e;
}
}  // namespace wh

namespace wh {
// W += sum_i scale_i * eq(z_i, .) over 2^n entries (Montgomery inputs)
int add_eq_points(whir_ctx* ctx, ef* d_w, int n, const std::vector<std::vector<ef>>& pts, const std::vector<ef>& scales,
                  int accumulate) {
  const int m = (int)pts.size();
  StageTimer timer(ctx, kStWeights);
  if (m == 0) {
    if (!accumulate) WH_TRY_CUDA(cudaMemsetAsync(d_w, 0, ((size_t)1 << n) * sizeof(ef), ctx->stream));
    return WHIR_OK;
  }
  const int lo_bits = std::min(n, 10);
  const size_t H = (size_t)1 << (n - lo_bits), Lc = (size_t)1 << lo_bits;
  WH_CHECK((H + Lc) * (size_t)m * sizeof(ef) <= ctx->arena_bytes, "too many constraints for the scratch arena");
  ef* hi = reinterpret_cast<ef*>(ctx->d_arena);
  ef* lo = hi + H * m;
  // the split tables of up to four points per launch (their hi and lo tables)
  const int hb = n - lo_bits;
  if (hb <= wk::kEqMultiCoords) {
    for (int c0 = 0; c0 < m; c0 += wk::kEqMultiTables / 2) {
      wk::EqMulti em;
      memset(&em, 0, sizeof(em));
      for (int c = c0; c < m && c < c0 + wk::kEqMultiTables / 2; c++) {
        const int th = em.count, tl = em.count + 1;
        em.h[th] = hb;
        em.zoff[th] = th * wk::kEqMultiCoords;
        em.out[th] = hi + H * c;
        em.scale[th] = scales[c];
        em.h[tl] = lo_bits;
        em.zoff[tl] = tl * wk::kEqMultiCoords;
        em.out[tl] = lo + Lc * c;
        em.scale[tl] = kb::ef_one();
        for (int i = 0; i < hb; i++) em.z[em.zoff[th] + i] = pts[c][i];
        for (int i = 0; i < lo_bits; i++) em.z[em.zoff[tl] + i] = pts[c][hb + i];
        em.count += 2;
      }
      WH_TRY_CUDA(wk::eq_tables_multi(em, ctx->stream));
    }
  } else {
    for (int c = 0; c < m; c++)
      WH_TRY(split_eq_tables(ctx, pts[c].data(), n, scales[c], lo_bits, hi + H * c, lo + Lc * c));
  }
  for (int c0 = 0; c0 < m; c0 += 16) {
    const int cnt = std::min(16, m - c0);
    WH_TRY_CUDA(wk::add_eq_batch(d_w, n, hi + H * c0, lo + Lc * c0, lo_bits, cnt, accumulate || c0 > 0, ctx->stream));
  }
  return WHIR_OK;
}

// W += sum_j g_j * vars_j^x (vars base field, Montgomery)
int add_select_vars(whir_ctx* ctx, ef* d_w, int n, const std::vector<uint32_t>& vars, const std::vector<ef>& g) {
  const int m = (int)vars.size();
  if (m == 0) return WHIR_OK;
  const int lo_bits = std::min(n, 10);
  const size_t Lc = (size_t)1 << lo_bits, H = (size_t)1 << (n - lo_bits);
  const size_t need = (size_t)m * 4 + (size_t)m * sizeof(ef) + (size_t)m * (Lc + H) * 4 + 64;
  WH_CHECK(need <= ctx->arena_bytes, "too many select constraints for the scratch arena");
  uint8_t* base = reinterpret_cast<uint8_t*>(ctx->d_arena);
  ef* d_g = reinterpret_cast<ef*>(base);
  uint32_t* d_vars = reinterpret_cast<uint32_t*>(d_g + m);
  uint32_t* pow_lo = d_vars + ((m + 3) & ~3);
  uint32_t* pow_hi = pow_lo + (size_t)m * Lc;
  std::vector<uint8_t> host((size_t)m * sizeof(ef) + (size_t)m * 4);
  memcpy(host.data(), g.data(), (size_t)m * sizeof(ef));
  memcpy(host.data() + (size_t)m * sizeof(ef), vars.data(), (size_t)m * 4);
  WH_TRY(upload(ctx, d_g, host.data(), host.size()));
  StageTimer timer(ctx, kStWeights);
  WH_TRY_CUDA(wk::select_tables(d_vars, m, n, lo_bits, pow_lo, pow_hi, ctx->stream));
  WH_TRY_CUDA(wk::add_select(d_w, n, pow_lo, pow_hi, lo_bits, d_g, m, ctx->stream));
  return WHIR_OK;
}
}  // namespace wh

extern "C" {

const char* whir_last_error(void) { return wh::last_error(); }
uint64_t whir_kernel_launches(void) { return wk::launches(); }

int whir_poseidon2_default_params(whir_poseidon2_params* p16, whir_poseidon2_params* p24) {
  wh::default_params(p16, p24);
  return WHIR_OK;
}

int whir_poseidon2_params_from_rng(uint64_t seed, uint32_t external_matrix, whir_poseidon2_params* p16,
                                   whir_poseidon2_params* p24) {
  WH_CHECK(external_matrix == WHIR_P2_MDS_MAT4 || external_matrix == WHIR_P2_HL_MAT4, "unknown external matrix");
  wh::params_from_rng(seed, external_matrix, p16, p24);
  return WHIR_OK;
}

int whir_rng_koalabear(uint64_t seed, uint32_t* out, size_t count) {
  WH_CHECK(out || count == 0, "null output");
  wh::SmallRng g(seed);
  for (size_t i = 0; i < count; i++) out[i] = g.field();
  return WHIR_OK;
}

int whir_ctx_create(int32_t device, const whir_poseidon2_params* p16, const whir_poseidon2_params* p24,
                    whir_ctx** out) {
  if (!out) return wh::set_error("null output"), WHIR_ERR_INVALID;
  *out = nullptr;
  if (device == -1) {
    // host-only context: Poseidon2 data, parameters and transcript, no device
    whir_poseidon2_params d16, d24;
    wh::default_params(&d16, &d24);
    if (!p16) p16 = &d16;
    if (!p24) p24 = &d24;
    WH_TRY(wh::validate_params(*p16, 16));
    WH_TRY(wh::validate_params(*p24, 24));
    WH_CHECK(p16->external_matrix == p24->external_matrix,
             "the width-16 and width-24 permutations must use the same external matrix");
    whir_ctx* c = new whir_ctx();
    c->device = -1;
    c->p16_params = *p16;
    c->p24_params = *p24;
    c->p16 = wh::to_consts(*p16);
    c->p24 = wh::to_consts(*p24);
    c->hp16 = wh::host_consts16(*p16);
    *out = c;
    return WHIR_OK;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    wh::set_error("no CUDA device");
    return WHIR_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return wh::set_error("device index out of range"), WHIR_ERR_INVALID;
  whir_poseidon2_params d16, d24;
  wh::default_params(&d16, &d24);
  if (!p16) p16 = &d16;
  if (!p24) p24 = &d24;
  WH_TRY(wh::validate_params(*p16, 16));
  WH_TRY(wh::validate_params(*p24, 24));
  WH_CHECK(p16->external_matrix == p24->external_matrix,
           "the width-16 and width-24 permutations must use the same external matrix");
  whir_ctx* c = new whir_ctx();
  c->device = device;
  c->p16_params = *p16;
  c->p24_params = *p24;
  c->p16 = wh::to_consts(*p16);
  c->p24 = wh::to_consts(*p24);
  c->hp16 = wh::host_consts16(*p16);
  auto fail = [&](int code) {
    whir_ctx_destroy(c);
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) return wh::set_error("cudaSetDevice failed"), fail(WHIR_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return wh::set_error("stream creation failed"), fail(WHIR_ERR_CUDA);
  c->own_stream = true;
  if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return wh::set_error("stream creation failed"), fail(WHIR_ERR_CUDA);
  for (cudaEvent_t& e : c->up_ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      return wh::set_error("event creation failed"), fail(WHIR_ERR_CUDA);
  {
    // the context's own pool, keeping freed blocks cached between proofs
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess)
      return wh::set_error("memory pool creation failed"), fail(WHIR_ERR_CUDA);
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  if (cudaMalloc(&c->tw_stage, wk::kDftStageTableWords * 4) != cudaSuccess || cudaMalloc(&c->d_partials, 8192 * sizeof(ef)) != cudaSuccess ||
      cudaMalloc(&c->d_small, 256 * sizeof(ef)) != cudaSuccess || cudaMalloc(&c->d_words, 64) != cudaSuccess ||
      cudaMalloc(&c->d_arena, kArenaBytes) != cudaSuccess)
    return wh::set_error("device allocation failed"), fail(WHIR_ERR_NOMEM);
  c->arena_bytes = kArenaBytes;
  if (cudaMemset(c->d_words, 0, 64) != cudaSuccess) return wh::set_error("device memset failed"), fail(WHIR_ERR_CUDA);
  if (wk::grind_reset(c->d_words, c->d_words + 1, c->d_words + 2, c->stream) != cudaSuccess)
    return wh::set_error("grind state initialisation failed"), fail(WHIR_ERR_CUDA);
  if (cudaHostAlloc(&c->h_pinned, kPinnedBytes, cudaHostAllocDefault) != cudaSuccess)
    return wh::set_error("pinned allocation failed"), fail(WHIR_ERR_NOMEM);
  c->pinned_bytes = kPinnedBytes / 2;
  c->h_open = static_cast<uint8_t*>(c->h_pinned) + kPinnedBytes / 2;
  c->open_bytes = kPinnedBytes / 2;
  if (cudaEventCreateWithFlags(&c->open_ev, cudaEventDisableTiming) != cudaSuccess)
    return wh::set_error("event creation failed"), fail(WHIR_ERR_CUDA);
  if (cudaHostAlloc(&c->h_mail, (wk::kMailWords + 32) * 4, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void**>(&c->d_mail), c->h_mail, 0) != cudaSuccess)
    return wh::set_error("mapped allocation failed"), fail(WHIR_ERR_NOMEM);
  memset(c->h_mail, 0, (wk::kMailWords + 32) * 4);
  // twiddle tables of every subgroup height (the stage tables come with them)
  if (cudaMalloc(&c->d_tr, wh::kDevTrWords * 4) != cudaSuccess)
    return wh::set_error("device allocation failed"), fail(WHIR_ERR_NOMEM);
  if (cudaMalloc(&c->tw_heights, wh::kDftLogHeights * wh::kDftTableWords * 4) != cudaSuccess)
    return wh::set_error("device allocation failed"), fail(WHIR_ERR_NOMEM);
  for (int lh = 0; lh < wh::kDftLogHeights; lh++) {
    uint32_t* lo = c->tw_heights + (size_t)lh * wh::kDftTableWords;
    if (wk::build_dft_tables(c->tw_stage, lo, lo + 4096, lh, c->stream) != cudaSuccess)
      return wh::set_error("DFT table build failed"), fail(WHIR_ERR_CUDA);
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return wh::set_error("initial sync failed"), fail(WHIR_ERR_CUDA);
  {
    const size_t gran = (size_t)2 << 20;
    auto up = [gran](size_t b) { return (b + gran - 1) / gran * gran; };
    c->fixed_device_bytes = up(wk::kDftStageTableWords * 4) + up(8192 * sizeof(ef)) + up(256 * sizeof(ef)) + up(64) +
                            up(kArenaBytes) + up((size_t)wh::kDftLogHeights * wh::kDftTableWords * 4) +
                            up(wh::kDevTrWords * 4);
  }
  *out = c;
  return WHIR_OK;
}

int whir_ctx_destroy(whir_ctx* c) {
  if (!c) return WHIR_OK;
  if (c->device < 0) {
    delete c;
    return WHIR_OK;
  }
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->tw_heights);
  cudaFree(c->d_tr);
  for (auto& rec : c->stage_events) {
    cudaEventDestroy(rec.second.first);
    cudaEventDestroy(rec.second.second);
  }
  for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
  }
  for (cudaEvent_t e : c->up_ev)
    if (e) cudaEventDestroy(e);
  if (c->open_ev) cudaEventDestroy(c->open_ev);
  cudaFree(c->tw_stage);
  cudaFree(c->d_partials);
  cudaFree(c->d_small);
  cudaFree(c->d_words);
  cudaFree(c->d_arena);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->h_mail) cudaFreeHost(c->h_mail);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (c->pool) cudaMemPoolDestroy(c->pool);
  delete c;
  return WHIR_OK;
}

int whir_ctx_set_stream(whir_ctx* ctx, void* stream) {
  WH_TRY(check_gpu(ctx));
  WH_TRY(sync(ctx));
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = (cudaStream_t)stream;
  ctx->own_stream = false;
  return WHIR_OK;
}

int whir_ctx_synchronize(whir_ctx* ctx) {
  WH_TRY(check_gpu(ctx));
  return sync(ctx);
}

int whir_ctx_set_profiling(whir_ctx* ctx, int32_t enable) {
  WH_TRY(check_gpu(ctx));
  ctx->profiling = enable != 0;
  return WHIR_OK;
}

int whir_ctx_stage_times(whir_ctx* ctx, double* ms, uint64_t* counts, int32_t cap, int32_t reset) {
  WH_TRY(check_gpu(ctx));
  WH_TRY(sync(ctx));
  for (auto& rec : ctx->stage_events) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, rec.second.first, rec.second.second) == cudaSuccess) {
      ctx->stage_ms[rec.first] += t;
      ctx->stage_launches[rec.first] += 1;
    }
    ctx->event_pool.push_back(rec.second.first);
    ctx->event_pool.push_back(rec.second.second);
  }
  ctx->stage_events.clear();
  for (int i = 0; i < wh::kStCount && i < cap; i++) {
    if (ms) ms[i] = ctx->stage_ms[i];
    if (counts) counts[i] = ctx->stage_launches[i];
  }
  if (reset)
    for (int i = 0; i < wh::kStCount; i++) {
      ctx->stage_ms[i] = 0.;
      ctx->stage_launches[i] = 0;
    }
  return wh::kStCount;
}

int whir_ctx_set_wait_spin(whir_ctx* ctx, int32_t microseconds) {
  WH_TRY(check_ctx(ctx));
  WH_CHECK(microseconds >= 0 && microseconds <= 100000, "spin time out of range");
  ctx->wait_spin_us.store(microseconds);
  return WHIR_OK;
}

int whir_ctx_set_grind_window(whir_ctx* ctx, int32_t mode) {
  WH_TRY(check_ctx(ctx));
  WH_CHECK(mode >= 0 && mode <= (wk::kGrindLeanSmall | wk::kGrindLeanLarge), "grind window mode must be 0 to 3");
  ctx->grind_window.store(mode);
  return WHIR_OK;
}

int whir_ctx_set_device_transcript(whir_ctx* ctx, int32_t enable) {
  WH_TRY(check_ctx(ctx));
  ctx->device_transcript = enable != 0;
  return WHIR_OK;
}

int whir_ctx_stage_work(whir_ctx* ctx, uint64_t* work, int32_t cap, int32_t reset) {
  WH_TRY(check_ctx(ctx));
  for (int i = 0; i < wh::kStCount && i < cap; i++)
    if (work) work[i] = ctx->stage_work[i];
  if (reset)
    for (int i = 0; i < wh::kStCount; i++) ctx->stage_work[i] = 0;
  return wh::kStCount;
}

int whir_poseidon2_permute(const whir_ctx* ctx, uint32_t* state, int32_t width) {
  WH_TRY(check_ctx(ctx));
  WH_CHECK(state && (width == 16 || width == 24), "width must be 16 or 24");
  WH_CHECK(canon_ok(state, (size_t)width), "state value out of range");
  if (width == 16) {
    wh::host_permute16(state, ctx->hp16);
  } else {
    uint32_t s[24];
    for (int i = 0; i < 24; i++) s[i] = state[i];
    p2::permute_canonical_rt<24, p2::RP24>(s, ctx->p24);
    for (int i = 0; i < 24; i++) state[i] = s[i];
  }
  return WHIR_OK;
}

int whir_config_new(const whir_protocol_params* params, int32_t n, whir_config* out) {
  WH_CHECK(params && out, "null argument");
  return wh::config_new(*params, n, out);
}

int whir_domain_separator(const whir_config* cfg, int32_t digest_elems, uint32_t* out, int32_t cap) {
  WH_CHECK(cfg, "null config");
  std::vector<uint32_t> v = wh::domain_separator(*cfg, digest_elems);
  if (out)
    for (int32_t i = 0; i < cap && i < (int32_t)v.size(); i++) out[i] = v[i];
  return (int)v.size();
}

void whir_challenger_init(whir_challenger* ch) {
  if (ch) memset(ch, 0, sizeof(*ch));
}

int whir_challenger_observe(const whir_ctx* ctx, whir_challenger* ch, const uint32_t* values, size_t n) {
  WH_TRY(check_ctx(ctx));
  WH_CHECK(ch && (values || n == 0), "null argument");
  WH_CHECK(canon_ok(values, n), "value out of range");
  wh::Chal c;
  c.load(*ch);
  for (size_t i = 0; i < n; i++) c.observe(ctx->hp16, kb::to_mont(values[i]));
  c.store(*ch);
  return WHIR_OK;
}

int whir_challenger_sample(const whir_ctx* ctx, whir_challenger* ch, uint32_t* out, size_t n) {
  WH_TRY(check_ctx(ctx));
  WH_CHECK(ch && (out || n == 0), "null argument");
  wh::Chal c;
  c.load(*ch);
  for (size_t i = 0; i < n; i++) out[i] = kb::from_mont(c.sample(ctx->hp16));
  c.store(*ch);
  return WHIR_OK;
}

int whir_challenger_sample_bits(const whir_ctx* ctx, whir_challenger* ch, int32_t bits, uint64_t* out) {
  WH_TRY(check_ctx(ctx));
  WH_CHECK(ch && out && bits >= 0 && bits < 31, "bad argument");
  wh::Chal c;
  c.load(*ch);
  *out = c.sample_bits(ctx->hp16, bits);
  c.store(*ch);
  return WHIR_OK;
}

int whir_challenger_grind(whir_ctx* ctx, whir_challenger* ch, int32_t bits, uint32_t* witness) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(ch && witness && bits >= 0, "bad argument");
  cudaSetDevice(ctx->device);
  wh::Chal c;
  c.load(*ch);
  if (bits == 0) {
    *witness = 0;
    return WHIR_OK;
  }
  WH_TRY(wh::grind(ctx, c, bits, witness));
  c.store(*ch);
  return WHIR_OK;
}

int whir_challenger_check_witness(const whir_ctx* ctx, whir_challenger* ch, int32_t bits, uint32_t witness) {
  WH_TRY(check_ctx(ctx));
  WH_CHECK(ch && bits >= 0 && bits < 31 && witness < kb::P, "bad argument");
  if (bits == 0) return 1;
  wh::Chal c;
  c.load(*ch);
  c.observe(ctx->hp16, kb::to_mont(witness));
  const int ok = c.sample_bits(ctx->hp16, bits) == 0;
  c.store(*ch);
  return ok;
}

int whir_device_alloc(whir_ctx* ctx, size_t bytes, void** d_ptr) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_ptr, "null argument");
  cudaSetDevice(ctx->device);
  WH_TRY_CUDA(cudaMalloc(d_ptr, bytes ? bytes : 1));
  return WHIR_OK;
}
int whir_device_free(whir_ctx* ctx, void* d_ptr) {
  WH_TRY(check_gpu(ctx));
  WH_TRY(sync(ctx));
  WH_TRY_CUDA(cudaFree(d_ptr));
  return WHIR_OK;
}
int whir_memcpy_h2d(whir_ctx* ctx, void* d_dst, const void* h_src, size_t bytes) {
  WH_TRY(check_gpu(ctx));
  WH_TRY_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return sync(ctx);
}
int whir_memcpy_d2h(whir_ctx* ctx, void* h_dst, const void* d_src, size_t bytes) {
  WH_TRY(check_gpu(ctx));
  WH_TRY_CUDA(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return sync(ctx);
}
int whir_monty_encode(whir_ctx* ctx, uint32_t* d, size_t n) {
  WH_TRY(check_gpu(ctx));
  WH_TRY_CUDA(wk::encode(d, n, ctx->stream));
  return WHIR_OK;
}
int whir_monty_decode(whir_ctx* ctx, uint32_t* d, size_t n) {
  WH_TRY(check_gpu(ctx));
  WH_TRY_CUDA(wk::decode(d, n, ctx->stream));
  return WHIR_OK;
}

int whir_dft_batch(whir_ctx* ctx, const uint32_t* d_chunks, int32_t log_chunk, int32_t log_width, int32_t log_blowup,
                   int32_t ext, uint32_t* d_out) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_chunks && d_out && log_chunk >= 0 && log_width >= 0 && log_width <= 12 && log_blowup >= 0 &&
               log_chunk + log_blowup <= 24,
           "bad DFT shape");
  const int lanes = ext ? 4 : 1;
  const int log_h = log_chunk + log_blowup;
  wk::DftTables t;
  WH_TRY(wh::ensure_dft_tables(ctx, log_h, &t));
  uint32_t* scratch = nullptr;
  const size_t bytes = ((size_t)1 << (log_h + log_width)) * 4 * lanes;
  WH_TRY_CUDA(wh::ctx_malloc(ctx, &scratch, bytes));
  const int s = wh::run_dft(ctx, d_chunks, d_out, scratch, log_chunk, log_width, log_blowup, lanes, t);
  cudaFreeAsync(scratch, ctx->stream);
  return s;
}

int whir_merkle_commit(whir_ctx* ctx, const uint32_t* d_rows, int32_t log_height, int32_t row_words,
                       int32_t leaf_hash, uint32_t* d_digests, uint32_t* root) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_rows && d_digests && log_height >= 0 && log_height <= 30 && row_words > 0 &&
               (leaf_hash == WHIR_LEAF_P24 || leaf_hash == WHIR_LEAF_P16 || leaf_hash == WHIR_LEAF_KECCAK),
           "bad Merkle arguments");
  WH_TRY(wh::run_merkle_leaves(ctx, d_rows, log_height, row_words, leaf_hash, d_digests));
  uint32_t posted = 0;
  WH_TRY(wh::run_merkle_upper(ctx, log_height, leaf_hash, d_digests, root ? &posted : nullptr));
  if (root) {
    const size_t h = (size_t)1 << log_height;
    uint32_t r[8];
    WH_TRY(wh::fetch_posted(ctx, posted, r, d_digests + (2 * h - 2) * 8, 32));
    for (int i = 0; i < 8; i++) root[i] = wh::digest_word_out(leaf_hash, r[i]);
  }
  return WHIR_OK;
}

int whir_merkle_commit_many(whir_ctx* ctx, int32_t count, const uint32_t* const* d_rows, const int32_t* log_heights,
                            int32_t row_words, int32_t leaf_hash, uint32_t* const* d_digests, uint32_t* roots) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(count >= 1 && count <= wk::kMaxManyTrees && d_rows && log_heights && d_digests && roots && row_words > 0 &&
               (leaf_hash == WHIR_LEAF_P24 || leaf_hash == WHIR_LEAF_P16),
           "bad batched Merkle arguments");
  int max_lh = 0;
  for (int i = 0; i < count; i++) {
    WH_CHECK(d_rows[i] && d_digests[i] && log_heights[i] >= 0 && log_heights[i] <= 30, "bad tree in the batch");
    WH_CHECK((reinterpret_cast<uintptr_t>(d_digests[i]) & 15) == 0, "digest arrays must be 16-byte aligned");
    max_lh = std::max(max_lh, (int)log_heights[i]);
  }
  // descriptors, then for every level the trees' first global nodes and the level's total
  const size_t stride = (size_t)count + 1;
  std::vector<wk::TreeDesc> desc((size_t)count);
  std::vector<unsigned long long> first(stride * (size_t)(max_lh + 1));
  std::vector<unsigned long long> totals((size_t)max_lh + 1);
  for (int l = 0; l <= max_lh; l++) {
    unsigned long long acc = 0;
    for (int i = 0; i < count; i++) {
      first[(size_t)l * stride + i] = acc;
      // level l of tree i is built by a level launch when it lies below the
      // tree's top (its levels above 2^kManyTopLevels nodes go to one CTA)
      if (l == 0 || log_heights[i] - l >= wk::kManyTopLevels) acc += 1ull << (log_heights[i] - l);
    }
    first[(size_t)l * stride + count] = acc;
    totals[l] = acc;
  }
  for (int i = 0; i < count; i++)
    desc[i] = wk::TreeDesc{d_rows[i], d_digests[i], first[i], log_heights[i], 0};
  const size_t desc_bytes = desc.size() * sizeof(wk::TreeDesc), first_bytes = first.size() * 8;
  WH_CHECK(desc_bytes + first_bytes + (size_t)count * 32 + 64 <= ctx->arena_bytes, "batch tables exceed the arena");
  uint8_t* base = static_cast<uint8_t*>(ctx->d_arena);
  auto* d_desc = reinterpret_cast<wk::TreeDesc*>(base);
  auto* d_first = reinterpret_cast<unsigned long long*>(base + desc_bytes);
  auto* d_roots = reinterpret_cast<uint32_t*>(base + desc_bytes + first_bytes);
  WH_TRY(wh::upload(ctx, d_desc, desc.data(), desc_bytes));
  WH_TRY(wh::upload(ctx, d_first, first.data(), first_bytes));
  {
    wh::StageTimer t(ctx, wh::kStLeaves);
    WH_TRY_CUDA(wk::merkle_many(d_desc, d_first, count, max_lh, totals.data(), row_words, leaf_hash, ctx->p16,
                                ctx->p24, reinterpret_cast<unsigned*>(ctx->d_words) + 13, d_roots, ctx->stream));
  }
  std::vector<uint32_t> r((size_t)count * 8);
  WH_TRY(wh::fetch(ctx, r.data(), d_roots, r.size() * 4));
  for (size_t k = 0; k < r.size(); k++) roots[k] = kb::from_mont(r[k]);
  return WHIR_OK;
}

int whir_keccak256(const uint8_t* data, size_t n, uint8_t* out32) {
  WH_CHECK((data || n == 0) && out32, "null argument");
  kk::K256 k;
  kk::k256_init(k);
  kk::k256_update(k, data, n);
  uint8_t out[32];
  kk::k256_final(k, out);
  memcpy(out32, out, 32);
  return WHIR_OK;
}

int whir_merkle_open(whir_ctx* ctx, const uint32_t* d_rows, const uint32_t* d_digests, int32_t log_height,
                     int32_t row_words, uint64_t index, uint32_t* row_out, uint32_t* path_out) {
  return whir_merkle_open_ex(ctx, d_rows, d_digests, log_height, row_words, WHIR_LEAF_P24, index, row_out, path_out);
}

int whir_merkle_open_ex(whir_ctx* ctx, const uint32_t* d_rows, const uint32_t* d_digests, int32_t log_height,
                        int32_t row_words, int32_t leaf_hash, uint64_t index, uint32_t* row_out,
                        uint32_t* path_out) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_rows && d_digests && row_out && path_out && index < (1ull << log_height) && row_words > 0 &&
               (leaf_hash == WHIR_LEAF_P24 || leaf_hash == WHIR_LEAF_P16 || leaf_hash == WHIR_LEAF_KECCAK),
           "bad opening arguments");
  uint64_t* d_idx = reinterpret_cast<uint64_t*>(ctx->d_arena);
  uint32_t* d_row = reinterpret_cast<uint32_t*>(d_idx + 8);
  uint32_t* d_path = d_row + row_words;
  WH_TRY(wh::upload(ctx, d_idx, &index, 8));
  WH_TRY_CUDA(wk::merkle_open(d_rows, d_digests, log_height, row_words, d_idx, 1, d_row, d_path, ctx->stream));
  std::vector<uint32_t> tmp((size_t)row_words + (size_t)log_height * 8);
  WH_TRY(wh::fetch(ctx, tmp.data(), d_row, tmp.size() * 4));
  for (int i = 0; i < row_words; i++) row_out[i] = kb::from_mont(tmp[i]);
  for (int i = 0; i < log_height * 8; i++) path_out[i] = wh::digest_word_out(leaf_hash, tmp[row_words + i]);
  return WHIR_OK;
}

int whir_eq_table(whir_ctx* ctx, const uint32_t* point, int32_t n, const uint32_t* scale, uint32_t* d_out) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK((point || n == 0) && scale && d_out && n >= 0 && n <= 30, "bad eq-table arguments");
  WH_CHECK(canon_ok(point, 4 * (size_t)n) && canon_ok(scale, 4), "value out of range");
  std::vector<ef> z(n);
  for (int i = 0; i < n; i++) z[i] = load_ef_canon(point + 4 * i);
  const int lo_bits = std::min(n, 10);
  ef* hi = reinterpret_cast<ef*>(ctx->d_arena);
  ef* lo = hi + ((size_t)1 << (n - lo_bits));
  WH_TRY(wh::split_eq_tables(ctx, z.data(), n, load_ef_canon(scale), lo_bits, hi, lo));
  WH_TRY_CUDA(wk::eq_outer(hi, lo, lo_bits, (size_t)1 << n, reinterpret_cast<ef*>(d_out), ctx->stream));
  return WHIR_OK;
}

static int eval_common(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* point, uint32_t* out,
                       int ext) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_evals && (point || n == 0) && out && n >= 0 && n <= 30, "bad evaluation arguments");
  WH_CHECK(canon_ok(point, 4 * (size_t)n), "value out of range");
  std::vector<ef> z(n > 0 ? n : 1);
  for (int i = 0; i < n; i++) z[i] = load_ef_canon(point + 4 * i);
  uint32_t posted = 0;
  WH_TRY(wh::dot_eq(ctx, d_evals, ext, 0, z.data(), n, &posted));
  ef r;
  WH_TRY(wh::fetch_posted(ctx, posted, &r, ctx->d_small, sizeof(ef)));
  WH_TRY(wh::check_dot(&r, sizeof(ef)));
  store_ef_canon(out, r);
  return WHIR_OK;
}

int whir_eval_base(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* point, uint32_t* out) {
  return eval_common(ctx, d_evals, n, point, out, 0);
}
int whir_eval_ext(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* point, uint32_t* out) {
  return eval_common(ctx, d_evals, n, point, out, 1);
}

int whir_fold_ext(whir_ctx* ctx, uint32_t* d_evals, int32_t n, const uint32_t* r) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_evals && r && n >= 1 && n <= 30 && canon_ok(r, 4), "bad fold arguments");
  WH_TRY(wh::run_fold(ctx, reinterpret_cast<ef*>(d_evals), nullptr, (size_t)1 << (n - 1), load_ef_canon(r)));
  return WHIR_OK;
}

int whir_fold_base(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* r, uint32_t* d_out) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_evals && d_out && r && n >= 1 && n <= 30 && canon_ok(r, 4), "bad fold arguments");
  WH_TRY_CUDA(wk::fold_base(d_evals, (size_t)1 << (n - 1), load_ef_canon(r), reinterpret_cast<ef*>(d_out), ctx->stream));
  return WHIR_OK;
}



int whir_fold_multi_base(whir_ctx* ctx, const uint32_t* d_evals, int32_t n, const uint32_t* rs, int32_t k,
                         uint32_t* d_out) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_evals && d_out && (rs || k == 0) && k >= 0 && k <= 6 && k <= n && n <= 30 && canon_ok(rs, 4 * (size_t)k),
           "bad fold arguments");
  std::vector<ef> r(k > 0 ? k : 1);
  for (int i = 0; i < k; i++) r[i] = load_ef_canon(rs + 4 * i);
  wk::EqSmall e = wh::eq_small_host(r.data(), k);
  WH_TRY_CUDA(wk::fold_multi_base(d_evals, k, (size_t)1 << (n - k), e, reinterpret_cast<ef*>(d_out), ctx->stream));
  return WHIR_OK;
}

int whir_sumcheck_coeffs(whir_ctx* ctx, const uint32_t* d_f, const uint32_t* d_w, int32_t n, uint32_t* c0,
                         uint32_t* c2) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_f && d_w && c0 && c2 && n >= 1 && n <= 30, "bad sumcheck arguments");
  WH_TRY_CUDA(wk::sumcheck_coeffs(reinterpret_cast<const ef*>(d_f), reinterpret_cast<const ef*>(d_w),
                                  (size_t)1 << (n - 1), ctx->d_partials, ctx->d_small, ctx->stream));
  ef r[2];
  WH_TRY(wh::fetch(ctx, r, ctx->d_small, sizeof(r)));
  store_ef_canon(c0, r[0]);
  store_ef_canon(c2, r[1]);
  return WHIR_OK;
}



int whir_sumcheck_coeffs_shaped(whir_ctx* ctx, const uint32_t* d_f, const uint32_t* d_w, int32_t n,
                                int32_t max_blocks, uint32_t* c0, uint32_t* c2) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_f && d_w && c0 && c2 && n >= 1 && n <= 30, "bad sumcheck arguments");
  // the partial sums take 2 * blocks of the context's 8192-entry buffer
  WH_CHECK(max_blocks >= 1 && max_blocks <= 4096, "max_blocks must be in [1, 4096]");
  WH_TRY_CUDA(wk::sumcheck_coeffs_capped(reinterpret_cast<const ef*>(d_f), reinterpret_cast<const ef*>(d_w),
                                         (size_t)1 << (n - 1), ctx->d_partials, (unsigned)max_blocks,
                                         ctx->d_small, ctx->stream));
  ef r[2];
  WH_TRY(wh::fetch(ctx, r, ctx->d_small, sizeof(r)));
  store_ef_canon(c0, r[0]);
  store_ef_canon(c2, r[1]);
  return WHIR_OK;
}

int whir_combine_eq(whir_ctx* ctx, uint32_t* d_w, int32_t n, const uint32_t* points, int32_t m,
                    const uint32_t* gamma_pows) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_w && n >= 0 && n <= 30 && m >= 0 && (m == 0 || (points && gamma_pows)), "bad combine arguments");
  WH_CHECK(canon_ok(points, 4 * (size_t)n * m) && canon_ok(gamma_pows, 4 * (size_t)m), "value out of range");
  std::vector<std::vector<ef>> pts(m, std::vector<ef>(n));
  std::vector<ef> sc(m);
  for (int c = 0; c < m; c++) {
    for (int i = 0; i < n; i++) pts[c][i] = load_ef_canon(points + 4 * ((size_t)c * n + i));
    sc[c] = load_ef_canon(gamma_pows + 4 * c);
  }
  return wh::add_eq_points(ctx, reinterpret_cast<ef*>(d_w), n, pts, sc, 1);
}

int whir_combine_select(whir_ctx* ctx, uint32_t* d_w, int32_t n, const uint32_t* vars, int32_t m,
                        const uint32_t* gamma_pows) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_w && n >= 0 && n <= 30 && m >= 0 && (m == 0 || (vars && gamma_pows)), "bad combine arguments");
  WH_CHECK(canon_ok(vars, (size_t)m) && canon_ok(gamma_pows, 4 * (size_t)m), "value out of range");
  std::vector<uint32_t> v(m);
  std::vector<ef> g(m);
  for (int j = 0; j < m; j++) {
    v[j] = kb::to_mont(vars[j]);
    g[j] = load_ef_canon(gamma_pows + 4 * j);
  }
  return wh::add_select_vars(ctx, reinterpret_cast<ef*>(d_w), n, v, g);
}

int whir_svo_partial_evals(whir_ctx* ctx, const uint32_t* d_poly, int32_t n, int32_t l, const uint32_t* point,
                           uint32_t* out, uint32_t* eval_out) {
  WH_TRY(check_gpu(ctx));
  WH_CHECK(d_poly && point && out && l >= 0 && l <= 8 && l <= n && n <= 30, "bad partial-evaluation arguments");
  WH_CHECK(canon_ok(point, 4 * (size_t)n), "value out of range");
  std::vector<ef> z(n > 0 ? n : 1);
  for (int i = 0; i < n; i++) z[i] = load_ef_canon(point + 4 * i);
  uint32_t posted = 0;
  WH_TRY(wh::dot_eq(ctx, d_poly, 0, l, z.data() + l, n - l, &posted));
  std::vector<ef> g((size_t)1 << l);
  WH_TRY(wh::fetch_posted(ctx, posted, g.data(), ctx->d_small, g.size() * sizeof(ef)));
  WH_TRY(wh::check_dot(g.data(), g.size() * sizeof(ef)));
  ef eval = kb::ef_zero();
  const std::vector<ef> e = wh::eq_host(z.data(), l);  // 2^l <= 256 entries
  for (size_t y = 0; y < g.size(); y++) {
    store_ef_canon(out + 4 * y, g[y]);
    eval = kb::ef_add(eval, kb::ef_mul(e[y], g[y]));
  }
  if (eval_out) store_ef_canon(eval_out, eval);
  return WHIR_OK;
}

}  // extern "C"
