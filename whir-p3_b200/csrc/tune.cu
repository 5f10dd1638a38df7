// Launch-shape tuner. The first time a shape runs, every candidate launch
// shape is timed with CUDA events on the calling context's stream and the
// fastest is cached for the process:
//   DFT:     four-step split (or the one-pass kernel), tile and CTA size of
//            each pass, timed pass by pass;
//   Merkle:  the leaf-digest kernel's batch width (threads per CTA and CTAs
//            per SM), the same for the two-level compression kernel, and
//            the kernel that finishes the top of the tree;
//   fold:    threads per CTA and CTAs per SM of the in-place fold.
// All candidates compute the same values (they only tile the same exact
// arithmetic differently), so tuning changes timing, never results.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <vector>

#include "host.h"

using kb::ef;

namespace {

struct Key {
  int kind, dev, a, b, c, d;
  bool operator<(const Key& o) const {
    return std::tie(kind, dev, a, b, c, d) < std::tie(o.kind, o.dev, o.a, o.b, o.c, o.d);
  }
};

std::mutex g_mu;  // guards g_table
std::map<Key, whir_tune_entry> g_table;
std::mutex g_session;  // one tuning session at a time in the process
std::atomic<int> g_mode{1};

bool lookup(const Key& k, whir_tune_entry* e) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_table.find(k);
  if (it == g_table.end()) return false;
  *e = it->second;
  return true;
}

void store(const Key& k, const whir_tune_entry& e) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.emplace(k, e);
}

whir_tune_entry entry_for(const Key& k) {
  whir_tune_entry e;
  memset(&e, 0, sizeof(e));
  e.kind = k.kind;
  e.device = k.dev;
  e.key[0] = k.a;
  e.key[1] = k.b;
  e.key[2] = k.c;
  e.key[3] = k.d;
  return e;
}

constexpr float kNever = 3.0e38f;
constexpr int kReps = 2;

// Times launch(i) for i < count, `reps` rounds, on the context's stream.
// ms[i] is the fastest round, or kNever when the launch failed.
int time_all(whir_ctx* ctx, int count, int reps, const std::function<cudaError_t(int)>& launch,
             std::vector<float>& ms) {
  ms.assign(count, kNever);
  std::vector<cudaEvent_t> ev((size_t)2 * count * reps, nullptr);
  for (cudaEvent_t& e : ev) WH_TRY_CUDA(cudaEventCreate(&e));
  std::vector<char> ok(count, 1);
  for (int r = 0; r < reps; r++)
    for (int i = 0; i < count; i++) {
      if (!ok[i]) continue;
      const size_t at = ((size_t)r * count + i) * 2;
      cudaEventRecord(ev[at], ctx->stream);
      if (launch(i) != cudaSuccess) {
        cudaGetLastError();
        ok[i] = 0;
      }
      cudaEventRecord(ev[at + 1], ctx->stream);
    }
  const cudaError_t se = cudaStreamSynchronize(ctx->stream);
  if (se == cudaSuccess)
    for (int r = 0; r < reps; r++)
      for (int i = 0; i < count; i++) {
        if (!ok[i]) continue;
        const size_t at = ((size_t)r * count + i) * 2;
        float t = 0.f;
        if (cudaEventElapsedTime(&t, ev[at], ev[at + 1]) == cudaSuccess) ms[i] = std::min(ms[i], t);
      }
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  WH_TRY_CUDA(se);
  return WHIR_OK;
}

wk::DftPlan plan_of(const whir_tune_entry& e) {
  return wk::DftPlan{e.choice[0], e.choice[1], e.choice[2], e.choice[3], e.choice[4], e.choice[5], e.choice[6]};
}

// Times every candidate plan of a DFT shape: one-pass plans whole, four-step
// plans pass by pass (each distinct pass variant once). The plan joins, for
// the best split, its fastest pass 1 and fastest pass 2.
int tune_dft(whir_ctx* ctx, const Key& k, const uint32_t* in, uint32_t* out, uint32_t* scratch, int log_chunk,
             int log_w, int log_blowup, int lanes, const wk::DftTables& t, wk::DftPlan* plan) {
  wk::DftPlan cand[256];
  int nc = 0;
  wk::dft_candidates(log_chunk, log_w, log_blowup, lanes, cand, &nc, 256);
  struct Run {
    wk::DftPlan p;
    int passes;
  };
  std::vector<Run> runs;
  std::set<std::tuple<int, int, int, int, int>> seen;
  for (int i = 0; i < nc; i++) {
    const wk::DftPlan& p = cand[i];
    if (p.log_h2 == 0) {
      if (seen.insert(std::make_tuple(0, p.log_t1, p.threads1, 0, 0)).second) runs.push_back({p, 3});
      continue;
    }
    if (seen.insert(std::make_tuple(p.log_h2, p.log_t1, p.threads1, p.reg1, 1)).second) runs.push_back({p, 1});
    if (seen.insert(std::make_tuple(p.log_h2, p.log_t2, p.threads2, p.reg2, 2)).second) runs.push_back({p, 2});
  }
  std::vector<float> ms;
  WH_TRY(time_all(ctx, (int)runs.size(), kReps,
                  [&](int i) {
                    return wk::dft_batch(in, out, scratch, log_chunk, log_w, log_blowup, lanes, t, runs[i].p,
                                         runs[i].passes, ctx->stream);
                  },
                  ms));
  const wk::DftPlan def = *plan;
  float best = kNever, t_def = 0.f;
  std::map<int, std::pair<int, int>> split;  // log_h2 -> (fastest pass-1 run, fastest pass-2 run)
  for (int i = 0; i < (int)runs.size(); i++) {
    const Run& r = runs[i];
    if (r.passes == 3) {
      if (ms[i] < best) {
        best = ms[i];
        *plan = r.p;
      }
      if (def.log_h2 == 0 && r.p.log_t1 == def.log_t1 && r.p.threads1 == def.threads1) t_def = ms[i];
      continue;
    }
    auto& s = split.emplace(r.p.log_h2, std::make_pair(-1, -1)).first->second;
    int& slot = r.passes == 1 ? s.first : s.second;
    if (slot < 0 || ms[i] < ms[slot]) slot = i;
    if (def.log_h2 == r.p.log_h2) {
      if (r.passes == 1 && r.p.log_t1 == def.log_t1 && r.p.threads1 == def.threads1 && r.p.reg1 == def.reg1)
        t_def += ms[i];
      if (r.passes == 2 && r.p.log_t2 == def.log_t2 && r.p.threads2 == def.threads2 && r.p.reg2 == def.reg2)
        t_def += ms[i];
    }
  }
  for (const auto& kv : split) {
    const int a = kv.second.first, b = kv.second.second;
    if (a < 0 || b < 0 || ms[a] >= kNever || ms[b] >= kNever) continue;
    const float tot = ms[a] + ms[b];
    if (tot < best) {
      best = tot;
      *plan = wk::DftPlan{kv.first,         runs[a].p.log_t1, runs[a].p.threads1, runs[b].p.log_t2,
                          runs[b].p.threads2, runs[a].p.reg1,   runs[b].p.reg2};
    }
  }
  if (best >= kNever) *plan = def;
  whir_tune_entry e = entry_for(k);
  e.choice[0] = plan->log_h2;
  e.choice[1] = plan->log_t1;
  e.choice[2] = plan->threads1;
  e.choice[3] = plan->log_t2;
  e.choice[4] = plan->threads2;
  e.choice[5] = plan->reg1;
  e.choice[6] = plan->reg2;
  e.candidates = (int)runs.size();
  e.ms_default = t_def;
  e.ms_best = best < kNever ? best : t_def;
  store(k, e);
  return WHIR_OK;
}

const wk::Shape kLeafShapes[] = {{128, 0, 0},  {128, 8, 0}, {128, 16, 0}, {256, 0, 0}, {256, 4, 0}, {256, 8, 0},
                                 {256, 16, 0}, {512, 0, 0}, {512, 2, 0},  {512, 4, 0}, {512, 8, 0}};
// variant: bit 0 the top kernel (cooperative subtrees / one CTA), bit 1 the
// two-level kernel's permutations one after the other instead of together,
// bit 2 the last two-level step with four-lane cooperative permutations
const wk::Shape kNodeShapes[] = {{128, 0, 0}, {128, 8, 0}, {128, 16, 0}, {256, 0, 0}, {256, 8, 0}, {256, 16, 0},
                                 {128, 0, 1}, {128, 8, 1}, {128, 16, 1}, {256, 0, 1}, {256, 8, 1}, {256, 16, 1},
                                 {128, 0, 2}, {128, 16, 2}, {256, 0, 2}, {256, 16, 2}, {128, 0, 3}, {256, 0, 3},
                                 {128, 0, 4}, {256, 0, 4}, {256, 16, 4}, {128, 0, 5}, {256, 0, 5}};
const wk::Shape kFoldShapes[] = {{128, 0, 0},  {128, 16, 0}, {256, 0, 0}, {256, 4, 0}, {256, 8, 0},
                                 {256, 16, 0}, {512, 0, 0},  {512, 2, 0}, {512, 4, 0}, {512, 8, 0}};

bool same(const wk::Shape& a, const wk::Shape& b) {
  return a.threads == b.threads && a.per_sm == b.per_sm && a.variant == b.variant;
}

// Looks up or tunes the shape for `k` among `shapes`; launch(s) runs shape s.
template <size_t N>
int pick_shape(whir_ctx* ctx, const Key& k, const wk::Shape (&shapes)[N], const wk::Shape& def,
               const std::function<cudaError_t(const wk::Shape&)>& launch, wk::Shape* out) {
  whir_tune_entry e;
  *out = def;
  if (lookup(k, &e)) {
    *out = wk::Shape{e.choice[0], e.choice[1], e.choice[2]};
    return WHIR_OK;
  }
  if (g_mode.load() != 1) return WHIR_OK;
  std::lock_guard<std::mutex> session(g_session);
  if (lookup(k, &e)) {
    *out = wk::Shape{e.choice[0], e.choice[1], e.choice[2]};
    return WHIR_OK;
  }
  std::vector<float> ms;
  WH_TRY(time_all(ctx, (int)N, kReps, [&](int i) { return launch(shapes[i]); }, ms));
  int bi = -1;
  float t_def = 0.f;
  for (int i = 0; i < (int)N; i++) {
    if (bi < 0 || ms[i] < ms[bi]) bi = i;
    if (same(shapes[i], def)) t_def = ms[i];
  }
  const bool found = bi >= 0 && ms[bi] < kNever;
  if (found) *out = shapes[bi];
  e = entry_for(k);
  e.choice[0] = out->threads;
  e.choice[1] = out->per_sm;
  e.choice[2] = out->variant;
  e.candidates = (int)N;
  e.ms_default = t_def;
  e.ms_best = found ? ms[bi] : t_def;
  store(k, e);
  return WHIR_OK;
}

}  // namespace

namespace wh {

int run_dft(whir_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t* scratch, int log_chunk, int log_w,
            int log_blowup, int lanes, const wk::DftTables& t) {
  const Key k{WHIR_TUNE_DFT, ctx->device, log_chunk, log_w, log_blowup, lanes};
  whir_tune_entry e;
  wk::DftPlan plan = wk::dft_default_plan(log_chunk, log_w, log_blowup, lanes);
  if (lookup(k, &e)) {
    plan = plan_of(e);
  } else if (g_mode.load() == 1 && wk::dft_plan_ok(plan, log_chunk, log_w, log_blowup, lanes)) {
    std::lock_guard<std::mutex> session(g_session);
    if (lookup(k, &e))
      plan = plan_of(e);
    else
      WH_TRY(tune_dft(ctx, k, in, out, scratch, log_chunk, log_w, log_blowup, lanes, t, &plan));
  }
  const cudaError_t ce =
      wk::dft_batch(in, out, scratch, log_chunk, log_w, log_blowup, lanes, t, plan, 3, ctx->stream);
  if (ce == cudaErrorInvalidValue) return wh::set_error("unsupported DFT shape"), WHIR_ERR_INVALID;
  WH_TRY_CUDA(ce);
  return WHIR_OK;
}

bool dft_plan_known(const whir_ctx* ctx, int log_chunk, int log_w, int log_blowup, int lanes, wk::DftPlan* plan) {
  const Key k{WHIR_TUNE_DFT, ctx->device, log_chunk, log_w, log_blowup, lanes};
  whir_tune_entry e;
  *plan = wk::dft_default_plan(log_chunk, log_w, log_blowup, lanes);
  if (lookup(k, &e)) {
    *plan = plan_of(e);
    return true;
  }
  // mode 1 would tune this shape on its first run; other modes use the default
  return g_mode.load() != 1 || !wk::dft_plan_ok(*plan, log_chunk, log_w, log_blowup, lanes);
}

int run_merkle_leaves(whir_ctx* ctx, const uint32_t* rows, int log_h, int row_words, int leaf_hash,
                      uint32_t* digests) {
  if (leaf_hash == WHIR_LEAF_KECCAK) {
    WH_TRY_CUDA(wk::keccak_leaves(rows, log_h, row_words, digests, ctx->stream));
    return WHIR_OK;
  }
  wk::Shape sh = wk::merkle_leaf_default();
  if (((size_t)1 << log_h) >= (size_t)wk::kMerkleLevelPairMin) {
    const Key k{WHIR_TUNE_MERKLE_LEAVES, ctx->device, log_h, row_words, leaf_hash, 0};
    WH_TRY(pick_shape(ctx, k, kLeafShapes, sh,
                      [&](const wk::Shape& s) {
                        return wk::merkle_leaves(rows, log_h, row_words, leaf_hash, digests, ctx->p16, ctx->p24, s,
                                                 ctx->stream);
                      },
                      &sh));
  }
  WH_TRY_CUDA(wk::merkle_leaves(rows, log_h, row_words, leaf_hash, digests, ctx->p16, ctx->p24, sh, ctx->stream));
  return WHIR_OK;
}

int run_merkle_upper(whir_ctx* ctx, int log_h, int leaf_hash, uint32_t* digests, uint32_t* posted_seq) {
  if (leaf_hash == WHIR_LEAF_KECCAK) {
    const uint32_t seq = posted_seq && ctx->h_mail ? mail_next(ctx) : 0u;
    int posted = 0;
    WH_TRY_CUDA(wk::keccak_upper(log_h, digests, seq ? ctx->d_mail : nullptr, seq, &posted, ctx->stream));
    if (posted_seq) *posted_seq = posted ? seq : 0u;
    return WHIR_OK;
  }
  unsigned* counter = reinterpret_cast<unsigned*>(ctx->d_words) + 10;
  wk::Shape sh = wk::merkle_node_default();
  // the two-level kernel runs only on levels wider than 2^15 nodes
  if (log_h > 15) {
    const Key k{WHIR_TUNE_MERKLE_NODES, ctx->device, log_h, 0, 0, 0};
    WH_TRY(pick_shape(ctx, k, kNodeShapes, sh,
                      [&](const wk::Shape& s) {
                        return wk::merkle_upper(log_h, digests, ctx->p16, s, counter, nullptr, 0u, nullptr,
                                                ctx->stream);
                      },
                      &sh));
  }
  const uint32_t seq = posted_seq && ctx->h_mail ? mail_next(ctx) : 0u;
  int posted = 0;
  WH_TRY_CUDA(wk::merkle_upper(log_h, digests, ctx->p16, sh, counter, seq ? ctx->d_mail : nullptr, seq, &posted,
                               ctx->stream));
  if (posted_seq) *posted_seq = posted ? seq : 0u;
  return WHIR_OK;
}

int run_fold(whir_ctx* ctx, ef* a, ef* b, size_t half, const ef& r) {
  wk::Shape sh = wk::fold_default();
  int lg = 0;
  while (((size_t)1 << lg) < half) lg++;
  // small folds are launch-latency bound; tune from 2^14 pairs up, on scratch
  // arrays (the fold is in place, so it cannot be repeated on the live data)
  if (lg >= 14) {
    const Key k{WHIR_TUNE_FOLD, ctx->device, lg, b ? 2 : 1, 0, 0};
    whir_tune_entry e;
    if (lookup(k, &e)) {
      sh = wk::Shape{e.choice[0], e.choice[1], e.choice[2]};
    } else if (g_mode.load() == 1) {
      const size_t n = 2 * half * (b ? 2 : 1);
      ef* tmp = nullptr;
      WH_TRY_CUDA(wh::ctx_malloc(ctx, &tmp, n * sizeof(ef)));
      cudaMemsetAsync(tmp, 0, n * sizeof(ef), ctx->stream);
      ef* ta = tmp;
      ef* tb = b ? tmp + 2 * half : nullptr;
      const int s = pick_shape(ctx, k, kFoldShapes, sh,
                               [&](const wk::Shape& x) { return wk::fold_ext(ta, tb, half, r, x, ctx->stream); }, &sh);
      cudaFreeAsync(tmp, ctx->stream);
      WH_TRY(s);
    }
  }
  WH_TRY_CUDA(wk::fold_ext(a, b, half, r, sh, ctx->stream));
  return WHIR_OK;
}

}  // namespace wh

namespace {
int tune_check_gpu(const whir_ctx* ctx) {
  WH_CHECK(ctx, "null context");
  if (ctx->device < 0) {
    wh::set_error("host-only context (device -1) cannot run device work");
    return WHIR_ERR_NO_DEVICE;
  }
  cudaSetDevice(ctx->device);
  return WHIR_OK;
}
}  // namespace

extern "C" {

int whir_tune_set_mode(int32_t mode) {
  WH_CHECK(mode == 0 || mode == 1, "tune mode must be 0 (fixed shapes) or 1 (tune on first use)");
  g_mode.store(mode);
  return WHIR_OK;
}

int whir_tune_get_mode(void) { return g_mode.load(); }

int whir_tune_entries(whir_tune_entry* out, int32_t cap) {
  WH_CHECK(cap >= 0 && (out || cap == 0), "bad arguments");
  std::lock_guard<std::mutex> lk(g_mu);
  int n = 0;
  for (const auto& kv : g_table) {
    if (n < cap) out[n] = kv.second;
    n++;
  }
  return n;
}

int whir_tune_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
  return WHIR_OK;
}

int whir_dft_plans(int32_t log_chunk, int32_t log_width, int32_t log_blowup, int32_t ext, int32_t* plans,
                   int32_t cap) {
  WH_CHECK(cap >= 0 && (plans || cap == 0), "bad arguments");
  wk::DftPlan cand[256];
  int nc = 0;
  wk::dft_candidates(log_chunk, log_width, log_blowup, ext ? 4 : 1, cand, &nc, 256);
  for (int i = 0; i < nc && i < cap; i++) {
    plans[7 * i] = cand[i].log_h2;
    plans[7 * i + 1] = cand[i].log_t1;
    plans[7 * i + 2] = cand[i].threads1;
    plans[7 * i + 3] = cand[i].log_t2;
    plans[7 * i + 4] = cand[i].threads2;
    plans[7 * i + 5] = cand[i].reg1;
    plans[7 * i + 6] = cand[i].reg2;
  }
  return nc;
}

int whir_dft_batch_plan(whir_ctx* ctx, const uint32_t* d_chunks, int32_t log_chunk, int32_t log_width,
                        int32_t log_blowup, int32_t ext, const int32_t* plan, uint32_t* d_out) {
  WH_TRY(tune_check_gpu(ctx));
  WH_CHECK(d_chunks && d_out && plan, "null argument");
  const int lanes = ext ? 4 : 1;
  const wk::DftPlan p{plan[0], plan[1], plan[2], plan[3], plan[4], plan[5], plan[6]};
  WH_CHECK(wk::dft_plan_ok(p, log_chunk, log_width, log_blowup, lanes), "invalid DFT plan for this shape");
  const int log_h = log_chunk + log_blowup;
  wk::DftTables t;
  WH_TRY(wh::ensure_dft_tables(ctx, log_h, &t));
  uint32_t* scratch = nullptr;
  if (p.log_h2 != 0)
    WH_TRY_CUDA(wh::ctx_malloc(ctx, &scratch, ((size_t)1 << (log_h + log_width)) * 4 * lanes));
  const cudaError_t e =
      wk::dft_batch(d_chunks, d_out, scratch, log_chunk, log_width, log_blowup, lanes, t, p, 3, ctx->stream);
  if (scratch) cudaFreeAsync(scratch, ctx->stream);
  WH_TRY_CUDA(e);
  return WHIR_OK;
}

int whir_merkle_commit_shaped(whir_ctx* ctx, const uint32_t* d_rows, int32_t log_height, int32_t row_words,
                              int32_t leaf_hash, const int32_t* shape, uint32_t* d_digests, uint32_t* root) {
  WH_TRY(tune_check_gpu(ctx));
  WH_CHECK(d_rows && d_digests && shape && log_height >= 0 && log_height <= 30 && row_words > 0 &&
               (leaf_hash == 0 || leaf_hash == 1),
           "bad Merkle arguments");
  const wk::Shape leaf{shape[0], shape[1], 0}, node{shape[2], shape[3], shape[4]};
  cudaError_t e = wk::merkle_leaves(d_rows, log_height, row_words, leaf_hash, d_digests, ctx->p16, ctx->p24, leaf,
                                    ctx->stream);
  if (e == cudaErrorInvalidValue) return wh::set_error("invalid Merkle shape"), WHIR_ERR_INVALID;
  WH_TRY_CUDA(e);
  e = wk::merkle_upper(log_height, d_digests, ctx->p16, node, reinterpret_cast<unsigned*>(ctx->d_words) + 10,
                      nullptr, 0u, nullptr, ctx->stream);
  if (e == cudaErrorInvalidValue) return wh::set_error("invalid Merkle shape"), WHIR_ERR_INVALID;
  WH_TRY_CUDA(e);
  if (root) {
    const size_t h = (size_t)1 << log_height;
    uint32_t r[8];
    WH_TRY(wh::fetch(ctx, r, d_digests + (2 * h - 2) * 8, 32));
    for (int i = 0; i < 8; i++) root[i] = kb::from_mont(r[i]);
  }
  return WHIR_OK;
}

int whir_fold_ext_shaped(whir_ctx* ctx, uint32_t* d_evals, int32_t n, const uint32_t* r, const int32_t* shape) {
  WH_TRY(tune_check_gpu(ctx));
  WH_CHECK(d_evals && r && shape && n >= 1 && n <= 30, "bad fold arguments");
  for (int i = 0; i < 4; i++) WH_CHECK(r[i] < kb::P, "non-canonical field element");
  const ef rm{{kb::to_mont(r[0]), kb::to_mont(r[1]), kb::to_mont(r[2]), kb::to_mont(r[3])}};
  const cudaError_t e = wk::fold_ext(reinterpret_cast<ef*>(d_evals), nullptr, (size_t)1 << (n - 1), rm,
                                     wk::Shape{shape[0], shape[1], 0}, ctx->stream);
  if (e == cudaErrorInvalidValue) return wh::set_error("invalid fold shape"), WHIR_ERR_INVALID;
  WH_TRY_CUDA(e);
  return WHIR_OK;
}

}  // extern "C"
