// Batched and served proving: a pool of worker threads, each owning one
// context (one CUDA stream) on the same device, takes commit+prove jobs from
// a queue. A job is admitted only when the device memory the pool would then
// hold fits the HBM budget, so requests that arrive while others are running
// start as soon as a worker and memory free up, and their kernels overlap on
// the device with the proofs already in flight. Every job runs the same code
// path as whir_commit_and_prove, so each proof is identical to the one the
// job would produce alone.
//
// Memory accounting. Each worker holds its context's fixed allocations
// (tables, scratch, arena) and its stream-ordered pool, which keeps what it
// has reserved between jobs. The pools reserve memory in chunks (32 MiB on
// B200, measured), so a job is charged its footprint plus one chunk. A worker
// counts as max(pool reservation, charge of its running job); admitting job j
// on worker w needs
//   fixed(all workers) + sum over other workers + max(reserved(w), charge(j)) <= budget.
// When that fails, idle workers' pools are trimmed (their cached blocks go
// back to the driver) and the check is repeated. The first queued job that
// fits is taken; a job passed over more than twice the worker count is
// waited for (no job behind it starts first). With nothing running, the
// oldest job starts even if it exceeds the budget on its own.
#include <stdio.h>

#include <chrono>
#include <condition_variable>
#include <algorithm>
#include <deque>
#include <mutex>
#include <thread>

#include "host.h"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

int ilog2u(uint64_t v) {
  int r = -1;
  while (v) {
    r++;
    v >>= 1;
  }
  return r;
}

}  // namespace

struct whir_batch {
  int device = 0;
  size_t budget = 0;
  size_t fixed = 0;                 // fixed device bytes of all worker contexts
  std::vector<size_t> running_fp;   // per worker: charge of its running job, 0 when idle
  uint32_t head_skips = 0;          // times the oldest job was passed over
  std::vector<whir_ctx*> ctxs;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work;  // workers wait for admissible work
  std::condition_variable cv_done;  // submitters wait for completions
  std::deque<whir_job*> queue;
  size_t pending = 0;  // submitted and not finished
  bool stop = false;
};

namespace wh {

// Peak device bytes of one commit+prove: polynomial, commitment tree and
// codeword, the two sumcheck arrays, and the largest round's pair of trees plus
// its DFT scratch. Context arenas are counted per worker, not per job.
size_t footprint(const whir_config& c, int poly_on_device) {
  const int n = c.num_variables, k0 = c.folding_factor_0;
  const uint64_t log_h0 = (uint64_t)(n + c.starting_log_inv_rate - k0);
  size_t poly = poly_on_device ? 0 : ((size_t)4 << n);
  size_t commit_rows = (size_t)4 << (log_h0 + k0);
  size_t commit_dig = ((size_t)2 << log_h0) * 32;
  size_t fw = 2 * ((size_t)16 << (n - k0));
  size_t peak_round = commit_rows;  // the commit DFT scratch
  size_t prev_tree = 0;
  int nv = n - k0;
  for (int r = 0; r < c.n_rounds; r++) {
    const whir_round_config& rc = c.rounds[r];
    const int ffn = ff_at(c, r + 1);
    const uint64_t new_dom = rc.domain_size >> rsr_at(c, r);
    const int log_h = ilog2u(new_dom) - ffn;
    const size_t rows = ((size_t)16 << ffn) << log_h;
    const size_t dig = ((size_t)2 << log_h) * 32;
    const size_t here = prev_tree + rows + dig + rows;  // previous tree, new tree, DFT scratch
    if (here > peak_round) peak_round = here;
    prev_tree = rows + dig;
    nv -= ffn;
  }
  return poly + commit_rows + commit_dig + fw + peak_round;
}

}  // namespace wh

namespace {

void run_job(whir_ctx* ctx, whir_job* j) {
  j->t_start_ms = now_ms();
  size_t words = 0;
  j->status = whir_commit_and_prove(ctx, &j->params, j->n, j->poly, j->poly_on_device, j->points, j->num_points,
                                    j->evals_out, j->proof_out, j->proof_cap, &words, j->checkpoint);
  j->proof_words = words;
  if (j->status != WHIR_OK) {
    snprintf(j->error, sizeof(j->error), "%s", whir_last_error());
  }
  j->t_done_ms = now_ms();
}

// the pool's reservation granule: a job may grow its worker's pool by up to
// one chunk beyond its footprint
constexpr size_t kPoolChunk = (size_t)32 << 20;
size_t charge(const whir_job* j) { return (size_t)j->footprint_bytes + kPoolChunk; }

uint64_t reserved(whir_ctx* c) {
  uint64_t v = 0;
  if (c->pool && cudaMemPoolGetAttribute(c->pool, cudaMemPoolAttrReservedMemCurrent, &v) != cudaSuccess) v = 0;
  return v;
}

// Bytes the pool holds apart from worker `idx`'s pool reservation; called
// with b->mu held.
size_t others(whir_batch* b, int idx) {
  size_t total = b->fixed;
  for (size_t w = 0; w < b->ctxs.size(); w++)
    if ((int)w != idx) total += std::max((size_t)reserved(b->ctxs[w]), b->running_fp[w]);
  return total;
}

whir_job* take(whir_batch* b, size_t i) {
  whir_job* j = b->queue[i];
  b->queue.erase(b->queue.begin() + (std::ptrdiff_t)i);
  b->head_skips = i == 0 ? 0 : b->head_skips + 1;
  return j;
}

// The job worker `idx` takes next, or null; called with b->mu held.
whir_job* pick(whir_batch* b, int idx) {
  if (b->queue.empty()) return nullptr;
  bool any_running = false;
  for (size_t v : b->running_fp) any_running |= v != 0;
  const bool head_only = b->head_skips > 2 * b->ctxs.size();
  for (int attempt = 0; attempt < 2; attempt++) {
    const size_t base = others(b, idx), mine = (size_t)reserved(b->ctxs[idx]);
    for (size_t i = 0; i < b->queue.size() && (i == 0 || !head_only); i++)
      if (base + std::max(mine, charge(b->queue[i])) <= b->budget) return take(b, i);
    if (attempt == 0) {
      // make room: idle workers (this one included) hand their cached
      // blocks back to the driver
      for (size_t w = 0; w < b->ctxs.size(); w++)
        if (b->running_fp[w] == 0 && b->ctxs[w]->pool) cudaMemPoolTrimTo(b->ctxs[w]->pool, 0);
    }
  }
  // nothing fits and nothing runs: the oldest job runs alone
  return any_running ? nullptr : take(b, 0);
}

void worker(whir_batch* b, int idx) {
  whir_ctx* ctx = b->ctxs[idx];
  // a worker whose thread cannot select the device fails every job it takes
  const cudaError_t dev_err = cudaSetDevice(b->device);
  for (;;) {
    whir_job* j = nullptr;
    {
      std::unique_lock<std::mutex> lk(b->mu);
      for (;;) {
        if (b->stop && b->queue.empty()) return;
        j = pick(b, idx);
        if (j) break;
        b->cv_work.wait(lk);
      }
      b->running_fp[idx] = charge(j);
    }
    if (dev_err == cudaSuccess) {
      run_job(ctx, j);
    } else {
      j->t_start_ms = j->t_done_ms = now_ms();
      j->status = WHIR_ERR_CUDA;
      snprintf(j->error, sizeof(j->error), "cudaSetDevice failed on the worker thread: %s",
               cudaGetErrorString(dev_err));
    }
    {
      std::lock_guard<std::mutex> lk(b->mu);
      b->running_fp[idx] = 0;
      j->done = 1;
      b->pending--;
    }
    b->cv_work.notify_all();
    b->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

int whir_job_footprint(const whir_protocol_params* params, int32_t n, int32_t poly_on_device, uint64_t* bytes) {
  WH_CHECK(params && bytes, "null argument");
  whir_config c;
  WH_TRY(wh::config_new(*params, n, &c));
  *bytes = wh::footprint(c, poly_on_device);
  return WHIR_OK;
}

int whir_batch_create(int32_t device, int32_t workers, const whir_poseidon2_params* p16,
                      const whir_poseidon2_params* p24, uint64_t hbm_budget_bytes, whir_batch** out) {
  WH_CHECK(out && workers >= 1 && workers <= 256 && hbm_budget_bytes > 0, "bad batch arguments");
  *out = nullptr;
  whir_batch* b = new whir_batch();
  b->device = device;
  b->budget = hbm_budget_bytes;
  for (int i = 0; i < workers; i++) {
    whir_ctx* c = nullptr;
    int s = whir_ctx_create(device, p16, p24, &c);
    if (s != WHIR_OK) {
      for (whir_ctx* x : b->ctxs) whir_ctx_destroy(x);
      delete b;
      return s;
    }
    b->ctxs.push_back(c);
    b->fixed += c->fixed_device_bytes;
  }
  b->running_fp.assign((size_t)workers, 0);
  for (int i = 0; i < workers; i++) b->threads.emplace_back(worker, b, i);
  *out = b;
  return WHIR_OK;
}

int whir_batch_memory(whir_batch* b, uint64_t* fixed_bytes, uint64_t* pool_reserved_bytes) {
  WH_CHECK(b, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  uint64_t r = 0;
  for (whir_ctx* c : b->ctxs) r += reserved(c);
  if (fixed_bytes) *fixed_bytes = b->fixed;
  if (pool_reserved_bytes) *pool_reserved_bytes = r;
  return WHIR_OK;
}

int whir_batch_set_device_transcript(whir_batch* b, int32_t enable) {
  WH_CHECK(b, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  for (whir_ctx* c : b->ctxs) WH_TRY(whir_ctx_set_device_transcript(c, enable));
  return WHIR_OK;
}

int whir_batch_set_wait_spin(whir_batch* b, int32_t microseconds) {
  WH_CHECK(b, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  for (whir_ctx* c : b->ctxs) WH_TRY(whir_ctx_set_wait_spin(c, microseconds));
  return WHIR_OK;
}

int whir_batch_set_grind_window(whir_batch* b, int32_t mode) {
  WH_CHECK(b, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  for (whir_ctx* c : b->ctxs) WH_TRY(whir_ctx_set_grind_window(c, mode));
  return WHIR_OK;
}

int whir_batch_destroy(whir_batch* b) {
  if (!b) return WHIR_OK;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->stop = true;
  }
  b->cv_work.notify_all();
  for (std::thread& t : b->threads) t.join();
  for (whir_ctx* c : b->ctxs) whir_ctx_destroy(c);
  delete b;
  return WHIR_OK;
}

int whir_batch_submit(whir_batch* b, whir_job* j) {
  WH_CHECK(b && j && j->proof_out && j->poly, "bad job");
  whir_config c;
  WH_TRY(wh::config_new(j->params, j->n, &c));
  j->footprint_bytes = wh::footprint(c, j->poly_on_device);
  j->error[0] = 0;
  j->done = 0;
  j->status = WHIR_OK;
  j->t_submit_ms = now_ms();
  {
    std::lock_guard<std::mutex> lk(b->mu);
    WH_CHECK(!b->stop, "batch is shutting down");
    b->queue.push_back(j);
    b->pending++;
  }
  b->cv_work.notify_all();
  return WHIR_OK;
}

int whir_batch_wait(whir_batch* b, whir_job* j, int32_t timeout_ms) {
  WH_CHECK(b && j, "null argument");
  std::unique_lock<std::mutex> lk(b->mu);
  auto pred = [&] { return j->done != 0; };
  if (timeout_ms < 0) {
    b->cv_done.wait(lk, pred);
  } else if (!b->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
    wh::set_error("timed out waiting for the job");
    return WHIR_ERR_NOT_FOUND;
  }
  return j->status;
}

int whir_batch_wait_all(whir_batch* b) {
  WH_CHECK(b, "null argument");
  std::unique_lock<std::mutex> lk(b->mu);
  b->cv_done.wait(lk, [&] { return b->pending == 0; });
  return WHIR_OK;
}

int whir_batch_run(whir_batch* b, whir_job* jobs, int32_t count) {
  WH_CHECK(b && (jobs || count == 0) && count >= 0, "bad arguments");
  for (int32_t i = 0; i < count; i++) WH_TRY(whir_batch_submit(b, &jobs[i]));
  WH_TRY(whir_batch_wait_all(b));
  for (int32_t i = 0; i < count; i++)
    if (jobs[i].status != WHIR_OK) return jobs[i].status;
  return WHIR_OK;
}

}  // extern "C"
