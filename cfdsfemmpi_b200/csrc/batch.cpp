// Batched time stepping of many independent instances (meshes, controls and
// solver options of their own) on one GPU.
//
// Each instance is an ordinary handle with its own stream; its Arnoldi chunks
// are replayed as CUDA graphs and its Newton/GMRES control stays on the host.
// A persistent pool of host threads drives the instances concurrently, so the
// GPU runs the small kernels of many instances side by side instead of one
// instance's latency-bound sequence at a time.  Host waits of batched handles
// sleep (blocking-sync events) so that dozens of threads can share a few cores.
//
// Schedule: instances are taken largest first (longest-processing-time
// order) and their streams get priorities by size (largest highest), so the
// longest dependent kernel chains are not slowed by the small instances;
// `concurrency` threads take part; `chunk` is the number of Arnoldi
// steps per graph; `depth` the number of chunks a handle keeps enqueued
// beyond the one whose state its host thread waits for (a sleeping thread
// wakes up tens of microseconds after its event, so small instances need
// more than one chunk in flight to keep their stream busy).  With all three
// set to 0 the batch autotunes: the first batch steps try candidate
// triples, one per step, scored by wall time per GMRES iteration of the
// step, and the best is kept for the rest of the run.  No knob changes any
// number an instance computes (kernels after GMRES convergence are no-ops and
// every reduction has a fixed order), so each instance's results are bitwise
// those of its own single-instance run.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/cfdgpu.h"
#include "internal.h"

struct cfdgpu_batch {
  int device = 0;
  std::vector<cfdgpu_handle *> h;
  std::vector<int> order;              // instance indices, largest system first
  std::vector<double> work;            // BSR blocks per instance
  // schedule
  struct Sched {
    int concurrency, chunk, depth;
  };
  Sched cur{0, 0, 0};                  // in use
  bool autotune = true, tuned = false;
  std::vector<Sched> candidates;
  size_t trial = 0;
  double best_cost = std::numeric_limits<double>::infinity();
  Sched best{0, 0, 0};
  std::vector<double> trial_cost;
  // worker pool
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_go, cv_done;
  uint64_t generation = 0;
  int finished = 0;
  bool quit = false;
  std::atomic<int> next{0};
  // arguments of the current step
  const double *tnow = nullptr, *tfact = nullptr;
  cfdgpu_step_stats *stats = nullptr;
  double *lat = nullptr;
  std::vector<int> rc;
  std::string err;
};

namespace {

void worker_main(cfdgpu_batch *b, int id)
{
  cudaSetDevice(b->device);
  uint64_t seen = 0;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(b->mu);
      b->cv_go.wait(lk, [&] { return b->quit || b->generation != seen; });
      if (b->quit) return;
      seen = b->generation;
    }
    if (id < b->cur.concurrency) {
      for (;;) {
        const int k = b->next.fetch_add(1);
        if (k >= (int)b->order.size()) break;
        const int i = b->order[k];
        const auto t0 = std::chrono::steady_clock::now();
        b->rc[i] = cfdgpu_step(b->h[i], b->tnow[i], b->tfact[i], &b->stats[i]);
        b->lat[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      }
    }
    {
      std::lock_guard<std::mutex> lk(b->mu);
      b->finished++;
    }
    b->cv_done.notify_one();
  }
}

int apply_schedule(cfdgpu_batch *b, cfdgpu_batch::Sched s)
{
  for (auto *h : b->h) {
    const int rc = cfdgpu::set_host_schedule(h, true, s.chunk, s.depth);
    if (rc) return rc;
  }
  b->cur = s;
  return 0;
}

void make_candidates(cfdgpu_batch *b)
{
  const int n = (int)b->h.size();
  const int all = std::min(n, (int)b->workers.size());
  std::vector<int> cs = {std::min(32, all), all};
  cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
  b->candidates.clear();
  for (int depth : {1, 2, 4})
    for (int ch : {4, 8})
      for (int c : cs) b->candidates.push_back({c, ch, depth});
}

}  // namespace

extern "C" {

int cfdgpu_batch_create(int count, const cfdgpu_mesh *meshes, const cfdgpu_control *ctrls,
                        const cfdgpu_solver_opts *opts, cfdgpu_batch **out)
{
  if (!out) return CFDGPU_EINVAL;
  *out = nullptr;
  if (count <= 0 || count > CFDGPU_BATCH_MAX || !meshes || !ctrls || !opts) return CFDGPU_EINVAL;
  cfdgpu_batch *b = new cfdgpu_batch();
  cudaGetDevice(&b->device);
  b->h.assign(count, nullptr);
  b->work.assign(count, 0.0);
  for (int i = 0; i < count; i++) {
    const int rc = cfdgpu_create(&meshes[i], &ctrls[i], &opts[i], &b->h[i]);
    if (rc) {
      b->err = "instance " + std::to_string(i) + ": " + (b->h[i] ? cfdgpu_last_error(b->h[i]) : "create failed");
      *out = b;   // the caller reads the message, then destroys
      return rc;
    }
    cfdgpu::handle_work(b->h[i], nullptr, &b->work[i]);
  }
  b->order.resize(count);
  for (int i = 0; i < count; i++) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int c) { return b->work[a] > b->work[c]; });
  // stream priorities by size: the largest systems have the longest chains
  // of dependent Arnoldi kernels, so their kernels go first and the small
  // instances fill the gaps
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  const int levels = least - greatest + 1;
  for (int k = 0; k < count && levels > 1; k++) {
    const int prio = greatest + (int)((int64_t)k * levels / count);
    const int rc = cfdgpu::set_stream_priority(b->h[b->order[k]], prio);
    if (rc) {
      b->err = "stream priority";
      *out = b;
      return rc;
    }
  }
  b->rc.assign(count, 0);
  const int nthreads = std::min(count, CFDGPU_BATCH_MAX_THREADS);
  for (int t = 0; t < nthreads; t++) b->workers.emplace_back(worker_main, b, t);
  make_candidates(b);
  const int rc = apply_schedule(b, b->candidates[0]);
  *out = b;
  return rc;
}

int cfdgpu_batch_destroy(cfdgpu_batch *b)
{
  if (!b) return CFDGPU_EINVAL;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->quit = true;
  }
  b->cv_go.notify_all();
  for (auto &t : b->workers) t.join();
  for (auto *h : b->h)
    if (h) cfdgpu_destroy(h);
  delete b;
  return 0;
}

const char *cfdgpu_batch_last_error(cfdgpu_batch *b) { return b ? b->err.c_str() : "null batch"; }

int cfdgpu_batch_size(cfdgpu_batch *b) { return b ? (int)b->h.size() : CFDGPU_EINVAL; }

cfdgpu_handle *cfdgpu_batch_handle(cfdgpu_batch *b, int i)
{
  if (!b || i < 0 || i >= (int)b->h.size()) return nullptr;
  return b->h[i];
}

int cfdgpu_batch_set_schedule(cfdgpu_batch *b, int concurrency, int chunk, int depth)
{
  if (!b || concurrency < 0 || chunk < 0 || chunk > 64 || depth < 0 || depth > CFDGPU_BATCH_MAX_DEPTH)
    return CFDGPU_EINVAL;
  if (concurrency == 0 && chunk == 0 && depth == 0) {
    b->autotune = true;
    b->tuned = false;
    b->trial = 0;
    b->best_cost = std::numeric_limits<double>::infinity();
    b->trial_cost.clear();
    return apply_schedule(b, b->candidates[0]);
  }
  if (concurrency == 0 || chunk == 0 || depth == 0) return CFDGPU_EINVAL;
  b->autotune = false;
  b->tuned = true;
  return apply_schedule(b, {std::min(concurrency, (int)b->workers.size()), chunk, depth});
}

int cfdgpu_batch_get_schedule(cfdgpu_batch *b, int *concurrency, int *chunk, int *depth, int *tuned)
{
  if (!b) return CFDGPU_EINVAL;
  if (concurrency) *concurrency = b->cur.concurrency;
  if (chunk) *chunk = b->cur.chunk;
  if (depth) *depth = b->cur.depth;
  if (tuned) *tuned = b->tuned ? 1 : 0;
  return 0;
}

int cfdgpu_batch_step(cfdgpu_batch *b, const double *timeNow, const double *timeFact, cfdgpu_step_stats *stats,
                      double *latency_ms)
{
  if (!b || !timeNow || !timeFact || !stats || !latency_ms) return CFDGPU_EINVAL;
  const auto t0 = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->tnow = timeNow;
    b->tfact = timeFact;
    b->stats = stats;
    b->lat = latency_ms;
    std::fill(b->rc.begin(), b->rc.end(), 0);
    b->next.store(0);
    b->finished = 0;
    b->generation++;
  }
  b->cv_go.notify_all();
  {
    std::unique_lock<std::mutex> lk(b->mu);
    b->cv_done.wait(lk, [&] { return b->finished == (int)b->workers.size(); });
  }
  const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  int first_bad = -1;
  for (int i = 0; i < (int)b->h.size(); i++)
    if (b->rc[i] && first_bad < 0) first_bad = i;
  if (first_bad >= 0) {
    b->err = "instance " + std::to_string(first_bad) + ": " + cfdgpu_last_error(b->h[first_bad]);
    return b->rc[first_bad];
  }
  if (b->autotune && !b->tuned) {
    double its = 0.0;
    for (int i = 0; i < (int)b->h.size(); i++)
      for (int k = 0; k < stats[i].newton_iters && k < CFDGPU_MAX_NEWTON; k++) its += stats[i].ksp_its[k];
    const double cost = wall / std::max(1.0, its);
    b->trial_cost.push_back(cost);
    if (cost < b->best_cost) {
      b->best_cost = cost;
      b->best = b->candidates[b->trial];
    }
    b->trial++;
    if (b->trial < b->candidates.size()) {
      const int rc = apply_schedule(b, b->candidates[b->trial]);
      if (rc) return rc;
    } else {
      b->tuned = true;
      const int rc = apply_schedule(b, b->best);
      if (rc) return rc;
    }
  }
  return 0;
}

}  // extern "C"
