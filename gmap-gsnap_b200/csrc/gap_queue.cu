/*
 * gap_queue.cu -- the stage-3 batching adapter for Dynprog_single_gap.
 *
 * GMAP's stage 3 runs one worker thread per read and calls
 * Dynprog_single_gap once per gap (src/stage3.c:9117, :9297, :9546), one
 * gap at a time.  A gap queue keeps that call shape -- one gap, its query
 * strings by pointer, a blocking call -- and aligns the gaps of all calling
 * threads together: a worker thread owning a context takes every waiting
 * gap (up to max_batch) as one gdp_single_gap_batch call once max_batch
 * gaps wait or the oldest has waited max_wait_us, and hands each caller its
 * own result and records.  Results do not depend on the batching.
 */
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>
#include "gdp.h"

namespace {

struct GapRequest {
  gdp_single_gap_t gap;
  const char *rseq, *rseq_uc;
  gdp_result_t *result;
  int8_t *path;
  gdp_rec_t *recs;
  int64_t max_recs;
  int64_t *nrecs;
  bool done = false;
  int rc = GDP_OK;
  std::chrono::steady_clock::time_point t0;
};

}  // namespace

struct gdp_gap_queue {
  gdp_ctx *ctx = nullptr;
  int64_t max_batch = 4096;
  std::chrono::microseconds max_wait{200};
  std::mutex mu;
  std::condition_variable work_cv, done_cv;
  std::deque<GapRequest *> waiting;
  bool stop = false;
  std::thread worker;
  int64_t st_batches = 0, st_gaps = 0, st_max_batch = 0;

  /* batch buffers, reused */
  std::vector<gdp_single_gap_t> gaps;
  std::vector<char> arena;
  std::vector<gdp_result_t> results;
  std::vector<int8_t> path;
  std::vector<gdp_rec_t> recs;

  void run () {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      work_cv.wait(lk, [&] { return stop || !waiting.empty(); });
      if (waiting.empty() && stop) return;
      /* wait for a full batch or the oldest request's deadline */
      const auto deadline = waiting.front()->t0 + max_wait;
      work_cv.wait_until(lk, deadline, [&] { return stop || (int64_t) waiting.size() >= max_batch; });
      std::vector<GapRequest *> batch;
      while (!waiting.empty() && (int64_t) batch.size() < max_batch) {
        batch.push_back(waiting.front());
        waiting.pop_front();
      }
      lk.unlock();
      align(batch);
      lk.lock();
      for (GapRequest *r : batch) r->done = true;
      st_batches++;
      st_gaps += (int64_t) batch.size();
      st_max_batch = std::max<int64_t>(st_max_batch, (int64_t) batch.size());
      done_cv.notify_all();
    }
  }

  void align (const std::vector<GapRequest *> &batch) {
    const int64_t n = (int64_t) batch.size();
    gaps.resize((size_t) n);
    int64_t bytes = 0, cap = 0;
    for (GapRequest *r : batch) {
      const int64_t rl = std::max(r->gap.rlength, 0);
      bytes += 2 * rl;
      cap += rl + std::max(r->gap.glength, 0) + 2;
    }
    arena.resize((size_t) std::max<int64_t>(bytes, 1));
    int64_t off = 0;
    for (int64_t i = 0; i < n; i++) {
      GapRequest *r = batch[(size_t) i];
      gdp_single_gap_t g = r->gap;
      const int64_t rl = std::max(g.rlength, 0);
      if (rl > 0) {
        memcpy(arena.data() + off, r->rseq, (size_t) rl);
        memcpy(arena.data() + off + rl, r->rseq_uc, (size_t) rl);
      }
      g.rseq = off;
      g.rseq_uc = off + rl;
      off += 2 * rl;
      gaps[(size_t) i] = g;
    }
    results.resize((size_t) n);
    path.resize((size_t) n);
    recs.resize((size_t) std::max<int64_t>(cap, 1));
    int64_t used = 0;
    const int rc = gdp_single_gap_batch(ctx, gaps.data(), n, arena.data(), bytes, results.data(), path.data(),
                                        recs.data(), (int64_t) recs.size(), &used);
    for (int64_t i = 0; i < n; i++) {
      GapRequest *r = batch[(size_t) i];
      r->rc = rc;
      if (rc != GDP_OK) continue;
      gdp_result_t res = results[(size_t) i];
      const int64_t k = res.nrecs;
      if (k > r->max_recs) {
        res.status = GDP_ERR_RECS;
        res.nrecs = 0;
      } else if (k > 0) {
        memcpy(r->recs, recs.data() + res.rec_offset, (size_t) k * sizeof(gdp_rec_t));
      }
      res.rec_offset = 0;
      *r->result = res;
      if (r->path) *r->path = path[(size_t) i];
      if (r->nrecs) *r->nrecs = res.nrecs;
    }
  }
};

extern "C" int
gdp_gap_queue_create (int device, int mode, int64_t max_batch, int64_t max_wait_us, const uint32_t *genome_blocks,
                      const uint32_t *alt_blocks, uint64_t genome_length, gdp_gap_queue **out) {
  if (out == nullptr || genome_blocks == nullptr || max_batch < 0 || max_wait_us < 0) return GDP_ERR_PARAM;
  gdp_gap_queue *q = new gdp_gap_queue();
  int rc = gdp_ctx_create(&q->ctx, device, mode, 0);
  if (rc == GDP_OK) rc = gdp_set_genome(q->ctx, genome_blocks, alt_blocks, genome_length);
  if (rc != GDP_OK) {
    if (q->ctx) gdp_ctx_destroy(q->ctx);
    delete q;
    return rc;
  }
  if (max_batch > 0) q->max_batch = max_batch;
  q->max_wait = std::chrono::microseconds(max_wait_us);
  q->worker = std::thread([q] { q->run(); });
  *out = q;
  return GDP_OK;
}

extern "C" int
gdp_gap_queue_setup (gdp_gap_queue *q, int user_open, int user_extend, int user_dynprog_p, int homopolymerp) {
  if (q == nullptr) return GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(q->mu);
  return gdp_single_setup(q->ctx, user_open, user_extend, user_dynprog_p, homopolymerp);
}

extern "C" int
gdp_gap_queue_align (gdp_gap_queue *q, const gdp_single_gap_t *gap, const char *rsequence, const char *rsequenceuc,
                     gdp_result_t *result, int8_t *path, gdp_rec_t *recs, int64_t max_recs, int64_t *nrecs) {
  if (q == nullptr || gap == nullptr || result == nullptr || max_recs < 0 || (max_recs > 0 && recs == nullptr) ||
      (gap->rlength > 0 && (rsequence == nullptr || rsequenceuc == nullptr)))
    return GDP_ERR_PARAM;
  GapRequest r;
  r.gap = *gap;
  r.rseq = rsequence;
  r.rseq_uc = rsequenceuc;
  r.result = result;
  r.path = path;
  r.recs = recs;
  r.max_recs = max_recs;
  r.nrecs = nrecs;
  r.t0 = std::chrono::steady_clock::now();
  std::unique_lock<std::mutex> lk(q->mu);
  if (q->stop) return GDP_ERR_PARAM;
  q->waiting.push_back(&r);
  q->work_cv.notify_one();
  q->done_cv.wait(lk, [&] { return r.done; });
  return r.rc;
}

extern "C" int
gdp_gap_queue_stats (gdp_gap_queue *q, int64_t *batches, int64_t *gaps, int64_t *max_batch) {
  if (q == nullptr) return GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(q->mu);
  if (batches) *batches = q->st_batches;
  if (gaps) *gaps = q->st_gaps;
  if (max_batch) *max_batch = q->st_max_batch;
  return GDP_OK;
}

extern "C" void
gdp_gap_queue_destroy (gdp_gap_queue *q) {
  if (q == nullptr) return;
  {
    std::lock_guard<std::mutex> lk(q->mu);
    q->stop = true;
  }
  q->work_cv.notify_all();
  if (q->worker.joinable()) q->worker.join();
  gdp_ctx_destroy(q->ctx);
  delete q;
}
