/*
 * serve.cu -- a continuous-batching request loop over the batch runtime.
 *
 * Requests (one or more alignment pairs each) arrive at any time from any
 * thread.  A request is admitted when the direction-matrix memory it needs
 * (the device words of its fills) fits into what the admitted, unfinished
 * requests leave of the budget.  Requests fall into two size classes by
 * their longest stretch -- short reads and long ones (long reads, cDNA
 * gaps) -- with
 * one arrival-order queue each, and a batch takes the admissible waiting
 * requests of one class: a lone long read needs ten times the time of a
 * short one, and a short request batched with it would wait for it.  Each
 * worker owns a context (its own CUDA streams and buffers, the resident
 * genome) and runs one batch at a time; some workers take short batches
 * only, the others long batches first and short ones when no long request
 * waits, and short batches compute on a higher stream priority.  With two
 * or more workers a new batch is copied in, planned and filled while
 * another traces back and copies out.  Every pair is independent, so a
 * request's results do not depend on what it was batched with.
 *
 * A load generator (gdp_server_drive) submits single-pair requests at
 * Poisson arrival times from the calling thread and records each one's
 * latency (submit to results on the host).
 */
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "gdp_internal.h"

namespace {

using clk = std::chrono::steady_clock;

double
secs_since (clk::time_point t0) {
  return std::chrono::duration<double>(clk::now() - t0).count();
}

/* pinned, grow-only host buffer */
struct Pinned {
  void *p = nullptr;
  size_t bytes = 0;
  bool ensure (size_t want) {
    if (want <= bytes) return true;
    /* geometric growth: freeing pinned memory waits for the device, which
       a worker should do rarely while other workers' batches run */
    const size_t grow = std::max(want + want / 4, 2 * bytes) + 4096;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    if (cudaHostAlloc(&p, grow, cudaHostAllocDefault) != cudaSuccess) return false;
    bytes = grow;
    return true;
  }
  ~Pinned () { if (p) cudaFreeHost(p); }
  template <class T> T *as () const { return (T *) p; }
};

struct Request {
  int64_t id = 0;
  /* owned copies (gdp_server_submit) or borrowed pool entries (the load generator) */
  std::vector<gdp_pair_t> own_pairs;
  std::vector<char> own_arena;
  const gdp_pair_t *pairs = nullptr;
  const char *arena = nullptr;
  int64_t n = 0;
  int64_t dir_bytes = 0;   /* direction-matrix bytes the request's fills hold */
  int cls = 0;             /* size class: 0 short, 1 long */
  int64_t rec_slots = 0;   /* traceback record capacity it needs */
  clk::time_point t_submit;
  double latency_ms = 0;
  /* outputs */
  std::vector<gdp_result_t> results;
  std::vector<gdp_rec_t> recs;
  gdp_result_t *result_out = nullptr;   /* borrowed requests: where the one result goes */
  double *latency_out = nullptr;
  int64_t *done_count = nullptr;        /* load generator: completions so far */
  bool keep_recs = true;
  int status = GDP_OK;
  bool done = false;
};

int64_t
request_dir_bytes (const gdp_pair_t *p, int64_t n) {
  int64_t w = 0;
  for (int64_t i = 0; i < n; i++) {
    const bool rerun = p[i].precision == 8 && (p[i].flags & GDP_FLAG_RERUN16);
    if (p[i].precision == 16 || rerun) w += (gdp_pair_words(&p[i], 16) + 3) & ~(int64_t) 3;
    if (p[i].precision == 8) w += (gdp_pair_words(&p[i], 32) + 3) & ~(int64_t) 3;
  }
  return w * 4;
}

int64_t
request_rec_slots (const gdp_pair_t *p, int64_t n) {
  int64_t k = 0;
  for (int64_t i = 0; i < n; i++)
    if (p[i].flags & GDP_FLAG_TRACEBACK) k += (int64_t) p[i].rlength + p[i].glength + 2;
  return k;
}

}  // namespace

struct gdp_server {
  int device = 0;
  std::vector<gdp_ctx *> ctx;
  std::vector<std::thread> workers;
  int64_t budget = 0;             /* direction-matrix bytes */
  int64_t max_batch_pairs = 0;
  int64_t max_batch_rec_bytes = (int64_t) 1 << 30;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue[2];   /* waiting requests per size class, in arrival order */
  int64_t short_max_length = 512;
  int short_workers = 0;          /* workers 0 .. short_workers-1 take short batches only */
  bool started = false;           /* a request was enqueued: the classes are fixed */
  int long_blocks_per_sm = 2;     /* grid cap of long batches (0: none) */
  std::unordered_map<int64_t, Request *> owned;   /* submitted through the public API */
  int64_t next_id = 0;
  int64_t reserved = 0;           /* bytes of admitted, unfinished requests */
  int64_t outstanding = 0;        /* requests not yet done */
  bool stop = false;
  /* statistics */
  int64_t st_batches = 0, st_pairs = 0, st_peak_reserved = 0, st_max_batch = 0;
  int64_t st_cls_batches[2] = {0, 0}, st_cls_pairs[2] = {0, 0};
  double st_busy_s = 0;

  void worker (int w);
  int class_of (const gdp_pair_t *p, int64_t n) const {
    for (int64_t i = 0; i < n; i++)
      if (p[i].rlength > short_max_length || p[i].glength > short_max_length) return 1;
    return 0;
  }
  /* the class worker w takes a batch of now, or -1 (caller holds mu) */
  int pick (int w) const {
    auto ready = [&](int c) { return !queue[c].empty() && reserved + queue[c].front()->dir_bytes <= budget; };
    if (short_workers > 0 && w < short_workers) return ready(0) ? 0 : -1;
    if (short_workers > 0 && ready(1)) return 1;
    if (ready(0)) return 0;
    return ready(1) ? 1 : -1;
  }
};

/* One worker: take the admitted head of the queue as a batch, align it on
   this worker's context, hand the results back. */
void
gdp_server::worker (int w) {
  gdp_ctx *c = ctx[w];
  cudaSetDevice(device);
  std::vector<Request *> batch;
  std::vector<gdp_pair_t> bpairs;
  std::vector<int64_t> first_pair;
  Pinned arena, results, recs;
  for (;;) {
    batch.clear();
    int64_t bytes = 0, npairs = 0, rec_slots = 0;
    int cls = -1;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || pick(w) >= 0; });
      cls = pick(w);
      if (cls < 0) {
        if (stop) return;
        continue;
      }
      std::deque<Request *> &q = queue[cls];
      while (!q.empty()) {
        Request *r = q.front();
        if (!batch.empty() && (npairs + r->n > max_batch_pairs || reserved + bytes + r->dir_bytes > budget ||
                               (rec_slots + r->rec_slots) * (int64_t) sizeof(gdp_rec_t) > max_batch_rec_bytes))
          break;
        q.pop_front();
        batch.push_back(r);
        bytes += r->dir_bytes;
        npairs += r->n;
        rec_slots += r->rec_slots;
      }
      reserved += bytes;
      st_peak_reserved = std::max(st_peak_reserved, reserved);
    }
    const clk::time_point t0 = clk::now();
    /* the batch's pairs, their sequences copied into one arena (windows the
       device extracts are only reserved) */
    bpairs.resize(npairs);
    first_pair.resize(batch.size());
    int64_t abytes = 0;
    {
      int64_t k = 0;
      for (size_t b = 0; b < batch.size(); b++) {
        first_pair[b] = k;
        for (int64_t i = 0; i < batch[b]->n; i++, k++) {
          const gdp_pair_t &p = batch[b]->pairs[i];
          abytes += 2 * (int64_t) p.rlength + 2 * (int64_t) p.glength + 32;
        }
      }
    }
    int rc = GDP_OK;
    if (!arena.ensure(std::max<int64_t>(abytes, 16)) || !results.ensure(std::max<int64_t>(npairs, 1) * sizeof(gdp_result_t)) ||
        !recs.ensure(std::max<int64_t>(rec_slots, 1) * sizeof(gdp_rec_t)))
      rc = GDP_ERR_CUDA;
    if (rc == GDP_OK) {
      char *a = arena.as<char>();
      int64_t off = 0, k = 0;
      for (Request *r : batch) {
        for (int64_t i = 0; i < r->n; i++, k++) {
          gdp_pair_t q = r->pairs[i];
          const gdp_pair_t &p = r->pairs[i];
          const int64_t rl = p.rlength > 0 ? p.rlength : 0, gl = p.glength > 0 ? p.glength : 0;
          q.rseq = off; memcpy(a + off, r->arena + p.rseq, rl); off += rl;
          if (p.rseq_uc == p.rseq) q.rseq_uc = q.rseq;
          else { q.rseq_uc = off; memcpy(a + off, r->arena + p.rseq_uc, rl); off += rl; }
          const bool gw = (p.flags & GDP_FLAG_GWINDOW) != 0;
          q.gseq = off;
          if (!gw) memcpy(a + off, r->arena + p.gseq, gl);
          off += gl;
          if (p.gseq_alt == p.gseq) q.gseq_alt = q.gseq;
          else { q.gseq_alt = off; if (!gw) memcpy(a + off, r->arena + p.gseq_alt, gl); off += gl; }
          off = (off + 15) & ~(int64_t) 15;
          bpairs[k] = q;
        }
      }
      int64_t used = 0;
      /* long batches below short ones on the device, and on part of each SM */
      rc = gdp_ctx_set_param(c, "wave_priority", cls == 0 ? 0 : (int64_t) 1 << 20);
      if (rc == GDP_OK) rc = gdp_ctx_set_param(c, "grid_blocks_per_sm", cls == 0 ? 0 : long_blocks_per_sm);
      if (rc == GDP_OK)
        rc = gdp_align_batch(c, bpairs.data(), npairs, a, off, results.as<gdp_result_t>(), recs.as<gdp_rec_t>(),
                           std::max<int64_t>(rec_slots, 1), &used);
    }
    const gdp_result_t *res = results.as<gdp_result_t>();
    const gdp_rec_t *rv = recs.as<gdp_rec_t>();
    for (size_t b = 0; b < batch.size(); b++) {
      Request *r = batch[b];
      r->status = rc;
      if (r->result_out) {
        gdp_result_t x = res[first_pair[b]];
        if (rc != GDP_OK) x.status = rc;
        x.rec_offset = -1;
        *r->result_out = x;
        continue;
      }
      r->results.assign(res + first_pair[b], res + first_pair[b] + r->n);
      int64_t nr = 0;
      for (gdp_result_t &x : r->results) {
        if (rc != GDP_OK) x.status = rc;
        nr += std::max(x.nrecs, 0);
      }
      if (r->keep_recs && rc == GDP_OK) {
        r->recs.resize(nr);
        int64_t o = 0;
        for (gdp_result_t &x : r->results) {
          if (x.nrecs > 0) memcpy(r->recs.data() + o, rv + x.rec_offset, x.nrecs * sizeof(gdp_rec_t));
          x.rec_offset = o;
          o += std::max(x.nrecs, 0);
        }
      }
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      const clk::time_point t1 = clk::now();
      for (Request *r : batch) {
        r->latency_ms = std::chrono::duration<double, std::milli>(t1 - r->t_submit).count();
        if (r->latency_out) *r->latency_out = r->latency_ms;
        if (r->done_count) (*r->done_count)++;
        r->done = true;
        outstanding--;
      }
      reserved -= bytes;
      st_batches++;
      st_pairs += npairs;
      st_max_batch = std::max(st_max_batch, npairs);
      st_cls_batches[cls]++;
      st_cls_pairs[cls] += npairs;
      st_busy_s += std::chrono::duration<double>(t1 - t0).count();
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

static void
server_enqueue (gdp_server *s, Request *r) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->t_submit = clk::now();
    r->cls = s->class_of(r->pairs, r->n);
    s->started = true;
    s->queue[r->cls].push_back(r);
    s->outstanding++;
  }
  /* the worker that takes this class may be any of them */
  s->cv_work.notify_all();
}

extern "C" int
gdp_server_create (int device, int mode, int nworkers, int64_t dir_budget_bytes, int64_t max_batch_pairs,
                   const uint32_t *genome_blocks, const uint32_t *alt_blocks, uint64_t genome_length,
                   gdp_server **out) {
  if (out == nullptr || nworkers < 1 || nworkers > 8) return GDP_ERR_PARAM;
  *out = nullptr;
  gdp_server *s = new gdp_server();
  s->device = device;
  s->budget = dir_budget_bytes > 0 ? dir_budget_bytes : ((int64_t) 40 << 30);
  s->max_batch_pairs = max_batch_pairs > 0 ? max_batch_pairs : 131072;
  for (int w = 0; w < nworkers; w++) {
    gdp_ctx *c = nullptr;
    int rc = gdp_ctx_create(&c, device, mode, 0);
    /* a worker's batch is one wave: the workers already overlap batches on
       the device, and a one-wave call hands its records out on its own
       thread */
    if (rc == GDP_OK) rc = gdp_ctx_set_param(c, "wave_pairs", std::max<int64_t>(s->max_batch_pairs, 16384));
    if (rc == GDP_OK) rc = gdp_ctx_set_param(c, "first_wave_pairs", std::max<int64_t>(s->max_batch_pairs, 16384));
    if (rc == GDP_OK && genome_blocks) rc = gdp_set_genome(c, genome_blocks, alt_blocks, genome_length);
    if (rc != GDP_OK) {
      if (c) gdp_ctx_destroy(c);
      for (gdp_ctx *x : s->ctx) gdp_ctx_destroy(x);
      delete s;
      return rc;
    }
    s->ctx.push_back(c);
  }
  /* short requests are most of a read mix: three workers in four take them */
  s->short_workers = nworkers >= 2 ? std::min(std::max(1, (3 * nworkers) / 4), nworkers - 1) : 0;
  for (int w = 0; w < nworkers; w++) s->workers.emplace_back(&gdp_server::worker, s, w);
  *out = s;
  return GDP_OK;
}

extern "C" int64_t
gdp_server_submit (gdp_server *s, const gdp_pair_t *pairs, int64_t npairs, const char *arena, int64_t arena_bytes) {
  if (s == nullptr || npairs <= 0 || pairs == nullptr || arena_bytes < 0) return -GDP_ERR_PARAM;
  Request *r = new Request();
  r->own_pairs.assign(pairs, pairs + npairs);
  r->own_arena.assign(arena, arena + arena_bytes);
  r->pairs = r->own_pairs.data();
  r->arena = r->own_arena.data();
  r->n = npairs;
  for (int64_t i = 0; i < npairs; i++) {
    const gdp_pair_t &p = pairs[i];
    const int64_t rl = std::max(p.rlength, 0), gl = std::max(p.glength, 0);
    const bool gw = (p.flags & GDP_FLAG_GWINDOW) != 0;
    if (p.rseq < 0 || p.rseq + rl > arena_bytes || p.rseq_uc < 0 || p.rseq_uc + rl > arena_bytes ||
        (!gw && (p.gseq < 0 || p.gseq + gl > arena_bytes || p.gseq_alt < 0 || p.gseq_alt + gl > arena_bytes))) {
      delete r;
      return -GDP_ERR_LEN;
    }
  }
  r->dir_bytes = request_dir_bytes(pairs, npairs);
  r->rec_slots = request_rec_slots(pairs, npairs);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    s->owned[r->id] = r;
    if (r->dir_bytes > s->budget) {
      /* can never be admitted */
      r->status = GDP_ERR_BUDGET;
      r->results.assign(npairs, gdp_result_t());
      for (gdp_result_t &x : r->results) { memset(&x, 0, sizeof(x)); x.status = GDP_ERR_BUDGET; }
      r->done = true;
      return r->id;
    }
  }
  server_enqueue(s, r);
  return r->id;
}

extern "C" int
gdp_server_wait (gdp_server *s, int64_t id, gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs,
                 int64_t *nrecs, double *latency_ms) {
  if (s == nullptr) return GDP_ERR_PARAM;
  Request *r = nullptr;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->owned.find(id);
    if (it == s->owned.end()) return GDP_ERR_PARAM;
    r = it->second;
    s->cv_done.wait(lk, [&] { return r->done; });
    s->owned.erase(it);
  }
  int rc = r->status;
  if (results) memcpy(results, r->results.data(), r->results.size() * sizeof(gdp_result_t));
  if (nrecs) *nrecs = (int64_t) r->recs.size();
  if (recs && !r->recs.empty()) {
    if ((int64_t) r->recs.size() > max_recs) rc = (rc == GDP_OK) ? GDP_ERR_RECS : rc;
    else memcpy(recs, r->recs.data(), r->recs.size() * sizeof(gdp_rec_t));
  }
  if (latency_ms) *latency_ms = r->latency_ms;
  delete r;
  return rc;
}

extern "C" int
gdp_server_drive (gdp_server *s, const gdp_pair_t *pool, int64_t npool, const char *arena, int64_t nrequests,
                  double rate, uint64_t seed, gdp_result_t *results_out, double *latency_ms, double *elapsed_s) {
  if (s == nullptr || pool == nullptr || npool <= 0 || nrequests <= 0 || rate <= 0 || latency_ms == nullptr)
    return GDP_ERR_PARAM;
  std::vector<Request> reqs(nrequests);
  std::vector<gdp_result_t> sink(results_out ? 0 : nrequests);
  int64_t ndone = 0;
  for (int64_t k = 0; k < nrequests; k++) {
    Request &r = reqs[k];
    r.id = -1 - k;
    r.pairs = pool + (k % npool);
    r.arena = arena;
    r.n = 1;
    r.dir_bytes = request_dir_bytes(r.pairs, 1);
    r.rec_slots = request_rec_slots(r.pairs, 1);
    r.result_out = results_out ? results_out + k : sink.data() + k;
    r.latency_out = latency_ms + k;
    r.keep_recs = false;
    r.done_count = &ndone;
    if (r.dir_bytes > s->budget) return GDP_ERR_BUDGET;
  }
  /* Poisson arrivals: exponential gaps from a seeded xorshift stream */
  uint64_t x = seed * 0x9E3779B97F4A7C15ull + 1;
  const clk::time_point t0 = clk::now();
  double t = 0;
  for (int64_t k = 0; k < nrequests; k++) {
    x ^= x << 13; x ^= x >> 7; x ^= x << 17;
    const double u = ((x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    t += -log(u) / rate;
    for (;;) {
      const double now = secs_since(t0);
      if (now >= t) break;
      if (t - now > 200e-6) std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    server_enqueue(s, &reqs[k]);
  }
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return ndone == nrequests; });
  }
  if (elapsed_s) *elapsed_s = secs_since(t0);
  int rc = GDP_OK;
  for (const Request &r : reqs)
    if (r.status != GDP_OK) rc = r.status;
  return rc;
}

extern "C" int
gdp_server_stats (gdp_server *s, int64_t *batches, int64_t *pairs, int64_t *max_batch_pairs,
                  int64_t *peak_reserved_bytes, double *busy_s) {
  if (s == nullptr) return GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(s->mu);
  if (batches) *batches = s->st_batches;
  if (pairs) *pairs = s->st_pairs;
  if (max_batch_pairs) *max_batch_pairs = s->st_max_batch;
  if (peak_reserved_bytes) *peak_reserved_bytes = s->st_peak_reserved;
  if (busy_s) *busy_s = s->st_busy_s;
  return GDP_OK;
}

extern "C" void
gdp_server_destroy (gdp_server *s) {
  if (s == nullptr) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (std::thread &t : s->workers) t.join();
  for (auto &kv : s->owned) delete kv.second;
  for (gdp_ctx *c : s->ctx) gdp_ctx_destroy(c);
  delete s;
}

extern "C" int
gdp_server_set_classes (gdp_server *s, int64_t short_max_length, int short_workers) {
  if (s == nullptr || short_max_length < 0 || short_workers < 0) return GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(s->mu);
  const int nw = (int) s->ctx.size();
  /* before the first request: a request keeps the class it got */
  if (s->started || (nw > 1 && short_workers >= nw)) return GDP_ERR_PARAM;
  s->short_max_length = short_max_length;
  s->short_workers = nw >= 2 ? short_workers : 0;
  return GDP_OK;
}

extern "C" int
gdp_server_class_of (gdp_server *s, const gdp_pair_t *pairs, int64_t npairs) {
  if (s == nullptr || pairs == nullptr || npairs <= 0) return -GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(s->mu);
  return s->class_of(pairs, npairs);
}

extern "C" int
gdp_server_class_stats (gdp_server *s, int64_t *batches, int64_t *pairs) {
  if (s == nullptr) return GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(s->mu);
  for (int c = 0; c < 2; c++) {
    if (batches) batches[c] = s->st_cls_batches[c];
    if (pairs) pairs[c] = s->st_cls_pairs[c];
  }
  return GDP_OK;
}
