/*
 * runtime.cu -- host runtime and C ABI of libgdp (include/gdp.h).
 *
 * A context owns a compute stream and two copy streams, the device copy of
 * the substitution tables (built as Dynprog_init builds them), an optional
 * resident genome, and grow-only device and pinned-host pools.
 *
 * Planning (host, O(n)): pairs are validated, binned by fill kind (lane
 * width W, variant, tie rule, pass) and ordered by work inside each bin
 * (bucketed), so that the threads of a warp run pairs of similar size;
 * direction storage and traceback record slots are laid out by prefix sums.
 * Execution enqueues one fill kernel per non-empty bin, the 8-bit pass of
 * rerun pairs over a device-compacted list, one traceback kernel, and a
 * device compaction of the Pair records (CUB scan + warp-per-pair gather).
 *
 * gdp_align_batch (host buffers) processes the batch in waves of at most
 * `wave` pairs with two in-flight slots: while the GPU fills wave i, the host
 * plans wave i+1, the copy streams move wave i+1's pairs in and wave i-1's
 * results and records out.
 *
 * 8-bit pairs flagged GDP_FLAG_RERUN16 follow the overflow contract: the
 * 16-bit fill runs first and records the largest in-band score; when that
 * reaches 127 the 8-bit fill would overflow too (its in-band scores are
 * never below the 16-bit ones unless it saturates at the top), so the
 * 16-bit outputs are kept.  Otherwise the 8-bit fill runs and its outputs
 * are kept unless it reaches 127 in the band, ends at or below -98, or its
 * traceback would read cells the 8-bit fill never wrote.
 */
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "gdp_internal.h"
#include "gdp_dropin_internal.h"
#include "fill_thread.cuh"
#include "traceback.cuh"
#include "traceback_warp.cuh"
#include "rec_runs.h"

#define GDP_VERSION "gdp-b200 0.2"

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure (size_t want) {
    if (want <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    /* a quarter of headroom (device buffers can be a large part of HBM, so
       no doubling) */
    size_t grow = want + want / 4 + 4096;
    cudaError_t e = cudaMalloc(&p, grow);
    if (e == cudaSuccess) bytes = grow;
    return e;
  }
  void release () { if (p) cudaFree(p); p = nullptr; bytes = 0; }
  template <class T> T *as () const { return (T *) p; }
};

struct HostBuf {   /* pinned host memory */
  void *p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure (size_t want) {
    if (want <= bytes) return cudaSuccess;
    /* grow geometrically, so that a buffer that keeps growing is
       reallocated rarely: freeing pinned memory waits for the device */
    const size_t grow = std::max(want + want / 4, 2 * bytes) + 4096;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaHostAlloc(&p, grow, cudaHostAllocMapped);
    if (e == cudaSuccess) bytes = grow;
    return e;
  }
  void release () { if (p) cudaFreeHost(p); p = nullptr; bytes = 0; }
  template <class T> T *as () const { return (T *) p; }
};

constexpr int NTHREADKINDS = 24;   /* one thread per pair: (W32, variant, late, pass) */
constexpr int NWARPKINDS = 18;     /* K lanes per pair (16-bit plain): 24 + (variant * 2 + late) * 3 + log2(K) - 3 */
constexpr int WARP_K[3] = {8, 16, 32};
constexpr int NWARP8KINDS = 18;    /* K lanes per pair, 8-bit pass of rerun pairs: 42 + (variant * 2 + late) * 3 + log2(K) - 2 */
constexpr int WARP8_K[3] = {4, 8, 16};
constexpr int NCTAKINDS = 24;      /* one CTA per pair (16-bit plain): 60 + (variant * 2 + late) * 4 + log2(NW) - 1 */
constexpr int NEARLY8KINDS = 6;    /* one thread per pair, 8-bit pass beside the 16-bit pass: 84 + variant * 2 + late */
constexpr int FIRST_WARP8 = NTHREADKINDS + NWARPKINDS;
constexpr int FIRST_CTA = FIRST_WARP8 + NWARP8KINDS;
constexpr int FIRST_EARLY8 = FIRST_CTA + NCTAKINDS;
constexpr int NKINDS = FIRST_EARLY8 + NEARLY8KINDS;
constexpr int CTA_NW[4] = {2, 4, 8, 16};

inline int kind_id (int w32, int variant, int late, int pass) {
  return (((w32 * 3 + variant) * 2 + late) * 2) + pass;
}

inline int warp_kind_id (int variant, int late, int kg) {
  return NTHREADKINDS + (variant * 2 + late) * 3 + kg;
}

inline int warp8_kind_id (int variant, int late, int kg) {
  return FIRST_WARP8 + (variant * 2 + late) * 3 + kg;
}

inline int cta_kind_id (int variant, int late, int nwi) {
  return FIRST_CTA + (variant * 2 + late) * 4 + nwi;
}

inline int early8_kind_id (int variant, int late) {
  return FIRST_EARLY8 + variant * 2 + late;
}

}  // namespace

/* Persistent host worker threads for the planner.  run(nt, f) calls f(t)
   for t = 0 .. nt-1, t = 0 on the caller, the rest on the pool's workers,
   and returns when all are done.  A context owns one pool, so contexts
   plan concurrently without sharing threads. */
class WorkPool {
 public:
  WorkPool () = default;
  WorkPool (const WorkPool &) = delete;
  WorkPool &operator= (const WorkPool &) = delete;
  ~WorkPool () {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }
  template <class F>
  void run (int nt, F &&f) {
    if (nt <= 1) { f(0); return; }
    std::unique_lock<std::mutex> g(m_);
    try {
      while ((int) th_.size() < nt - 1) th_.emplace_back([this] { work(); });
    } catch (...) {
      /* fewer threads than asked: the caller and the threads there are take
         every index all the same */
    }
    fn_ = [&f] (int t) { f(t); };
    next_ = 1;
    nt_ = nt;
    left_ = nt - 1;
    g.unlock();
    cv_.notify_all();
    f(0);
    g.lock();
    while (next_ < nt_) {   /* indices no worker has taken yet */
      const int t = next_++;
      g.unlock();
      f(t);
      g.lock();
      --left_;
    }
    done_.wait(g, [this] { return left_ == 0; });
    nt_ = next_ = 0;
    fn_ = nullptr;
  }
 private:
  void work () {
    std::unique_lock<std::mutex> g(m_);
    for (;;) {
      cv_.wait(g, [this] { return stop_ || next_ < nt_; });
      if (stop_) return;
      const int t = next_++;
      std::function<void(int)> fn = fn_;
      g.unlock();
      fn(t);
      g.lock();
      if (--left_ == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  std::function<void(int)> fn_;
  int next_ = 0, nt_ = 0, left_ = 0;
  bool stop_ = false;
};

/* Host side of a plan (pinned so its upload is asynchronous). */
struct PlanHost {
  int64_t n = 0;
  int64_t nlists = 0;
  HostBuf lists, meta, status, rec_off;
  int64_t start[NKINDS + 2] = {0};
  /* entries of each kind's list, then of the traceback list (jump-late
     pairs first), then its jump-late and its jump-early part */
  int32_t counts[NKINDS + 3] = {0};
  int maxY[NKINDS] = {0};
  int maxMin[NKINDS] = {0};   /* per kind: the largest min(rlength, glength) */
  int64_t dir_words = 0, total_recs = 0;
  int64_t nwindow = 0;   /* pairs whose genome window the device extracts */
  /* planner scratch, kept from plan to plan (grown, never shrunk) */
  std::vector<uint32_t> k16, k8, keys, keys2;
  std::vector<int32_t> vals, vals2, tbl;
  void release () { lists.release(); meta.release(); status.release(); rec_off.release(); }
};

template <class T>
static inline T *grow (std::vector<T> &v, int64_t n) {
  if ((int64_t) v.size() < n) v.resize((size_t) n);
  return v.data();
}

/* Device side of a plan. */
struct PlanDev {
  DevBuf lists, work, counts, work_counts, status, meta0, meta, rec_off, dirs, hdump;
  DevBuf slots;        /* records, rlength + glength + 2 per traceback pair */
  DevBuf nrec_scan;    /* int64 exclusive scan of records per pair */
  DevBuf total;        /* int64 record total of the plan */
  DevBuf cub_tmp;
  DevBuf sel_tmp;      /* temporary storage of the 8-bit pass selection */
  DevBuf sel_tmp_late; /* the same for the jump-late chain */
  void release () {
    lists.release(); work.release(); counts.release(); work_counts.release(); status.release();
    meta0.release(); meta.release(); rec_off.release(); dirs.release(); hdump.release();
    slots.release(); nrec_scan.release(); total.release(); cub_tmp.release(); sel_tmp.release();
    sel_tmp_late.release();
  }
};

struct gdp_plan {
  PlanHost h;
  PlanDev d;
  /* optional CUDA graph of the plan's launches for one set of device pointers */
  bool use_graph = false;
  cudaGraphExec_t gexec = nullptr;
  const void *gkey[4] = {nullptr, nullptr, nullptr, nullptr};
  int64_t glaunches = 0;
};

/* Host-side phase timing of the wave pipeline, compiled in only with
   -DGDP_HOST_TRACE (a diagnostic build): one line per phase on stderr. */
#ifdef GDP_HOST_TRACE
#include <chrono>
#define GDP_TRACE_BEGIN(v) const auto v = std::chrono::steady_clock::now()
#define GDP_TRACE_END(v, what) \
  fprintf(stderr, "gdp-trace %s %.3f ms\n", what, \
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - v).count())
/* device-side timeline: an event recorded on a stream, printed at the end
   of gdp_align_batch as milliseconds from the batch's first event */
struct GdpTraceEv { char what[48]; cudaEvent_t ev; std::chrono::steady_clock::time_point host; };
static std::vector<GdpTraceEv> gdp_tev;
static std::mutex gdp_tev_mu;
#define GDP_TEV(stream, fmt, arg) do { \
    GdpTraceEv t_; snprintf(t_.what, sizeof(t_.what), fmt, (long long) (arg)); \
    cudaEventCreate(&t_.ev); cudaEventRecord(t_.ev, stream); t_.host = std::chrono::steady_clock::now(); \
    std::lock_guard<std::mutex> tg_(gdp_tev_mu); gdp_tev.push_back(t_); } while (0)
#else
#define GDP_TRACE_BEGIN(v) (void) 0
#define GDP_TRACE_END(v, what) (void) 0
#define GDP_TEV(stream, fmt, arg) (void) 0
#endif

/* One in-flight wave of gdp_align_batch; NSLOTS waves are in flight. */
constexpr int NSLOTS = 3;
struct Slot {
  PlanHost h;
  PlanDev d;
  DevBuf pairs, results, recs;
  /* the stream the wave's kernels run on (one of the context's wave
     streams) and the slot's own scratch, so consecutive waves overlap on
     the device (one wave's tail beside the next wave's start) */
  cudaStream_t cs = nullptr;
  DevBuf scratch, scratch8, scratch_late;
  HostBuf total;           /* pinned int64: records of the wave */
  /* the record-run transport (rec_runs.h): the wave's encoded records, each
     pair's stream offset, and their pinned host copies */
  DevBuf enc, enc_off;
  HostBuf h_enc, h_encoff, enc_total;
  bool runs = false;       /* the wave's records leave as runs */
  bool expand = false;     /* its runs are on their way to the host, not yet rebuilt */
  cudaEvent_t h2d_done = nullptr, comp_done = nullptr, out_done = nullptr, total_ready = nullptr;
  int64_t first = 0, count = 0, rec_base = 0;
  bool busy = false;
};

#define GDP_MAX_WAVE_STREAMS 6
/* side streams of a compute stream for the lane-group / CTA / early 8-bit
   kinds (one more takes the jump-late chain) */
#define GDP_NSIDE 6
struct gdp_ctx {
  int device = 0;
  cudaStream_t wave_stream[GDP_MAX_WAVE_STREAMS] = {};   /* gdp_align_batch's compute, highest priority first */
  int nwave = 0;
  int wave_prio = 0;     /* first wave stream of a batch: 0 = the highest priority */
  int grid_limit = 0;    /* fill and traceback grids: at most this many blocks per SM (0: no limit) */
  int nsm = 148;
  cudaStream_t stream = nullptr;        /* compute */
  cudaStream_t h2d = nullptr, d2h = nullptr;
  /* side[0] takes the early 8-bit kinds, side[1 .. GDP_NSIDE-1] the
     one-warp/one-CTA-per-pair fill kinds (each kind beside the others and
     beside the thread kinds), side[GDP_NSIDE] the jump-late thread kinds and
     their 8-bit passes, a chain of its own beside the jump-early one */
  cudaStream_t side[GDP_NSIDE + 1] = {};
  /* the side streams of the wave streams, each at its wave stream's
     priority: a wave's lane-group, CTA and early 8-bit kinds run beside its
     thread kinds with the same priority, and waves on different streams do
     not queue behind one another's side kernels */
  cudaStream_t wave_side[GDP_MAX_WAVE_STREAMS][GDP_NSIDE + 1] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[GDP_NSIDE + 1] = {};
  gdp_tables_t *h_tab = nullptr;
  gdp_tables_t *d_tab = nullptr;
  int reach_from[4] = {0, 0, 0, 0};   /* FillParams::reach_from of h_tab */
  int lower_slack[4] = {0, 0, 0, 0};  /* FillParams::lower_slack4 of h_tab */
  int packed_len = -1;                 /* FillParams::packed_len of h_tab */
  int tab_mn = 0, tab_mx = 0;          /* FillParams::tab_mn / tab_mx of h_tab */
  uint32_t *d_genome = nullptr, *d_genomealt = nullptr;
  uint64_t genome_len = 0;
  int64_t budget = 0;
  int64_t wave = 131072;
  int64_t first_wave = 0;   /* pairs of the first wave (0: wave / 2, at least 16,384) */
  int warp_min_x = 512;     /* pairs with at least this many lanes (rows; lower: columns) ... */
  int warp_max_sweep = 496; /* ... and at most this sweep width per block go one warp per pair */
  bool tb_warp = true;      /* tracebacks with one warp per pair (false: one thread per pair) */
  int group_slack = 48;     /* lane groups of K lanes take sweeps up to 17 K - group_slack columns */
  int plan_threads = 8;     /* host threads of the planner */
  bool check_groups = false; /* the 8-bit pass of rerun pairs on lane groups (false: one thread per pair) ... */
  int check_min_x = 1 << 30; /* ... or only for pairs with at least this many rows (lower: columns) */
  gdpi_single_cfg single;   /* Dynprog_single_setup's user penalties */
  DevBuf arena, scratch, scratch8, scratch_late;
  Slot slot[NSLOTS];
  WorkPool pool;            /* the planner's host threads */
  WorkPool xpool;           /* the copy-out side's host threads (record-run expansion) */
  int record_runs = 0;      /* gdp_align_batch's records as runs: 0 never, 1 every wave, 2 the later waves */
  int runs_from_wave = 5;   /* record_runs 2: the first wave whose records leave as runs */
  int64_t last_d2h = 0;     /* bytes the last gdp_align_batch copied device to host */
  std::atomic<int64_t> launches{0};
  std::string err;
  std::mutex mu;
  /* optional per-launch timing: (kernel id, start, stop) */
  bool profiling = false;
  struct Timed { int id; cudaEvent_t a, b; };
  std::vector<Timed> timed;
  double prof_ms[128] = {0};
  int64_t prof_n[128] = {0};
};

/* kernel ids for profiling: 0..NKINDS-1 fill kinds, then traceback, init,
   integer probe, rerun compaction, record compaction */
#define PROF_TB (NKINDS)
#define PROF_INIT (NKINDS + 1)
#define PROF_PEAK (NKINDS + 2)
#define PROF_RERUN (NKINDS + 3)
#define PROF_RECS (NKINDS + 4)
#define PROF_WINDOW (NKINDS + 5)
#define NPROF (NKINDS + 6)
static const char *
kernel_name (int id) {
  static char buf[NPROF][48];
  if (id == PROF_TB) return "traceback";
  if (id == PROF_INIT) return "init_results_kernel";
  if (id == PROF_PEAK) return "int_peak_kernel";
  if (id == PROF_RERUN) return "rerun_select";
  if (id == PROF_RECS) return "compact_records_kernel";
  if (id == PROF_WINDOW) return "window_kernel";
  if (id >= FIRST_EARLY8) {
    const int c = id - FIRST_EARLY8, variant = c / 2, late = c & 1;
    snprintf(buf[id], sizeof(buf[id]), "fill_thread<W32,%s,%s,8bit-check-early>",
             variant == 0 ? "full" : variant == 1 ? "upper" : "lower", late ? "late" : "early");
    return buf[id];
  }
  if (id >= FIRST_CTA) {
    const int c = id - FIRST_CTA, vl = c / 4, variant = vl / 2, late = vl & 1;
    snprintf(buf[id], sizeof(buf[id]), "fill_cta<W16,%s,%s,%dwarps>",
             variant == 0 ? "full" : variant == 1 ? "upper" : "lower", late ? "late" : "early", CTA_NW[c % 4]);
    return buf[id];
  }
  if (id >= FIRST_WARP8) {
    const int c = id - FIRST_WARP8, vl = c / 3, variant = vl / 2, late = vl & 1;
    snprintf(buf[id], sizeof(buf[id]), "fill_warp<W32,%s,%s,%dlanes,8bit-check>",
             variant == 0 ? "full" : variant == 1 ? "upper" : "lower", late ? "late" : "early", WARP8_K[c % 3]);
    return buf[id];
  }
  if (id >= NTHREADKINDS) {
    const int c = id - NTHREADKINDS, vl = c / 3, variant = vl / 2, late = vl & 1;
    snprintf(buf[id], sizeof(buf[id]), "fill_warp<W16,%s,%s,%dlanes>",
             variant == 0 ? "full" : variant == 1 ? "upper" : "lower", late ? "late" : "early", WARP_K[c % 3]);
    return buf[id];
  }
  const int pass = id & 1, late = (id >> 1) & 1, vw = id >> 2, variant = vw % 3, w32 = vw / 3;
  /* full-band 16-bit thread kinds run the packed fill (fill_packed_kernel) */
  snprintf(buf[id], sizeof(buf[id]), "%s<W%d,%s,%s,%s>", (!w32 && variant == 0) ? "fill_packed" : "fill_thread",
           w32 ? 32 : 16,
           variant == 0 ? "full" : variant == 1 ? "upper" : "lower", late ? "late" : "early",
           pass ? (w32 ? "8bit-check" : "16bit-track") : "plain");
  return buf[id];
}

static void
prof_begin (gdp_ctx *ctx, cudaEvent_t *a, cudaStream_t s = nullptr) {
  if (!ctx->profiling) return;
  cudaEventCreate(a);
  cudaEventRecord(*a, s ? s : ctx->stream);
}

static void
prof_end (gdp_ctx *ctx, int id, cudaEvent_t a, cudaStream_t s = nullptr) {
  if (!ctx->profiling) return;
  cudaEvent_t b;
  cudaEventCreate(&b);
  cudaEventRecord(b, s ? s : ctx->stream);
  ctx->timed.push_back({id, a, b});
}

/* Per mismatch type, the smallest row and column index at which a score
   can reach 127 under h_tab.  Every score is a path score from the matrix
   corner.  The corner itself scores one table entry in the upper and lower
   fills (their row and column 0 profiles meet the 'N' row or class 4 at
   (0, 0), src/dynprog_simd.c:7879, :8782), so a score at (r, c) is at most
   min(r, c) + 1 times the table's largest entry: a 42 x 42 exact match of
   an upper fill scores 3 + 42 * 3 = 129. */
static void
update_reach (gdp_ctx *ctx) {
  for (int mt = 0; mt < 4; mt++) {
    int mx = -32768;
    for (int a = 0; a < 128; a++)
      for (int b = 0; b < 128; b++) mx = std::max(mx, (int) ctx->h_tab->pd[mt][a][b]);
    ctx->reach_from[mt] = (mx <= 0) ? (1 << 30) : std::max(0, (127 + mx - 1) / mx - 1);
    /* lower fills: the 16-bit corner profile ('N') against the 8-bit one
       (character code 4), for each query class (FillParams::lower_slack4) */
    int slack = 0;
    for (int k = 0; k < 5; k++) {
      const int q = "ACGTN"[k];
      slack = std::max(slack, (int) ctx->h_tab->pd[mt][q]['N'] - (int) ctx->h_tab->pd[mt][q][4]);
    }
    ctx->lower_slack[mt] = std::min(slack, 255);
  }
  ctx->packed_len = gdp_packed_len_of(ctx->h_tab);
  ctx->tab_mn = ctx->tab_mx = 0;
  for (int mt = 0; mt < 4; mt++)
    for (int a = 0; a < 128; a++)
      for (int b = 0; b < 128; b++) {
        ctx->tab_mn = std::min(ctx->tab_mn, (int) ctx->h_tab->pd[mt][a][b]);
        ctx->tab_mx = std::max(ctx->tab_mx, (int) ctx->h_tab->pd[mt][a][b]);
      }
  const char *pe = getenv("GDP_PACKED");   /* 0: every pair on the one-lane-per-register fill */
  if (pe && atoi(pe) == 0) ctx->packed_len = -1;
}

static int
set_err (gdp_ctx *ctx, const char *what, cudaError_t e) {
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  if (ctx) ctx->err = buf;
  return GDP_ERR_CUDA;
}

#define CK(ctx, call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return set_err((ctx), #call, e_); } while (0)

extern "C" const char *
gdp_version (void) {
  return GDP_VERSION;
}

static void
slot_release (Slot &sl) {
  if (sl.cs) cudaStreamSynchronize(sl.cs);
  sl.d.release();
  sl.h.release();
  sl.pairs.release(); sl.results.release(); sl.recs.release(); sl.total.release();
  sl.enc.release(); sl.enc_off.release(); sl.h_enc.release(); sl.h_encoff.release(); sl.enc_total.release();
  if (sl.h2d_done) cudaEventDestroy(sl.h2d_done);
  if (sl.comp_done) cudaEventDestroy(sl.comp_done);
  if (sl.out_done) cudaEventDestroy(sl.out_done);
  if (sl.total_ready) cudaEventDestroy(sl.total_ready);
  sl.h2d_done = sl.comp_done = sl.out_done = sl.total_ready = nullptr;
  sl.cs = nullptr;
  sl.scratch.release();
  sl.scratch8.release();
  sl.scratch_late.release();
}

extern "C" void
gdp_ctx_destroy (gdp_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->h2d) cudaStreamSynchronize(ctx->h2d);
  if (ctx->d2h) cudaStreamSynchronize(ctx->d2h);
  for (auto &t : ctx->timed) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
  for (int s = 0; s < NSLOTS; s++) slot_release(ctx->slot[s]);
  for (int k = 0; k < GDP_MAX_WAVE_STREAMS; k++)
    if (ctx->wave_stream[k]) {
      cudaStreamSynchronize(ctx->wave_stream[k]);
      cudaStreamDestroy(ctx->wave_stream[k]);
    }
  ctx->arena.release(); ctx->scratch.release(); ctx->scratch8.release(); ctx->scratch_late.release();
  gdpi_single_release(&ctx->single);
  if (ctx->d_tab) cudaFree(ctx->d_tab);
  if (ctx->d_genome) cudaFree(ctx->d_genome);
  if (ctx->d_genomealt) cudaFree(ctx->d_genomealt);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->h2d) cudaStreamDestroy(ctx->h2d);
  if (ctx->d2h) cudaStreamDestroy(ctx->d2h);
  for (int k = 0; k <= GDP_NSIDE; k++) {
    if (ctx->side[k]) cudaStreamDestroy(ctx->side[k]);
    if (ctx->join_ev[k]) cudaEventDestroy(ctx->join_ev[k]);
  }
  for (int w = 0; w < GDP_MAX_WAVE_STREAMS; w++)
    for (int k = 0; k <= GDP_NSIDE; k++)
      if (ctx->wave_side[w][k]) cudaStreamDestroy(ctx->wave_side[w][k]);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  free(ctx->h_tab);
  delete ctx;
}

extern "C" int
gdp_ctx_create (gdp_ctx **out, int device, int mode, int64_t budget) {
  *out = nullptr;
  if (mode < 0 || mode > 6) return GDP_ERR_PARAM;
  gdp_ctx *ctx = new gdp_ctx();
  ctx->device = device;
  ctx->budget = budget > 0 ? budget : (int64_t) 40 << 30;
  if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return GDP_ERR_CUDA; }
  cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device);
  bool ok = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming) == cudaSuccess;
  for (int k = 0; ok && k <= GDP_NSIDE; k++)
    ok = cudaStreamCreateWithFlags(&ctx->side[k], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&ctx->join_ev[k], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    gdp_ctx_destroy(ctx);
    return GDP_ERR_CUDA;
  }
  /* Wave streams, one per stream priority from the highest down: wave k of
     a batch computes on stream min(k, last), so when waves overlap the
     pending blocks of an older wave go before a younger wave's. */
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  ctx->nwave = std::max(1, std::min(GDP_MAX_WAVE_STREAMS, least - greatest + 1));
  for (int k = 0; k < ctx->nwave; k++) {
    ok = cudaStreamCreateWithPriority(&ctx->wave_stream[k], cudaStreamNonBlocking, greatest + k) == cudaSuccess;
    for (int q = 0; ok && q <= GDP_NSIDE; q++)
      ok = cudaStreamCreateWithPriority(&ctx->wave_side[k][q], cudaStreamNonBlocking, greatest + k) == cudaSuccess;
    if (!ok) {
      gdp_ctx_destroy(ctx);
      return GDP_ERR_CUDA;
    }
  }
  for (int s = 0; s < NSLOTS; s++) {
    Slot &sl = ctx->slot[s];
    cudaEventCreateWithFlags(&sl.h2d_done, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&sl.comp_done, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&sl.out_done, cudaEventDisableTiming);
    /* the copy-out thread sleeps on this one while the planner uses the cores */
    cudaEventCreateWithFlags(&sl.total_ready, cudaEventDisableTiming | cudaEventBlockingSync);
  }
  ctx->h_tab = (gdp_tables_t *) malloc(sizeof(gdp_tables_t));
  gdp_build_tables(ctx->h_tab, mode);
  update_reach(ctx);
  if (cudaMalloc(&ctx->d_tab, sizeof(gdp_tables_t)) != cudaSuccess ||
      cudaMemcpy(ctx->d_tab, ctx->h_tab, sizeof(gdp_tables_t), cudaMemcpyHostToDevice) != cudaSuccess) {
    gdp_ctx_destroy(ctx);
    return GDP_ERR_CUDA;
  }
  const char *w = getenv("GDP_WAVE_PAIRS");
  if (w && atol(w) > 0) ctx->wave = atol(w);
  const char *wx = getenv("GDP_WARP_MIN_X");
  if (wx && atoi(wx) > 0) ctx->warp_min_x = atoi(wx);
  ctx->plan_threads = (int) std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const char *pt = getenv("GDP_PLAN_THREADS");
  if (pt && atoi(pt) > 0) ctx->plan_threads = atoi(pt);
  const char *tw = getenv("GDP_TB_WARP");
  if (tw && *tw) ctx->tb_warp = atoi(tw) != 0;
  *out = ctx;
  return GDP_OK;
}

extern "C" int
gdp_debug_tables (int mode, int16_t *pd, uint8_t *cons, int8_t *nt2int) {
  if (mode < 0 || mode > 6) return GDP_ERR_PARAM;
  gdp_tables_t *t = (gdp_tables_t *) malloc(sizeof(gdp_tables_t));
  if (!t) return GDP_ERR_PARAM;
  gdp_build_tables(t, mode);
  if (pd) memcpy(pd, t->pd, sizeof(t->pd));
  if (cons) memcpy(cons, t->cons, sizeof(t->cons));
  if (nt2int) memcpy(nt2int, t->nt2int, sizeof(t->nt2int));
  free(t);
  return GDP_OK;
}

extern "C" const char *
gdp_last_error (gdp_ctx *ctx) {
  return ctx ? ctx->err.c_str() : "";
}

extern "C" int64_t
gdp_launch_count (gdp_ctx *ctx) {
  return ctx ? ctx->launches.load() : 0;
}

extern "C" void *
gdp_ctx_stream (gdp_ctx *ctx) {
  return (void *) ctx->stream;
}

extern "C" int
gdp_profile_enable (gdp_ctx *ctx, int on) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->profiling = on != 0;
  return GDP_OK;
}

static void
prof_collect (gdp_ctx *ctx) {
  if (ctx->timed.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  for (auto &t : ctx->timed) {
    float f = 0.f;
    cudaEventElapsedTime(&f, t.a, t.b);
    ctx->prof_ms[t.id] += f;
    ctx->prof_n[t.id] += 1;
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  ctx->timed.clear();
}

extern "C" int
gdp_profile_read (gdp_ctx *ctx, int id, char *name, int name_cap, double *ms, int64_t *launches) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (id < 0 || id >= NPROF) return GDP_ERR_PARAM;
  prof_collect(ctx);
  if (name && name_cap > 0) snprintf(name, name_cap, "%s", kernel_name(id));
  if (ms) *ms = ctx->prof_ms[id];
  if (launches) *launches = ctx->prof_n[id];
  return GDP_OK;
}

extern "C" int
gdp_profile_reset (gdp_ctx *ctx) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  prof_collect(ctx);
  for (int i = 0; i < 128; i++) { ctx->prof_ms[i] = 0; ctx->prof_n[i] = 0; }
  return GDP_OK;
}

/*
 * Integer issue-rate probe: every thread runs 16 independent dependency
 * chains of 32-bit add / min-max / multiply-add, so the SMs issue integer
 * lane-ops as fast as their pipes allow.  Used as the roofline denominator
 * of the integer-bound fill.  kind 0: add + min/max, kind 1: multiply-add,
 * kind 2: both interleaved.  Each chain step counts as 2 lane-ops.
 */
__global__ void __launch_bounds__(256)
int_peak_kernel (int *out, int iters, int kind, int seed) {
  int a[16];
#pragma unroll
  for (int k = 0; k < 16; k++) a[k] = seed + k * 7 + threadIdx.x;
  const int b = seed | 1, c = seed ^ 0x5a5a;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      if (kind == 0) {
        a[k] = max(a[k] + b, c - k);
      } else if (kind == 1) {
        a[k] = a[k] * b + c;
        a[k] = a[k] * c + b;
      } else {
        if (k & 1) a[k] = max(a[k] + b, c - k);
        else { a[k] = a[k] * b + c; a[k] = a[k] * c + b; }
      }
    }
  }
  int s = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) s ^= a[k];
  if (s == 0x7fffffff) out[0] = s;
}

/* Returns integer lane-ops per second of the fastest probe kind. */
extern "C" double
gdp_measure_int_peak (gdp_ctx *ctx) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  int *d = nullptr;
  if (cudaMalloc(&d, 4) != cudaSuccess) return 0.0;
  const int blocks = ctx->nsm * 8, threads = 256, iters = 4096;
  double best = 0.0;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  for (int kind = 0; kind < 3; kind++) {
    for (int rep = 0; rep < 3; rep++) {
      cudaEventRecord(a, ctx->stream);
      int_peak_kernel<<<blocks, threads, 0, ctx->stream>>>(d, iters, kind, 12345 + rep);
      cudaEventRecord(b, ctx->stream);
      cudaEventSynchronize(b);
      ctx->launches++;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      const double ops = (double) blocks * threads * iters * 16 * 2;
      if (ms > 0 && ops / (ms * 1e-3) > best) best = ops / (ms * 1e-3);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  return best;
}

extern "C" int
gdp_sync (gdp_ctx *ctx) {
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GDP_OK;
}

extern "C" int
gdp_set_genome (gdp_ctx *ctx, const uint32_t *blocks, const uint32_t *altblocks, uint64_t len) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  size_t words = (size_t) ((len + 31) / 32) * 3;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->d_genome) cudaFree(ctx->d_genome);
  if (ctx->d_genomealt) cudaFree(ctx->d_genomealt);
  ctx->d_genome = ctx->d_genomealt = nullptr;
  ctx->genome_len = 0;
  CK(ctx, cudaMalloc(&ctx->d_genome, words * 4));
  CK(ctx, cudaMemcpy(ctx->d_genome, blocks, words * 4, cudaMemcpyHostToDevice));
  if (altblocks) {
    CK(ctx, cudaMalloc(&ctx->d_genomealt, words * 4));
    CK(ctx, cudaMemcpy(ctx->d_genomealt, altblocks, words * 4, cudaMemcpyHostToDevice));
  }
  ctx->genome_len = len;
  return GDP_OK;
}

/* ------------------------------------------------------------------ */
/* Planning                                                            */
/* ------------------------------------------------------------------ */

static int
validate (const gdp_pair_t &p, int64_t arena_bytes, uint64_t genome_len) {
  if (p.variant < GDP_FULL || p.variant > GDP_LOWER) return GDP_ERR_PARAM;
  if (p.precision != 8 && p.precision != 16) return GDP_ERR_PARAM;
  if (p.mismatchtype < 0 || p.mismatchtype > 3) return GDP_ERR_PARAM;
  if (p.open < -127 || p.open > 0 || p.extend < -127 || p.extend > 0) return GDP_ERR_PARAM;
  if (p.genestrand < 0 || p.genestrand > 2) return GDP_ERR_PARAM;
  if ((p.xflags & ~(GDP_XFLAG_SEGMENT | GDP_XFLAG_SEGMENT_REV)) ||
      (p.xflags & (GDP_XFLAG_SEGMENT | GDP_XFLAG_SEGMENT_REV)) == (GDP_XFLAG_SEGMENT | GDP_XFLAG_SEGMENT_REV))
    return GDP_ERR_PARAM;
  if (p.rlength <= 0 || p.glength <= 0 || p.rlength > (1 << 20) || p.glength > (1 << 20)) return GDP_ERR_LEN;
  if (p.lband < 0 || p.uband < 0) return GDP_ERR_BAND;
  if (arena_bytes >= 0) {
    if (p.rseq < 0 || p.rseq + p.rlength > arena_bytes || p.rseq_uc < 0 || p.rseq_uc + p.rlength > arena_bytes ||
        p.gseq < 0 || p.gseq + p.glength > arena_bytes || p.gseq_alt < 0 || p.gseq_alt + p.glength > arena_bytes)
      return GDP_ERR_LEN;
  }
  if (p.flags & GDP_FLAG_TRACEBACK) {
    if (p.tb_r < 0 || p.tb_c < 0 || p.tb_r > p.rlength || p.tb_c > p.glength) return GDP_ERR_BAND;
  }
  if (p.flags & (GDP_FLAG_ENDPOINT | GDP_FLAG_ENDPOINT_QEND)) {
    /* the end-gap searches scan an upper and a lower fill at the pair's
       own precision */
    if (p.variant == GDP_FULL || (p.flags & GDP_FLAG_RERUN16) ||
        ((p.flags & GDP_FLAG_ENDPOINT) && (p.flags & GDP_FLAG_ENDPOINT_QEND)))
      return GDP_ERR_PARAM;
  }
  if (p.flags & GDP_FLAG_GWINDOW) {
    /* the window's positions inside [chroffset, chrhigh) must be resident */
    const int64_t g0 = (p.flags & GDP_FLAG_REVP) ? (int64_t) p.genomeoffset - (p.glength - 1) : p.genomeoffset;
    const int64_t g1 = g0 + p.glength - 1;
    int64_t lo, hi;
    if (p.watsonp) { lo = (int64_t) p.chroffset + g0; hi = (int64_t) p.chroffset + g1; }
    else { lo = (int64_t) p.chrhigh - g1; hi = (int64_t) p.chrhigh - g0; }
    if (p.xflags & GDP_XFLAG_SEGMENT) {
      /* Genome_get_segment_right stars positions at and above chrhigh,
         Genome_get_segment_left those below chroffset */
      if (p.watsonp) hi = std::min<int64_t>(hi, (int64_t) p.chrhigh - 1);
      else lo = std::max<int64_t>(lo, p.chroffset);
    } else if (p.xflags & GDP_XFLAG_SEGMENT_REV) {
      /* the mirrored segment: left on the plus strand, right on the minus */
      if (p.watsonp) lo = std::max<int64_t>(lo, p.chroffset);
      else hi = std::min<int64_t>(hi, (int64_t) p.chrhigh - 1);
    } else {
      lo = std::max<int64_t>(lo, p.chroffset);
      hi = std::min<int64_t>(hi, (int64_t) p.chrhigh - 1);
    }
    if (lo <= hi && lo < 0) return GDP_ERR_NOGENOME;
    if (genome_len == 0 || (lo <= hi && (uint64_t) hi >= genome_len)) return GDP_ERR_NOGENOME;
  }
  return GDP_OK;
}

/* Sort key of a pair's fill inside its kind (25 bits): wider bands first,
   inside one band width (lband + uband) by lband, and then longer pairs
   first (more lanes, so more blocks, and with them about as many swept
   columns).  Threads that share the band width and run the same block in lock
   step are in the same column phase at the same step: the phase of the j-th
   swept column of a block depends on j and lband + uband only, while the
   sweep is not cut at column 0.  The sweeps of the first blocks are cut at
   column 0 by lband, so pairs of one lband stay in phase there too. */
static inline uint32_t
work_key (const gdp_pair_t &p, int W) {
  gdp_geom_t g;
  gdp_geom_of(&p, W, &g);
  const int lanes = std::min(511, g.X);
  const int lb = (p.variant == GDP_FULL) ? p.lband : 0;
  const int band = std::min(255, lb + g.band_hi);
  return (uint32_t) (255 - band) << 17 | (uint32_t) std::min(255, lb) << 9 | (uint32_t) (511 - lanes);
}
#define KEY_KIND_SHIFT 25   /* sort key = kind << 25 | work key */
#define KEY_GROUP_SHIFT 17  /* entries with equal key >> 17 share kind and band width: the padded groups
                               (sorted by lband inside, so most warps hold one lband without the padding
                               of a group per lband) */
#define KEY_BITS 32         /* kinds below 128 */

/* Kinds whose warps are padded to pairs of one band width: the 16-bit
   one-thread-per-pair fills, which run phase-specialised columns. */
static inline bool
padded_kind (int k) {
  return k < NTHREADKINDS && ((k >> 2) / 3) == 0;
}

/* Runs f(lo, hi, t) over [0, n) split into `nt` contiguous chunks, one
   pool thread per chunk. */
template <class F>
static void
parallel_chunks (WorkPool &pool, int64_t n, int nt, F f) {
  pool.run(nt, [&](int t) { f(n * t / nt, n * (t + 1) / nt, t); });
}

/* Stable LSD radix sort of (key, value)[0..n) by the low KEY_BITS bits of key,
   11 bits per pass, `nt` pool threads (per-thread histograms, then each
   thread scatters its own chunk in order).  k2/v2 are scratch of n. */
static void
radix_sort (WorkPool &pool, uint32_t *key, int32_t *val, uint32_t *k2, int32_t *v2, int64_t n, int nt) {
  constexpr int B = 2048;
  uint32_t *const key0 = key;
  int32_t *const val0 = val;
  std::vector<int64_t> hist((size_t) nt * B);
  for (int shift = 0; shift < KEY_BITS; shift += 11) {
    std::fill(hist.begin(), hist.end(), 0);
    parallel_chunks(pool, n, nt, [&](int64_t lo, int64_t hi, int t) {
      int64_t *h = hist.data() + (size_t) t * B;
      for (int64_t i = lo; i < hi; i++) h[(key[i] >> shift) & (B - 1)]++;
    });
    int64_t sum = 0;
    for (int d = 0; d < B; d++)
      for (int t = 0; t < nt; t++) {
        const int64_t c = hist[(size_t) t * B + d];
        hist[(size_t) t * B + d] = sum;
        sum += c;
      }
    parallel_chunks(pool, n, nt, [&](int64_t lo, int64_t hi, int t) {
      int64_t *h = hist.data() + (size_t) t * B;
      for (int64_t i = lo; i < hi; i++) {
        const int64_t at = h[(key[i] >> shift) & (B - 1)]++;
        k2[at] = key[i];
        v2[at] = val[i];
      }
    });
    std::swap(key, k2);
    std::swap(val, v2);
  }
  /* an odd number of passes leaves the sorted data in the scratch arrays */
  if (key != key0) {
    parallel_chunks(pool, n, nt, [&](int64_t lo, int64_t hi, int) {
      memcpy(key0 + lo, key + lo, (size_t) (hi - lo) * sizeof(uint32_t));
      memcpy(val0 + lo, val + lo, (size_t) (hi - lo) * sizeof(int32_t));
    });
  }
}

/* Fills ph for pairs[0..n) (pinned host buffers).  arena_bytes < 0 skips the
   arena bound checks (device-resident callers). */
static int
plan_build (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t n, int64_t arena_bytes, PlanHost &ph) {
  ph.n = n;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = ph.meta.ensure(std::max<int64_t>(n, 1) * sizeof(gdp_meta_t));
  if (e == cudaSuccess) e = ph.status.ensure(std::max<int64_t>(n, 1) * sizeof(int32_t));
  if (e == cudaSuccess) e = ph.rec_off.ensure(std::max<int64_t>(n, 1) * sizeof(int64_t));
  if (e != cudaSuccess) return set_err(ctx, "pinned plan buffers", e);
  gdp_meta_t *meta = ph.meta.as<gdp_meta_t>();
  int32_t *status = ph.status.as<int32_t>();
  int64_t *rec_off = ph.rec_off.as<int64_t>();
  const int nt = (int) std::max<int64_t>(1, std::min<int64_t>(ctx->plan_threads, n / 8192));
  /* per chunk: sums of direction words, record slots, fill entries,
     tracebacks, device windows, and the largest swept dimension per kind */
  struct Chunk { int64_t words = 0, recs = 0, entries = 0, ntb = 0, nwindow = 0; int maxY[NKINDS] = {0}, maxMin[NKINDS] = {0}; };
  std::vector<Chunk> ch(nt);
  uint32_t *k16 = grow(ph.k16, n), *k8 = grow(ph.k8, n);   /* fill keys of each pair (~0u: none) */
  const uint64_t glen = ctx->genome_len;
  /* pass 1: validate, route, size (meta.dir16 / dir8 and rec_off hold sizes) */
  parallel_chunks(ctx->pool, n, nt, [&](int64_t lo, int64_t hi, int t) {
    Chunk &c = ch[t];
    for (int64_t i = lo; i < hi; i++) {
      const gdp_pair_t &p = pairs[i];
      gdp_meta_t &m = meta[i];
      m.dir16 = m.dir8 = -1;
      m.maxh16 = -32768; m.status8 = 0; m.final8 = 0; m.final16 = 0;
      rec_off[i] = 0;
      k16[i] = k8[i] = ~0u;
      const int st = validate(p, arena_bytes, glen);
      status[i] = st;
      if (st != GDP_OK) continue;
      if (p.flags & GDP_FLAG_GWINDOW) c.nwindow++;
      const int late = (p.flags & GDP_FLAG_JUMP_LATE) ? 1 : 0;
      const bool rerun = p.precision == 8 && (p.flags & GDP_FLAG_RERUN16);
      const int Y = (p.variant == GDP_LOWER) ? p.rlength : p.glength;
      if (p.precision == 16 || rerun) {
        gdp_geom_t g16;
        gdp_geom_of(&p, 16, &g16);
        const int sweep = 15 + g16.band_hi + (p.variant == GDP_FULL ? p.lband : 0);
        int k = kind_id(0, p.variant, late, rerun ? 1 : 0);
        const bool endpoint = (p.flags & (GDP_FLAG_ENDPOINT | GDP_FLAG_ENDPOINT_QEND)) != 0;
        if (!rerun && !endpoint && g16.X >= ctx->warp_min_x) {   /* endpoint searches: one thread per pair */
          if (sweep <= ctx->warp_max_sweep) {
            /* the smallest lane group whose blocks do not overlap in time */
            int kg = 2;
            for (int q = 0; q < 2; q++)
              if (sweep <= WARP_K[q] * 17 - ctx->group_slack) { kg = q; break; }
            k = warp_kind_id(p.variant, late, kg);
          } else {
            /* enough lanes that a lane's next block starts after its last one ends */
            for (int nwi = 0; nwi < 4; nwi++) {
              if (sweep + 16 < CTA_NW[nwi] * 32 * 17 - 16) { k = cta_kind_id(p.variant, late, nwi); break; }
            }
          }
        }
        m.dir16 = (gdp_pair_words(&p, 16) + 3) & ~(int64_t) 3;   /* keep pairs 16-byte aligned */
        c.words += m.dir16;
        k16[i] = (uint32_t) k << KEY_KIND_SHIFT | work_key(p, 16);
        c.entries++;
        c.maxY[k] = std::max(c.maxY[k], Y);
        c.maxMin[k] = std::max(c.maxMin[k], std::min(p.rlength, p.glength));
      }
      if (p.precision == 8) {
        int k = kind_id(1, p.variant, late, rerun ? 1 : 0);
        gdp_geom_t g8;
        gdp_geom_of(&p, 32, &g8);
        if (rerun && (ctx->check_groups || g8.X >= ctx->check_min_x)) {
          /* the 8-bit pass runs for few pairs, and its time is that of the
             longest: lane groups give a long pair K lanes */
          const int sweep8 = 31 + g8.band_hi + (p.variant == GDP_FULL ? p.lband : 0);
          for (int q = 0; q < 3; q++)
            if (sweep8 <= WARP8_K[q] * 33 - ctx->group_slack) { k = warp8_kind_id(p.variant, late, q); break; }
        } else if (rerun && std::min(p.rlength, p.glength) < ctx->reach_from[p.mismatchtype & 3]) {
          /* no score of this pair can reach 127 (a score is at most
             min(r, c) times the largest table entry), so its 8-bit pass
             does not wait for the 16-bit pass: it runs beside it */
          k = early8_kind_id(p.variant, late);
        }
        m.dir8 = (gdp_pair_words(&p, 32) + 3) & ~(int64_t) 3;
        c.words += m.dir8;
        k8[i] = (uint32_t) k << KEY_KIND_SHIFT | work_key(p, 32);
        c.entries++;
        c.maxY[k] = std::max(c.maxY[k], Y);
        c.maxMin[k] = std::max(c.maxMin[k], std::min(p.rlength, p.glength));
      }
      if (p.flags & GDP_FLAG_TRACEBACK) {
        rec_off[i] = (int64_t) p.rlength + p.glength + 2;
        c.recs += rec_off[i];
        c.ntb++;
      }
    }
  });
  /* chunk bases */
  std::vector<int64_t> wbase(nt), rbase(nt), ebase(nt), tbase(nt);
  int64_t words = 0, recs = 0, entries = 0, ntb = 0, nwindow = 0;
  int maxY[NKINDS] = {0};
  int maxMin[NKINDS] = {0};   /* per kind: the largest min(rlength, glength) */
  for (int t = 0; t < nt; t++) {
    wbase[t] = words; rbase[t] = recs; ebase[t] = entries; tbase[t] = ntb;
    words += ch[t].words; recs += ch[t].recs; entries += ch[t].entries; ntb += ch[t].ntb;
    nwindow += ch[t].nwindow;
    for (int k = 0; k < NKINDS; k++) {
      maxY[k] = std::max(maxY[k], ch[t].maxY[k]);
      maxMin[k] = std::max(maxMin[k], ch[t].maxMin[k]);
    }
  }
  /* pass 2: sizes to offsets, fill entries in pair order */
  uint32_t *keys = grow(ph.keys, entries);
  int32_t *vals = grow(ph.vals, entries);
  int32_t *tbl = grow(ph.tbl, ntb);
  parallel_chunks(ctx->pool, n, nt, [&](int64_t lo, int64_t hi, int t) {
    int64_t w = wbase[t], r = rbase[t], en = ebase[t], tb = tbase[t];
    for (int64_t i = lo; i < hi; i++) {
      if (status[i] != GDP_OK) continue;
      gdp_meta_t &m = meta[i];
      if (m.dir16 >= 0) { const int64_t sz = m.dir16; m.dir16 = w; w += sz; }
      if (m.dir8 >= 0) { const int64_t sz = m.dir8; m.dir8 = w; w += sz; }
      if (k16[i] != ~0u) { keys[en] = k16[i]; vals[en] = (int32_t) i; en++; }
      if (k8[i] != ~0u) { keys[en] = k8[i]; vals[en] = (int32_t) i; en++; }
      if (pairs[i].flags & GDP_FLAG_TRACEBACK) {
        const int64_t sz = rec_off[i];
        rec_off[i] = r;
        r += sz;
        tbl[tb++] = (int32_t) i;
      }
    }
  });
  static_assert(NKINDS < (1 << (KEY_BITS - KEY_KIND_SHIFT)), "kind ids fit in the sort key");
  radix_sort(ctx->pool, keys, vals, grow(ph.keys2, entries), grow(ph.vals2, entries), entries, nt);
  /* padded kinds: every band-width group starts a warp (-1 = no pair) */
  int64_t groups = 0;
  for (int64_t i = 0; i < entries; i++) {
    const bool group_end = (i + 1 == entries) || (keys[i + 1] >> KEY_GROUP_SHIFT) != (keys[i] >> KEY_GROUP_SHIFT);
    if (group_end && padded_kind((int) (keys[i] >> KEY_KIND_SHIFT))) groups++;
  }
  e = ph.lists.ensure((size_t) std::max<int64_t>(entries + 31 * groups + ntb, 1) * sizeof(int32_t));
  if (e != cudaSuccess) return set_err(ctx, "pinned plan lists", e);
  int32_t *lists = ph.lists.as<int32_t>();
  int64_t pos = 0, ei = 0;
  for (int k = 0; k < NKINDS; k++) {
    ph.start[k] = pos;
    const bool pad = padded_kind(k);
    while (ei < entries && (int) (keys[ei] >> KEY_KIND_SHIFT) == k) {
      lists[pos++] = vals[ei];
      if (pad && ((ei + 1 == entries) || (keys[ei + 1] >> KEY_GROUP_SHIFT) != (keys[ei] >> KEY_GROUP_SHIFT)))
        while ((pos - ph.start[k]) & 31) lists[pos++] = -1;
      ei++;
    }
    ph.counts[k] = (int32_t) (pos - ph.start[k]);
    ph.maxY[k] = maxY[k];
    ph.maxMin[k] = maxMin[k];
  }
  ph.start[NKINDS] = pos;
  ph.counts[NKINDS] = (int32_t) ntb;
  /* the traceback list: jump-late pairs first (each part in pair order), so
     that each fill chain can trace its own pairs back */
  int64_t nlate = 0;
  for (int64_t t = 0; t < ntb; t++)
    if (pairs[tbl[t]].flags & GDP_FLAG_JUMP_LATE) lists[pos + nlate++] = tbl[t];
  for (int64_t t = 0, e2 = nlate; t < ntb; t++)
    if (!(pairs[tbl[t]].flags & GDP_FLAG_JUMP_LATE)) lists[pos + e2++] = tbl[t];
  ph.counts[NKINDS + 1] = (int32_t) nlate;
  ph.counts[NKINDS + 2] = (int32_t) (ntb - nlate);
  pos += ntb;
  ph.start[NKINDS + 1] = pos;
  ph.nlists = pos;
  ph.dir_words = words;
  ph.total_recs = recs;
  ph.nwindow = nwindow;
  return GDP_OK;
}

/* Device buffers for ph and the async upload of the plan on stream s. */
static int
plan_upload (gdp_ctx *ctx, const PlanHost &ph, PlanDev &pd, bool hdump, cudaStream_t s) {
  const int64_t n = std::max<int64_t>(ph.n, 1);
  const size_t nl = (size_t) std::max<int64_t>(ph.nlists, 1);
  CK(ctx, pd.lists.ensure(nl * sizeof(int32_t)));
  CK(ctx, pd.work.ensure(nl * sizeof(int32_t)));
  CK(ctx, pd.counts.ensure((NKINDS + 3) * sizeof(int32_t)));
  CK(ctx, pd.work_counts.ensure(NKINDS * sizeof(int32_t)));
  CK(ctx, pd.status.ensure(n * sizeof(int32_t)));
  CK(ctx, pd.meta0.ensure(n * sizeof(gdp_meta_t)));
  CK(ctx, pd.meta.ensure(n * sizeof(gdp_meta_t)));
  CK(ctx, pd.rec_off.ensure(n * sizeof(int64_t)));
  CK(ctx, pd.dirs.ensure(std::max<int64_t>(ph.dir_words, 4) * sizeof(uint32_t)));
  CK(ctx, pd.total.ensure(sizeof(int64_t)));
  if (hdump) CK(ctx, pd.hdump.ensure(std::max<int64_t>(ph.dir_words, 4) * 8 * sizeof(int16_t)));
  if (ph.nlists > 0)
    CK(ctx, cudaMemcpyAsync(pd.lists.p, ph.lists.p, ph.nlists * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(pd.counts.p, ph.counts, (NKINDS + 3) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (ph.n > 0) {
    CK(ctx, cudaMemcpyAsync(pd.status.p, ph.status.p, ph.n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CK(ctx, cudaMemcpyAsync(pd.meta0.p, ph.meta.p, ph.n * sizeof(gdp_meta_t), cudaMemcpyHostToDevice, s));
    CK(ctx, cudaMemcpyAsync(pd.rec_off.p, ph.rec_off.p, ph.n * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  }
  return GDP_OK;
}

extern "C" void
gdp_plan_destroy (gdp_plan *pl) {
  if (!pl) return;
  if (pl->gexec) cudaGraphExecDestroy(pl->gexec);
  pl->d.release();
  pl->h.release();
  delete pl;
}

extern "C" int
gdp_plan_create (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t npairs, gdp_plan **plan) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  gdp_plan *pl = new gdp_plan();
  int rc = plan_build(ctx, pairs, npairs, -1, pl->h);
  if (rc == GDP_OK) rc = plan_upload(ctx, pl->h, pl->d, false, ctx->stream);
  if (rc == GDP_OK) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = set_err(ctx, "plan upload", e);
  }
  if (rc != GDP_OK) {
    gdp_plan_destroy(pl);
    return rc;
  }
  *plan = pl;
  return GDP_OK;
}

extern "C" int64_t gdp_plan_total_recs (const gdp_plan *pl) { return pl->h.total_recs; }
extern "C" int64_t gdp_plan_rec_offset (const gdp_plan *pl, int64_t i) { return pl->h.rec_off.as<int64_t>()[i]; }
extern "C" int64_t gdp_plan_dir_bytes (const gdp_plan *pl) { return pl->h.dir_words * 4; }

/* ------------------------------------------------------------------ */
/* Execution                                                           */
/* ------------------------------------------------------------------ */

/* Zeroed results, the planner's metadata copied to the working copy, and
   the 8-bit pass counters cleared: all on the SMs, so that no copy engine
   (busy with another wave's records) sits on the compute stream. */
__global__ void
init_results_kernel (gdp_result_t *res, const int32_t *status, const gdp_pair_t *pairs, int64_t n,
                     const gdp_meta_t *meta0, gdp_meta_t *meta, int32_t *work_counts, int nwork) {
  if (blockIdx.x == 0 && (int) threadIdx.x < nwork) work_counts[threadIdx.x] = 0;
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
    meta[i] = meta0[i];
    gdp_result_t r;
    r.status = status[i];
    r.score = 0;
    r.precision = pairs[i].precision;
    r.rerun = 0;
    r.tb_score = r.nmatches = r.nmismatches = r.nopens = r.nindels = 0;
    r.nrecs = 0;
    r.rec_offset = 0;
    r.end_score = r.end_r = r.end_c = r.end_found = 0;
    res[i] = r;
  }
}

__global__ void
gather_nrecs_kernel (const gdp_result_t *res, int64_t n, int64_t *out) {
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
    out[i] = res[i].nrecs;
}

/* Copies each pair's records from its slot range to the dense position
   given by the exclusive scan (one warp per pair), points the pair's
   result at it (offset relative to the batch), and writes the total. */
__global__ void
compact_records_kernel (gdp_result_t *res, const int64_t *slot_off, const gdp_rec_t *slots,
                        const int64_t *scan, int64_t n, gdp_rec_t *out, int64_t *total, int64_t *total_host) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  for (int64_t i = warp; i < n; i += nwarps) {
    const int nr = res[i].nrecs;
    const int64_t dst = scan[i];
    /* the pair's records as one run of 32-bit words, so a warp's stores
       are contiguous */
    static_assert(sizeof(gdp_rec_t) % 4 == 0, "records are whole words");
    constexpr int RW = sizeof(gdp_rec_t) / 4;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(slots + slot_off[i]);
    uint32_t *to = reinterpret_cast<uint32_t *>(out + dst);
    for (int k = lane; k < nr * RW; k += 32) to[k] = src[k];
    if (lane == 0) {
      res[i].rec_offset = dst;
      if (i == n - 1) {
        *total = dst + nr;
        if (total_host) {
          *(volatile int64_t *) total_host = dst + nr;
          __threadfence_system();
        }
      }
    }
  }
}

/* A thread-per-pair kind.  Full-band 16-bit plain fills and 16-bit passes
   run the packed fill first; the one-lane-per-register kernel follows only
   when the kind holds pairs too long for it (their scores could pass the
   packed range). */
template <int W, int V, bool L, int M>
static int launch_fill (FillParams P, int grid, cudaStream_t s, int max_min_len) {
  if constexpr (W == 16 && V == GDP_FULL && M != 2) {
    if (P.packed_len >= 0) {
      fill_packed_kernel<L, M><<<grid, 128, 0, s>>>(P);
      if (max_min_len <= P.packed_len) return 1;
      fill_thread_kernel<W, V, L, M><<<grid, 128, 0, s>>>(P);
      return 2;
    }
  }
  fill_thread_kernel<W, V, L, M><<<grid, 128, 0, s>>>(P);
  return 1;
}

/* Returns the number of kernels launched. */
static int
launch_kind (int k, FillParams P, int grid, cudaStream_t s, int max_min_len) {
  const int pass = k & 1, late = (k >> 1) & 1, vw = k >> 2, variant = vw % 3, w32 = vw / 3;
#define GDP_CASE(W32, VAR, LATE)                                                                   \
  if (w32 == W32 && variant == VAR && late == LATE) {                                             \
    if (W32) return pass ? launch_fill<32, VAR, LATE, 2>(P, grid, s, max_min_len) : launch_fill<32, VAR, LATE, 0>(P, grid, s, max_min_len); \
    return pass ? launch_fill<16, VAR, LATE, 1>(P, grid, s, max_min_len) : launch_fill<16, VAR, LATE, 0>(P, grid, s, max_min_len);          \
  }
  GDP_CASE(0, 0, false) GDP_CASE(0, 0, true) GDP_CASE(0, 1, false) GDP_CASE(0, 1, true)
  GDP_CASE(0, 2, false) GDP_CASE(0, 2, true) GDP_CASE(1, 0, false) GDP_CASE(1, 0, true)
  GDP_CASE(1, 1, false) GDP_CASE(1, 1, true) GDP_CASE(1, 2, false) GDP_CASE(1, 2, true)
#undef GDP_CASE
  return 0;
}

/* Grid cap of the fill and traceback kernels: k blocks per SM, or fewer
   under the context's grid_limit (a footprint cap that leaves SMs' block
   slots to other contexts' kernels: the grid-stride kernels then take more
   items per block). */
static inline int64_t
grid_cap (const gdp_ctx *ctx, int k) {
  return (int64_t) ctx->nsm * (ctx->grid_limit > 0 ? std::min(k, ctx->grid_limit) : k);
}

static inline int
fill_grid (gdp_ctx *ctx, int64_t count) {
  return (int) std::max<int64_t>(1, std::min<int64_t>((count + 127) / 128, grid_cap(ctx, 16)));
}

/* warp kinds: K lanes per pair, 128 / K pairs per block of 128 */
static inline int
warp_grid (gdp_ctx *ctx, int64_t count, int K) {
  const int per_block = 128 / K;
  return (int) std::max<int64_t>(1, std::min<int64_t>((count + per_block - 1) / per_block, grid_cap(ctx, 16)));
}

template <int V, bool L>
static void launch_cta (int nwi, FillParams P, int grid, cudaStream_t s) {
  switch (CTA_NW[nwi]) {
  case 2: fill_cta_kernel<V, L, 2><<<grid, 64, 0, s>>>(P); break;
  case 4: fill_cta_kernel<V, L, 4><<<grid, 128, 0, s>>>(P); break;
  case 8: fill_cta_kernel<V, L, 8><<<grid, 256, 0, s>>>(P); break;
  default: fill_cta_kernel<V, L, 16><<<grid, 512, 0, s>>>(P); break;
  }
}

static void
launch_cta_kind (int k, FillParams P, int grid, cudaStream_t s) {
  const int c = k - FIRST_CTA, vl = c / 4, variant = vl / 2, late = vl & 1, nwi = c % 4;
  if (variant == GDP_FULL) { if (late) launch_cta<GDP_FULL, true>(nwi, P, grid, s); else launch_cta<GDP_FULL, false>(nwi, P, grid, s); }
  else if (variant == GDP_UPPER) { if (late) launch_cta<GDP_UPPER, true>(nwi, P, grid, s); else launch_cta<GDP_UPPER, false>(nwi, P, grid, s); }
  else { if (late) launch_cta<GDP_LOWER, true>(nwi, P, grid, s); else launch_cta<GDP_LOWER, false>(nwi, P, grid, s); }
}

template <int V, bool L>
static void launch_warp (int kg, FillParams P, int grid, cudaStream_t s) {
  switch (WARP_K[kg]) {
  case 8: fill_warp_kernel<V, L, 8><<<grid, 128, 0, s>>>(P); break;
  case 16: fill_warp_kernel<V, L, 16><<<grid, 128, 0, s>>>(P); break;
  default: fill_warp_kernel<V, L, 32><<<grid, 128, 0, s>>>(P); break;
  }
}

template <int V, bool L>
static void launch_warp8 (int kg, FillParams P, int grid, cudaStream_t s) {
  switch (WARP8_K[kg]) {
  case 4: fill_warp_kernel<V, L, 4, 32, 2><<<grid, 128, 0, s>>>(P); break;
  case 8: fill_warp_kernel<V, L, 8, 32, 2><<<grid, 128, 0, s>>>(P); break;
  default: fill_warp_kernel<V, L, 16, 32, 2><<<grid, 128, 0, s>>>(P); break;
  }
}

static void
launch_warp8_kind (int k, FillParams P, int grid, cudaStream_t s) {
  const int c = k - FIRST_WARP8, vl = c / 3, variant = vl / 2, late = vl & 1, kg = c % 3;
  if (variant == GDP_FULL) { if (late) launch_warp8<GDP_FULL, true>(kg, P, grid, s); else launch_warp8<GDP_FULL, false>(kg, P, grid, s); }
  else if (variant == GDP_UPPER) { if (late) launch_warp8<GDP_UPPER, true>(kg, P, grid, s); else launch_warp8<GDP_UPPER, false>(kg, P, grid, s); }
  else { if (late) launch_warp8<GDP_LOWER, true>(kg, P, grid, s); else launch_warp8<GDP_LOWER, false>(kg, P, grid, s); }
}

/* the 8-bit pass of rerun pairs that cannot reach 127, one thread per pair,
   beside the 16-bit pass */
static void
launch_early8_kind (int k, FillParams P, int grid, cudaStream_t s) {
  const int c = k - FIRST_EARLY8, variant = c / 2, late = c & 1;
  if (variant == GDP_FULL) { if (late) launch_fill<32, GDP_FULL, true, 2>(P, grid, s, 0); else launch_fill<32, GDP_FULL, false, 2>(P, grid, s, 0); }
  else if (variant == GDP_UPPER) { if (late) launch_fill<32, GDP_UPPER, true, 2>(P, grid, s, 0); else launch_fill<32, GDP_UPPER, false, 2>(P, grid, s, 0); }
  else { if (late) launch_fill<32, GDP_LOWER, true, 2>(P, grid, s, 0); else launch_fill<32, GDP_LOWER, false, 2>(P, grid, s, 0); }
}

static void
launch_warp_kind (int k, FillParams P, int grid, cudaStream_t s) {
  const int c = k - NTHREADKINDS, vl = c / 3, variant = vl / 2, late = vl & 1, kg = c % 3;
  if (variant == GDP_FULL) { if (late) launch_warp<GDP_FULL, true>(kg, P, grid, s); else launch_warp<GDP_FULL, false>(kg, P, grid, s); }
  else if (variant == GDP_UPPER) { if (late) launch_warp<GDP_UPPER, true>(kg, P, grid, s); else launch_warp<GDP_UPPER, false>(kg, P, grid, s); }
  else { if (late) launch_warp<GDP_LOWER, true>(kg, P, grid, s); else launch_warp<GDP_LOWER, false>(kg, P, grid, s); }
}

/* The traceback launch over the plan's traceback list on stream ks: part 0
   the whole list, 1 its jump-late pairs, 2 its jump-early pairs. */
static int
launch_traceback (gdp_ctx *ctx, const PlanHost &ph, PlanDev &pd, const gdp_pair_t *d_pairs, const char *d_arena,
                  gdp_result_t *d_res, gdp_rec_t *d_slots, cudaStream_t ks, int part = 0) {
  const int64_t count = ph.counts[NKINDS + part];
  if (count <= 0) return GDP_OK;
  TbParams T;
  T.pairs = d_pairs; T.arena = d_arena;
  T.list = pd.lists.as<int32_t>() + ph.start[NKINDS] + (part == 2 ? ph.counts[NKINDS + 1] : 0);
  T.count = pd.counts.as<int32_t>() + NKINDS + part;
  T.dirs = pd.dirs.as<uint32_t>(); T.meta = pd.meta.as<gdp_meta_t>(); T.res = d_res; T.recs = d_slots;
  T.rec_off = pd.rec_off.as<int64_t>();
  T.genome = ctx->d_genome; T.genomealt = ctx->d_genomealt;
  T.genome_base = 0;
  T.genome_len = ctx->genome_len;
  T.tab = ctx->d_tab;
  cudaEvent_t ev = nullptr;
  prof_begin(ctx, &ev, ks);
  if (ctx->tb_warp) {
    const int g = (int) std::max<int64_t>(1, std::min<int64_t>((count + 3) / 4, grid_cap(ctx, 16)));
    traceback_warp_kernel<<<g, 128, 0, ks>>>(T);
  } else {
    traceback_kernel<<<fill_grid(ctx, count), 128, 0, ks>>>(T);
  }
  prof_end(ctx, PROF_TB, ev, ks);
  ctx->launches++;
  CK(ctx, cudaGetLastError());
  return GDP_OK;
}

/* Enqueues fills and tracebacks of a planned batch on the compute stream.
   d_slots receives records at the plan's slot offsets. */
static int
plan_run (gdp_ctx *ctx, const PlanHost &ph, PlanDev &pd, const gdp_pair_t *d_pairs, const char *d_arena,
          gdp_result_t *d_res, gdp_rec_t *d_slots, cudaStream_t stream = nullptr, DevBuf *scratch_buf = nullptr,
          DevBuf *scratch8_buf = nullptr, DevBuf *scratch_late_buf = nullptr) {
  cudaStream_t s = stream ? stream : ctx->stream;
  cudaStream_t *side_s = ctx->side;
  for (int w = 0; w < ctx->nwave; w++)
    if (s == ctx->wave_stream[w]) side_s = ctx->wave_side[w];
  DevBuf &scratch = scratch_buf ? *scratch_buf : ctx->scratch;
  DevBuf &scratch8 = scratch8_buf ? *scratch8_buf : ctx->scratch8;   /* the early 8-bit kinds' own */
  DevBuf &scratch_late = scratch_late_buf ? *scratch_late_buf : ctx->scratch_late;   /* the jump-late chain's */
  const int64_t n = ph.n;
  if (n == 0) return GDP_OK;
  cudaEvent_t ev0 = nullptr;
  prof_begin(ctx, &ev0, s);
  static_assert(NKINDS <= 256, "one block clears every 8-bit pass counter");
  init_results_kernel<<<(int) std::min<int64_t>((n + 255) / 256, 4096), 256, 0, s>>>(
      d_res, pd.status.as<int32_t>(), d_pairs, n, pd.meta0.as<gdp_meta_t>(), pd.meta.as<gdp_meta_t>(),
      pd.work_counts.as<int32_t>(), NKINDS);
  prof_end(ctx, PROF_INIT, ev0, s);
  ctx->launches++;
  CK(ctx, cudaGetLastError());
  if (ph.nwindow > 0) {
    cudaEvent_t evw = nullptr;
    prof_begin(ctx, &evw, s);
    window_kernel<<<(int) std::min<int64_t>(n, (int64_t) ctx->nsm * 16), 256, 0, s>>>(
        d_pairs, pd.status.as<int32_t>(), n, const_cast<char *>(d_arena), ctx->d_genome,
        ctx->d_genomealt ? ctx->d_genomealt : ctx->d_genome, ctx->genome_len);
    prof_end(ctx, PROF_WINDOW, evw, s);
    ctx->launches++;
    CK(ctx, cudaGetLastError());
  }
  /* the jump-late chain runs beside the jump-early one (below) unless
     per-launch timing is on or a grid footprint cap is set; only then does
     it need a scratch of its own */
  const bool two_chains = !ctx->profiling && ctx->grid_limit == 0;
  size_t need = 0, need8 = 0, need_late = 0;
  for (int k = 0; k < NTHREADKINDS; k++) {
    if (!ph.counts[k]) continue;
    size_t &nd = (((k >> 1) & 1) && two_chains) ? need_late : need;
    nd = std::max(nd, (size_t) (ph.maxY[k] + 1) * (size_t) fill_grid(ctx, ph.counts[k]) * 128 * sizeof(int2));
  }
  for (int k = FIRST_EARLY8; k < NKINDS; k++) {
    if (!ph.counts[k]) continue;
    need8 = std::max(need8, (size_t) (ph.maxY[k] + 1) * (size_t) fill_grid(ctx, ph.counts[k]) * 128 * sizeof(int2));
  }
  CK(ctx, scratch.ensure(std::max<size_t>(need, 64)));
  if (need8 > 0) CK(ctx, scratch8.ensure(need8));
  if (need_late > 0) CK(ctx, scratch_late.ensure(need_late));
  /* 16-bit and plain passes first, then the 8-bit passes of rerun pairs.
     The one-warp / one-CTA-per-pair kinds (no scratch) go first, on side
     streams, so that they run beside the one-thread-per-pair kinds and
     beside one another.  Those form two chains: the jump-early kinds share the scratch
     and stay in order on the main stream, the jump-late kinds have a
     scratch of their own and stay in order on the third side stream.  A
     pair's 8-bit pass waits only for its own 16-bit pass, so each chain's
     8-bit pass (few pairs, a few blocks per SM) runs beside the other
     chain's 16-bit pass instead of after it.  With per-launch timing on,
     both chains stay on the main stream, so that each kernel's events
     time it alone; so they do under a grid footprint cap (grid_limit),
     which bounds the blocks per SM of one launch at a time. */
  bool forked = false, forked_late = false;
  int side = 0;
  CK(ctx, cudaEventRecord(ctx->fork_ev, s));
  for (int round = 0; round < 2; round++) {
    if (round == 1 && forked) {
      for (int q = 0; q < GDP_NSIDE; q++) {
        CK(ctx, cudaEventRecord(ctx->join_ev[q], side_s[q]));
        CK(ctx, cudaStreamWaitEvent(s, ctx->join_ev[q], 0));
      }
    }
    for (int kk = 0; kk < NKINDS; kk++) {
      const int k = (round == 0) ? (kk + NTHREADKINDS) % NKINDS : kk;
      const bool warp = k >= NTHREADKINDS && k < FIRST_WARP8;
      const bool warp8 = k >= FIRST_WARP8 && k < FIRST_CTA;
      const bool cta = k >= FIRST_CTA && k < FIRST_EARLY8;
      const bool early8 = k >= FIRST_EARLY8;
      const bool thread = !warp && !warp8 && !cta && !early8;
      const int w32 = thread ? (k >> 2) / 3 : 0, pass = thread ? (k & 1) : 0;
      const bool second = (w32 == 1 && pass == 1) || warp8;
      if ((round == 0) == second || !ph.counts[k]) continue;
      /* the jump-late chain: thread kinds and lane-group 8-bit passes of
         jump-late pairs */
      const bool late_chain = (thread && ((k >> 1) & 1)) || (warp8 && (((k - FIRST_WARP8) / 3) & 1));
      if (late_chain && !forked_late && two_chains) {
        CK(ctx, cudaStreamWaitEvent(side_s[GDP_NSIDE], ctx->fork_ev, 0));
        forked_late = true;
      }
      cudaStream_t ks = (late_chain && two_chains) ? side_s[GDP_NSIDE] : s;
      const int grid = cta ? (int) std::max<int64_t>(1, std::min<int64_t>(ph.counts[k], grid_cap(ctx, 8)))
                     : warp ? warp_grid(ctx, ph.counts[k], WARP_K[(k - NTHREADKINDS) % 3])
                     : warp8 ? warp_grid(ctx, ph.counts[k], WARP8_K[(k - FIRST_WARP8) % 3])
                             : fill_grid(ctx, ph.counts[k]);
      FillParams P;
      P.pairs = d_pairs; P.arena = d_arena;
      P.list = pd.lists.as<int32_t>() + ph.start[k];
      P.count = pd.counts.as<int32_t>() + k;
      if (second) {
        /* only the pairs whose 16-bit maximum stayed below 127 run the 8-bit
           pass; the selection keeps the planner's order, so a warp's pairs
           share band width and lband as in the other passes */
        const NeedsPass8 need{pd.meta.as<gdp_meta_t>()};
        DevBuf &sel_tmp = (late_chain && two_chains) ? pd.sel_tmp_late : pd.sel_tmp;
        size_t tmp = 0;
        CK(ctx, cub::DeviceSelect::If(nullptr, tmp, P.list, pd.work.as<int32_t>() + ph.start[k],
                                      pd.work_counts.as<int32_t>() + k, (int) ph.counts[k], need, ks));
        CK(ctx, sel_tmp.ensure(std::max<size_t>(tmp, 16)));
        cudaEvent_t evc = nullptr;
        prof_begin(ctx, &evc, ks);
        CK(ctx, cub::DeviceSelect::If(sel_tmp.p, tmp, P.list, pd.work.as<int32_t>() + ph.start[k],
                                      pd.work_counts.as<int32_t>() + k, (int) ph.counts[k], need, ks));
        prof_end(ctx, PROF_RERUN, evc, ks);
        ctx->launches++;
        P.list = pd.work.as<int32_t>() + ph.start[k];
        P.count = pd.work_counts.as<int32_t>() + k;
      }
      P.dirs = pd.dirs.as<uint32_t>();
      P.hdump = pd.hdump.as<int16_t>();
      P.meta = pd.meta.as<gdp_meta_t>();
      P.res = d_res;
      P.scratch = early8 ? scratch8.as<int2>()
                         : ((late_chain && two_chains) ? scratch_late.as<int2>() : scratch.as<int2>());
      P.nslots = (int64_t) grid * 128;
      P.scratch_rows = ph.maxY[k] + 1;
      P.tab = ctx->d_tab;
      P.reach_from4 = 0;
      P.lower_slack4 = 0;
      P.packed_len = ctx->packed_len;
      P.tab_mn = ctx->tab_mn;
      P.tab_mx = ctx->tab_mx;
      for (int q = 0; q < 4; q++) {
        P.reach_from4 |= (uint32_t) std::min(ctx->reach_from[q], 255) << (8 * q);
        P.lower_slack4 |= (uint32_t) ctx->lower_slack[q] << (8 * q);
      }
      if (warp || cta || early8) {
        if (!forked) {
          for (int q = 0; q < GDP_NSIDE; q++) CK(ctx, cudaStreamWaitEvent(side_s[q], ctx->fork_ev, 0));
          forked = true;
        }
        if (early8) {
          /* the early 8-bit kinds share one scratch: they stay in order on
             one side stream */
          ks = side_s[0];
        } else {
          /* each lane-group / CTA kind on a side stream of its own (round
             robin): a few long pairs leave most of the GPU idle, and their
             kinds, one after another, took the sum of their latencies.
             Under a grid footprint cap two side streams, as the cap
             assumes. */
          ks = side_s[1 + side % (ctx->grid_limit > 0 ? 2 : GDP_NSIDE - 1)];
          side++;
        }
      }
      cudaEvent_t ev = nullptr;
      prof_begin(ctx, &ev, ks);
      int nlaunch = 1;
      if (cta) launch_cta_kind(k, P, grid, ks);
      else if (warp) launch_warp_kind(k, P, grid, ks);
      else if (warp8) launch_warp8_kind(k, P, grid, ks);
      else if (early8) launch_early8_kind(k, P, grid, ks);
      else nlaunch = launch_kind(k, P, grid, ks, ph.maxMin[k]);
      prof_end(ctx, k, ev, ks);
      ctx->launches += nlaunch;
      CK(ctx, cudaGetLastError());
    }
  }
  /* The 8-bit outcome of rerun pairs, after both of their passes, then
     the tracebacks.  With the two chains, the jump-late pairs' outcomes and
     tracebacks run on the jump-late chain's stream once it and the side
     kinds are done, beside the jump-early chain's tail (its 8-bit pass
     holds few pairs and leaves most of the GPU idle); the jump-early ones
     follow on the plan's stream. */
  cudaStream_t late_s = forked_late ? side_s[GDP_NSIDE] : s;
  if (forked_late && forked)
    for (int q = 0; q < GDP_NSIDE; q++) CK(ctx, cudaStreamWaitEvent(late_s, ctx->join_ev[q], 0));
  for (int k = 0; k < NKINDS; k++) {
    const bool check8 = (k < NTHREADKINDS && (k >> 2) / 3 == 1 && (k & 1)) || (k >= FIRST_WARP8 && k < FIRST_CTA) ||
                        k >= FIRST_EARLY8;
    if (!check8 || !ph.counts[k]) continue;
    const int late = (k < NTHREADKINDS) ? ((k >> 1) & 1)
                   : (k < FIRST_CTA) ? (((k - FIRST_WARP8) / 3) & 1) : ((k - FIRST_EARLY8) & 1);
    cudaStream_t as = late ? late_s : s;
    const int ag = (int) std::max<int64_t>(1, std::min<int64_t>((ph.counts[k] + 255) / 256, (int64_t) ctx->nsm * 8));
    apply_rerun8_kernel<<<ag, 256, 0, as>>>(pd.lists.as<int32_t>() + ph.start[k], pd.counts.as<int32_t>() + k,
                                            pd.meta.as<gdp_meta_t>(), d_res);
    ctx->launches++;
    CK(ctx, cudaGetLastError());
  }
  int rc = GDP_OK;
  if (forked_late) {
    rc = launch_traceback(ctx, ph, pd, d_pairs, d_arena, d_res, d_slots, late_s, 1);
    if (rc == GDP_OK) rc = launch_traceback(ctx, ph, pd, d_pairs, d_arena, d_res, d_slots, s, 2);
    CK(ctx, cudaEventRecord(ctx->join_ev[GDP_NSIDE], late_s));
    CK(ctx, cudaStreamWaitEvent(s, ctx->join_ev[GDP_NSIDE], 0));
  } else {
    rc = launch_traceback(ctx, ph, pd, d_pairs, d_arena, d_res, d_slots, s, 0);
  }
  return rc;
}

/* Dense records after plan_run: scan of nrecs, gather into `out`, total in
   pd.total. */
static int
compact_records (gdp_ctx *ctx, const PlanHost &ph, PlanDev &pd, gdp_result_t *d_res, const gdp_rec_t *d_slots,
                 gdp_rec_t *out, int64_t *total_host = nullptr, cudaStream_t stream = nullptr) {
  cudaStream_t s = stream ? stream : ctx->stream;
  const int64_t n = ph.n;
  if (n == 0) return GDP_OK;
  CK(ctx, pd.nrec_scan.ensure((2 * n + 1) * sizeof(int64_t)));
  int64_t *counts = pd.nrec_scan.as<int64_t>() + n;
  gather_nrecs_kernel<<<(int) std::min<int64_t>((n + 255) / 256, 4096), 256, 0, s>>>(d_res, n, counts);
  ctx->launches++;
  size_t tmp = 0;
  CK(ctx, cub::DeviceScan::ExclusiveSum(nullptr, tmp, counts, pd.nrec_scan.as<int64_t>(), (int) n, s));
  CK(ctx, pd.cub_tmp.ensure(std::max<size_t>(tmp, 16)));
  CK(ctx, cub::DeviceScan::ExclusiveSum(pd.cub_tmp.p, tmp, counts, pd.nrec_scan.as<int64_t>(), (int) n, s));
  ctx->launches++;
  cudaEvent_t ev = nullptr;
  prof_begin(ctx, &ev, s);
  const int grid = (int) std::max<int64_t>(1, std::min<int64_t>((n * 32 + 255) / 256, (int64_t) ctx->nsm * 16));
  compact_records_kernel<<<grid, 256, 0, s>>>(d_res, pd.rec_off.as<int64_t>(), d_slots,
                                              pd.nrec_scan.as<int64_t>(), n, out, pd.total.as<int64_t>(),
                                              total_host);
  prof_end(ctx, PROF_RECS, ev, s);
  ctx->launches++;
  CK(ctx, cudaGetLastError());
  return GDP_OK;
}

/* The record-run stream length of each pair of a wave (one thread per
   pair, its records as compacted); len[n] = 0, so that the exclusive scan's
   last entry is the total. */
__global__ void __launch_bounds__(128)
run_size_kernel (const gdp_result_t *res, const gdp_pair_t *pairs, const char *arena, const gdp_rec_t *recs,
                 int64_t n, int64_t *len) {
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t) gridDim.x * blockDim.x) {
    int64_t l = 0;
    if (i < n) {
      const int nr = res[i].nrecs;
      if (nr > 0) {
        const gdp_pair_t p = pairs[i];
        l = rec_encode(run_seqs(p, arena), recs + res[i].rec_offset, nr, (p.flags & GDP_FLAG_GWINDOW) != 0,
                       nullptr);
      }
    }
    len[i] = l;
  }
}

/* Writes each pair's stream at off[i]; the total goes to a mapped host
   word. */
__global__ void __launch_bounds__(128)
run_write_kernel (const gdp_result_t *res, const gdp_pair_t *pairs, const char *arena, const gdp_rec_t *recs,
                  int64_t n, const int64_t *off, uint8_t *out, int64_t *total_host) {
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
    const int nr = res[i].nrecs;
    if (nr > 0) {
      const gdp_pair_t p = pairs[i];
      rec_encode(run_seqs(p, arena), recs + res[i].rec_offset, nr, (p.flags & GDP_FLAG_GWINDOW) != 0, out + off[i]);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *(volatile int64_t *) total_host = off[n];
    __threadfence_system();
  }
}

/* Encodes a wave's compacted records as runs, on its compute stream. */
static int
encode_runs (gdp_ctx *ctx, Slot &sl, const char *d_arena) {
  const int64_t n = sl.count;
  cudaStream_t s = sl.cs;
  CK(ctx, sl.enc_off.ensure((2 * n + 2) * sizeof(int64_t)));
  CK(ctx, sl.enc.ensure(std::max<int64_t>(sl.h.total_recs, 1) * (1 + (int64_t) sizeof(gdp_rec_t))));
  CK(ctx, sl.enc_total.ensure(sizeof(int64_t)));
  *(volatile int64_t *) sl.enc_total.p = 0;
  int64_t *total_dev = nullptr;
  CK(ctx, cudaHostGetDevicePointer((void **) &total_dev, sl.enc_total.p, 0));
  int64_t *len = sl.enc_off.as<int64_t>() + n + 1, *off = sl.enc_off.as<int64_t>();
  const gdp_result_t *res = sl.results.as<gdp_result_t>();
  const gdp_pair_t *pairs = sl.pairs.as<gdp_pair_t>();
  const gdp_rec_t *recs = sl.recs.as<gdp_rec_t>();
  const int grid = (int) std::max<int64_t>(1, std::min<int64_t>((n + 128) / 128, (int64_t) ctx->nsm * 16));
  run_size_kernel<<<grid, 128, 0, s>>>(res, pairs, d_arena, recs, n, len);
  ctx->launches++;
  size_t tmp = 0;
  CK(ctx, cub::DeviceScan::ExclusiveSum(nullptr, tmp, len, off, (int) (n + 1), s));
  CK(ctx, sl.d.cub_tmp.ensure(std::max<size_t>(tmp, 16)));
  CK(ctx, cub::DeviceScan::ExclusiveSum(sl.d.cub_tmp.p, tmp, len, off, (int) (n + 1), s));
  ctx->launches++;
  run_write_kernel<<<grid, 128, 0, s>>>(res, pairs, d_arena, recs, n, off, sl.enc.as<uint8_t>(), total_dev);
  ctx->launches++;
  CK(ctx, cudaGetLastError());
  return GDP_OK;
}

extern "C" int
gdp_plan_execute (gdp_ctx *ctx, gdp_plan *pl, const gdp_pair_t *d_pairs, const char *d_arena,
                  gdp_result_t *d_results, gdp_rec_t *d_recs) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  if (!pl->use_graph || ctx->profiling) return plan_run(ctx, pl->h, pl->d, d_pairs, d_arena, d_results, d_recs);
  const void *key[4] = {d_pairs, d_arena, d_results, d_recs};
  if (pl->gexec && memcmp(key, pl->gkey, sizeof(key)) == 0) {
    CK(ctx, cudaGraphLaunch(pl->gexec, ctx->stream));
    ctx->launches += pl->glaunches;
    return GDP_OK;
  }
  /* run once (this call's work; it also sizes every buffer), then capture
     the same launches for the next calls with these pointers */
  const int64_t l0 = ctx->launches;
  int rc = plan_run(ctx, pl->h, pl->d, d_pairs, d_arena, d_results, d_recs);
  if (rc != GDP_OK) return rc;
  const int64_t nl = ctx->launches - l0;
  if (pl->gexec) { cudaGraphExecDestroy(pl->gexec); pl->gexec = nullptr; }
  cudaGraph_t g = nullptr;
  CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  rc = plan_run(ctx, pl->h, pl->d, d_pairs, d_arena, d_results, d_recs);
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  ctx->launches -= nl;   /* captured, not launched */
  if (rc != GDP_OK) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) return set_err(ctx, "plan capture", e);
  e = cudaGraphInstantiate(&pl->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { pl->gexec = nullptr; return set_err(ctx, "plan graph", e); }
  memcpy(pl->gkey, key, sizeof(key));
  pl->glaunches = nl;
  return GDP_OK;
}

extern "C" int
gdp_plan_use_graph (gdp_plan *pl, int on) {
  if (pl == nullptr) return GDP_ERR_PARAM;
  pl->use_graph = on != 0;
  if (!pl->use_graph && pl->gexec) { cudaGraphExecDestroy(pl->gexec); pl->gexec = nullptr; }
  return GDP_OK;
}

/* ------------------------------------------------------------------ */
/* Tunable routing parameters and the autotuner                        */
/* ------------------------------------------------------------------ */

/* The record-run codec on the host (rec_runs.h), for callers that move
   records elsewhere and for tests. */
extern "C" int64_t
gdp_runs_encode (const gdp_pair_t *pair, const char *arena, const gdp_rec_t *recs, int32_t nrecs, uint8_t *out) {
  if (pair == nullptr || arena == nullptr || nrecs < 0 || (nrecs > 0 && recs == nullptr)) return -GDP_ERR_PARAM;
  return rec_encode(run_seqs(*pair, arena), recs, nrecs, (pair->flags & GDP_FLAG_GWINDOW) != 0, out);
}

extern "C" int
gdp_runs_decode (const gdp_pair_t *pair, const char *arena, const uint8_t *in, int64_t len, gdp_rec_t *recs,
                 int32_t nrecs) {
  if (pair == nullptr || arena == nullptr || nrecs < 0 || len < 0 || (len > 0 && in == nullptr) ||
      (nrecs > 0 && recs == nullptr))
    return GDP_ERR_PARAM;
  return rec_decode(run_seqs(*pair, arena), in, len, recs, nrecs) ? GDP_OK : GDP_ERR_PARAM;
}

extern "C" int
gdp_ctx_set_param (gdp_ctx *ctx, const char *name, int64_t value) {
  if (ctx == nullptr || name == nullptr) return GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!strcmp(name, "warp_min_x") && value >= 1) ctx->warp_min_x = (int) value;
  else if (!strcmp(name, "warp_max_sweep") && value >= 1) ctx->warp_max_sweep = (int) std::min<int64_t>(value, 32 * 17 - 16);
  else if (!strcmp(name, "group_slack") && value >= 16 && value <= 128) ctx->group_slack = (int) value;
  else if (!strcmp(name, "tb_warp")) ctx->tb_warp = value != 0;
  else if (!strcmp(name, "check_groups")) ctx->check_groups = value != 0;
  else if (!strcmp(name, "check_min_x") && value >= 1) ctx->check_min_x = (int) std::min<int64_t>(value, 1 << 30);
  else if (!strcmp(name, "wave_pairs") && value >= 1) ctx->wave = value;
  else if (!strcmp(name, "first_wave_pairs") && value >= 0) ctx->first_wave = value;
  else if (!strcmp(name, "wave_priority") && value >= 0)
    ctx->wave_prio = (int) std::min<int64_t>(value, std::max(ctx->nwave - 1, 0));
  else if (!strcmp(name, "grid_blocks_per_sm") && value >= 0) ctx->grid_limit = (int) std::min<int64_t>(value, 64);
  else if (!strcmp(name, "record_runs") && value >= 0 && value <= 2) ctx->record_runs = (int) value;
  else if (!strcmp(name, "runs_from_wave") && value >= 0) ctx->runs_from_wave = (int) std::min<int64_t>(value, 1 << 20);
  else return GDP_ERR_PARAM;
  return GDP_OK;
}

extern "C" int
gdp_ctx_get_param (gdp_ctx *ctx, const char *name, int64_t *value) {
  if (ctx == nullptr || name == nullptr || value == nullptr) return GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!strcmp(name, "warp_min_x")) *value = ctx->warp_min_x;
  else if (!strcmp(name, "warp_max_sweep")) *value = ctx->warp_max_sweep;
  else if (!strcmp(name, "group_slack")) *value = ctx->group_slack;
  else if (!strcmp(name, "tb_warp")) *value = ctx->tb_warp ? 1 : 0;
  else if (!strcmp(name, "check_groups")) *value = ctx->check_groups ? 1 : 0;
  else if (!strcmp(name, "check_min_x")) *value = ctx->check_min_x;
  else if (!strcmp(name, "wave_pairs")) *value = ctx->wave;
  else if (!strcmp(name, "first_wave_pairs")) *value = ctx->first_wave;
  else if (!strcmp(name, "wave_priority")) *value = ctx->wave_prio;
  else if (!strcmp(name, "grid_blocks_per_sm")) *value = ctx->grid_limit;
  else if (!strcmp(name, "record_runs")) *value = ctx->record_runs;
  else if (!strcmp(name, "runs_from_wave")) *value = ctx->runs_from_wave;
  else if (!strcmp(name, "last_d2h_bytes")) *value = ctx->last_d2h;
  else return GDP_ERR_PARAM;
  return GDP_OK;
}

/* Device time of one plan execution of a sample under the current routing
   (best of `reps` after one warm-up), or a negative status. */
static double
tune_trial (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t n, const gdp_pair_t *d_pairs, const char *d_arena,
            gdp_result_t *d_res, DevBuf &recs, int reps) {
  gdp_plan pl;
  int rc = plan_build(ctx, pairs, n, -1, pl.h);
  if (rc == GDP_OK) rc = plan_upload(ctx, pl.h, pl.d, false, ctx->stream);
  if (rc != GDP_OK) return -rc;
  if (recs.ensure(std::max<int64_t>(pl.h.total_recs, 1) * sizeof(gdp_rec_t)) != cudaSuccess) return -GDP_ERR_CUDA;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 1e30;
  for (int r = 0; r <= reps && rc == GDP_OK; r++) {
    cudaEventRecord(a, ctx->stream);
    rc = plan_run(ctx, pl.h, pl.d, d_pairs, d_arena, d_res, recs.as<gdp_rec_t>());
    cudaEventRecord(b, ctx->stream);
    if (cudaEventSynchronize(b) != cudaSuccess) rc = GDP_ERR_CUDA;
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (r > 0) best = std::min(best, (double) ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  pl.d.release();
  pl.h.release();
  return rc == GDP_OK ? best : -rc;
}

extern "C" int
gdp_autotune (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t npairs, const char *arena, int64_t arena_bytes,
              double *best_ms) {
  if (ctx == nullptr || pairs == nullptr || npairs <= 0 || arena == nullptr || arena_bytes <= 0) return GDP_ERR_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  const bool prof = ctx->profiling;
  ctx->profiling = false;
  DevBuf dp, da, dr, drec;
  CK(ctx, dp.ensure(npairs * sizeof(gdp_pair_t)));
  CK(ctx, da.ensure(arena_bytes));
  CK(ctx, dr.ensure(npairs * sizeof(gdp_result_t)));
  CK(ctx, cudaMemcpyAsync(dp.p, pairs, npairs * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, ctx->stream));
  CK(ctx, cudaMemcpyAsync(da.p, arena, arena_bytes, cudaMemcpyHostToDevice, ctx->stream));
  /* coordinate descent over the routing knobs, each from a small set */
  struct Knob { int *v; std::vector<int> cand; };
  int tbw = ctx->tb_warp ? 1 : 0, cg = ctx->check_groups ? 1 : 0;
  std::vector<Knob> knobs = {
    {&ctx->warp_min_x, {128, 256, 512, 1024, 2048, 1 << 30}},
    {&ctx->group_slack, {16, 32, 48, 80}},
    {&ctx->warp_max_sweep, {272, 400, 496, 528}},
    {&tbw, {1, 0}},
    {&cg, {1, 0}},
    {&ctx->check_min_x, {96, 128, 160, 224, 1 << 30}},
  };
  double best = tune_trial(ctx, pairs, npairs, dp.as<gdp_pair_t>(), da.as<char>(), dr.as<gdp_result_t>(), drec, 2);
  int rc = best < 0 ? (int) -best : GDP_OK;
  for (size_t k = 0; k < knobs.size() && rc == GDP_OK; k++) {
    const int keep = *knobs[k].v;
    int choice = keep;
    for (int c : knobs[k].cand) {
      if (c == keep) continue;
      *knobs[k].v = c;
      ctx->tb_warp = tbw != 0;
      ctx->check_groups = cg != 0;
      const double t = tune_trial(ctx, pairs, npairs, dp.as<gdp_pair_t>(), da.as<char>(), dr.as<gdp_result_t>(), drec, 2);
      if (t < 0) { rc = (int) -t; break; }
      if (t < best * 0.98) { best = t; choice = c; }
    }
    *knobs[k].v = choice;
    ctx->tb_warp = tbw != 0;
    ctx->check_groups = cg != 0;
  }
  ctx->profiling = prof;
  if (best_ms) *best_ms = best;
  return rc;
}

/* ------------------------------------------------------------------ */
/* Host-buffer path: waves with overlapped planning and copies         */
/* ------------------------------------------------------------------ */

/* Enqueues wave (first, count) in slot sl: copy-in on the h2d stream, work
   on the compute stream, results out on the d2h stream.  Records leave once
   the host knows their count (slot_finish). */
static int
slot_launch (gdp_ctx *ctx, Slot &sl, const gdp_pair_t *pairs, int64_t first, int64_t count,
             int64_t arena_bytes, gdp_result_t *results, cudaEvent_t arena_ready, int wave_index) {
  /* the slot's host plan buffers are free once their last upload ended */
  GDP_TRACE_BEGIN(t0);
  CK(ctx, cudaEventSynchronize(sl.h2d_done));
  GDP_TRACE_END(t0, "wait_h2d");
  GDP_TRACE_BEGIN(t1);
  int rc = plan_build(ctx, pairs + first, count, arena_bytes, sl.h);
  GDP_TRACE_END(t1, "plan");
  if (rc != GDP_OK) return rc;
  sl.first = first;
  sl.count = count;
  /* the slot's device buffers are free once the last wave's copies out
     ended: the copy-in stream waits for that on the device */
  CK(ctx, cudaStreamWaitEvent(ctx->h2d, sl.out_done, 0));
  CK(ctx, sl.pairs.ensure(std::max<int64_t>(count, 1) * sizeof(gdp_pair_t)));
  CK(ctx, sl.results.ensure(std::max<int64_t>(count, 1) * sizeof(gdp_result_t)));
  CK(ctx, sl.d.slots.ensure(std::max<int64_t>(sl.h.total_recs, 1) * sizeof(gdp_rec_t)));
  CK(ctx, sl.recs.ensure(std::max<int64_t>(sl.h.total_recs, 1) * sizeof(gdp_rec_t)));
  CK(ctx, sl.total.ensure(sizeof(int64_t)));
  GDP_TEV(ctx->h2d, "h2d_begin %lld", first);
  CK(ctx, cudaMemcpyAsync(sl.pairs.p, pairs + first, count * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, ctx->h2d));
  rc = plan_upload(ctx, sl.h, sl.d, false, ctx->h2d);
  if (rc != GDP_OK) return rc;
  CK(ctx, cudaEventRecord(sl.h2d_done, ctx->h2d));
  GDP_TEV(ctx->h2d, "h2d_end %lld", first);
  sl.cs = ctx->wave_stream[std::min(ctx->wave_prio + wave_index, ctx->nwave - 1)];
  CK(ctx, cudaStreamWaitEvent(sl.cs, sl.h2d_done, 0));
  if (arena_ready) CK(ctx, cudaStreamWaitEvent(sl.cs, arena_ready, 0));
  GDP_TEV(sl.cs, "comp_begin %lld", first);
  rc = plan_run(ctx, sl.h, sl.d, sl.pairs.as<gdp_pair_t>(), ctx->arena.as<char>(), sl.results.as<gdp_result_t>(),
                sl.d.slots.as<gdp_rec_t>(), sl.cs, &sl.scratch, &sl.scratch8, &sl.scratch_late);
  if (rc != GDP_OK) return rc;
  /* the count reaches the host through a mapped pinned word written by the
     compaction kernel, not a copy on the compute stream (a copy engine busy
     with an earlier wave's records would hold the stream up) */
  int64_t *total_dev = nullptr;
  CK(ctx, cudaHostGetDevicePointer((void **) &total_dev, sl.total.p, 0));
  *(volatile int64_t *) sl.total.p = 0;
  rc = compact_records(ctx, sl.h, sl.d, sl.results.as<gdp_result_t>(), sl.d.slots.as<gdp_rec_t>(),
                       sl.recs.as<gdp_rec_t>(), total_dev, sl.cs);
  if (rc != GDP_OK) return rc;
  /* runs only pay where the host holds the genome characters: not for a
     wave whose every pair has its window written on the device */
  sl.runs = false;
  /* record_runs 1: every wave; 2: the waves from runs_from_wave on.  The
     last waves' records cross PCIe after the device has finished, so they
     set the batch's end: as runs they leave at once and the host rebuilds
     them while the earlier waves' plain records are still crossing; the
     first waves stay plain, so that rebuilding does not take the cores
     from the planner of the waves that follow */
  if (ctx->record_runs == 1 || (ctx->record_runs == 2 && wave_index >= ctx->runs_from_wave))
    for (int64_t i = first; i < first + count && !sl.runs; i++) sl.runs = !(pairs[i].flags & GDP_FLAG_GWINDOW);
  if (sl.runs) {
    rc = encode_runs(ctx, sl, ctx->arena.as<char>());
    if (rc != GDP_OK) return rc;
  }
  GDP_TEV(sl.cs, "comp_end %lld", first);
  CK(ctx, cudaEventRecord(sl.total_ready, sl.cs));
  CK(ctx, cudaEventRecord(sl.comp_done, sl.cs));
  return GDP_OK;
}

/* Adds the wave's first record (its base in the batch) to the record
   offsets of the wave's results, on the copy-out stream before they leave. */
__global__ void
add_rec_base_kernel (gdp_result_t *res, int64_t n, int64_t base) {
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
    res[i].rec_offset += base;
}

/* Waits for the wave's record count and queues its results and records
   out (records at *base).  The copy stream takes waves in order, so a wave
   still computing never holds up the copies of an earlier one.  A wave
   whose records travel as runs (rec_runs.h) copies its streams out instead
   and rebuilds the records into recs on the context's host threads before
   the slot is free again. */
static int
slot_finish (gdp_ctx *ctx, Slot &sl, const gdp_pair_t *pairs, const char *arena, gdp_result_t *results,
             gdp_rec_t *recs, int64_t max_recs, int64_t *base, bool *overflow) {
  GDP_TRACE_BEGIN(t0);
  CK(ctx, cudaEventSynchronize(sl.total_ready));
  GDP_TRACE_END(t0, "wait_total");
  CK(ctx, cudaStreamWaitEvent(ctx->d2h, sl.comp_done, 0));
  if (*base != 0 && sl.count > 0) {
    add_rec_base_kernel<<<(int) std::min<int64_t>((sl.count + 255) / 256, (int64_t) ctx->nsm * 4), 256, 0, ctx->d2h>>>(
        sl.results.as<gdp_result_t>(), sl.count, *base);
    ctx->launches++;
    CK(ctx, cudaGetLastError());
  }
  CK(ctx, cudaMemcpyAsync(results + sl.first, sl.results.p, sl.count * sizeof(gdp_result_t), cudaMemcpyDeviceToHost,
                          ctx->d2h));
  ctx->last_d2h += sl.count * (int64_t) sizeof(gdp_result_t);
  const int64_t total = sl.h.n > 0 ? *(volatile int64_t *) sl.total.p : 0;
  bool expand = false;
  if (total > 0) {
    if (recs == nullptr || *base + total > max_recs) {
      *overflow = true;
    } else if (sl.runs) {
      const int64_t bytes = *(volatile int64_t *) sl.enc_total.p;
      CK(ctx, sl.h_enc.ensure(std::max<int64_t>(bytes, 16)));
      CK(ctx, sl.h_encoff.ensure((sl.count + 1) * sizeof(int64_t)));
      GDP_TEV(ctx->d2h, "runs_begin %lld", sl.first);
      CK(ctx, cudaMemcpyAsync(sl.h_enc.p, sl.enc.p, bytes, cudaMemcpyDeviceToHost, ctx->d2h));
      CK(ctx, cudaMemcpyAsync(sl.h_encoff.p, sl.enc_off.p, (sl.count + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                              ctx->d2h));
      GDP_TEV(ctx->d2h, "runs_end %lld", sl.first);
      ctx->last_d2h += bytes + (sl.count + 1) * (int64_t) sizeof(int64_t);
      expand = true;
    } else {
      GDP_TEV(ctx->d2h, "recs_begin %lld", sl.first);
      CK(ctx, cudaMemcpyAsync(recs + *base, sl.recs.p, total * sizeof(gdp_rec_t), cudaMemcpyDeviceToHost, ctx->d2h));
      GDP_TEV(ctx->d2h, "recs_end %lld", sl.first);
      ctx->last_d2h += total * (int64_t) sizeof(gdp_rec_t);
    }
  }
  CK(ctx, cudaEventRecord(sl.out_done, ctx->d2h));
  sl.rec_base = *base;
  *base += total;
  sl.expand = expand;
  return GDP_OK;
}

/* Rebuilds a wave's records from its runs into recs, on the copy-out
   side's host threads, once its copies out are done. */
static int
slot_expand (gdp_ctx *ctx, Slot &sl, const gdp_pair_t *pairs, const char *arena, const gdp_result_t *results,
             gdp_rec_t *recs) {
  if (!sl.expand) return GDP_OK;
  sl.expand = false;
  GDP_TRACE_BEGIN(t1);
  CK(ctx, cudaEventSynchronize(sl.out_done));
  const gdp_pair_t *wp = pairs + sl.first;
  const gdp_result_t *wr = results + sl.first;
  const uint8_t *enc = sl.h_enc.as<uint8_t>();
  const int64_t *off = sl.h_encoff.as<int64_t>();
  const int64_t n = sl.count;
  const int nt = (int) std::max<int64_t>(1, std::min<int64_t>(ctx->plan_threads, n / 4096));
  std::atomic<int> bad{0};
  parallel_chunks(ctx->xpool, n, nt, [&](int64_t lo, int64_t hi, int) {
    for (int64_t i = lo; i < hi; i++) {
      const int nr = wr[i].nrecs;
      if (nr <= 0) continue;
      if (!rec_decode(run_seqs(wp[i], arena), enc + off[i], off[i + 1] - off[i], recs + wr[i].rec_offset, nr))
        bad.store(1);
    }
  });
  GDP_TRACE_END(t1, "expand");
  if (bad.load()) return set_err(ctx, "record runs: a stream did not rebuild its records", cudaErrorUnknown);
  return GDP_OK;
}

extern "C" int
gdp_align_batch (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t n, const char *arena, int64_t arena_bytes,
                 gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs, int64_t *nrecs_used) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  if (nrecs_used) *nrecs_used = 0;
  ctx->last_d2h = 0;
  if (n <= 0) return GDP_OK;
  /* the previous batch may still be reading the arena */
  for (int s = 0; s < NSLOTS; s++) CK(ctx, cudaEventSynchronize(ctx->slot[s].out_done));
  for (int k = 0; k < ctx->nwave; k++) CK(ctx, cudaStreamSynchronize(ctx->wave_stream[k]));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  CK(ctx, ctx->arena.ensure(std::max<int64_t>(arena_bytes, 16)));
  const int64_t wave = std::max<int64_t>(1, ctx->wave);
#ifdef GDP_HOST_TRACE
  for (auto &t : gdp_tev) cudaEventDestroy(t.ev);
  gdp_tev.clear();
  const auto host0 = std::chrono::steady_clock::now();
  GDP_TEV(ctx->h2d, "batch_begin %lld", 0);
#endif
  /* The arena goes to the device as a growing prefix: before each wave, the
     bytes up to the end of that wave's sequences that are not there yet.
     With pairs in arena order the first wave starts after its own
     sequences, not the whole arena. */
  int64_t copied = 0;
  auto arena_upto = [&](int64_t lo, int64_t hi) -> int {
    hi = std::min(std::max<int64_t>(hi, 0), arena_bytes);
    if (hi > copied) {
      GDP_TEV(ctx->h2d, "arena_begin %lld", lo);
      CK(ctx, cudaMemcpyAsync(ctx->arena.as<char>() + copied, arena + copied, hi - copied, cudaMemcpyHostToDevice,
                              ctx->h2d));
      GDP_TEV(ctx->h2d, "arena_end %lld", lo);
      copied = hi;
    }
    return GDP_OK;
  };
  /* A short first wave gets the pipeline going: the first holds half a
     wave and each next one twice the one before, up to a full wave, so the
     copies out start early and never wait long for the next wave. */
  int64_t wave_cap = std::min(wave, ctx->first_wave > 0 ? ctx->first_wave : std::max<int64_t>(16384, wave / 2));
  /* A wave also ends before its direction words would pass the context's
     budget (an upper bound per pair: every block sweeps at most
     W + lband + uband columns).  One pass finds the count and the end of the
     wave's sequences in the arena (*hi). */
  auto pair_bytes = [&](const gdp_pair_t &p) -> int64_t {
    const int64_t X = std::max(p.variant == GDP_LOWER ? p.glength : p.rlength, 0);
    const int64_t band = std::max(p.lband, 0) + std::max(p.uband, 0);
    int64_t b = 0;
    if (p.precision == 16 || (p.flags & GDP_FLAG_RERUN16)) b += (X / 16 + 1) * (16 + band) * 8;
    if (p.precision == 8) b += (X / 32 + 1) * (32 + band) * 16;
    return b;
  };
  auto pair_end = [&](const gdp_pair_t &p) -> int64_t {
    const int64_t rl = std::max(p.rlength, 0), gl = std::max(p.glength, 0);
    return std::max(std::max(p.rseq + rl, p.rseq_uc + rl), std::max(p.gseq + gl, p.gseq_alt + gl));
  };
  /* The scan runs on the planner's threads, chunk by chunk; the first chunk
     that would pass the budget is then walked pair by pair. */
  auto wave_count = [&](int64_t first, int64_t cap, int64_t *hi) -> int64_t {
    const int64_t m = std::min(cap, n - first);
    const int nt = (int) std::max<int64_t>(1, std::min<int64_t>(ctx->plan_threads, m / 16384));
    std::vector<int64_t> cbytes(nt, 0), chi(nt, 0);
    parallel_chunks(ctx->pool, m, nt, [&](int64_t lo, int64_t hi_, int t) {
      int64_t b = 0, h = 0;
      for (int64_t i = lo; i < hi_; i++) {
        b += pair_bytes(pairs[first + i]);
        h = std::max(h, pair_end(pairs[first + i]));
      }
      cbytes[t] = b;
      chi[t] = h;
    });
    int64_t bytes = 0, h = 0, k = 0;
    for (int t = 0; t < nt; t++) {
      const int64_t lo = m * t / nt, hi_ = m * (t + 1) / nt;
      if (bytes + cbytes[t] <= ctx->budget) {
        bytes += cbytes[t];
        h = std::max(h, chi[t]);
        k = hi_;
        continue;
      }
      for (int64_t i = lo; i < hi_; i++) {
        const int64_t b = pair_bytes(pairs[first + i]);
        if (i > 0 && bytes + b > ctx->budget) break;
        bytes += b;
        h = std::max(h, pair_end(pairs[first + i]));
        k = i + 1;
      }
      break;
    }
    *hi = h;
    return std::max<int64_t>(k, 1);
  };
  int64_t base = 0;
  bool overflow = false;
  int rc = GDP_OK;
  /* Waves are launched NSLOTS deep by this thread, which plans the next
     wave while earlier ones compute.  A copy-out thread takes the launched
     waves in order: it waits for a wave's record count and at once queues
     its results and records out, then frees the slot. */
  std::mutex m;
  std::condition_variable cv;
  std::deque<int> launched;          /* slots launched, not yet handed out, oldest first */
  std::deque<int> to_expand;         /* slots handed out whose runs wait to be rebuilt */
  bool all_launched = false, outs_done = false, have_expander = false;
  int out_rc = GDP_OK;
  /* A wave whose records travel as runs is rebuilt on the host after its
     copies; an expander thread does that, so the copy-out thread queues
     the next waves' copies meanwhile.  The slot stays busy until then. */
  auto expand_one = [&](int k) {
    Slot &o = ctx->slot[k];
    {
      std::lock_guard<std::mutex> g(m);
      if (out_rc != GDP_OK) o.expand = false;
    }
    const int r = slot_expand(ctx, o, pairs, arena, results, recs);
    std::lock_guard<std::mutex> g(m);
    if (r != GDP_OK) out_rc = r;
    o.busy = false;
    cv.notify_all();
  };
  auto hand_out = [&](int k) {
    Slot &o = ctx->slot[k];
    const int r = out_rc == GDP_OK ? slot_finish(ctx, o, pairs, arena, results, recs, max_recs, &base, &overflow)
                                   : out_rc;
    bool inline_expand = false;
    {
      std::lock_guard<std::mutex> g(m);
      if (r != GDP_OK) out_rc = r;
      launched.pop_front();
      if (o.expand && r == GDP_OK) {
        if (have_expander) to_expand.push_back(k);
        else inline_expand = true;
      } else {
        o.expand = false;
        o.busy = false;
      }
      cv.notify_all();
    }
    if (inline_expand) expand_one(k);
  };
  auto copy_out_loop = [&] {
    cudaSetDevice(ctx->device);
    for (;;) {
      int k;
      {
        std::unique_lock<std::mutex> g(m);
        cv.wait(g, [&] { return !launched.empty() || all_launched; });
        if (launched.empty()) return;
        k = launched.front();
      }
      hand_out(k);
    }
  };
  auto expand_loop = [&] {
    cudaSetDevice(ctx->device);
    for (;;) {
      int k;
      {
        std::unique_lock<std::mutex> g(m);
        cv.wait(g, [&] { return !to_expand.empty() || outs_done; });
        if (to_expand.empty()) return;
        k = to_expand.front();
        to_expand.pop_front();
      }
      expand_one(k);
    }
  };
  /* a batch of one wave hands out on this thread (and so does any batch
     when no thread can be started) */
  std::thread copy_out, expander;
  if (n > wave_cap) {
    try {
      copy_out = std::thread(copy_out_loop);
    } catch (...) {
    }
    if (copy_out.joinable() && ctx->record_runs) {
      try {
        expander = std::thread(expand_loop);
        std::lock_guard<std::mutex> g(m);
        have_expander = true;
      } catch (...) {
      }
    }
  }
  int cur = 0, wave_index = 0;
  for (int64_t first = 0; first < n;) {
    if (copy_out.joinable()) {
      /* every slot in flight: wait until the oldest has handed its records out */
      std::unique_lock<std::mutex> g(m);
      cv.wait(g, [&] { return !ctx->slot[cur].busy || out_rc != GDP_OK; });
      if (out_rc != GDP_OK) break;
    } else {
      /* no copy-out thread (a batch meant for one wave, cut by the budget) */
      while (ctx->slot[cur].busy && out_rc == GDP_OK) hand_out(launched.front());
      if (out_rc != GDP_OK) break;
    }
    int64_t hi = 0;
    const int64_t count = wave_count(first, std::min(wave_cap, n - first), &hi);
    wave_cap = std::min(wave, 2 * wave_cap);
    rc = arena_upto(first, hi);
    if (rc != GDP_OK) break;
    rc = slot_launch(ctx, ctx->slot[cur], pairs, first, count, arena_bytes, results, nullptr, wave_index++);
    if (rc != GDP_OK) break;
    first += count;
    {
      std::lock_guard<std::mutex> g(m);
      ctx->slot[cur].busy = true;
      launched.push_back(cur);
    }
    cv.notify_all();
    cur = (cur + 1) % NSLOTS;
  }
  {
    std::lock_guard<std::mutex> g(m);
    all_launched = true;
  }
  cv.notify_all();
  if (copy_out.joinable()) copy_out.join();
  else copy_out_loop();
  {
    std::lock_guard<std::mutex> g(m);
    outs_done = true;
  }
  cv.notify_all();
  if (expander.joinable()) expander.join();
  if (rc == GDP_OK) rc = out_rc;
  GDP_TRACE_BEGIN(tdrain);
  cudaError_t e = cudaStreamSynchronize(ctx->d2h);
  cudaError_t e2 = cudaSuccess;
  for (int k = 0; k < ctx->nwave; k++) {
    const cudaError_t ek = cudaStreamSynchronize(ctx->wave_stream[k]);
    if (e2 == cudaSuccess) e2 = ek;
  }
  GDP_TRACE_END(tdrain, "drain");
#ifdef GDP_HOST_TRACE
  fprintf(stderr, "gdp-trace host_enqueue_done %.3f ms\n",
          std::chrono::duration<double, std::milli>(tdrain - host0).count());
  for (auto &t : gdp_tev) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, gdp_tev[0].ev, t.ev);
    fprintf(stderr, "gdp-tev %8.3f %s (host %.3f)\n", ms, t.what,
            std::chrono::duration<double, std::milli>(t.host - gdp_tev[0].host).count());
  }
#endif
  if (rc == GDP_OK && e != cudaSuccess) rc = set_err(ctx, "batch copies", e);
  if (rc == GDP_OK && e2 != cudaSuccess) rc = set_err(ctx, "batch kernels", e2);
  /* record offsets are batch-wide: add_rec_base_kernel moved each wave's */
  if (rc == GDP_OK && overflow) rc = GDP_ERR_RECS;
  if (nrecs_used) *nrecs_used = base;
  return rc;
}

/*
 * One batch over several contexts (one per GPU, or several on one GPU).
 * Pairs are independent, so the batch splits into contiguous shards of
 * about equal band cells, one per context, each run by gdp_align_batch
 * from its own host thread; no data crosses between devices.  A shard
 * gets only its own part of the arena: its pairs' offsets are rebased to
 * the shard's first sequence byte (rounded down to 256, which keeps every
 * sequence's alignment).  Shard k's records start at the record slots
 * (rlength + glength + 2 per traceback pair) of the pairs before it, and
 * its results' rec_offset count from recs.
 */
extern "C" int
gdp_align_batch_multi (gdp_ctx *const *ctxs, int nctx, const gdp_pair_t *pairs, int64_t n, const char *arena,
                       int64_t arena_bytes, gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs,
                       int64_t *nrecs_used) {
  if (nrecs_used) *nrecs_used = 0;
  if (ctxs == nullptr || nctx < 1 || n < 0 || (n > 0 && (pairs == nullptr || results == nullptr))) return GDP_ERR_PARAM;
  for (int k = 0; k < nctx; k++)
    if (ctxs[k] == nullptr) return GDP_ERR_PARAM;
  if (n == 0) return GDP_OK;
  std::vector<int64_t> work(n + 1, 0), slots(n + 1, 0);
  for (int64_t i = 0; i < n; i++) {
    const gdp_pair_t &p = pairs[i];
    const int64_t rl = std::max(p.rlength, 0), gl = std::max(p.glength, 0);
    const int64_t band = std::max(p.lband, 0) + std::max(p.uband, 0) + 1;
    work[i + 1] = work[i] + 1 + (p.variant == GDP_LOWER ? gl : rl) * std::min<int64_t>(band, rl + gl + 1);
    slots[i + 1] = slots[i] + ((p.flags & GDP_FLAG_TRACEBACK) ? rl + gl + 2 : 0);
  }
  if (slots[n] > 0 && (recs == nullptr || max_recs < slots[n])) return GDP_ERR_RECS;
  std::vector<int64_t> first(nctx + 1, n);
  first[0] = 0;
  for (int k = 1; k < nctx; k++) {
    const int64_t target = work[n] / nctx * k;
    first[k] = std::max(first[k - 1], (int64_t) (std::lower_bound(work.begin(), work.end(), target) - work.begin()));
    first[k] = std::min(first[k], n);
  }
  std::vector<int> rc(nctx, GDP_OK);
  std::vector<int64_t> used(nctx, 0);
  auto run = [&](int k) {
    const int64_t lo = first[k], hi = first[k + 1], m = hi - lo;
    if (m <= 0) return;
    int64_t alo = (int64_t) 1 << 62, ahi = 0;
    for (int64_t i = lo; i < hi; i++) {
      const gdp_pair_t &p = pairs[i];
      const int64_t rl = std::max(p.rlength, 0), gl = std::max(p.glength, 0);
      alo = std::min(alo, std::min(std::min(p.rseq, p.rseq_uc), std::min(p.gseq, p.gseq_alt)));
      ahi = std::max(ahi, std::max(std::max(p.rseq + rl, p.rseq_uc + rl), std::max(p.gseq + gl, p.gseq_alt + gl)));
    }
    alo = std::min(std::max<int64_t>(alo, 0), arena_bytes) & ~(int64_t) 255;
    ahi = std::min(std::max(ahi, alo), arena_bytes);
    /* offsets out of the arena stay out of the shard's arena, so they fail
       validation as they would in one batch */
    std::vector<gdp_pair_t> sp(pairs + lo, pairs + hi);
    for (gdp_pair_t &p : sp) {
      p.rseq -= alo; p.rseq_uc -= alo; p.gseq -= alo; p.gseq_alt -= alo;
    }
    rc[k] = gdp_align_batch(ctxs[k], sp.data(), m, arena + alo, ahi - alo, results + lo,
                            slots[n] > 0 ? recs + slots[lo] : nullptr, slots[hi] - slots[lo], &used[k]);
    for (int64_t i = lo; i < hi; i++) results[i].rec_offset += slots[lo];
  };
  /* shard k > 0 on a thread of its own; a shard whose thread cannot be
     started runs on this thread after shard 0 */
  std::vector<std::thread> th;
  std::vector<int> inline_shards;
  for (int k = 1; k < nctx; k++) {
    try {
      th.emplace_back(run, k);
    } catch (...) {
      inline_shards.push_back(k);
    }
  }
  run(0);
  for (int k : inline_shards) run(k);
  for (auto &t : th) t.join();
  int64_t end = 0;
  for (int k = 0; k < nctx; k++) {
    if (rc[k] != GDP_OK) return rc[k];
    if (first[k + 1] > first[k] && used[k] > 0) end = slots[first[k]] + used[k];
  }
  if (nrecs_used) *nrecs_used = end;
  return GDP_OK;
}

/* ------------------------------------------------------------------ */
/* Parity/debug: dense dump of the compare domain                      */
/* ------------------------------------------------------------------ */

extern "C" int
gdp_fill_dump (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t n, const char *arena, int64_t arena_bytes,
               const int64_t *dense_offsets, int16_t *H, int8_t *dN, int8_t *dE, int8_t *dF,
               gdp_result_t *results) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::vector<gdp_pair_t> pp(pairs, pairs + n);
  for (auto &p : pp) p.flags &= ~GDP_FLAG_TRACEBACK;
  gdp_plan pl;
  int rc = plan_build(ctx, pp.data(), n, arena_bytes, pl.h);
  cudaStream_t s = ctx->stream;
  DevBuf dpairs, dres;
  for (int k = 0; k < NSLOTS; k++) cudaEventSynchronize(ctx->slot[k].out_done);
  /* without H the fills run exactly as in production: no score dump, so
     the steady and half-width column bodies take their columns */
  if (rc == GDP_OK) rc = plan_upload(ctx, pl.h, pl.d, H != nullptr, s);
  if (rc == GDP_OK) {
    cudaError_t e = ctx->arena.ensure(std::max<int64_t>(arena_bytes, 16));
    if (e == cudaSuccess) e = dpairs.ensure(std::max<int64_t>(n, 1) * sizeof(gdp_pair_t));
    if (e == cudaSuccess) e = dres.ensure(std::max<int64_t>(n, 1) * sizeof(gdp_result_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->arena.p, arena, arena_bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dpairs.p, pp.data(), n * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) rc = set_err(ctx, "dump staging", e);
  }
  if (rc == GDP_OK)
    rc = plan_run(ctx, pl.h, pl.d, dpairs.as<gdp_pair_t>(), ctx->arena.as<char>(), dres.as<gdp_result_t>(), nullptr);
  std::vector<uint32_t> words(std::max<int64_t>(pl.h.dir_words, 1));
  std::vector<int16_t> hs(H != nullptr ? std::max<int64_t>(pl.h.dir_words, 1) * 8 : 0);
  std::vector<gdp_meta_t> meta(std::max<int64_t>(n, 1));
  if (rc == GDP_OK) {
    cudaError_t e = cudaMemcpyAsync(results, dres.p, n * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(words.data(), pl.d.dirs.p, pl.h.dir_words * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && H != nullptr)
      e = cudaMemcpyAsync(hs.data(), pl.d.hdump.p, pl.h.dir_words * 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(meta.data(), pl.d.meta.p, n * sizeof(gdp_meta_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = set_err(ctx, "dump copy", e);
  }
  if (rc == GDP_OK) {
    for (int64_t i = 0; i < n; i++) {
      const gdp_pair_t &p = pp[i];
      if (results[i].status != GDP_OK) continue;
      const int W = results[i].precision == 8 ? 32 : 16;
      const int64_t base = (W == 16) ? meta[i].dir16 : meta[i].dir8;
      gdp_geom_t g;
      gdp_geom_of(&p, W, &g);
      std::vector<int64_t> boff((g.X / W) + 2, 0);
      for (int b = 0; b * W <= g.X; b++) boff[b + 1] = boff[b] + gdp_block_words(&g, b * W);
      const int R = p.rlength + 1;
      for (int c = 1; c <= p.glength; c++) {
        int lo, hi;
        if (p.variant == GDP_FULL) { lo = c - p.uband; hi = c + p.lband; }
        else if (p.variant == GDP_UPPER) { lo = c - p.uband; hi = c; }
        else { lo = c; hi = c + p.lband; }
        lo = std::max(lo, 1); hi = std::min(hi, p.rlength);
        for (int r = lo; r <= hi; r++) {
          const int x = (p.variant == GDP_LOWER) ? c : r, y = (p.variant == GDP_LOWER) ? r : c;
          const int b = x / W, lane = x - b * W;
          int y0, y1;
          gdp_block_sweep(&g, b * W, &y0, &y1);
          const int64_t at = dense_offsets[i] + (int64_t) c * R + r;
          if (y < y0 || y > y1) continue;
          const int64_t col = base + boff[b] + (int64_t) (y - y0) * (W / 8);
          const uint32_t w = words[col + gdp_dir_word(W, lane)];
          const int sh = gdp_dir_bit(W, lane);
          const int nh = (w >> sh) & 1, nv = (w >> (8 + sh)) & 1, ee = (w >> (16 + sh)) & 1, ff = (w >> (24 + sh)) & 1;
          if (H) H[at] = hs[col * 8 + lane];
          if (dN) dN[at] = (int8_t) (nv ? -2 : nh ? -1 : 0);
          if (dE) dE[at] = (int8_t) (ee ? -1 : 0);
          if (dF) dF[at] = (int8_t) (ff ? -2 : 0);
        }
      }
    }
  }
  pl.d.release();
  pl.h.release();
  dpairs.release();
  dres.release();
  return rc;
}

/* ------------------------------------------------------------------ */
/* Single-pair fill and traceback for the reference-signature entry    */
/* points (dropin.cu)                                                  */
/* ------------------------------------------------------------------ */


struct gdpi_fill {
  gdp_pair_t pair;
  gdp_plan pl;
  DevBuf dpairs, darena, dres, dlist, drecs, drecoff, dgenome, dgenomealt;
  std::vector<uint32_t> words;     /* host copy of the pair's direction words */
  std::vector<int16_t> scores;     /* host copy of the swept cells' scores (8 per word) */
  gdp_result_t res;
  gdp_meta_t meta;
};

gdpi_fill *gdpi_fill_new () { return new gdpi_fill(); }

int
gdpi_fill_run (gdp_ctx *ctx, gdpi_fill *f, const gdp_pair_t *p, const char *arena, int64_t arena_bytes) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  f->pair = *p;
  f->pair.flags &= ~GDP_FLAG_TRACEBACK;
  f->res.status = GDP_ERR_PARAM;
  cudaStream_t s = ctx->stream;
  int rc = plan_build(ctx, &f->pair, 1, arena_bytes, f->pl.h);
  if (rc == GDP_OK) rc = plan_upload(ctx, f->pl.h, f->pl.d, true, s);
  if (rc == GDP_OK) {
    cudaError_t e = f->dpairs.ensure(sizeof(gdp_pair_t));
    if (e == cudaSuccess) e = f->darena.ensure(std::max<int64_t>(arena_bytes, 16));
    if (e == cudaSuccess) e = f->dres.ensure(sizeof(gdp_result_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(f->dpairs.p, &f->pair, sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(f->darena.p, arena, arena_bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) rc = set_err(ctx, "single-pair staging", e);
  }
  if (rc == GDP_OK)
    rc = plan_run(ctx, f->pl.h, f->pl.d, f->dpairs.as<gdp_pair_t>(), f->darena.as<char>(), f->dres.as<gdp_result_t>(), nullptr);
  if (rc == GDP_OK) {
    const int64_t nw = std::max<int64_t>(f->pl.h.dir_words, 1);
    if ((int64_t) f->words.size() < nw) f->words.resize(nw);
    if ((int64_t) f->scores.size() < nw * 8) f->scores.resize(nw * 8);
    cudaError_t e = cudaMemcpyAsync(&f->res, f->dres.p, sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&f->meta, f->pl.d.meta.p, sizeof(gdp_meta_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && f->pl.h.dir_words > 0)
      e = cudaMemcpyAsync(f->words.data(), f->pl.d.dirs.p, f->pl.h.dir_words * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && f->pl.h.dir_words > 0)
      e = cudaMemcpyAsync(f->scores.data(), f->pl.d.hdump.p, f->pl.h.dir_words * 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = set_err(ctx, "single-pair results", e);
  }
  if (rc != GDP_OK) f->res.status = rc;
  return rc;
}

const uint32_t *gdpi_fill_words (const gdpi_fill *f) { return f->words.data(); }
const int16_t *gdpi_fill_scores (const gdpi_fill *f) { return f->scores.data(); }
int gdpi_fill_width (const gdpi_fill *f) { return f->res.precision == 8 ? 32 : 16; }
int64_t gdpi_fill_base (const gdpi_fill *f) { return f->res.precision == 8 ? f->meta.dir8 : f->meta.dir16; }
const gdp_result_t *gdpi_fill_result (const gdpi_fill *f) { return &f->res; }
const gdp_pair_t *gdpi_fill_pair (const gdpi_fill *f) { return &f->pair; }

int
gdpi_traceback_one (gdp_ctx *ctx, gdpi_fill *f, const gdp_pair_t *p, const char *arena, int64_t arena_bytes,
                    const uint32_t *gblocks, const uint32_t *galtblocks, uint64_t gbase, uint64_t glen,
                    gdp_result_t *res, std::vector<gdp_rec_t> *recs) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const int64_t cap = (int64_t) p->rlength + p->glength + 2;
  const size_t gwords = (size_t) ((glen + 31) / 32) * 3;
  const int32_t one[2] = {0, 1};
  const int64_t zero = 0;
  if (f->res.status != GDP_OK) return GDP_ERR_PARAM;   /* no usable fill behind this traceback */
  gdp_pair_t q = *p;
  q.flags |= GDP_FLAG_TRACEBACK;
  CK(ctx, f->dpairs.ensure(sizeof(gdp_pair_t)));
  CK(ctx, f->darena.ensure(std::max<int64_t>(arena_bytes, 16)));
  CK(ctx, f->dlist.ensure(2 * sizeof(int32_t)));
  CK(ctx, f->drecs.ensure(cap * sizeof(gdp_rec_t)));
  CK(ctx, f->drecoff.ensure(sizeof(int64_t)));
  CK(ctx, cudaMemcpyAsync(f->dpairs.p, &q, sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(f->darena.p, arena, arena_bytes, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(f->dlist.p, one, sizeof(one), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(f->drecoff.p, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(f->dres.p, &f->res, sizeof(gdp_result_t), cudaMemcpyHostToDevice, s));
  if (gblocks && gwords > 0) {
    CK(ctx, f->dgenome.ensure(gwords * 4));
    CK(ctx, f->dgenomealt.ensure(gwords * 4));
    CK(ctx, cudaMemcpyAsync(f->dgenome.p, gblocks, gwords * 4, cudaMemcpyHostToDevice, s));
    CK(ctx, cudaMemcpyAsync(f->dgenomealt.p, galtblocks ? galtblocks : gblocks, gwords * 4, cudaMemcpyHostToDevice, s));
  }
  TbParams T;
  T.pairs = f->dpairs.as<gdp_pair_t>();
  T.arena = f->darena.as<char>();
  T.list = f->dlist.as<int32_t>();
  T.count = f->dlist.as<int32_t>() + 1;
  T.dirs = f->pl.d.dirs.as<uint32_t>();
  T.meta = f->pl.d.meta.as<gdp_meta_t>();
  T.res = f->dres.as<gdp_result_t>();
  T.recs = f->drecs.as<gdp_rec_t>();
  T.rec_off = f->drecoff.as<int64_t>();
  T.genome = (gblocks && gwords > 0) ? f->dgenome.as<uint32_t>() : nullptr;
  T.genomealt = (gblocks && gwords > 0) ? f->dgenomealt.as<uint32_t>() : nullptr;
  T.genome_base = gbase;
  T.genome_len = glen;
  T.tab = ctx->d_tab;
  if (ctx->tb_warp) traceback_warp_kernel<<<1, 32, 0, s>>>(T);
  else traceback_kernel<<<1, 32, 0, s>>>(T);
  ctx->launches++;
  CK(ctx, cudaGetLastError());
  CK(ctx, cudaMemcpyAsync(res, f->dres.p, sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s));
  CK(ctx, cudaStreamSynchronize(s));
  recs->resize(std::max(res->nrecs, 0));
  if (res->nrecs > 0) {
    CK(ctx, cudaMemcpy(recs->data(), f->drecs.p, res->nrecs * sizeof(gdp_rec_t), cudaMemcpyDeviceToHost));
  }
  return GDP_OK;
}

void
gdpi_fill_free (gdpi_fill *f) {
  if (!f) return;
  f->pl.d.release();
  f->pl.h.release();
  f->dpairs.release(); f->darena.release(); f->dres.release(); f->dlist.release();
  f->drecs.release(); f->drecoff.release(); f->dgenome.release(); f->dgenomealt.release();
  delete f;
}

/* Replaces the context's substitution / consistency tables with the
   caller's own (a GMAP process that ran Dynprog_init). */
int
gdpi_set_tables (gdp_ctx *ctx, const gdp_tables_t *t) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  memcpy(ctx->h_tab, t, sizeof(gdp_tables_t));
  update_reach(ctx);
  CK(ctx, cudaMemcpyAsync(ctx->d_tab, ctx->h_tab, sizeof(gdp_tables_t), cudaMemcpyHostToDevice, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GDP_OK;
}

int
gdpi_plan_reuse (gdp_ctx *ctx, gdp_plan **plan, const gdp_pair_t *pairs, int64_t n) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  if (*plan == nullptr) *plan = new gdp_plan();
  gdp_plan *pl = *plan;
  int rc = plan_build(ctx, pairs, n, -1, pl->h);
  if (rc == GDP_OK) rc = plan_upload(ctx, pl->h, pl->d, false, ctx->stream);
  return rc;
}

int
gdpi_plan_reuse_dump (gdp_ctx *ctx, gdp_plan **plan, const gdp_pair_t *pairs, int64_t n) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  if (*plan == nullptr) *plan = new gdp_plan();
  gdp_plan *pl = *plan;
  int rc = plan_build(ctx, pairs, n, -1, pl->h);
  if (rc == GDP_OK) rc = plan_upload(ctx, pl->h, pl->d, true, ctx->stream);
  return rc;
}

const int16_t *
gdpi_plan_scores (const gdp_plan *plan) {
  return plan->d.hdump.as<int16_t>();
}

const gdp_meta_t *
gdpi_plan_meta (const gdp_plan *plan) {
  return plan->d.meta.as<gdp_meta_t>();
}

void
gdpi_single_release (gdpi_single_cfg *c) {
  for (int k = 0; k < gdpi_single_cfg::NBUF; k++) {
    if (c->dbuf[k]) cudaFree(c->dbuf[k]);
    if (c->hbuf[k]) cudaFreeHost(c->hbuf[k]);
    c->dbuf[k] = c->hbuf[k] = nullptr;
    c->dcap[k] = c->hcap[k] = 0;
  }
  if (c->plan) gdp_plan_destroy(c->plan);
  if (c->dump_plan) gdp_plan_destroy(c->dump_plan);
  c->plan = c->dump_plan = nullptr;
}

int
gdpi_view_of (gdp_ctx *ctx, gdpi_view *v) {
  if (ctx == nullptr || v == nullptr) return GDP_ERR_PARAM;
  v->device = ctx->device;
  v->stream = ctx->stream;
  v->d_tab = ctx->d_tab;
  v->d_genome = ctx->d_genome;
  v->d_genomealt = ctx->d_genomealt ? ctx->d_genomealt : ctx->d_genome;
  v->has_alt = ctx->d_genomealt != nullptr;
  v->genome_len = ctx->genome_len;
  v->budget = ctx->budget;
  v->nsm = ctx->nsm;
  v->single = &ctx->single;
  return GDP_OK;
}

void
gdpi_count_launch (gdp_ctx *ctx) {
  ctx->launches++;
}

int
gdpi_fail (gdp_ctx *ctx, const char *what, cudaError_t e) {
  return set_err(ctx, what, e);
}

/* ------------------------------------------------------------------ */
/* End-gap endpoint search: merging the two halves                     */
/* ------------------------------------------------------------------ */

extern "C" int
gdp_endpoint_combine (const gdp_result_t *upper, const gdp_result_t *lower, int jump_late, int qend, int precision,
                      int rlength, int *finalscore, int *bestr, int *bestc) {
  if (upper == nullptr || lower == nullptr || finalscore == nullptr || bestr == nullptr || bestc == nullptr)
    return GDP_ERR_PARAM;
  /* the reference scans each row's lower cells (c < r) before its upper
     cells (c >= r): row-then-column order over both halves */
  const gdp_result_t *best = nullptr;
  for (const gdp_result_t *h : {lower, upper}) {
    if (!h->end_found) continue;
    if (best == nullptr || h->end_score > best->end_score) { best = h; continue; }
    if (h->end_score < best->end_score) continue;
    const bool later = (h->end_r > best->end_r) || (h->end_r == best->end_r && h->end_c > best->end_c);
    if (jump_late ? later : !later) best = h;
  }
  if (best != nullptr) {
    *finalscore = best->end_score;
    *bestr = best->end_r;
    *bestc = best->end_c;
  } else if (qend) {
    *finalscore = precision == 8 ? -128 : -32768;   /* NEG_INFINITY_8 / _16 */
    *bestr = rlength;
    *bestc = 0;
  } else {
    *finalscore = 0;
    *bestr = 0;
    *bestc = 0;
  }
  return GDP_OK;
}
