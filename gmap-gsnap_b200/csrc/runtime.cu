/*
 * runtime.cu -- host runtime and C ABI of libgdp (include/gdp.h).
 *
 * A context owns a CUDA stream, the device copy of the substitution tables
 * (built as Dynprog_init builds them), an optional resident genome, and
 * growable device buffers.  A batch is planned on the host: pairs are
 * validated, binned by fill kind (lane width W, variant, tie rule, pass)
 * and sorted by work within each bin so that the threads of a warp run
 * pairs of similar size; direction storage and traceback record slots are
 * laid out by prefix sums.  Execution enqueues one fill kernel per
 * non-empty bin and one traceback kernel, all on the context stream.
 *
 * 8-bit pairs flagged GDP_FLAG_RERUN16 follow the overflow contract: the
 * 16-bit fill runs first and records the largest in-band score; when that
 * reaches 127 the 8-bit fill would overflow too (its in-band scores are
 * never below the 16-bit ones unless it saturates at the top), so the
 * 16-bit outputs are kept.  Otherwise the 8-bit fill runs and its outputs
 * are kept unless it reaches 127 in the band or ends at or below -98.
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "gdp_internal.h"
#include "fill_thread.cuh"
#include "traceback.cuh"

#define GDP_VERSION "gdp-b200 0.1"

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure (size_t want) {
    if (want <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t grow = want + want / 4 + 4096;
    cudaError_t e = cudaMalloc(&p, grow);
    if (e == cudaSuccess) bytes = grow;
    return e;
  }
  void release () { if (p) cudaFree(p); p = nullptr; bytes = 0; }
};

constexpr int NKINDS = 24;   /* (W32, variant, late, pass) */

inline int kind_id (int w32, int variant, int late, int pass) {
  return (((w32 * 3 + variant) * 2 + late) * 2) + pass;
}

}  // namespace

struct gdp_ctx {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  gdp_tables_t *h_tab = nullptr;
  gdp_tables_t *d_tab = nullptr;
  uint32_t *d_genome = nullptr, *d_genomealt = nullptr;
  uint64_t genome_len = 0;
  int64_t budget = 0;
  DevBuf pairs, arena, results, recs, scratch;
  std::atomic<int64_t> launches{0};
  std::string err;
  std::mutex mu;
  /* optional per-launch timing: (kernel id, start, stop) */
  bool profiling = false;
  struct Timed { int id; cudaEvent_t a, b; };
  std::vector<Timed> timed;
  double prof_ms[32] = {0};
  int64_t prof_n[32] = {0};
};

/* kernel ids for profiling: 0..23 fill kinds, 24 traceback, 25 init */
static const char *
kernel_name (int id) {
  static char buf[32][48];
  if (id == 24) return "traceback_kernel";
  if (id == 25) return "init_results_kernel";
  if (id == 26) return "int_peak_kernel";
  const int pass = id & 1, late = (id >> 1) & 1, vw = id >> 2, variant = vw % 3, w32 = vw / 3;
  snprintf(buf[id], sizeof(buf[id]), "fill_thread<W%d,%s,%s,%s>", w32 ? 32 : 16,
           variant == 0 ? "full" : variant == 1 ? "upper" : "lower", late ? "late" : "early",
           pass ? (w32 ? "8bit-check" : "16bit-track") : "plain");
  return buf[id];
}

static void
prof_begin (gdp_ctx *ctx, int id, cudaEvent_t *a) {
  (void) id;
  if (!ctx->profiling) return;
  cudaEventCreate(a);
  cudaEventRecord(*a, ctx->stream);
}

static void
prof_end (gdp_ctx *ctx, int id, cudaEvent_t a) {
  if (!ctx->profiling) return;
  cudaEvent_t b;
  cudaEventCreate(&b);
  cudaEventRecord(b, ctx->stream);
  ctx->timed.push_back({id, a, b});
}

struct gdp_plan {
  int64_t n = 0;
  std::vector<int32_t> lists;          /* kinds' lists, then the traceback list */
  int64_t start[NKINDS + 2] = {0};
  int32_t counts[NKINDS + 1] = {0};
  int maxY[NKINDS] = {0};
  std::vector<gdp_meta_t> meta;
  std::vector<int64_t> rec_off;
  std::vector<int32_t> status;
  int64_t dir_words = 0, total_recs = 0;
  /* device copies */
  int32_t *d_lists = nullptr, *d_counts = nullptr, *d_status = nullptr;
  gdp_meta_t *d_meta0 = nullptr, *d_meta = nullptr;
  int64_t *d_rec_off = nullptr;
  uint32_t *d_dirs = nullptr;
  int16_t *d_hdump = nullptr;          /* debug: scores of every swept cell */
};

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

extern "C" int
gdp_ctx_create (gdp_ctx **out, int device, int mode, int64_t budget) {
  *out = nullptr;
  if (mode < 0 || mode > 6) return GDP_ERR_PARAM;
  gdp_ctx *ctx = new gdp_ctx();
  ctx->device = device;
  ctx->budget = budget > 0 ? budget : (int64_t) 40 << 30;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { delete ctx; return GDP_ERR_CUDA; }
  cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return GDP_ERR_CUDA; }
  ctx->h_tab = (gdp_tables_t *) malloc(sizeof(gdp_tables_t));
  gdp_build_tables(ctx->h_tab, mode);
  if (cudaMalloc(&ctx->d_tab, sizeof(gdp_tables_t)) != cudaSuccess ||
      cudaMemcpy(ctx->d_tab, ctx->h_tab, sizeof(gdp_tables_t), cudaMemcpyHostToDevice) != cudaSuccess) {
    gdp_ctx_destroy(ctx);
    return GDP_ERR_CUDA;
  }
  *out = ctx;
  return GDP_OK;
}

extern "C" void
gdp_ctx_destroy (gdp_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->pairs.release(); ctx->arena.release(); ctx->results.release();
  ctx->recs.release(); ctx->scratch.release();
  if (ctx->d_tab) cudaFree(ctx->d_tab);
  if (ctx->d_genome) cudaFree(ctx->d_genome);
  if (ctx->d_genomealt) cudaFree(ctx->d_genomealt);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  free(ctx->h_tab);
  delete ctx;
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

extern "C" int
gdp_profile_read (gdp_ctx *ctx, int id, char *name, int name_cap, double *ms, int64_t *launches) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (id < 0 || id >= 27) return GDP_ERR_PARAM;
  if (!ctx->timed.empty()) {
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
  if (name && name_cap > 0) snprintf(name, name_cap, "%s", kernel_name(id));
  if (ms) *ms = ctx->prof_ms[id];
  if (launches) *launches = ctx->prof_n[id];
  return GDP_OK;
}

extern "C" int
gdp_profile_reset (gdp_ctx *ctx) {
  double dummy;
  gdp_profile_read(ctx, 0, nullptr, 0, &dummy, nullptr);
  std::lock_guard<std::mutex> lk(ctx->mu);
  for (int i = 0; i < 32; i++) { ctx->prof_ms[i] = 0; ctx->prof_n[i] = 0; }
  return GDP_OK;
}

/*
 * Integer issue-rate probe: every thread runs 16 independent dependency
 * chains of 32-bit add / min-max / multiply-add, so the SMs issue integer
 * lane-ops as fast as their pipes allow.  Used as the roofline denominator
 * of the integer-bound fill.  kind 0: IADD3 + IMNMX (ALU pipe), kind 1:
 * IMAD (FMA pipe), kind 2: both interleaved.
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
        a[k] = max(a[k] + b, c - k);          /* 2 ops */
      } else if (kind == 1) {
        a[k] = a[k] * b + c;                  /* 1 op (IMAD) */
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
  size_t words = (size_t) ((len + 31) / 32) * 3;
  cudaSetDevice(ctx->device);
  if (ctx->d_genome) cudaFree(ctx->d_genome);
  if (ctx->d_genomealt) cudaFree(ctx->d_genomealt);
  ctx->d_genome = ctx->d_genomealt = nullptr;
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
validate (const gdp_pair_t &p) {
  if (p.variant < GDP_FULL || p.variant > GDP_LOWER) return GDP_ERR_PARAM;
  if (p.precision != 8 && p.precision != 16) return GDP_ERR_PARAM;
  if (p.mismatchtype < 0 || p.mismatchtype > 3) return GDP_ERR_PARAM;
  if (p.open < -127 || p.open > 0 || p.extend < -127 || p.extend > 0) return GDP_ERR_PARAM;
  if (p.genestrand < 0 || p.genestrand > 2) return GDP_ERR_PARAM;
  if (p.rlength <= 0 || p.glength <= 0 || p.rlength > (1 << 20) || p.glength > (1 << 20)) return GDP_ERR_LEN;
  if (p.lband < 0 || p.uband < 0) return GDP_ERR_BAND;
  if (p.flags & GDP_FLAG_TRACEBACK) {
    if (p.tb_r < 0 || p.tb_c < 0 || p.tb_r > p.rlength || p.tb_c > p.glength) return GDP_ERR_BAND;
  }
  return GDP_OK;
}

static int64_t
work_of (const gdp_pair_t &p, int W) {
  return gdp_pair_words(&p, W);
}

static void
plan_free_device (gdp_plan *pl) {
  cudaFree(pl->d_lists); cudaFree(pl->d_counts); cudaFree(pl->d_status);
  cudaFree(pl->d_meta0); cudaFree(pl->d_meta); cudaFree(pl->d_rec_off);
  cudaFree(pl->d_dirs); cudaFree(pl->d_hdump);
  pl->d_lists = pl->d_counts = pl->d_status = nullptr;
  pl->d_meta0 = pl->d_meta = nullptr;
  pl->d_rec_off = nullptr; pl->d_dirs = nullptr; pl->d_hdump = nullptr;
}

static int
plan_build (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t n, bool hdump, gdp_plan **out) {
  gdp_plan *pl = new gdp_plan();
  pl->n = n;
  pl->meta.resize(n);
  pl->rec_off.assign(n, 0);
  pl->status.assign(n, GDP_OK);
  std::vector<std::vector<std::pair<int64_t, int32_t>>> bins(NKINDS);
  std::vector<int32_t> tb;
  int64_t words = 0, recs = 0;
  for (int64_t i = 0; i < n; i++) {
    const gdp_pair_t &p = pairs[i];
    gdp_meta_t &m = pl->meta[i];
    m.dir16 = m.dir8 = -1;
    m.maxh16 = -32768; m.status8 = 0; m.final8 = 0; m.pad = 0;
    int st = validate(p);
    pl->status[i] = st;
    if (st != GDP_OK) continue;
    const int late = (p.flags & GDP_FLAG_JUMP_LATE) ? 1 : 0;
    const bool rerun = p.precision == 8 && (p.flags & GDP_FLAG_RERUN16);
    gdp_geom_t g16, g8;
    gdp_geom_of(&p, 16, &g16);
    gdp_geom_of(&p, 32, &g8);
    if (p.precision == 16 || rerun) {
      m.dir16 = words;
      words += (gdp_pair_words(&p, 16) + 3) & ~(int64_t) 3;   /* keep blocks 16-byte aligned */
      bins[kind_id(0, p.variant, late, rerun ? 1 : 0)].push_back({work_of(p, 16), (int32_t) i});
    }
    if (p.precision == 8) {
      m.dir8 = words;
      words += (gdp_pair_words(&p, 32) + 3) & ~(int64_t) 3;
      bins[kind_id(1, p.variant, late, rerun ? 1 : 0)].push_back({work_of(p, 32), (int32_t) i});
    }
    if (p.flags & GDP_FLAG_TRACEBACK) {
      pl->rec_off[i] = recs;
      recs += (int64_t) p.rlength + p.glength + 2;
      tb.push_back((int32_t) i);
    }
  }
  pl->dir_words = words;
  pl->total_recs = recs;
  int64_t at = 0;
  for (int k = 0; k < NKINDS; k++) {
    auto &b = bins[k];
    std::stable_sort(b.begin(), b.end(), [](const std::pair<int64_t, int32_t> &a,
                                            const std::pair<int64_t, int32_t> &c) { return a.first > c.first; });
    pl->start[k] = at;
    pl->counts[k] = (int32_t) b.size();
    int maxY = 0;
    for (auto &e : b) {
      pl->lists.push_back(e.second);
      const gdp_pair_t &p = pairs[e.second];
      maxY = std::max(maxY, p.variant == GDP_LOWER ? p.rlength : p.glength);
    }
    pl->maxY[k] = maxY;
    at += (int64_t) b.size();
  }
  pl->start[NKINDS] = at;
  pl->counts[NKINDS] = (int32_t) tb.size();
  for (int32_t i : tb) pl->lists.push_back(i);
  pl->start[NKINDS + 1] = at + (int64_t) tb.size();

  cudaSetDevice(ctx->device);
  const size_t nl = std::max<size_t>(pl->lists.size(), 1);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_lists, nl * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_counts, (NKINDS + 1) * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_status, std::max<int64_t>(n, 1) * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_meta0, std::max<int64_t>(n, 1) * sizeof(gdp_meta_t));
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_meta, std::max<int64_t>(n, 1) * sizeof(gdp_meta_t));
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_rec_off, std::max<int64_t>(n, 1) * sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_dirs, std::max<int64_t>(words, 4) * sizeof(uint32_t));
  if (e == cudaSuccess && hdump) e = cudaMalloc(&pl->d_hdump, std::max<int64_t>(words, 4) * 8 * sizeof(int16_t));
  if (e == cudaSuccess && !pl->lists.empty())
    e = cudaMemcpy(pl->d_lists, pl->lists.data(), pl->lists.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pl->d_counts, pl->counts, (NKINDS + 1) * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n > 0) {
    e = cudaMemcpy(pl->d_status, pl->status.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pl->d_meta0, pl->meta.data(), n * sizeof(gdp_meta_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pl->d_rec_off, pl->rec_off.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    plan_free_device(pl);
    delete pl;
    return set_err(ctx, "plan allocation", e);
  }
  *out = pl;
  return GDP_OK;
}

extern "C" int
gdp_plan_create (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t npairs, gdp_plan **plan) {
  return plan_build(ctx, pairs, npairs, false, plan);
}

extern "C" void
gdp_plan_destroy (gdp_plan *pl) {
  if (!pl) return;
  plan_free_device(pl);
  delete pl;
}

extern "C" int64_t gdp_plan_total_recs (const gdp_plan *pl) { return pl->total_recs; }
extern "C" int64_t gdp_plan_rec_offset (const gdp_plan *pl, int64_t i) { return pl->rec_off[i]; }
extern "C" int64_t gdp_plan_dir_bytes (const gdp_plan *pl) { return pl->dir_words * 4; }

/* ------------------------------------------------------------------ */
/* Execution                                                           */
/* ------------------------------------------------------------------ */

__global__ void
init_results_kernel (gdp_result_t *res, const int32_t *status, const gdp_pair_t *pairs, int64_t n) {
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
    gdp_result_t r;
    r.status = status[i];
    r.score = 0;
    r.precision = pairs[i].precision;
    r.rerun = 0;
    r.tb_score = r.nmatches = r.nmismatches = r.nopens = r.nindels = 0;
    r.nrecs = 0;
    r.rec_offset = 0;
    res[i] = r;
  }
}

typedef void (*fill_fn)(FillParams);

template <int W, int V, bool L, int M>
static void launch_fill (FillParams P, int grid, cudaStream_t s) {
  fill_thread_kernel<W, V, L, M><<<grid, 128, 0, s>>>(P);
}

static void
launch_kind (int k, FillParams P, int grid, cudaStream_t s) {
  const int pass = k & 1, late = (k >> 1) & 1, vw = k >> 2, variant = vw % 3, w32 = vw / 3;
#define GDP_CASE(W32, VAR, LATE)                                                                   \
  if (w32 == W32 && variant == VAR && late == LATE) {                                             \
    if (W32) { if (pass) launch_fill<32, VAR, LATE, 2>(P, grid, s); else launch_fill<32, VAR, LATE, 0>(P, grid, s); } \
    else { if (pass) launch_fill<16, VAR, LATE, 1>(P, grid, s); else launch_fill<16, VAR, LATE, 0>(P, grid, s); }     \
    return;                                                                                        \
  }
  GDP_CASE(0, 0, false) GDP_CASE(0, 0, true) GDP_CASE(0, 1, false) GDP_CASE(0, 1, true)
  GDP_CASE(0, 2, false) GDP_CASE(0, 2, true) GDP_CASE(1, 0, false) GDP_CASE(1, 0, true)
  GDP_CASE(1, 1, false) GDP_CASE(1, 1, true) GDP_CASE(1, 2, false) GDP_CASE(1, 2, true)
#undef GDP_CASE
}

static int
plan_run (gdp_ctx *ctx, gdp_plan *pl, const gdp_pair_t *d_pairs, const char *d_arena,
          gdp_result_t *d_res, gdp_rec_t *d_recs) {
  cudaStream_t s = ctx->stream;
  const int64_t n = pl->n;
  if (n == 0) return GDP_OK;
  cudaEvent_t ev0 = nullptr;
  prof_begin(ctx, 25, &ev0);
  init_results_kernel<<<(int) std::min<int64_t>((n + 255) / 256, 4096), 256, 0, s>>>(d_res, pl->d_status, d_pairs, n);
  prof_end(ctx, 25, ev0);
  ctx->launches++;
  CK(ctx, cudaMemcpyAsync(pl->d_meta, pl->d_meta0, n * sizeof(gdp_meta_t), cudaMemcpyDeviceToDevice, s));
  /* scratch for the largest kind */
  size_t need = 0;
  for (int k = 0; k < NKINDS; k++) {
    if (!pl->counts[k]) continue;
    const int64_t grid = std::min<int64_t>((pl->counts[k] + 127) / 128, (int64_t) ctx->nsm * 16);
    need = std::max(need, (size_t) (pl->maxY[k] + 1) * (size_t) grid * 128 * sizeof(int2));
  }
  CK(ctx, ctx->scratch.ensure(std::max<size_t>(need, 64)));
  /* 16-bit and plain passes first, then the 8-bit passes of rerun pairs */
  for (int round = 0; round < 2; round++) {
    for (int k = 0; k < NKINDS; k++) {
      const int w32 = (k >> 2) / 3, pass = k & 1;
      const bool second = (w32 == 1 && pass == 1);
      if ((round == 0) == second || !pl->counts[k]) continue;
      const int grid = (int) std::min<int64_t>((pl->counts[k] + 127) / 128, (int64_t) ctx->nsm * 16);
      FillParams P;
      P.pairs = d_pairs; P.arena = d_arena;
      P.list = pl->d_lists + pl->start[k];
      P.count = pl->d_counts + k;
      P.dirs = pl->d_dirs;
      P.hdump = pl->d_hdump;
      P.meta = pl->d_meta;
      P.res = d_res;
      P.scratch = (int2 *) ctx->scratch.p;
      P.nslots = (int64_t) grid * 128;
      P.scratch_rows = pl->maxY[k] + 1;
      P.tab = ctx->d_tab;
      cudaEvent_t ev = nullptr;
      prof_begin(ctx, k, &ev);
      launch_kind(k, P, grid, s);
      prof_end(ctx, k, ev);
      ctx->launches++;
      CK(ctx, cudaGetLastError());
    }
  }
  if (pl->counts[NKINDS] > 0) {
    TbParams T;
    T.pairs = d_pairs; T.arena = d_arena;
    T.list = pl->d_lists + pl->start[NKINDS];
    T.count = pl->d_counts + NKINDS;
    T.dirs = pl->d_dirs; T.meta = pl->d_meta; T.res = d_res; T.recs = d_recs;
    T.rec_off = pl->d_rec_off;
    T.genome = ctx->d_genome; T.genomealt = ctx->d_genomealt;
    T.genome_len = ctx->genome_len;
    T.tab = ctx->d_tab;
    const int grid = (int) std::min<int64_t>((pl->counts[NKINDS] + 127) / 128, (int64_t) ctx->nsm * 16);
    cudaEvent_t ev = nullptr;
    prof_begin(ctx, 24, &ev);
    traceback_kernel<<<grid, 128, 0, s>>>(T);
    prof_end(ctx, 24, ev);
    ctx->launches++;
    CK(ctx, cudaGetLastError());
  }
  return GDP_OK;
}

extern "C" int
gdp_plan_execute (gdp_ctx *ctx, gdp_plan *pl, const gdp_pair_t *d_pairs, const char *d_arena,
                  gdp_result_t *d_results, gdp_rec_t *d_recs) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  return plan_run(ctx, pl, d_pairs, d_arena, d_results, d_recs);
}

/* Uploads pairs/arena, runs, and leaves results on the device. */
static int
stage_and_run (gdp_ctx *ctx, gdp_plan *pl, const gdp_pair_t *pairs, int64_t n,
               const char *arena, int64_t arena_bytes) {
  cudaStream_t s = ctx->stream;
  CK(ctx, ctx->pairs.ensure(std::max<int64_t>(n, 1) * sizeof(gdp_pair_t)));
  CK(ctx, ctx->arena.ensure(std::max<int64_t>(arena_bytes, 16)));
  CK(ctx, ctx->results.ensure(std::max<int64_t>(n, 1) * sizeof(gdp_result_t)));
  CK(ctx, ctx->recs.ensure(std::max<int64_t>(pl->total_recs, 1) * sizeof(gdp_rec_t)));
  CK(ctx, cudaMemcpyAsync(ctx->pairs.p, pairs, n * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->arena.p, arena, arena_bytes, cudaMemcpyHostToDevice, s));
  return plan_run(ctx, pl, (const gdp_pair_t *) ctx->pairs.p, (const char *) ctx->arena.p,
                  (gdp_result_t *) ctx->results.p, (gdp_rec_t *) ctx->recs.p);
}

extern "C" int
gdp_align_batch (gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t n, const char *arena, int64_t arena_bytes,
                 gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs, int64_t *nrecs_used) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  gdp_plan *pl = nullptr;
  int rc = plan_build(ctx, pairs, n, false, &pl);
  if (rc != GDP_OK) return rc;
  cudaStream_t s = ctx->stream;
  rc = stage_and_run(ctx, pl, pairs, n, arena, arena_bytes);
  if (rc == GDP_OK) {
    cudaError_t e = cudaMemcpyAsync(results, ctx->results.p, n * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = set_err(ctx, "results", e);
  }
  if (rc == GDP_OK) {
    /* compact the records in push order per pair */
    int64_t used = 0;
    for (int64_t i = 0; i < n; i++) used += results[i].nrecs;
    if (recs == nullptr || used > max_recs) {
      rc = (used == 0) ? GDP_OK : GDP_ERR_RECS;
    } else if (used > 0) {
      std::vector<gdp_rec_t> all(pl->total_recs);
      cudaError_t e = cudaMemcpyAsync(all.data(), ctx->recs.p, pl->total_recs * sizeof(gdp_rec_t),
                                      cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) {
        rc = set_err(ctx, "records", e);
      } else {
        int64_t at = 0;
        for (int64_t i = 0; i < n; i++) {
          const int nr = results[i].nrecs;
          if (nr > 0) memcpy(recs + at, all.data() + pl->rec_off[i], nr * sizeof(gdp_rec_t));
          results[i].rec_offset = at;
          at += nr;
        }
      }
    }
    if (nrecs_used) *nrecs_used = used;
  }
  gdp_plan_destroy(pl);
  return rc;
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
  gdp_plan *pl = nullptr;
  int rc = plan_build(ctx, pp.data(), n, true, &pl);
  if (rc != GDP_OK) return rc;
  cudaStream_t s = ctx->stream;
  rc = stage_and_run(ctx, pl, pp.data(), n, arena, arena_bytes);
  std::vector<uint32_t> words(std::max<int64_t>(pl->dir_words, 1));
  std::vector<int16_t> hs(std::max<int64_t>(pl->dir_words, 1) * 8);
  std::vector<gdp_meta_t> meta(std::max<int64_t>(n, 1));
  if (rc == GDP_OK) {
    cudaError_t e = cudaMemcpyAsync(results, ctx->results.p, n * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(words.data(), pl->d_dirs, pl->dir_words * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hs.data(), pl->d_hdump, pl->dir_words * 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(meta.data(), pl->d_meta, n * sizeof(gdp_meta_t), cudaMemcpyDeviceToHost, s);
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
          const int64_t widx = base + boff[b] + (int64_t) (y - y0) * (W / 8) + (lane >> 3);
          const uint32_t w = words[widx];
          const int sh = lane & 7;
          const int nh = (w >> sh) & 1, nv = (w >> (8 + sh)) & 1, ee = (w >> (16 + sh)) & 1, ff = (w >> (24 + sh)) & 1;
          if (H) H[at] = hs[(base + boff[b] + (int64_t) (y - y0) * (W / 8)) * 8 + lane];
          if (dN) dN[at] = (int8_t) (nv ? -2 : nh ? -1 : 0);
          if (dE) dE[at] = (int8_t) (ee ? -1 : 0);
          if (dF) dF[at] = (int8_t) (ff ? -2 : 0);
        }
      }
    }
  }
  gdp_plan_destroy(pl);
  return rc;
}
