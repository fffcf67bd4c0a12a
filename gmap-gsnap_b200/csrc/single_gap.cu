/*
 * single_gap.cu -- Dynprog_single_gap (src/dynprog_single.c:428-675) for a
 * batch of gaps: the single-gap step of GMAP's stage 3 (src/stage3.c:9117,
 * :9297, :9546), which fills the gap between two aligned blocks of a read
 * and traces it back.
 *
 * Per gap, the reference (1) returns no pairs when a length is out of range,
 * (2) reads the genome segment, (3) for equal lengths takes the ungapped
 * diagonal when it has at most one mismatch (single_gap_simple, :345-425),
 * and otherwise (4) widens the band with Dynprog_compute_bands
 * (src/dynprog.c:1246), fills with Dynprog_simd_8 or _16 by the use8p_size
 * rule (src/dynprog.c:1021-1024) and traces back from (rlength, glength).
 *
 * The batch runs that as two device phases around one host decision:
 *   - the caller's arena goes to the device once, with room for the genome
 *     segments of the gaps that need a fill behind it;
 *   - phase 1: one warp per equal-length gap walks its diagonal
 *     (single_simple_kernel) and writes the simple path's records;
 *   - the host reads which gaps took the simple path;
 *   - phase 2: the other gaps run as full-band pairs of the batch planner
 *     (gdp_plan_create / gdp_plan_execute), their segments read from the
 *     resident genome by the fill's window step (GDP_XFLAG_SEGMENT), cut
 *     into plans whose direction storage stays within the context budget.
 * Results and records come back per gap in the order of the List the
 * reference returns.
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <vector>
#include "gdp.h"
#include "gdp_internal.h"
#include "gdp_dropin_internal.h"
#include "genome_chars.cuh"

namespace {

/* Comparison characters (src/comp.h:5-8) and scores (src/scores.h:4-5). */
constexpr char COMP_DYNPROG_MATCH = '*', COMP_AMBIGUOUS = ':', COMP_MISMATCH = ' ';
constexpr int SCORE_MATCH = 1, SCORE_MISMATCH = -3;
constexpr int NEG_INFINITY_32 = -32768;   /* src/dynprog.h:158 */

struct SimpleOut {
  int32_t simple;              /* 1: the diagonal is the gap's alignment */
  int32_t score, nmatch, nmismatch, nrecs;
};

/*
 * single_gap_simple (src/dynprog_single.c:345-425) for one gap per warp:
 * query position q against segment position q (genomic coordinate
 * genomeoffset + q).  A '*' genome character (past the chromosome) pushes
 * nothing and scores nothing; an exact match against the genome or the
 * alternate genome scores MATCH ('*'), a consistent pair
 * (Dynprog_consistent_p) MATCH (':'), anything else MISMATCH (' ').  The path is taken when at most one position mismatched
 * and at least one pair was pushed (Pairpool_push drops negative
 * positions).  Records are written head first: the reference pushes from
 * the first position, so its List starts at the last one.
 */
__device__ __forceinline__ int
simple_class (const gdp_pair_t &p, const char *ruc, int q, const uint32_t *genome, const uint32_t *genomealt,
              uint64_t glen, const gdp_tables_t *tab, char *c2, char *c2a, bool *pushed) {
  *c2 = segment_char(p, p.genomeoffset + q, genome, genomealt, glen, c2a);
  *pushed = false;
  if (*c2 == '*') return 0;
  *pushed = (p.queryoffset + q >= 0) && (p.genomeoffset + q >= 0);
  const char c1uc = ruc[q];
  if (c1uc == *c2 || c1uc == *c2a) return 1;
  if (tab->cons[p.genestrand][c1uc & 127][*c2 & 127] || tab->cons[p.genestrand][c1uc & 127][*c2a & 127]) return 2;
  return 3;
}

__global__ void __launch_bounds__(256)
single_simple_kernel (const gdp_pair_t *cand, int64_t n, const char *arena, const int64_t *rec_off, gdp_rec_t *recs,
                      SimpleOut *out, const uint32_t *genome, const uint32_t *genomealt, uint64_t glen,
                      const gdp_tables_t *tab) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    const gdp_pair_t p = cand[i];
    const char *ruc = arena + p.rseq_uc;
    int nmatch = 0, nmis = 0, npush = 0;
    for (int q0 = 0; q0 < p.rlength && nmis <= 1; q0 += 32) {
      const int q = q0 + lane;
      int cls = 0;
      bool pushed = false;
      if (q < p.rlength) {
        char c2, c2a;
        cls = simple_class(p, ruc, q, genome, genomealt, glen, tab, &c2, &c2a, &pushed);
      }
      nmatch += __popc(__ballot_sync(0xffffffffu, cls == 1 || cls == 2));
      nmis += __popc(__ballot_sync(0xffffffffu, cls == 3));
      npush += __popc(__ballot_sync(0xffffffffu, pushed));
    }
    const bool simple = nmis <= 1 && npush > 0;
    if (lane == 0) {
      SimpleOut o;
      o.simple = simple ? 1 : 0;
      o.score = SCORE_MATCH * nmatch + SCORE_MISMATCH * nmis;
      o.nmatch = nmatch;
      o.nmismatch = nmis;
      o.nrecs = simple ? npush : 0;
      out[i] = o;
    }
    if (!simple) continue;
    const char *rs = arena + p.rseq;
    gdp_rec_t *dst = recs + rec_off[i];
    int before = 0;   /* records pushed at positions below this chunk */
    for (int q0 = 0; q0 < p.rlength; q0 += 32) {
      const int q = q0 + lane;
      int cls = 0;
      bool pushed = false;
      char c2 = 0, c2a = 0;
      if (q < p.rlength) cls = simple_class(p, ruc, q, genome, genomealt, glen, tab, &c2, &c2a, &pushed);
      const unsigned m = __ballot_sync(0xffffffffu, pushed);
      if (pushed) {
        gdp_rec_t r;
        r.querypos = p.queryoffset + q;
        r.genomepos = p.genomeoffset + q;
        r.cdna = rs[q];
        r.comp = cls == 1 ? COMP_DYNPROG_MATCH : cls == 2 ? COMP_AMBIGUOUS : COMP_MISMATCH;
        r.genome = c2;
        r.genomealt = c2a;
        dst[npush - 1 - (before + __popc(m & below))] = r;
      }
      before += __popc(m);
    }
  }
}

/* Stream-ordered device buffers of one call, freed on every return path. */
struct CallBufs {
  cudaStream_t s;
  std::vector<void *> held;
  explicit CallBufs (cudaStream_t st) : s(st) {}
  template <class T> cudaError_t get (T **p, int64_t count) {
    void *q = nullptr;
    cudaError_t e = cudaMallocAsync(&q, (size_t) std::max<int64_t>(count, 1) * sizeof(T), s);
    if (e == cudaSuccess) held.push_back(q);
    *p = (T *) q;
    return e;
  }
  ~CallBufs () { for (void *q : held) cudaFreeAsync(q, s); cudaStreamSynchronize(s); }
};

/* The reference's choices for one gap (src/dynprog_single.c:453-481, :612-617). */
struct GapSetup {
  int mismatchtype, open, extend, lband, uband, precision;
};

GapSetup
gap_setup (const gdp_single_gap_t &g, const gdpi_single_cfg &cfg) {
  GapSetup s;
  /* DEFECT_HIGHQ 0.003, DEFECT_MEDQ 0.014 (src/dynprog.h:58-59); single-gap
     penalties SINGLE_OPEN_* / SINGLE_EXTEND_* (src/dynprog.h:61-67) */
  static const int open_q[3] = {-8, -7, -6}, extend_q[3] = {-3, -2, -1}, mismatch_q[3] = {-3, -2, -1};
  const int q = g.defect_rate < 0.003 ? 0 : g.defect_rate < 0.014 ? 1 : 2;
  s.mismatchtype = q;   /* HIGHQ, MEDQ, LOWQ */
  s.open = cfg.user_p ? cfg.user_open : open_q[q];
  s.extend = cfg.user_p ? cfg.user_extend : extend_q[q];
  /* Dynprog_compute_bands */
  if (!g.widebandp) {
    s.lband = s.uband = g.extraband_single;
  } else if (g.glength >= g.rlength) {
    s.uband = g.glength - g.rlength + g.extraband_single;
    s.lband = g.extraband_single;
  } else {
    s.lband = g.rlength - g.glength + g.extraband_single;
    s.uband = g.extraband_single;
  }
  /* use8p_size[mismatchtype] = NEG_INFINITY_8 / MISMATCH_* - 1 */
  const int use8p = (-128) / mismatch_q[q] - 1;
  s.precision = (g.rlength < use8p && g.glength < use8p) ? 8 : 16;
  return s;
}

/* Whether the resident genome holds every position the gap's segment reads
   from the genome (positions outside the chromosome read as '*'). */
bool
segment_resident (const gdp_single_gap_t &g, uint64_t genome_len) {
  if (genome_len == 0) return false;
  const int64_t g0 = g.goffset, g1 = (int64_t) g.goffset + g.glength - 1;
  int64_t lo, hi;
  if (g.watsonp) {
    lo = (int64_t) g.chroffset + g0;
    hi = std::min<int64_t>((int64_t) g.chroffset + g1, (int64_t) g.chrhigh - 1);
  } else {
    lo = std::max<int64_t>((int64_t) g.chrhigh - g1, g.chroffset);
    hi = (int64_t) g.chrhigh - g0;
  }
  return lo > hi || (lo >= 0 && (uint64_t) hi < genome_len);
}

gdp_pair_t
base_pair (const gdp_single_gap_t &g) {
  gdp_pair_t p;
  memset(&p, 0, sizeof(p));
  p.rseq = g.rseq; p.rseq_uc = g.rseq_uc;
  p.rlength = g.rlength; p.glength = g.glength;
  p.variant = GDP_FULL;
  p.tb_r = g.rlength; p.tb_c = g.glength;
  p.queryoffset = g.roffset; p.genomeoffset = g.goffset;
  p.chroffset = g.chroffset; p.chrhigh = g.chrhigh;
  p.watsonp = g.watsonp; p.genestrand = g.genestrand;
  p.xflags = GDP_XFLAG_SEGMENT;
  p.dynprogindex = g.dynprogindex;
  return p;
}

}  // namespace

#define SCK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return gdpi_fail(ctx, #call, e_); } while (0)

extern "C" int
gdp_single_setup (gdp_ctx *ctx, int user_open, int user_extend, int user_dynprog_p, int homopolymerp) {
  gdpi_view v;
  if (gdpi_view_of(ctx, &v) != GDP_OK) return GDP_ERR_PARAM;
  if (homopolymerp) return GDP_ERR_PARAM;
  if (user_dynprog_p && (user_open < -127 || user_open > 0 || user_extend < -127 || user_extend > 0))
    return GDP_ERR_PARAM;
  v.single->user_open = user_open;
  v.single->user_extend = user_extend;
  v.single->user_p = user_dynprog_p != 0;
  return GDP_OK;
}

extern "C" int
gdp_single_gap_batch (gdp_ctx *ctx, const gdp_single_gap_t *gaps, int64_t n, const char *arena, int64_t arena_bytes,
                      gdp_result_t *results, int8_t *path, gdp_rec_t *recs, int64_t max_recs, int64_t *nrecs_used) {
  gdpi_view v;
  if (gdpi_view_of(ctx, &v) != GDP_OK || n < 0 || (n > 0 && (gaps == nullptr || results == nullptr)) ||
      arena_bytes < 0 || (arena_bytes > 0 && arena == nullptr) || max_recs < 0 || (max_recs > 0 && recs == nullptr))
    return GDP_ERR_PARAM;
  if (nrecs_used) *nrecs_used = 0;
  if (n == 0) return GDP_OK;
  SCK(cudaSetDevice(v.device));
  cudaStream_t s = v.stream;

  /* host decisions: NULL paths, simple candidates, fills */
  std::vector<int8_t> kind((size_t) n, GDP_SINGLE_NULL);
  std::vector<int64_t> cand, fill;
  for (int64_t i = 0; i < n; i++) {
    const gdp_single_gap_t &g = gaps[i];
    gdp_result_t &r = results[i];
    memset(&r, 0, sizeof(r));
    if (g.rlength <= 0 || g.glength <= 0 || g.rlength > g.max_rlength || g.glength > g.max_glength) {
      r.tb_score = NEG_INFINITY_32;
      continue;
    }
    if (g.rseq < 0 || g.rseq + g.rlength > arena_bytes || g.rseq_uc < 0 || g.rseq_uc + g.rlength > arena_bytes) {
      r.status = GDP_ERR_LEN;
      continue;
    }
    if (g.genestrand < 0 || g.genestrand > 2) { r.status = GDP_ERR_PARAM; continue; }
    if (!segment_resident(g, v.genome_len)) { r.status = GDP_ERR_NOGENOME; continue; }
    kind[i] = GDP_SINGLE_DP;
    if (g.glength == g.rlength) cand.push_back(i); else fill.push_back(i);
  }

  CallBufs B(s);
  /* the arena, followed by the segments of the gaps that may need a fill */
  const int64_t seg_base = (arena_bytes + 15) / 16 * 16;
  int64_t seg_bytes = 0;
  for (int64_t i = 0; i < n; i++)
    if (kind[i] == GDP_SINGLE_DP) seg_bytes += (int64_t) gaps[i].glength * (v.has_alt ? 2 : 1);
  char *d_arena = nullptr;
  SCK(B.get(&d_arena, seg_base + seg_bytes));
  if (arena_bytes > 0) SCK(cudaMemcpyAsync(d_arena, arena, arena_bytes, cudaMemcpyHostToDevice, s));

  /* phase 1: the ungapped diagonal of the equal-length gaps */
  std::vector<SimpleOut> sout(cand.size());
  std::vector<int64_t> soff(cand.size() + 1, 0);
  gdp_rec_t *d_srecs = nullptr;
  if (!cand.empty()) {
    std::vector<gdp_pair_t> cp(cand.size());
    for (size_t k = 0; k < cand.size(); k++) {
      cp[k] = base_pair(gaps[cand[k]]);
      soff[k + 1] = soff[k] + gaps[cand[k]].rlength;
    }
    gdp_pair_t *d_cp = nullptr;
    int64_t *d_soff = nullptr;
    SimpleOut *d_sout = nullptr;
    SCK(B.get(&d_cp, (int64_t) cand.size()));
    SCK(B.get(&d_soff, (int64_t) cand.size()));
    SCK(B.get(&d_sout, (int64_t) cand.size()));
    SCK(B.get(&d_srecs, soff.back()));
    SCK(cudaMemcpyAsync(d_cp, cp.data(), cp.size() * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
    SCK(cudaMemcpyAsync(d_soff, soff.data(), cand.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    const int64_t blocks = std::min<int64_t>(((int64_t) cand.size() + 7) / 8, (int64_t) v.nsm * 8);
    single_simple_kernel<<<(int) blocks, 256, 0, s>>>(d_cp, (int64_t) cand.size(), d_arena, d_soff, d_srecs, d_sout,
                                                       v.d_genome, v.d_genomealt, v.genome_len, v.d_tab);
    gdpi_count_launch(ctx);
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(sout.data(), d_sout, cand.size() * sizeof(SimpleOut), cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    for (size_t k = 0; k < cand.size(); k++) {
      if (sout[k].simple) kind[cand[k]] = GDP_SINGLE_SIMPLE;
      else fill.push_back(cand[k]);
    }
    std::sort(fill.begin(), fill.end());
  }

  /* phase 2: fills and tracebacks of the rest, in plans within the budget */
  std::vector<gdp_pair_t> fp(fill.size());
  {
    int64_t seg = seg_base;
    for (size_t k = 0; k < fill.size(); k++) {
      const gdp_single_gap_t &g = gaps[fill[k]];
      const GapSetup st = gap_setup(g, *v.single);
      gdp_pair_t p = base_pair(g);
      p.lband = st.lband; p.uband = st.uband;
      p.precision = (int8_t) st.precision;
      p.mismatchtype = (int8_t) st.mismatchtype;
      p.open = (int16_t) st.open; p.extend = (int16_t) st.extend;
      p.flags = GDP_FLAG_TRACEBACK | GDP_FLAG_GWINDOW | (g.jump_late_p ? GDP_FLAG_JUMP_LATE : 0);
      p.gseq = seg;
      p.gseq_alt = v.has_alt ? seg + g.glength : seg;
      seg += (int64_t) g.glength * (v.has_alt ? 2 : 1);
      fp[k] = p;
    }
  }
  std::vector<gdp_result_t> fres(fill.size());
  std::vector<gdp_rec_t> frecs;
  std::vector<int64_t> frec_base(fill.size(), 0);
  for (size_t k0 = 0; k0 < fill.size();) {
    /* one plan: gaps k0..k1 while their direction bytes stay in the budget */
    size_t k1 = k0;
    int64_t bytes = 0;
    while (k1 < fill.size()) {
      const int64_t b = gdp_pair_words(&fp[k1], fp[k1].precision == 8 ? 32 : 16) * 4;
      if (k1 > k0 && bytes + b > v.budget) break;
      bytes += b;
      k1++;
    }
    const int64_t m = (int64_t) (k1 - k0);
    gdp_plan *pl = nullptr;
    int rc = gdp_plan_create(ctx, fp.data() + k0, m, &pl);
    if (rc != GDP_OK) return rc;
    const int64_t nr = gdp_plan_total_recs(pl);
    gdp_pair_t *d_fp = nullptr;
    gdp_result_t *d_fres = nullptr;
    gdp_rec_t *d_frecs = nullptr;
    cudaError_t e = B.get(&d_fp, m);
    if (e == cudaSuccess) e = B.get(&d_fres, m);
    if (e == cudaSuccess) e = B.get(&d_frecs, nr);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_fp, fp.data() + k0, m * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { gdp_plan_destroy(pl); return gdpi_fail(ctx, "single-gap fill buffers", e); }
    rc = gdp_plan_execute(ctx, pl, d_fp, d_arena, d_fres, d_frecs);
    if (rc != GDP_OK) { gdp_plan_destroy(pl); return rc; }
    const size_t base = frecs.size();
    frecs.resize(base + (size_t) nr);
    e = cudaMemcpyAsync(fres.data() + k0, d_fres, m * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && nr > 0)
      e = cudaMemcpyAsync(frecs.data() + base, d_frecs, nr * sizeof(gdp_rec_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    gdp_plan_destroy(pl);
    if (e != cudaSuccess) return gdpi_fail(ctx, "single-gap fill results", e);
    for (int64_t k = 0; k < m; k++) frec_base[k0 + k] = (int64_t) base;
    k0 = k1;
  }

  /* simple records */
  std::vector<gdp_rec_t> srecs((size_t) soff.back());
  if (!cand.empty() && soff.back() > 0) {
    SCK(cudaMemcpyAsync(srecs.data(), d_srecs, soff.back() * sizeof(gdp_rec_t), cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
  }

  /* assemble per gap, in gap order */
  std::vector<int64_t> cand_of((size_t) n, -1), fill_of((size_t) n, -1);
  for (size_t k = 0; k < cand.size(); k++) cand_of[cand[k]] = (int64_t) k;
  for (size_t k = 0; k < fill.size(); k++) fill_of[fill[k]] = (int64_t) k;
  int64_t used = 0;
  for (int64_t i = 0; i < n; i++) {
    gdp_result_t &r = results[i];
    const gdp_rec_t *src = nullptr;
    int32_t cnt = 0;
    if (kind[i] == GDP_SINGLE_SIMPLE) {
      const SimpleOut &o = sout[cand_of[i]];
      r.tb_score = o.score; r.nmatches = o.nmatch; r.nmismatches = o.nmismatch;
      cnt = o.nrecs;
      src = srecs.data() + soff[cand_of[i]];
    } else if (kind[i] == GDP_SINGLE_DP) {
      const int64_t k = fill_of[i];
      r = fres[k];
      cnt = (r.status == GDP_OK) ? r.nrecs : 0;
      src = frecs.data() + frec_base[k] + r.rec_offset;
    }
    r.rec_offset = used;
    r.nrecs = cnt;
    if (cnt > 0) {
      if (used + cnt > max_recs) {
        r.status = GDP_ERR_RECS;
        r.nrecs = 0;
      } else {
        memcpy(recs + used, src, (size_t) cnt * sizeof(gdp_rec_t));
        used += cnt;
      }
    }
    if (path) path[i] = kind[i];
  }
  if (nrecs_used) *nrecs_used = used;
  return GDP_OK;
}
