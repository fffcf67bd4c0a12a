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
#include <cub/device/device_scan.cuh>
#include <algorithm>
#include <climits>
#include <cstring>
#include <thread>
#include <vector>
#include "gdp.h"
#include "gdp_internal.h"
#include "gdp_dropin_internal.h"
#include "gap_work.h"
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
 * (Dynprog_consistent_p) MATCH (':'), anything else MISMATCH (' ').  The
 * path is taken when at most one position mismatched and at least one pair
 * was pushed (Pairpool_push drops negative positions).  Records are written
 * head first: the reference pushes from the first position, so its List
 * starts at the last one.
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

/* Where a gap's outcome lives. */
enum { SRC_NULL = 0, SRC_SIMPLE = 1, SRC_FILL = 2, SRC_ERROR = 3 };
struct GapSrc {
  int32_t kind;
  int32_t idx;     /* SRC_SIMPLE: candidate index; SRC_FILL: fill index; SRC_ERROR: the status */
};

__global__ void __launch_bounds__(256)
single_count_kernel (const GapSrc *src, int64_t n, const SimpleOut *sout, const gdp_result_t *fres, int64_t *count) {
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t) gridDim.x * blockDim.x) {
    int64_t c = 0;
    if (i < n) {
      const GapSrc g = src[i];
      if (g.kind == SRC_SIMPLE) c = sout[g.idx].nrecs;
      else if (g.kind == SRC_FILL && fres[g.idx].status == GDP_OK) c = fres[g.idx].nrecs;
    }
    count[i] = c;   /* count[n] = 0: the scan's last entry is the total */
  }
}

/*
 * Final results and records in gap order, one warp per gap: the gap's
 * records go to out[off[i] ..) (a gap with records that would pass
 * max_recs gets GDP_ERR_RECS and none), and *used gets the end of the
 * records written.
 */
__global__ void __launch_bounds__(256)
single_gather_kernel (const GapSrc *src, int64_t n, const int64_t *off, int64_t max_recs, const SimpleOut *sout,
                      const gdp_rec_t *srecs, const int64_t *soff, const gdp_result_t *fres,
                      const gdp_rec_t *const *fslots, gdp_result_t *res, gdp_rec_t *out,
                      unsigned long long *used) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    const GapSrc g = src[i];
    gdp_result_t r;
    memset(&r, 0, sizeof(r));
    const gdp_rec_t *from = nullptr;
    int64_t cnt = 0;
    if (g.kind == SRC_NULL) {
      r.tb_score = NEG_INFINITY_32;
    } else if (g.kind == SRC_ERROR) {
      r.status = g.idx;
    } else if (g.kind == SRC_SIMPLE) {
      const SimpleOut o = sout[g.idx];
      r.tb_score = o.score; r.nmatches = o.nmatch; r.nmismatches = o.nmismatch;
      cnt = o.nrecs;
      from = srecs + soff[g.idx];
    } else {
      r = fres[g.idx];
      cnt = (r.status == GDP_OK) ? r.nrecs : 0;
      from = fslots[g.idx] + r.rec_offset;
    }
    const int64_t o = off[i];
    if (cnt > 0 && o + cnt > max_recs) {
      r.status = GDP_ERR_RECS;
      cnt = 0;
    }
    r.nrecs = (int32_t) cnt;
    r.rec_offset = o;
    /* a record is three 32-bit words */
    const uint32_t *fw = reinterpret_cast<const uint32_t *>(from);
    uint32_t *ow = reinterpret_cast<uint32_t *>(out + o);
    for (int64_t w = lane; w < 3 * cnt; w += 32) ow[w] = fw[w];
    if (lane == 0) {
      res[i] = r;
      if (cnt > 0) atomicMax(used, (unsigned long long) (o + cnt));
    }
  }
}

/* The context's grow-only working buffers: device slot k, pinned host slot k. */
enum { D_ARENA, D_CAND, D_SOFF, D_SOUT, D_SRECS, D_FILL, D_FRES, D_SLOTS, D_SRC, D_COUNT, D_OFF, D_FSLOT, D_RES,
       D_OUT, D_USED, D_TMP };
enum { H_CAND, H_SOFF, H_SOUT, H_FILL, H_FSEG, H_SRC, H_FSLOT, H_WORDS };

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

gdp_pair_t
fill_pair (const gdp_single_gap_t &g, const gdpi_single_cfg &cfg, int64_t seg, bool has_alt) {
  const GapSetup st = gap_setup(g, cfg);
  gdp_pair_t p = base_pair(g);
  p.lband = st.lband; p.uband = st.uband;
  p.precision = (int8_t) st.precision;
  p.mismatchtype = (int8_t) st.mismatchtype;
  p.open = (int16_t) st.open; p.extend = (int16_t) st.extend;
  p.flags = GDP_FLAG_TRACEBACK | GDP_FLAG_GWINDOW | (g.jump_late_p ? GDP_FLAG_JUMP_LATE : 0);
  p.gseq = seg;
  p.gseq_alt = has_alt ? seg + g.glength : seg;
  return p;
}

/* An upper bound of a fill's direction words: (rlength / W + 1) blocks of
   at most W + lband + uband swept columns, W / 8 words each. */
int64_t
words_bound (const gdp_pair_t &p) {
  const int W = p.precision == 8 ? 32 : 16;
  return ((int64_t) p.rlength / W + 1) * ((int64_t) W + p.lband + p.uband) * (W / 8);
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
  if (n > INT32_MAX) return GDP_ERR_LEN;   /* gap indices are 32-bit on the device */
  if (n == 0) return GDP_OK;
  SCK(cudaSetDevice(v.device));
  cudaStream_t s = v.stream;

  /* host decisions: NULL paths, simple candidates, fills */
  std::vector<int8_t> kind((size_t) n), cls((size_t) n);   /* cls: 0 no fill, 1 diagonal candidate, 2 fill */
  par_for(n, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; i++) {
      const gdp_single_gap_t &g = gaps[i];
      gdp_result_t &r = results[i];
      memset(&r, 0, sizeof(r));
      kind[i] = GDP_SINGLE_NULL;
      cls[i] = 0;
      if (g.rlength <= 0 || g.glength <= 0 || g.rlength > g.max_rlength || g.glength > g.max_glength) {
        r.tb_score = NEG_INFINITY_32;
      } else if (g.rseq < 0 || g.rseq + g.rlength > arena_bytes || g.rseq_uc < 0 ||
                 g.rseq_uc + g.rlength > arena_bytes) {
        r.status = GDP_ERR_LEN;
      } else if (g.genestrand < 0 || g.genestrand > 2) {
        r.status = GDP_ERR_PARAM;
      } else if (!segment_resident(g, v.genome_len)) {
        r.status = GDP_ERR_NOGENOME;
      } else {
        kind[i] = GDP_SINGLE_DP;
        cls[i] = (g.glength == g.rlength) ? 1 : 2;
      }
    }
  });
  std::vector<int64_t> cand, fill;
  std::vector<int32_t> where((size_t) n, -1);   /* a gap's candidate or fill index */
  int64_t seg_bytes = 0;
  for (int64_t i = 0; i < n; i++) {
    if (cls[i] == 1) { where[i] = (int32_t) cand.size(); cand.push_back(i); }
    else if (cls[i] == 2) { where[i] = (int32_t) fill.size(); fill.push_back(i); }
    if (cls[i] != 0) seg_bytes += (int64_t) gaps[i].glength * (v.has_alt ? 2 : 1);
  }

  gdpi_single_cfg *C = v.single;
  /* the arena, followed by the segments of the gaps that may need a fill */
  const int64_t seg_base = (arena_bytes + 15) / 16 * 16;
  char *d_arena = nullptr;
  SCK(dev_slot(C, D_ARENA, &d_arena, seg_base + seg_bytes));
  if (arena_bytes > 0) SCK(cudaMemcpyAsync(d_arena, arena, arena_bytes, cudaMemcpyHostToDevice, s));

  /* fill descriptors: the gaps that are not candidates first; the
     candidates whose diagonal does not hold join after phase 1 */
  const int64_t nc = (int64_t) cand.size();
  const int64_t nf_max = (int64_t) fill.size() + nc;
  gdp_pair_t *fp = nullptr;
  int64_t *fseg = nullptr;
  SCK(host_slot(C, H_FILL, &fp, nf_max));
  SCK(host_slot(C, H_FSEG, &fseg, nf_max + 1));
  const int64_t mult = v.has_alt ? 2 : 1;
  fseg[0] = seg_base;
  for (size_t k = 0; k < fill.size(); k++) fseg[k + 1] = fseg[k] + gaps[fill[k]].glength * mult;

  /* phase 1: the ungapped diagonal of the equal-length gaps */
  gdp_rec_t *d_srecs = nullptr;
  int64_t *d_soff = nullptr;
  SimpleOut *d_sout = nullptr;
  SimpleOut *sout = nullptr;
  if (nc > 0) {
    gdp_pair_t *cp = nullptr, *d_cp = nullptr;
    int64_t *soff = nullptr;
    SCK(host_slot(C, H_CAND, &cp, nc));
    SCK(host_slot(C, H_SOFF, &soff, nc + 1));
    SCK(host_slot(C, H_SOUT, &sout, nc));
    soff[0] = 0;
    for (int64_t k = 0; k < nc; k++) soff[k + 1] = soff[k] + gaps[cand[k]].rlength;
    par_for(nc, [&](int64_t lo, int64_t hi) {
      for (int64_t k = lo; k < hi; k++) cp[k] = base_pair(gaps[cand[k]]);
    });
    SCK(dev_slot(C, D_CAND, &d_cp, nc));
    SCK(dev_slot(C, D_SOFF, &d_soff, nc));
    SCK(dev_slot(C, D_SOUT, &d_sout, nc));
    SCK(dev_slot(C, D_SRECS, &d_srecs, soff[nc]));
    SCK(cudaMemcpyAsync(d_cp, cp, nc * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
    SCK(cudaMemcpyAsync(d_soff, soff, nc * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    const int64_t blocks = std::min<int64_t>((nc + 7) / 8, (int64_t) v.nsm * 8);
    single_simple_kernel<<<(int) blocks, 256, 0, s>>>(d_cp, nc, d_arena, d_soff, d_srecs, d_sout, v.d_genome,
                                                       v.d_genomealt, v.genome_len, v.d_tab);
    gdpi_count_launch(ctx);
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(sout, d_sout, nc * sizeof(SimpleOut), cudaMemcpyDeviceToHost, s));
  }
  /* while the diagonal runs: the other fills' descriptors */
  par_for((int64_t) fill.size(), [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; k++) fp[k] = fill_pair(gaps[fill[k]], *C, fseg[k], v.has_alt);
  });
  if (nc > 0) {
    SCK(cudaStreamSynchronize(s));
    for (int64_t k = 0; k < nc; k++) {
      const int64_t i = cand[k];
      if (sout[k].simple) {
        kind[i] = GDP_SINGLE_SIMPLE;
      } else {
        const int64_t f = (int64_t) fill.size();
        fp[f] = fill_pair(gaps[i], *C, fseg[f], v.has_alt);
        fseg[f + 1] = fseg[f] + gaps[i].glength * mult;
        where[i] = (int32_t) f;
        fill.push_back(i);
      }
    }
  }

  /* phase 2: fills and tracebacks, in plans within the budget */
  const int64_t nf = (int64_t) fill.size();
  gdp_pair_t *d_fp = nullptr;
  gdp_result_t *d_fres = nullptr;
  gdp_rec_t *d_slots = nullptr;
  const gdp_rec_t **fslot = nullptr, **d_fslot = nullptr;
  SCK(host_slot(C, H_FSLOT, &fslot, nf));
  int64_t slot_total = 0, bound = 0;   /* record slots (rlength + glength + 2 each), direction words */
  for (int64_t k = 0; k < nf; k++) {
    slot_total += (int64_t) fp[k].rlength + fp[k].glength + 2;
    bound += words_bound(fp[k]);
  }
  SCK(dev_slot(C, D_FILL, &d_fp, nf));
  SCK(dev_slot(C, D_FRES, &d_fres, nf));
  SCK(dev_slot(C, D_SLOTS, &d_slots, slot_total));
  if (nf > 0) SCK(cudaMemcpyAsync(d_fp, fp, nf * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
  int64_t slot_used = 0;
  for (int64_t k0 = 0; k0 < nf;) {
    /* one plan: gaps k0..k1 while their direction bytes stay in the budget */
    int64_t k1 = nf;
    if (bound * 4 > v.budget) {
      int64_t bytes = 0;
      for (k1 = k0; k1 < nf; k1++) {
        const int64_t b = gdp_pair_words(&fp[k1], fp[k1].precision == 8 ? 32 : 16) * 4;
        if (k1 > k0 && bytes + b > v.budget) break;
        bytes += b;
      }
    }
    int rc = gdpi_plan_reuse(ctx, &C->plan, fp + k0, k1 - k0);
    if (rc != GDP_OK) return rc;
    const int64_t nr = gdp_plan_total_recs(C->plan);
    if (slot_used + nr > slot_total) return GDP_ERR_RECS;   /* the planner's bound is the one above */
    rc = gdp_plan_execute(ctx, C->plan, d_fp + k0, d_arena, d_fres + k0, d_slots + slot_used);
    if (rc != GDP_OK) return rc;
    for (int64_t k = k0; k < k1; k++) fslot[k] = d_slots + slot_used;
    slot_used += nr;
    if (k1 < nf) SCK(cudaStreamSynchronize(s));   /* the plan's buffers are reused by the next plan */
    k0 = k1;
  }

  /* results and records in gap order, on the device */
  GapSrc *src = nullptr, *d_src = nullptr;
  SCK(host_slot(C, H_SRC, &src, n));
  par_for(n, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; i++) {
      GapSrc g{SRC_NULL, 0};
      if (kind[i] == GDP_SINGLE_NULL) {
        if (results[i].status != GDP_OK) g = GapSrc{SRC_ERROR, results[i].status};
      } else {
        g = GapSrc{kind[i] == GDP_SINGLE_SIMPLE ? SRC_SIMPLE : SRC_FILL, where[i]};
      }
      src[i] = g;
      if (path) path[i] = kind[i];
    }
  });
  int64_t *d_count = nullptr, *d_off = nullptr, *words = nullptr;
  gdp_result_t *d_res = nullptr;
  gdp_rec_t *d_out = nullptr;
  unsigned long long *d_used = nullptr;
  SCK(host_slot(C, H_WORDS, &words, 2));
  SCK(dev_slot(C, D_SRC, &d_src, n));
  SCK(dev_slot(C, D_COUNT, &d_count, n + 1));
  SCK(dev_slot(C, D_OFF, &d_off, n + 1));
  SCK(dev_slot(C, D_FSLOT, &d_fslot, nf));
  SCK(dev_slot(C, D_RES, &d_res, n));
  SCK(dev_slot(C, D_USED, &d_used, 1));
  SCK(cudaMemcpyAsync(d_src, src, n * sizeof(GapSrc), cudaMemcpyHostToDevice, s));
  if (nf > 0) SCK(cudaMemcpyAsync(d_fslot, fslot, nf * sizeof(gdp_rec_t *), cudaMemcpyHostToDevice, s));
  SCK(cudaMemsetAsync(d_used, 0, sizeof(unsigned long long), s));
  const int cblocks = (int) std::min<int64_t>((n + 256) / 256, (int64_t) v.nsm * 8);
  single_count_kernel<<<cblocks, 256, 0, s>>>(d_src, n, d_sout, d_fres, d_count);
  gdpi_count_launch(ctx);
  SCK(cudaGetLastError());
  size_t tmp_bytes = 0;
  SCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_count, d_off, n + 1, s));
  char *d_tmp = nullptr;
  SCK(dev_slot(C, D_TMP, &d_tmp, (int64_t) tmp_bytes));
  SCK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_count, d_off, n + 1, s));
  /* the records end where the scan does, or earlier when max_recs cuts them */
  SCK(cudaMemcpyAsync(&words[0], d_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  SCK(dev_slot(C, D_OUT, &d_out, std::min(words[0], max_recs)));
  const int gblocks = (int) std::min<int64_t>((n + 7) / 8, (int64_t) v.nsm * 8);
  single_gather_kernel<<<gblocks, 256, 0, s>>>(d_src, n, d_off, max_recs, d_sout, d_srecs, d_soff, d_fres, d_fslot,
                                                d_res, d_out, d_used);
  gdpi_count_launch(ctx);
  SCK(cudaGetLastError());
  SCK(cudaMemcpyAsync(results, d_res, n * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaMemcpyAsync(&words[1], d_used, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  const int64_t used = words[1];
  if (used > 0) {
    SCK(cudaMemcpyAsync(recs, d_out, used * sizeof(gdp_rec_t), cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
  }
  if (nrecs_used) *nrecs_used = used;
  return GDP_OK;
}
