/*
 * end_gap.cu -- Dynprog_end5_gap / Dynprog_end3_gap (src/dynprog_end.c:
 * 1293-1650, :1923-2245) for a batch of end gaps.
 *
 * An end gap aligns the part of a read beyond its last aligned block
 * against the genome that follows it (end 3) or precedes it (end 5).  The
 * reference fills an upper and a lower matrix, scans them for the best
 * endpoint, and traces back from that cell through one of the two.  Here
 * the host makes every decision the reference makes -- penalties by defect
 * rate, length cuts, bands, precision, which endpoint search -- and the
 * device does the work, with the caller's arena and every intermediate
 * result resident in device memory:
 *
 *   1. every gap's upper and lower fill as pairs of the batch planner, with
 *      the endpoint search fused in (GDP_FLAG_ENDPOINT / _QEND) and the
 *      genome segment read from the resident genome (GDP_FLAG_GWINDOW with
 *      the end's segment rule); only the search's results come back;
 *   2. the host merges each gap's halves (gdp_endpoint_combine) into the
 *      reference's best cell;
 *   3. per gap one fill and its traceback from the best cell: through the
 *      upper fill when bestc >= bestr, else the lower.  The fill of step 3
 *      is the one of step 1 again (fills are deterministic), so no
 *      direction storage is kept between the steps;
 *   4. on the device, the reference's last steps: no pairs and score 0
 *      when nmatches + 1 < nmismatches (QUERYEND_GAP, BEST_LOCAL), else
 *      the List in the reference's order (its head is the first pair the
 *      traceback pushed) without its leading indel pairs, reversed once
 *      more for end 5; the records are compacted in gap order and copied
 *      out once.
 *
 * The query.  The reference fills end 3 with rsequenceuc and traces back
 * with rsequence and rsequenceuc; this library's fills read the pair's
 * rseq.  The substitution tables score a lower-case query letter as its
 * upper-case letter (Dynprog_init's PREUC), so filling with rsequence gives
 * the same matrices whenever rsequenceuc is rsequence upper-cased, which is
 * how GMAP passes them (queryuc_ptr).
 */
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>
#include <string.h>
#include <algorithm>
#include <vector>

#include "gdp.h"
#include "gdp_internal.h"
#include "gdp_dropin_internal.h"
#include "gap_work.h"

namespace {

/* The reference's choices for one gap. */
struct EndSetup {
  bool null_result;   /* no pairs, score and counts 0, no device work */
  int rlength, glength;
  int open, extend, lband, uband, precision;
  bool qend;          /* the last-row search (QUERYEND_INDELS) */
};

EndSetup
end_setup (const gdp_end_gap_t &g, const gdpi_single_cfg &cfg) {
  EndSetup s;
  memset(&s, 0, sizeof(s));
  /* ENDQ; END_OPEN_* / END_EXTEND_* by defect rate (src/dynprog_end.c:88-94,
     DEFECT_HIGHQ 0.003, DEFECT_MEDQ 0.014) */
  if (cfg.end_user_p) { s.open = cfg.end_open; s.extend = cfg.end_extend; }
  else if (g.defect_rate < 0.003) { s.open = -10; s.extend = -2; }
  else if (g.defect_rate < 0.014) { s.open = -8; s.extend = -2; }
  else { s.open = -6; s.extend = -2; }
  s.rlength = g.rlength;
  s.glength = g.glength;
  /* the length checks, in the reference's order */
  if (s.rlength <= 0) { s.null_result = true; return s; }
  if (s.rlength > g.max_rlength) s.rlength = g.max_rlength;
  if (g.end == 5 && g.goffset < 0) { s.null_result = true; return s; }
  if (s.glength <= 0) { s.null_result = true; return s; }
  if (s.glength > g.max_glength) s.glength = g.max_glength;
  /* Dynprog_compute_bands: wide bands for QUERYEND_GAP / BEST_LOCAL, not
     for QUERYEND_INDELS (src/dynprog.c:1246-1261) */
  s.qend = (g.endalign == GDP_QUERYEND_INDELS);
  const int x = g.extraband_end;
  if (s.qend) {
    s.lband = s.uband = x;
  } else if (s.glength >= s.rlength) {
    s.uband = s.glength - s.rlength + x;
    s.lband = x;
  } else {
    s.lband = s.rlength - s.glength + x;
    s.uband = x;
  }
  /* use8p_size[ENDQ] = NEG_INFINITY_8 / MISMATCH_ENDQ - 1 = 24, with || */
  s.precision = (s.rlength < 24 || s.glength < 24) ? 8 : 16;
  return s;
}

/* One fill of a gap: the upper or the lower matrix, the gap's genome
   segment at `seg` in the device arena. */
gdp_pair_t
end_pair (const gdp_end_gap_t &g, const EndSetup &s, int variant, int64_t seg, bool has_alt) {
  gdp_pair_t p;
  memset(&p, 0, sizeof(p));
  const bool end5 = (g.end == 5);
  /* end 5 points at the query's last character and reads backwards */
  p.rseq = end5 ? g.rseq - (s.rlength - 1) : g.rseq;
  p.rseq_uc = end5 ? g.rseq_uc - (s.rlength - 1) : g.rseq_uc;
  p.gseq = seg;
  p.gseq_alt = has_alt ? seg + s.glength : seg;
  p.rlength = s.rlength;
  p.glength = s.glength;
  p.variant = (int8_t) variant;
  if (variant == GDP_UPPER) p.uband = s.uband;
  else p.lband = s.lband;
  p.precision = (int8_t) s.precision;
  p.mismatchtype = GDP_ENDQ;
  p.open = (int16_t) s.open;
  p.extend = (int16_t) s.extend;
  /* end 5 runs its fills with revp and the tie rule reversed */
  const bool late = end5 ? !g.jump_late_p : (g.jump_late_p != 0);
  p.flags = (int8_t) (GDP_FLAG_GWINDOW | (end5 ? GDP_FLAG_REVP : 0) | (late ? GDP_FLAG_JUMP_LATE : 0));
  p.queryoffset = g.roffset;
  p.genomeoffset = g.goffset;
  p.chroffset = g.chroffset;
  p.chrhigh = g.chrhigh;
  p.watsonp = g.watsonp;
  p.genestrand = g.genestrand;
  p.xflags = end5 ? GDP_XFLAG_SEGMENT_REV : GDP_XFLAG_SEGMENT;
  p.dynprogindex = g.dynprogindex;
  return p;
}

/* An upper bound of a fill's direction words: (rlength / W + 1) blocks of
   at most W + lband + uband swept columns, W / 8 words each. */
int64_t
words_bound (const gdp_pair_t &p) {
  const int W = p.precision == 8 ? 32 : 16;
  return ((int64_t) p.rlength / W + 1) * ((int64_t) W + p.lband + p.uband) * (W / 8);
}

/* What the device post-processing needs of a traced gap. */
struct TbInfo {
  int8_t end5;      /* the List is reversed once more */
  int8_t reject;    /* QUERYEND_GAP / BEST_LOCAL: nmatches + 1 < nmismatches empties it */
  int16_t pad;
};

__device__ __forceinline__ bool
rejected (const gdp_result_t &r, const TbInfo &t) {
  return t.reject && r.nmatches + 1 < r.nmismatches;
}

/*
 * Per traced gap, one warp: the number of leading indel pairs of its List
 * (the records in push order, which List_reverse puts at the head), and
 * how many records the gap keeps; count[n] = 0, so that the scan's last
 * entry is the total.
 */
__global__ void __launch_bounds__(256)
end_count_kernel (const gdp_result_t *res, const TbInfo *info, const gdp_rec_t *const *slots, int64_t n,
                  int32_t *first, int64_t *count) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  for (int64_t k = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5; k <= n; k += nwarps) {
    if (k == n) {
      if (lane == 0) count[n] = 0;
      continue;
    }
    const gdp_result_t r = res[k];
    int f = 0, keep = 0;
    if (r.status == GDP_OK && !rejected(r, info[k]) && r.nrecs > 0) {
      const gdp_rec_t *rec = slots[k] + r.rec_offset;
      f = r.nrecs;
      for (int base = 0; base < r.nrecs; base += 32) {
        const int j = base + lane;
        const bool indel = j < r.nrecs && rec[j].comp == '-';
        const unsigned stop = __ballot_sync(0xffffffffu, !indel);
        if (stop) {
          f = min(base + __ffs(stop) - 1, r.nrecs);
          break;
        }
      }
      keep = r.nrecs - f;
    }
    if (lane == 0) {
      first[k] = f;
      count[k] = keep;
    }
  }
}

/*
 * Per traced gap, one warp: its kept records to out[off[k] ..), reversed
 * for end 5 (a gap whose records would pass max_recs gets GDP_ERR_RECS and
 * none), and its final result: nrecs and rec_offset of the compacted
 * records, score and traceback score 0 when the List was rejected.  *used
 * gets the end of the records written.
 */
__global__ void __launch_bounds__(256)
end_gather_kernel (gdp_result_t *res, const TbInfo *info, const gdp_rec_t *const *slots, const int32_t *first,
                   const int64_t *count, const int64_t *off, int64_t n, int64_t max_recs, gdp_rec_t *out,
                   unsigned long long *used) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  for (int64_t k = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nwarps) {
    gdp_result_t r = res[k];
    const TbInfo t = info[k];
    int64_t cnt = count[k];
    const int64_t o = off[k];
    if (cnt > 0 && o + cnt > max_recs) {
      r.status = GDP_ERR_RECS;
      cnt = 0;
    }
    if (cnt > 0) {
      const gdp_rec_t *src = slots[k] + r.rec_offset + first[k];
      for (int64_t j = lane; j < cnt; j += 32) out[o + j] = t.end5 ? src[cnt - 1 - j] : src[j];
    }
    __syncwarp();
    if (lane == 0) {
      if (r.status == GDP_OK && rejected(r, t)) r.score = r.tb_score = 0;   /* the counts stay */
      else if (r.status == GDP_OK) r.score = r.tb_score;
      r.nrecs = (int32_t) cnt;
      r.rec_offset = o;
      res[k] = r;
      if (cnt > 0) atomicMax(used, (unsigned long long) (o + cnt));
    }
  }
}

/* The context's working slots of the end-gap batch. */
enum { D_ARENA, D_P1, D_R1, D_P2, D_R2, D_SLOTS, D_FSLOT, D_INFO, D_FIRST, D_COUNT, D_OFF, D_OUT, D_USED, D_TMP };
enum { H_P1, H_R1, H_P2, H_FSLOT, H_INFO, H_WORDS, H_R2 };

}  // namespace

#define SCK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return gdpi_fail(ctx, #call, e_); } while (0)

/* Runs pairs d_p[0..n) (host copies in hp) as plans whose direction words
   stay within the context budget, results to d_res, records (when the
   pairs trace back) into d_slots from *slot_used on; slot_base[k] gets the
   records' base of pair k (may be NULL). */
static int
run_plans (gdp_ctx *ctx, const gdpi_view &v, const gdp_pair_t *hp, const gdp_pair_t *d_p, int64_t n,
           char *d_arena, gdp_result_t *d_res, gdp_rec_t *d_slots, int64_t slot_cap, int64_t *slot_used,
           const gdp_rec_t **slot_base) {
  gdpi_single_cfg *C = v.single;
  int64_t bound = 0;
  for (int64_t k = 0; k < n; k++) bound += words_bound(hp[k]);
  for (int64_t k0 = 0; k0 < n;) {
    /* one plan: pairs k0..k1 while their direction bytes stay in the budget */
    int64_t k1 = n;
    if (bound * 4 > v.budget) {
      int64_t bytes = 0;
      for (k1 = k0; k1 < n; k1++) {
        const int64_t b = gdp_pair_words(&hp[k1], hp[k1].precision == 8 ? 32 : 16) * 4;
        if (k1 > k0 && bytes + b > v.budget) break;
        bytes += b;
      }
    }
    int rc = gdpi_plan_reuse(ctx, &C->plan, hp + k0, k1 - k0);
    if (rc != GDP_OK) return rc;
    const int64_t nr = gdp_plan_total_recs(C->plan);
    if (*slot_used + nr > slot_cap) return GDP_ERR_RECS;   /* the caller's bound is the planner's */
    rc = gdp_plan_execute(ctx, C->plan, d_p + k0, d_arena, d_res + k0, d_slots + *slot_used);
    if (rc != GDP_OK) return rc;
    if (slot_base)
      for (int64_t k = k0; k < k1; k++) slot_base[k] = d_slots + *slot_used;
    *slot_used += nr;
    if (k1 < n) SCK(cudaStreamSynchronize(v.stream));   /* the plan's buffers are reused by the next plan */
    k0 = k1;
  }
  return GDP_OK;
}

extern "C" int
gdp_end_setup (gdp_ctx *ctx, int user_open, int user_extend, int user_dynprog_p) {
  gdpi_view v;
  if (gdpi_view_of(ctx, &v) != GDP_OK) return GDP_ERR_PARAM;
  if (user_dynprog_p && (user_open < -127 || user_open > 0 || user_extend < -127 || user_extend > 0))
    return GDP_ERR_PARAM;
  v.single->end_open = user_open;
  v.single->end_extend = user_extend;
  v.single->end_user_p = user_dynprog_p != 0;
  return GDP_OK;
}

extern "C" int
gdp_end_gap_batch (gdp_ctx *ctx, const gdp_end_gap_t *gaps, int64_t n, const char *arena, int64_t arena_bytes,
                   gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs, int64_t *nrecs_used) {
  gdpi_view v;
  if (gdpi_view_of(ctx, &v) != GDP_OK || n < 0 || (n > 0 && (gaps == nullptr || results == nullptr)) ||
      arena_bytes < 0 || (arena_bytes > 0 && arena == nullptr) || max_recs < 0 || (max_recs > 0 && recs == nullptr))
    return GDP_ERR_PARAM;
  if (nrecs_used) *nrecs_used = 0;
  if (n == 0) return GDP_OK;
  SCK(cudaSetDevice(v.device));
  cudaStream_t s = v.stream;
  gdpi_single_cfg *C = v.single;

  /* the reference's decisions, per gap */
  std::vector<EndSetup> st((size_t) n);
  std::vector<int8_t> fills((size_t) n, 0);
  par_for(n, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; i++) {
      const gdp_end_gap_t &g = gaps[i];
      memset(&results[i], 0, sizeof(gdp_result_t));
      st[i] = end_setup(g, *C);
      if (g.end != 5 && g.end != 3) { results[i].status = GDP_ERR_PARAM; continue; }
      if (g.endalign == GDP_QUERYEND_NOGAPS || g.endalign < 0 || g.endalign > GDP_BEST_LOCAL) {
        results[i].status = GDP_ERR_PARAM;
        continue;
      }
      if (st[i].null_result || g.require_pos_score_p) continue;
      /* the query bytes the fills read must lie in the arena */
      const int64_t r0 = (g.end == 5) ? g.rseq - (st[i].rlength - 1) : g.rseq;
      const int64_t u0 = (g.end == 5) ? g.rseq_uc - (st[i].rlength - 1) : g.rseq_uc;
      if (r0 < 0 || u0 < 0 || r0 + st[i].rlength > arena_bytes || u0 + st[i].rlength > arena_bytes) {
        results[i].status = GDP_ERR_LEN;
        continue;
      }
      fills[i] = 1;
    }
  });
  std::vector<int64_t> fill;   /* the gaps with fills, in gap order */
  for (int64_t i = 0; i < n; i++)
    if (fills[i]) fill.push_back(i);
  const int64_t nf = (int64_t) fill.size();
  if (nf == 0) return GDP_OK;

  /* the arena on the device, then each filled gap's genome segment (and its
     alternate), written there by the fills' window step */
  const int64_t mult = v.has_alt ? 2 : 1;
  const int64_t seg_base = (arena_bytes + 15) / 16 * 16;
  std::vector<int64_t> seg((size_t) nf + 1);
  seg[0] = seg_base;
  for (int64_t k = 0; k < nf; k++) seg[k + 1] = seg[k] + ((int64_t) st[fill[k]].glength * mult + 15) / 16 * 16;
  char *d_arena = nullptr;
  SCK(dev_slot(C, D_ARENA, &d_arena, seg[nf]));
  if (arena_bytes > 0) SCK(cudaMemcpyAsync(d_arena, arena, arena_bytes, cudaMemcpyHostToDevice, s));

  /* run 1: the upper and lower fill of every gap with the endpoint search */
  gdp_pair_t *p1 = nullptr, *d_p1 = nullptr;
  gdp_result_t *r1 = nullptr, *d_r1 = nullptr;
  gdp_rec_t *d_slots = nullptr;
  SCK(host_slot(C, H_P1, &p1, 2 * nf));
  SCK(host_slot(C, H_R1, &r1, 2 * nf));
  SCK(dev_slot(C, D_P1, &d_p1, 2 * nf));
  SCK(dev_slot(C, D_R1, &d_r1, 2 * nf));
  par_for(nf, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; k++) {
      const int64_t i = fill[k];
      const int search = st[i].qend ? GDP_FLAG_ENDPOINT_QEND : GDP_FLAG_ENDPOINT;
      for (int h = 0; h < 2; h++) {
        gdp_pair_t p = end_pair(gaps[i], st[i], h == 0 ? GDP_UPPER : GDP_LOWER, seg[k], v.has_alt);
        p.flags = (int8_t) (p.flags | search);
        p1[2 * k + h] = p;
      }
    }
  });
  SCK(cudaMemcpyAsync(d_p1, p1, 2 * nf * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
  SCK(dev_slot(C, D_SLOTS, &d_slots, 1));
  int64_t slot_used = 0;
  int rc = run_plans(ctx, v, p1, d_p1, 2 * nf, d_arena, d_r1, d_slots, 1, &slot_used, nullptr);
  if (rc != GDP_OK) return rc;
  SCK(cudaMemcpyAsync(r1, d_r1, 2 * nf * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));

  /* each gap's best cell, and the pair that traces back from it */
  gdp_pair_t *p2 = nullptr;
  TbInfo *info = nullptr;
  SCK(host_slot(C, H_P2, &p2, nf));
  SCK(host_slot(C, H_INFO, &info, nf));
  std::vector<int64_t> gap2((size_t) nf, -1);
  int64_t n2 = 0, slot_total = 0;
  for (int64_t k = 0; k < nf; k++) {
    const int64_t i = fill[k];
    const gdp_result_t &up = r1[2 * k], &lo = r1[2 * k + 1];
    gdp_result_t &res = results[i];
    if (up.status != GDP_OK || lo.status != GDP_OK) {
      res.status = up.status != GDP_OK ? up.status : lo.status;
      continue;
    }
    const gdp_end_gap_t &g = gaps[i];
    const bool late = (g.end == 5) ? !g.jump_late_p : (g.jump_late_p != 0);
    int fs = 0, br = 0, bc = 0;
    gdp_endpoint_combine(&up, &lo, late ? 1 : 0, st[i].qend ? 1 : 0, st[i].precision, st[i].rlength, &fs, &br,
                         &bc);
    res.end_score = fs;
    res.end_r = br;
    res.end_c = bc;
    res.end_found = (up.end_found || lo.end_found) ? 1 : 0;
    res.precision = st[i].precision;
    gdp_pair_t p = end_pair(g, st[i], bc >= br ? GDP_UPPER : GDP_LOWER, seg[k], v.has_alt);
    p.flags = (int8_t) (p.flags | GDP_FLAG_TRACEBACK);
    p.tb_r = br;
    p.tb_c = bc;
    p2[n2] = p;
    info[n2].end5 = (g.end == 5) ? 1 : 0;
    info[n2].reject = (g.endalign == GDP_QUERYEND_GAP || g.endalign == GDP_BEST_LOCAL) ? 1 : 0;
    info[n2].pad = 0;
    gap2[n2++] = i;
    slot_total += (int64_t) p.rlength + p.glength + 2;
  }
  if (n2 == 0) return GDP_OK;

  /* run 2: one fill and traceback per gap from its best cell */
  gdp_pair_t *d_p2 = nullptr;
  gdp_result_t *d_r2 = nullptr, *r2 = nullptr;
  const gdp_rec_t **fslot = nullptr, **d_fslot = nullptr;
  TbInfo *d_info = nullptr;
  SCK(dev_slot(C, D_P2, &d_p2, n2));
  SCK(dev_slot(C, D_R2, &d_r2, n2));
  SCK(dev_slot(C, D_INFO, &d_info, n2));
  SCK(dev_slot(C, D_SLOTS, &d_slots, slot_total));
  SCK(host_slot(C, H_FSLOT, &fslot, n2));
  SCK(host_slot(C, H_R2, &r2, n2));
  SCK(cudaMemcpyAsync(d_p2, p2, n2 * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
  SCK(cudaMemcpyAsync(d_info, info, n2 * sizeof(TbInfo), cudaMemcpyHostToDevice, s));
  slot_used = 0;
  rc = run_plans(ctx, v, p2, d_p2, n2, d_arena, d_r2, d_slots, slot_total, &slot_used, fslot);
  if (rc != GDP_OK) return rc;

  /* the reference's last steps and the compaction, on the device */
  int32_t *d_first = nullptr;
  int64_t *d_count = nullptr, *d_off = nullptr, *words = nullptr;
  gdp_rec_t *d_out = nullptr;
  unsigned long long *d_used = nullptr;
  SCK(dev_slot(C, D_FSLOT, &d_fslot, n2));
  SCK(dev_slot(C, D_FIRST, &d_first, n2));
  SCK(dev_slot(C, D_COUNT, &d_count, n2 + 1));
  SCK(dev_slot(C, D_OFF, &d_off, n2 + 1));
  SCK(dev_slot(C, D_USED, &d_used, 1));
  SCK(host_slot(C, H_WORDS, &words, 2));
  SCK(cudaMemcpyAsync(d_fslot, fslot, n2 * sizeof(gdp_rec_t *), cudaMemcpyHostToDevice, s));
  SCK(cudaMemsetAsync(d_used, 0, sizeof(unsigned long long), s));
  const int wblocks = (int) std::min<int64_t>((n2 + 1 + 7) / 8, (int64_t) v.nsm * 8);
  end_count_kernel<<<wblocks, 256, 0, s>>>(d_r2, d_info, d_fslot, n2, d_first, d_count);
  gdpi_count_launch(ctx);
  SCK(cudaGetLastError());
  size_t tmp_bytes = 0;
  SCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_count, d_off, n2 + 1, s));
  char *d_tmp = nullptr;
  SCK(dev_slot(C, D_TMP, &d_tmp, (int64_t) tmp_bytes));
  SCK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_count, d_off, n2 + 1, s));
  SCK(cudaMemcpyAsync(&words[0], d_off + n2, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  SCK(dev_slot(C, D_OUT, &d_out, std::min(words[0], max_recs)));
  end_gather_kernel<<<wblocks, 256, 0, s>>>(d_r2, d_info, d_fslot, d_first, d_count, d_off, n2, max_recs, d_out,
                                            d_used);
  gdpi_count_launch(ctx);
  SCK(cudaGetLastError());
  SCK(cudaMemcpyAsync(r2, d_r2, n2 * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaMemcpyAsync(&words[1], d_used, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  const int64_t used = (int64_t) words[1];
  if (used > 0) {
    SCK(cudaMemcpyAsync(recs, d_out, used * sizeof(gdp_rec_t), cudaMemcpyDeviceToHost, s));
  }
  par_for(n2, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; k++) {
      const gdp_result_t &t = r2[k];
      gdp_result_t &res = results[gap2[k]];
      res.status = t.status;
      if (t.status != GDP_OK && t.status != GDP_ERR_RECS) continue;
      res.score = t.score;
      res.tb_score = t.tb_score;
      res.nmatches = t.nmatches;
      res.nmismatches = t.nmismatches;
      res.nopens = t.nopens;
      res.nindels = t.nindels;
      res.nrecs = t.nrecs;
      res.rec_offset = t.nrecs > 0 ? t.rec_offset : 0;
    }
  });
  if (used > 0) SCK(cudaStreamSynchronize(s));
  if (nrecs_used) *nrecs_used = used;
  return GDP_OK;
}
