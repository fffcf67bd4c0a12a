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
 * device does the work in two batch runs:
 *
 *   1. every gap's upper and lower fill, with the endpoint search fused in
 *      (GDP_FLAG_ENDPOINT / _QEND) and the genome segment read from the
 *      resident genome (GDP_FLAG_GWINDOW with the end's segment rule);
 *   2. for every gap with a traceback, one fill and its traceback from the
 *      best cell (gdp_endpoint_combine merges the halves of run 1): through
 *      the upper fill when bestc >= bestr, else the lower.  The fill of run
 *      2 is the one of run 1 again (fills are deterministic), so no
 *      direction storage is kept between the runs.
 *
 * The host then applies the reference's last steps: no pairs and score 0
 * when nmatches + 1 < nmismatches (QUERYEND_GAP, BEST_LOCAL), else the
 * List in the reference's order (its head is the first pair the traceback
 * pushed) without its leading indel pairs.
 *
 * The query.  The reference fills end 3 with rsequenceuc and traces back
 * with rsequence and rsequenceuc; this library's fills read the pair's
 * rseq.  The substitution tables score a lower-case query letter as its
 * upper-case letter (Dynprog_init's PREUC), so filling with rsequence gives
 * the same matrices whenever rsequenceuc is rsequence upper-cased, which is
 * how GMAP passes them (queryuc_ptr).
 */
#include <cuda_runtime.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "gdp_internal.h"
#include "gdp_dropin_internal.h"

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
   segment at `seg` in the staging arena. */
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

void
null_result (gdp_result_t &r, int status) {
  memset(&r, 0, sizeof(r));
  r.status = status;
}

}  // namespace

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
      arena_bytes < 0 || (arena_bytes > 0 && arena == nullptr))
    return GDP_ERR_PARAM;
  if (nrecs_used) *nrecs_used = 0;
  if (n == 0) return GDP_OK;
  const gdpi_single_cfg &cfg = *v.single;

  /* the reference's decisions; staging arena = the caller's bytes, then a
     genome segment (and its alternate) per gap with fills */
  std::vector<EndSetup> st(n);
  std::vector<int64_t> seg(n, -1);
  int64_t stage = (arena_bytes + 15) & ~(int64_t) 15;
  int64_t nfill = 0;
  for (int64_t i = 0; i < n; i++) {
    const gdp_end_gap_t &g = gaps[i];
    st[i] = end_setup(g, cfg);
    if (g.end != 5 && g.end != 3) { null_result(results[i], GDP_ERR_PARAM); continue; }
    if (g.endalign == GDP_QUERYEND_NOGAPS || g.endalign < 0 || g.endalign > GDP_BEST_LOCAL) {
      null_result(results[i], GDP_ERR_PARAM);
      continue;
    }
    null_result(results[i], GDP_OK);
    if (st[i].null_result || g.require_pos_score_p) continue;
    /* the query bytes the fills read must lie in the arena */
    const int64_t r0 = (g.end == 5) ? g.rseq - (st[i].rlength - 1) : g.rseq;
    const int64_t u0 = (g.end == 5) ? g.rseq_uc - (st[i].rlength - 1) : g.rseq_uc;
    if (r0 < 0 || u0 < 0 || r0 + st[i].rlength > arena_bytes || u0 + st[i].rlength > arena_bytes) {
      results[i].status = GDP_ERR_LEN;
      continue;
    }
    seg[i] = stage;
    stage += ((int64_t) st[i].glength * (v.has_alt ? 2 : 1) + 15) & ~(int64_t) 15;
    nfill++;
  }
  if (nfill == 0) return GDP_OK;
  std::vector<char> buf(std::max<int64_t>(stage, 16), 0);
  if (arena_bytes > 0) memcpy(buf.data(), arena, arena_bytes);

  /* run 1: the upper and lower fills with the endpoint search */
  std::vector<gdp_pair_t> p1;
  std::vector<int64_t> gap_of;
  p1.reserve(2 * nfill);
  for (int64_t i = 0; i < n; i++) {
    if (seg[i] < 0) continue;
    const int search = st[i].qend ? GDP_FLAG_ENDPOINT_QEND : GDP_FLAG_ENDPOINT;
    for (int variant : {GDP_UPPER, GDP_LOWER}) {
      gdp_pair_t p = end_pair(gaps[i], st[i], variant, seg[i], v.has_alt);
      p.flags = (int8_t) (p.flags | search);
      p1.push_back(p);
    }
    gap_of.push_back(i);
  }
  std::vector<gdp_result_t> r1(p1.size());
  int rc = gdp_align_batch(ctx, p1.data(), (int64_t) p1.size(), buf.data(), stage, r1.data(), nullptr, 0, nullptr);
  if (rc != GDP_OK) return rc;

  /* the best cell of each gap, and run 2: its traceback */
  std::vector<gdp_pair_t> p2;
  std::vector<int64_t> gap2;
  int64_t slots = 0;
  for (size_t k = 0; k < gap_of.size(); k++) {
    const int64_t i = gap_of[k];
    const gdp_result_t &up = r1[2 * k], &lo = r1[2 * k + 1];
    gdp_result_t &res = results[i];
    if (up.status != GDP_OK || lo.status != GDP_OK) {
      res.status = up.status != GDP_OK ? up.status : lo.status;
      continue;
    }
    const bool end5 = (gaps[i].end == 5);
    const bool late = end5 ? !gaps[i].jump_late_p : (gaps[i].jump_late_p != 0);
    int fs = 0, br = 0, bc = 0;
    gdp_endpoint_combine(&up, &lo, late ? 1 : 0, st[i].qend ? 1 : 0, st[i].precision, st[i].rlength, &fs, &br,
                         &bc);
    res.end_score = fs;
    res.end_r = br;
    res.end_c = bc;
    res.end_found = (up.end_found || lo.end_found) ? 1 : 0;
    res.precision = st[i].precision;
    gdp_pair_t p = end_pair(gaps[i], st[i], bc >= br ? GDP_UPPER : GDP_LOWER, seg[i], v.has_alt);
    p.flags = (int8_t) (p.flags | GDP_FLAG_TRACEBACK);
    p.tb_r = br;
    p.tb_c = bc;
    p2.push_back(p);
    gap2.push_back(i);
    slots += (int64_t) p.rlength + p.glength + 2;
  }
  int64_t out = 0;
  if (!p2.empty()) {
    std::vector<gdp_result_t> r2(p2.size());
    std::vector<gdp_rec_t> tb(std::max<int64_t>(slots, 1));
    int64_t used = 0;
    rc = gdp_align_batch(ctx, p2.data(), (int64_t) p2.size(), buf.data(), stage, r2.data(), tb.data(),
                         (int64_t) tb.size(), &used);
    if (rc != GDP_OK) return rc;
    bool cut = false;
    for (size_t k = 0; k < p2.size(); k++) {
      const int64_t i = gap2[k];
      const gdp_result_t &t = r2[k];
      gdp_result_t &res = results[i];
      if (t.status != GDP_OK) { res.status = t.status; continue; }
      res.nmatches = t.nmatches;
      res.nmismatches = t.nmismatches;
      res.nopens = t.nopens;
      res.nindels = t.nindels;
      const int endalign = gaps[i].endalign;
      if ((endalign == GDP_QUERYEND_GAP || endalign == GDP_BEST_LOCAL) && t.nmatches + 1 < t.nmismatches) {
        res.score = res.tb_score = 0;   /* no pairs; the counts stay */
        continue;
      }
      res.score = res.tb_score = t.tb_score;
      /* the List after List_reverse starts with the first pair pushed; its
         leading indel pairs go.  End 3 returns that List, end 5 its
         reverse. */
      const gdp_rec_t *r = tb.data() + t.rec_offset;
      int first = 0;
      while (first < t.nrecs && r[first].comp == '-') first++;
      const int keep = t.nrecs - first;
      if (cut || (keep > 0 && (recs == nullptr || out + keep > max_recs))) {
        cut = true;
        if (keep > 0) res.status = GDP_ERR_RECS;
        continue;
      }
      if (gaps[i].end == 5) std::reverse_copy(r + first, r + t.nrecs, recs + out);
      else if (keep > 0) memcpy(recs + out, r + first, (size_t) keep * sizeof(gdp_rec_t));
      res.nrecs = keep;
      res.rec_offset = out;
      out += keep;
    }
  }
  if (nrecs_used) *nrecs_used = out;
  return GDP_OK;
}
