/*
 * cdna_gap.cu -- Dynprog_cdna_gap (src/dynprog_cdna.c:786-1290) for a batch
 * of gaps.
 *
 * A cDNA gap is a gap between two aligned blocks of a read where the read
 * holds more bases than the genome (extra material in the read): the query
 * stretch left of the gap and the one right of it are each aligned against
 * the genome stretch between the blocks -- the left one forwards from the
 * left block, the right one backwards from the right block -- and the best
 * bridge between the two alignments is chosen.  The reference fills an
 * upper and a lower matrix per side, searches all combinations of a left
 * and a right end cell for the best sum of scores plus a gap penalty
 * (bridge_cdna_gap_{8,16}_ud, src/dynprog_cdna.c:123-651), traces both
 * sides back from those cells and joins them with a cDNA insertion or a gap
 * holder.  Here, per batch:
 *
 *   1. on the host, the reference's decisions: length checks, penalties by
 *      defect rate, bands, precision;
 *   2. on the device, the four fills of every gap as pairs of the batch
 *      planner, their genome segments written from the resident genome,
 *      with every swept cell's score kept; a kernel lays each fill's scores
 *      out densely, (genome column, query row);
 *   3. the bridge search, one thread block per gap: each thread scans its
 *      share of (left column, right column) combinations over both bands,
 *      and the block keeps the best score, ties broken by the reference's
 *      scan order (the last best for jump late, the first for jump early);
 *   4. both tracebacks as pairs of the planner (a fill and a traceback from
 *      the chosen cell each);
 *   5. one warp per gap writes the reference's List: the right traceback
 *      reversed, the cDNA insertion or the gap holder, the left traceback.
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
#include "genome_chars.cuh"

namespace {

constexpr int CDNA_OPEN = -10, CDNA_EXTEND = -7;   /* CDNA_OPEN_* / CDNA_EXTEND_* (src/dynprog_cdna.c:31-37) */
constexpr int INSERT_PAIRS = 9;                    /* src/dynprog_cdna.c:39 */
constexpr char SHORTGAP_COMP = '~';                /* src/comp.h:10 */
constexpr int NEG8 = -128, NEG16 = -32768;         /* NEG_INFINITY_8 / _16 */

/* The reference's choices for one gap. */
struct CdnaSetup {
  int8_t fill;        /* the gap runs its fills */
  int8_t advance;     /* the reference advances dynprogindex */
  int8_t precision;
  int8_t mismatchtype;
  int32_t lbandL, ubandL, lbandR, ubandR;
};

CdnaSetup
cdna_setup (const gdp_cdna_gap_t &g) {
  CdnaSetup s;
  memset(&s, 0, sizeof(s));
  if (g.glength <= 1) return s;                       /* NULL, dynprogindex unchanged */
  s.advance = 1;
  if (g.glength > g.max_glength || g.rlengthR > g.max_rlength || g.rlengthL > g.max_rlength) return s;
  if (g.rlengthL <= 0 || g.rlengthR <= 0) return s;   /* no fill the planner would take */
  /* DEFECT_HIGHQ 0.003, DEFECT_MEDQ 0.014 */
  const int q = g.defect_rate < 0.003 ? 0 : g.defect_rate < 0.014 ? 1 : 2;
  s.mismatchtype = (int8_t) q;
  /* use8p_size[mismatchtype] = NEG_INFINITY_8 / MISMATCH_* - 1: 41, 63, 127 */
  const int use8p = (q == 0) ? 41 : (q == 1) ? 63 : 127;
  s.precision = (g.glength < use8p || (g.rlengthL < use8p && g.rlengthR <= use8p)) ? 8 : 16;
  /* Dynprog_compute_bands(extraband_paired, widebandp) per side */
  const int x = g.extraband_paired;
  if (g.glength >= g.rlengthL) { s.ubandL = g.glength - g.rlengthL + x; s.lbandL = x; }
  else { s.lbandL = g.rlengthL - g.glength + x; s.ubandL = x; }
  if (g.glength >= g.rlengthR) { s.ubandR = g.glength - g.rlengthR + x; s.lbandR = x; }
  else { s.lbandR = g.rlengthR - g.glength + x; s.ubandR = x; }
  s.fill = 1;
  return s;
}

/* One fill of a gap: side 0 the left stretch against the segment read
   forwards from goffset, side 1 the right stretch against the mirrored
   segment read backwards from goffset + glength - 1. */
gdp_pair_t
cdna_pair (const gdp_cdna_gap_t &g, const CdnaSetup &s, int side, int variant, int64_t seg, bool has_alt) {
  gdp_pair_t p;
  memset(&p, 0, sizeof(p));
  const int to_r = g.rev_roffsetR - g.roffsetL;
  if (side == 0) {
    p.rseq = g.rseq;
    p.rseq_uc = g.rseq_uc;
    p.rlength = g.rlengthL;
    p.queryoffset = g.roffsetL;
    p.genomeoffset = g.goffset;
    p.flags = (int8_t) (GDP_FLAG_GWINDOW | (g.jump_late_p ? GDP_FLAG_JUMP_LATE : 0));
    p.xflags = GDP_XFLAG_SEGMENT;
    if (variant == GDP_UPPER) p.uband = s.ubandL;
    else p.lband = s.lbandL;
  } else {
    /* rev_rsequenceR: the query's character at rev_roffsetR, read backwards */
    p.rseq = g.rseq + to_r - (g.rlengthR - 1);
    p.rseq_uc = g.rseq_uc + to_r - (g.rlengthR - 1);
    p.rlength = g.rlengthR;
    p.queryoffset = g.rev_roffsetR;
    p.genomeoffset = g.goffset + g.glength - 1;
    p.flags = (int8_t) (GDP_FLAG_GWINDOW | GDP_FLAG_REVP | (g.jump_late_p ? 0 : GDP_FLAG_JUMP_LATE));
    p.xflags = GDP_XFLAG_SEGMENT_REV;
    if (variant == GDP_UPPER) p.uband = s.ubandR;
    else p.lband = s.lbandR;
  }
  p.gseq = seg;
  p.gseq_alt = has_alt ? seg + g.glength : seg;
  p.glength = g.glength;
  p.variant = (int8_t) variant;
  p.precision = s.precision;
  p.mismatchtype = s.mismatchtype;
  p.open = CDNA_OPEN;
  p.extend = CDNA_EXTEND;
  p.chroffset = g.chroffset;
  p.chrhigh = g.chrhigh;
  p.watsonp = g.watsonp;
  p.genestrand = g.genestrand;
  p.dynprogindex = g.dynprogindex;
  return p;
}

/* Where a fill's dense scores live: (glength + 1) columns of (rlength + 1)
   rows, score(c, r) at base + c * (rlength + 1) + r. */
struct DenseFill {
  int64_t base;
  int32_t rlength, glength;
};

__global__ void __launch_bounds__(256)
dense_clear_kernel (int16_t *dense, int64_t n) {
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
    dense[i] = (int16_t) NEG16;
}

/*
 * One warp per fill: the scores its fill kept for every swept cell (lane l
 * of the word-column at word offset w is at scores[w * 8 + l]) go to the
 * dense (genome column, query row) layout.  Lanes are query rows in the
 * upper fill and genome columns in the lower fill.
 */
__global__ void __launch_bounds__(256)
dense_scatter_kernel (const gdp_pair_t *pairs, const gdp_result_t *res, const gdp_meta_t *meta,
                      const int16_t *scores, const DenseFill *fills, int64_t n, int16_t *dense) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  for (int64_t k = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nwarps) {
    if (res[k].status != GDP_OK) continue;
    const gdp_pair_t p = pairs[k];
    const int W = (res[k].precision == 8) ? 32 : 16;
    const int64_t base = (W == 16) ? meta[k].dir16 : meta[k].dir8;
    if (base < 0) continue;
    const DenseFill f = fills[k];
    const bool lower = (p.variant == GDP_LOWER);
    gdp_geom_t g;
    gdp_geom_of(&p, W, &g);
    /* W = 16: two word-columns per warp step (lanes 0-15 and 16-31) */
    const int per = 32 / W, l = lane % W, sub = lane / W;
    int64_t boff = 0;
    for (int xlo = 0; xlo <= g.X; xlo += W) {
      int y0, y1;
      gdp_block_sweep(&g, xlo, &y0, &y1);
      const int x = xlo + l;
      for (int y = y0 + sub; y <= y1; y += per) {
        const int16_t v = scores[(base + boff + (int64_t) (y - y0) * (W / 8)) * 8 + l];
        const int c = lower ? x : y, r = lower ? y : x;
        if (x <= g.X && c <= f.glength && r <= f.rlength) dense[f.base + (int64_t) c * (f.rlength + 1) + r] = v;
      }
      boff += gdp_block_words(&g, xlo);
    }
  }
}

/* A gap's bridge search: its four dense fills (left upper, left lower,
   right upper, right lower) and the search's parameters. */
struct BridgeIn {
  int64_t fill[4];
  int32_t glength, rlengthL, rlengthR;
  int32_t lbandL, ubandL, lbandR, ubandR;
  int32_t open, leftoffset, rightoffset;
  int32_t late, neg;
};
struct BridgeOut {
  int32_t found, score, rL, cL, rR, cR, outside;
};

__device__ __forceinline__ bool
bridge_better (bool late, int s, int64_t key, int bs, int64_t bkey) {
  return s > bs || (s == bs && (late ? key > bkey : key < bkey));
}

/*
 * bridge_cdna_gap_{8,16}_ud (src/dynprog_cdna.c:123-651) for one gap per
 * block.  The reference scans left columns cL up, right columns cR from
 * glength - cL down, left rows rL up and right rows rR up, and keeps a
 * candidate when its score is >= (jump late) or > (jump early) the best so
 * far, starting from NEG_INFINITY: the result is the best score, at the
 * last (late) or first (early) place in that order among the cells that
 * reach it, provided it passes the start.  The gap penalty is 0 for the
 * first cR of each cL and `open` for the others (the reference's loop
 * resets it to open - extend, to which its increment adds extend).  Reads
 * of cells outside a dense fill (rows past its rlength) are counted in
 * `outside`: the reference reads stale scratch there.
 */
__global__ void __launch_bounds__(256)
bridge_kernel (const BridgeIn *in, const int16_t *dense, BridgeOut *out, int64_t n) {
  __shared__ int s_score[256];
  __shared__ long long s_key[256];
  __shared__ int s_outside[256];
  for (int64_t gi = blockIdx.x; gi < n; gi += gridDim.x) {
    const BridgeIn b = in[gi];
    const bool late = b.late != 0;
    const int G = b.glength, RL = b.rlengthL, RR = b.rlengthR;
    const int16_t *Lup = dense + b.fill[0], *Llo = dense + b.fill[1];
    const int16_t *Rup = dense + b.fill[2], *Rlo = dense + b.fill[3];
    int best = INT_MIN, outside = 0;
    long long bkey = -1;
    for (int cL = 1; cL < G; cL++) {
      for (int cR = G - cL - (int) threadIdx.x; cR >= 0; cR -= (int) blockDim.x) {
        const int pen = (cR == G - cL) ? 0 : b.open;
        const int rloL = max(1, cL - b.ubandL), rhighL = min(cL + b.lbandL, RL - 1);
        const int rloR = max(1, cR - b.ubandR), rhighR = min(cR + b.lbandR, RR - 1);
        /* left rows: the upper part runs to cL - 1, the lower part on to rhighL */
        const int rLend = max(rhighL, cL - 1);
        for (int rL = rloL; rL <= rLend; rL++) {
          if (rL >= cL && rL > rhighL) break;
          if (rL > RL) { outside++; continue; }
          const int scoreL = (rL < cL) ? Lup[(int64_t) cL * (RL + 1) + rL] : Llo[(int64_t) cL * (RL + 1) + rL];
          const int bound = b.rightoffset - b.leftoffset - rL;
          /* right rows: the upper part while rR < cR and rR < bound, then
             the lower part while rR <= rhighR and rR < bound */
          const int uend = max(rloR, min(cR, bound));
          for (int rR = rloR; rR < uend; rR++) {
            if (rR > RR) { outside++; continue; }
            const int s = scoreL + Rup[(int64_t) cR * (RR + 1) + rR] + pen;
            const long long key = (((long long) cL * (G + 1) + (G - cR)) * (RL + 1) + rL) * (RR + 1) + rR;
            if ((late ? s >= b.neg : s > b.neg) && bridge_better(late, s, key, best, bkey)) { best = s; bkey = key; }
          }
          for (int rR = uend; rR <= rhighR && rR < bound; rR++) {
            const int s = scoreL + Rlo[(int64_t) cR * (RR + 1) + rR] + pen;
            const long long key = (((long long) cL * (G + 1) + (G - cR)) * (RL + 1) + rL) * (RR + 1) + rR;
            if ((late ? s >= b.neg : s > b.neg) && bridge_better(late, s, key, best, bkey)) { best = s; bkey = key; }
          }
        }
      }
    }
    s_score[threadIdx.x] = best;
    s_key[threadIdx.x] = bkey;
    s_outside[threadIdx.x] = outside;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if ((int) threadIdx.x < w) {
        const int o = threadIdx.x + w;
        if (s_key[o] >= 0 && (s_key[threadIdx.x] < 0 ||
                              bridge_better(late, s_score[o], s_key[o], s_score[threadIdx.x], s_key[threadIdx.x]))) {
          s_score[threadIdx.x] = s_score[o];
          s_key[threadIdx.x] = s_key[o];
        }
        s_outside[threadIdx.x] += s_outside[o];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      BridgeOut o;
      o.outside = s_outside[0];
      o.found = s_key[0] >= 0 ? 1 : 0;
      o.score = s_score[0];
      long long k = s_key[0] >= 0 ? s_key[0] : 0;
      o.rR = (int) (k % (RR + 1)); k /= (RR + 1);
      o.rL = (int) (k % (RL + 1)); k /= (RL + 1);
      o.cR = G - (int) (k % (G + 1)); k /= (G + 1);
      o.cL = (int) k;
      out[gi] = o;
    }
    __syncthreads();
  }
}

/* A traced gap's assembly: its best cells and the results of its right
   (r2[2k]) and left (r2[2k + 1]) traceback. */
struct AsmIn {
  int32_t gap;
  int32_t rL, cL, rR, cR;
};

/* the middle of the List: a cDNA insertion (queryjump == genomejump ==
   INSERT_PAIRS) or a gap holder */
__device__ __forceinline__ void
cdna_jumps (const gdp_cdna_gap_t &g, const AsmIn &a, int *qj, int *gj) {
  const int rev_goffset = g.goffset + g.glength - 1;
  *qj = (g.rev_roffsetR - a.rR) - (g.roffsetL + a.rL) + 1;
  *gj = (rev_goffset - a.cR) - (g.goffset + a.cL) + 1;
}

/* Pairpool_push drops pairs with a negative position (src/pairpool.c:189-191) */
__device__ __forceinline__ int
cdna_middle_count (const gdp_cdna_gap_t &g, const AsmIn &a) {
  int qj, gj;
  cdna_jumps(g, a, &qj, &gj);
  if (qj != INSERT_PAIRS || gj != INSERT_PAIRS) return 1;
  const int rev_goffset = g.goffset + g.glength - 1;
  int n = 0;
  for (int k = g.rev_roffsetR - a.rR; k >= g.roffsetL + a.rL; k--) n += (k >= 0 && rev_goffset - a.cR + 1 >= 0);
  for (int k = rev_goffset - a.cR; k >= g.goffset + a.cL; k--) n += (g.roffsetL + a.rL >= 0 && k >= 0);
  return n;
}

__global__ void __launch_bounds__(256)
cdna_count_kernel (const gdp_cdna_gap_t *gaps, const AsmIn *as, const gdp_result_t *r2, int64_t n, int64_t *count) {
  for (int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += (int64_t) gridDim.x * blockDim.x) {
    int64_t c = 0;
    if (k < n) {
      const gdp_result_t &R = r2[2 * k], &L = r2[2 * k + 1];
      if (R.status == GDP_OK && L.status == GDP_OK) {
        const AsmIn a = as[k];
        c = (int64_t) R.nrecs + L.nrecs + cdna_middle_count(gaps[a.gap], a);
        if (c == 1) c = 0;   /* a List of the gap holder alone is returned as NULL */
      }
    }
    count[k] = c;
  }
}

/*
 * One warp per traced gap: the reference's List, head first -- the right
 * traceback's records reversed (its List_reverse), the middle in push
 * order, the left traceback's records in push order (the final
 * List_reverse undoes the pushes onto the front) -- to out[off[k] ..),
 * and the gap's result.
 */
__global__ void __launch_bounds__(256)
cdna_gather_kernel (const gdp_cdna_gap_t *gaps, const AsmIn *as, const gdp_result_t *r2,
                    const gdp_rec_t *const *slots, const int64_t *count, const int64_t *off, int64_t n,
                    int64_t max_recs, const char *arena, const uint32_t *genome, const uint32_t *genomealt,
                    uint64_t genome_len, gdp_rec_t *out, gdp_result_t *res, unsigned long long *used) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  for (int64_t k = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nwarps) {
    const AsmIn a = as[k];
    const gdp_cdna_gap_t g = gaps[a.gap];
    const gdp_result_t R = r2[2 * k], L = r2[2 * k + 1];
    gdp_result_t r;
    memset(&r, 0, sizeof(r));
    r.status = (R.status != GDP_OK) ? R.status : L.status;
    r.precision = R.precision;
    int64_t cnt = count[k];
    const int64_t o = off[k];
    if (r.status == GDP_OK && cnt > 0 && o + cnt > max_recs) {
      r.status = GDP_ERR_RECS;
      cnt = 0;
    }
    int qj, gj;
    cdna_jumps(g, a, &qj, &gj);
    const bool insert = (qj == INSERT_PAIRS && gj == INSERT_PAIRS);
    if (r.status == GDP_OK || r.status == GDP_ERR_RECS) {
      r.tb_score = R.tb_score + L.tb_score;
      r.nmatches = R.nmatches + L.nmatches;
      r.nmismatches = R.nmismatches + L.nmismatches;
      r.nopens = R.nopens + L.nopens;
      r.nindels = R.nindels + L.nindels;
      r.end_found = insert ? 0 : 1;   /* incompletep */
    }
    if (r.status == GDP_OK && cnt > 0) {
      const gdp_rec_t *rr = slots[2 * k] + R.rec_offset, *lr = slots[2 * k + 1] + L.rec_offset;
      gdp_rec_t *w = out + o;
      for (int j = lane; j < R.nrecs; j += 32) w[j] = rr[R.nrecs - 1 - j];
      w += R.nrecs;
      if (lane == 0) {
        if (!insert) {
          gdp_rec_t h;
          h.querypos = -1 - qj;
          h.genomepos = gj;
          h.cdna = ' '; h.comp = '\0'; h.genome = ' '; h.genomealt = ' ';
          *w++ = h;
        } else {
          const int rev_goffset = g.goffset + g.glength - 1;
          for (int q = g.rev_roffsetR - a.rR; q >= g.roffsetL + a.rL; q--) {
            const int gp = rev_goffset - a.cR + 1;
            if (q < 0 || gp < 0) continue;
            gdp_rec_t x;
            x.querypos = q; x.genomepos = gp;
            x.cdna = arena[g.rseq + (q - g.roffsetL)]; x.comp = SHORTGAP_COMP; x.genome = ' '; x.genomealt = ' ';
            *w++ = x;
          }
          gdp_pair_t pp;
          memset(&pp, 0, sizeof(pp));
          pp.chroffset = g.chroffset; pp.chrhigh = g.chrhigh; pp.watsonp = g.watsonp;
          for (int gp = rev_goffset - a.cR; gp >= g.goffset + a.cL; gp--) {
            const int q = g.roffsetL + a.rL;
            if (q < 0 || gp < 0) continue;
            char alt;
            char c2 = genomic_char(pp, gp, genome, genomealt, 0, genome_len, &alt);
            if (c2 == 0) { c2 = 'N'; alt = 'N'; }
            gdp_rec_t x;
            x.querypos = q; x.genomepos = gp;
            x.cdna = ' '; x.comp = SHORTGAP_COMP; x.genome = c2; x.genomealt = alt;
            *w++ = x;
          }
        }
      }
      const int mid = cdna_middle_count(g, a);
      w = out + o + R.nrecs + mid;
      for (int j = lane; j < L.nrecs; j += 32) w[j] = lr[j];
    }
    __syncwarp();
    if (lane == 0) {
      r.nrecs = (int32_t) cnt;
      r.rec_offset = o;
      res[k] = r;
      if (cnt > 0) atomicMax(used, (unsigned long long) (o + cnt));
    }
  }
}

/* Slots of the context's gap working memory this solver uses. */
enum { D_ARENA, D_P1, D_R1, D_FILLS, D_DENSE, D_BIN, D_BOUT, D_P2, D_R2, D_SLOTS, D_FSLOT, D_GAPS, D_AS, D_COUNT,
       D_OFF, D_OUT, D_TMP, D_USED };
enum { H_P1, H_FILLS, H_BIN, H_BOUT, H_P2, H_FSLOT, H_AS, H_R2, H_WORDS };

}  // namespace

#define SCK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return gdpi_fail(ctx, #call, e_); } while (0)

/* Runs pairs d_p[0..n) (host copies hp) as planner plans whose direction
   words stay within the context budget, results to d_res, records into
   d_slots from *slot_used on (slot_base[k]: the base of pair k's records;
   may be NULL when the pairs trace nothing back). */
static int
cdna_run_plans (gdp_ctx *ctx, const gdpi_view &v, gdp_plan **plan, const gdp_pair_t *hp, const gdp_pair_t *d_p,
                int64_t n, char *d_arena, gdp_result_t *d_res, gdp_rec_t *d_slots, int64_t slot_cap,
                int64_t *slot_used, const gdp_rec_t **slot_base) {
  for (int64_t k0 = 0; k0 < n;) {
    int64_t k1 = k0, bytes = 0;
    for (; k1 < n; k1++) {
      const int64_t b = gdp_pair_words(&hp[k1], hp[k1].precision == 8 ? 32 : 16) * 4;
      if (k1 > k0 && bytes + b > v.budget) break;
      bytes += b;
    }
    int rc = gdpi_plan_reuse(ctx, plan, hp + k0, k1 - k0);
    if (rc != GDP_OK) return rc;
    const int64_t nr = gdp_plan_total_recs(*plan);
    if (*slot_used + nr > slot_cap) return GDP_ERR_RECS;
    rc = gdp_plan_execute(ctx, *plan, d_p + k0, d_arena, d_res + k0, d_slots + *slot_used);
    if (rc != GDP_OK) return rc;
    if (slot_base)
      for (int64_t k = k0; k < k1; k++) slot_base[k] = d_slots + *slot_used;
    *slot_used += nr;
    if (k1 < n) SCK(cudaStreamSynchronize(v.stream));
    k0 = k1;
  }
  return GDP_OK;
}

extern "C" int
gdp_cdna_gap_batch (gdp_ctx *ctx, const gdp_cdna_gap_t *gaps, int64_t n, const char *arena, int64_t arena_bytes,
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

  /* the reference's decisions */
  std::vector<CdnaSetup> st((size_t) n);
  std::vector<int64_t> fill;
  for (int64_t i = 0; i < n; i++) {
    const gdp_cdna_gap_t &g = gaps[i];
    memset(&results[i], 0, sizeof(gdp_result_t));
    st[i] = cdna_setup(g);
    if (!st[i].fill) continue;
    if (g.genestrand < 0 || g.genestrand > 2) { results[i].status = GDP_ERR_PARAM; continue; }
    /* the query bytes the fills and the insertion read must lie in the arena */
    const int64_t to_r = (int64_t) g.rev_roffsetR - g.roffsetL;
    const int64_t lo = std::min<int64_t>(0, to_r - (g.rlengthR - 1));
    const int64_t hi = std::max<int64_t>(g.rlengthL, to_r + 1);
    if (g.rseq + lo < 0 || g.rseq_uc + lo < 0 || g.rseq + hi > arena_bytes || g.rseq_uc + hi > arena_bytes) {
      results[i].status = GDP_ERR_LEN;
      continue;
    }
    fill.push_back(i);
  }
  const int64_t nf = (int64_t) fill.size();
  if (nf == 0) return GDP_OK;

  /* the arena, then each gap's two genome segments (and their alternates) */
  const int64_t mult = v.has_alt ? 2 : 1;
  const int64_t seg_base = (arena_bytes + 15) / 16 * 16;
  std::vector<int64_t> seg((size_t) nf + 1);
  seg[0] = seg_base;
  for (int64_t k = 0; k < nf; k++) seg[k + 1] = seg[k] + 2 * ((gaps[fill[k]].glength * mult + 15) / 16 * 16);
  char *d_arena = nullptr;
  SCK(dev_slot(C, D_ARENA, &d_arena, seg[nf]));
  if (arena_bytes > 0) SCK(cudaMemcpyAsync(d_arena, arena, arena_bytes, cudaMemcpyHostToDevice, s));

  /* run 1, in chunks whose dense scores stay within 2 GB: the four fills
     with their scores, the dense layout, the bridge */
  gdp_pair_t *p1 = nullptr, *d_p1 = nullptr;
  gdp_result_t *d_r1 = nullptr;
  DenseFill *fl = nullptr, *d_fl = nullptr;
  BridgeIn *bin = nullptr, *d_bin = nullptr;
  BridgeOut *bout = nullptr, *d_bout = nullptr;
  int16_t *d_dense = nullptr;
  gdp_rec_t *d_dummy = nullptr;
  SCK(host_slot(C, H_BOUT, &bout, nf));
  SCK(dev_slot(C, D_SLOTS, &d_dummy, 1));
  const int64_t dense_cap = (int64_t) 1 << 30;   /* int16 scores per chunk */
  for (int64_t k0 = 0; k0 < nf;) {
    int64_t k1 = k0, cells = 0;
    for (; k1 < nf; k1++) {
      const gdp_cdna_gap_t &g = gaps[fill[k1]];
      const int64_t c = 2 * (int64_t) (g.glength + 1) * ((int64_t) g.rlengthL + g.rlengthR + 2);
      if (k1 > k0 && cells + c > dense_cap) break;
      cells += c;
    }
    const int64_t m = k1 - k0;
    SCK(host_slot(C, H_P1, &p1, 4 * m));
    SCK(host_slot(C, H_FILLS, &fl, 4 * m));
    SCK(host_slot(C, H_BIN, &bin, m));
    int64_t at = 0;
    for (int64_t j = 0; j < m; j++) {
      const int64_t i = fill[k0 + j];
      const gdp_cdna_gap_t &g = gaps[i];
      const CdnaSetup &su = st[i];
      const int64_t sg = seg[k0 + j], half = (g.glength * mult + 15) / 16 * 16;
      p1[4 * j + 0] = cdna_pair(g, su, 0, GDP_UPPER, sg, v.has_alt);
      p1[4 * j + 1] = cdna_pair(g, su, 0, GDP_LOWER, sg, v.has_alt);
      p1[4 * j + 2] = cdna_pair(g, su, 1, GDP_UPPER, sg + half, v.has_alt);
      p1[4 * j + 3] = cdna_pair(g, su, 1, GDP_LOWER, sg + half, v.has_alt);
      for (int f = 0; f < 4; f++) {
        fl[4 * j + f].base = at;
        fl[4 * j + f].rlength = f < 2 ? g.rlengthL : g.rlengthR;
        fl[4 * j + f].glength = g.glength;
        bin[j].fill[f] = at;
        at += (int64_t) (g.glength + 1) * ((f < 2 ? g.rlengthL : g.rlengthR) + 1);
      }
      BridgeIn &b = bin[j];
      b.glength = g.glength; b.rlengthL = g.rlengthL; b.rlengthR = g.rlengthR;
      b.lbandL = su.lbandL; b.ubandL = su.ubandL; b.lbandR = su.lbandR; b.ubandR = su.ubandR;
      b.open = CDNA_OPEN; b.leftoffset = g.roffsetL; b.rightoffset = g.rev_roffsetR;
      b.late = g.jump_late_p ? 1 : 0;
      b.neg = su.precision == 8 ? NEG8 : NEG16;
    }
    SCK(dev_slot(C, D_P1, &d_p1, 4 * m));
    SCK(dev_slot(C, D_R1, &d_r1, 4 * m));
    SCK(dev_slot(C, D_FILLS, &d_fl, 4 * m));
    SCK(dev_slot(C, D_BIN, &d_bin, m));
    SCK(dev_slot(C, D_BOUT, &d_bout, m));
    SCK(dev_slot(C, D_DENSE, &d_dense, at));
    SCK(cudaMemcpyAsync(d_p1, p1, 4 * m * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
    SCK(cudaMemcpyAsync(d_fl, fl, 4 * m * sizeof(DenseFill), cudaMemcpyHostToDevice, s));
    SCK(cudaMemcpyAsync(d_bin, bin, m * sizeof(BridgeIn), cudaMemcpyHostToDevice, s));
    int rc = gdpi_plan_reuse_dump(ctx, &C->dump_plan, p1, 4 * m);
    if (rc != GDP_OK) return rc;
    rc = gdp_plan_execute(ctx, C->dump_plan, d_p1, d_arena, d_r1, d_dummy);
    if (rc != GDP_OK) return rc;
    const int cg = (int) std::min<int64_t>((at + 255) / 256, (int64_t) v.nsm * 16);
    dense_clear_kernel<<<cg, 256, 0, s>>>(d_dense, at);
    gdpi_count_launch(ctx);
    const int sg = (int) std::min<int64_t>((4 * m + 7) / 8, (int64_t) v.nsm * 8);
    dense_scatter_kernel<<<sg, 256, 0, s>>>(d_p1, d_r1, gdpi_plan_meta(C->dump_plan), gdpi_plan_scores(C->dump_plan),
                                            d_fl, 4 * m, d_dense);
    gdpi_count_launch(ctx);
    bridge_kernel<<<(int) std::min<int64_t>(m, (int64_t) v.nsm * 8), 256, 0, s>>>(d_bin, d_dense, d_bout, m);
    gdpi_count_launch(ctx);
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(bout + k0, d_bout, m * sizeof(BridgeOut), cudaMemcpyDeviceToHost, s));
    /* the fills' statuses, for gaps whose fills failed */
    std::vector<gdp_result_t> r1((size_t) 4 * m);
    SCK(cudaMemcpyAsync(r1.data(), d_r1, 4 * m * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    for (int64_t j = 0; j < m; j++) {
      gdp_result_t &res = results[fill[k0 + j]];
      for (int f = 0; f < 4 && res.status == GDP_OK; f++) res.status = r1[4 * j + f].status;
      const BridgeOut &o = bout[k0 + j];
      if (res.status == GDP_OK && (!o.found || o.outside)) res.status = GDP_ERR_BAND;
      res.score = o.score;
      res.precision = st[fill[k0 + j]].precision;
    }
    k0 = k1;
  }

  /* run 2: the right and the left traceback of each bridged gap */
  gdp_pair_t *p2 = nullptr, *d_p2 = nullptr;
  AsmIn *as = nullptr, *d_as = nullptr;
  SCK(host_slot(C, H_P2, &p2, 2 * nf));
  SCK(host_slot(C, H_AS, &as, nf));
  std::vector<int64_t> gap2;
  int64_t n2 = 0, slot_total = 0;
  for (int64_t k = 0; k < nf; k++) {
    const int64_t i = fill[k];
    if (results[i].status != GDP_OK) continue;
    const gdp_cdna_gap_t &g = gaps[i];
    const CdnaSetup &su = st[i];
    const BridgeOut &o = bout[k];
    const int64_t half = (g.glength * mult + 15) / 16 * 16;
    gdp_pair_t r = cdna_pair(g, su, 1, o.cR >= o.rR ? GDP_UPPER : GDP_LOWER, seg[k] + half, v.has_alt);
    gdp_pair_t l = cdna_pair(g, su, 0, o.cL >= o.rL ? GDP_UPPER : GDP_LOWER, seg[k], v.has_alt);
    r.flags = (int8_t) (r.flags | GDP_FLAG_TRACEBACK);
    l.flags = (int8_t) (l.flags | GDP_FLAG_TRACEBACK);
    r.tb_r = o.rR; r.tb_c = o.cR;
    l.tb_r = o.rL; l.tb_c = o.cL;
    p2[2 * n2] = r;
    p2[2 * n2 + 1] = l;
    as[n2].gap = (int32_t) i;
    as[n2].rL = o.rL; as[n2].cL = o.cL; as[n2].rR = o.rR; as[n2].cR = o.cR;
    slot_total += (int64_t) r.rlength + r.glength + 2 + (int64_t) l.rlength + l.glength + 2;
    gap2.push_back(i);
    n2++;
  }
  if (n2 == 0) return GDP_OK;
  gdp_result_t *d_r2 = nullptr, *r2 = nullptr;
  gdp_rec_t *d_slots = nullptr;
  const gdp_rec_t **fslot = nullptr, **d_fslot = nullptr;
  gdp_cdna_gap_t *d_gaps = nullptr;
  SCK(dev_slot(C, D_P2, &d_p2, 2 * n2));
  SCK(dev_slot(C, D_R2, &d_r2, 2 * n2));
  SCK(dev_slot(C, D_SLOTS, &d_slots, slot_total));
  SCK(dev_slot(C, D_AS, &d_as, n2));
  SCK(dev_slot(C, D_GAPS, &d_gaps, n));
  SCK(host_slot(C, H_FSLOT, &fslot, 2 * n2));
  SCK(host_slot(C, H_R2, &r2, n2));
  SCK(cudaMemcpyAsync(d_p2, p2, 2 * n2 * sizeof(gdp_pair_t), cudaMemcpyHostToDevice, s));
  SCK(cudaMemcpyAsync(d_as, as, n2 * sizeof(AsmIn), cudaMemcpyHostToDevice, s));
  SCK(cudaMemcpyAsync(d_gaps, gaps, n * sizeof(gdp_cdna_gap_t), cudaMemcpyHostToDevice, s));
  int64_t slot_used = 0;
  int rc = cdna_run_plans(ctx, v, &C->plan, p2, d_p2, 2 * n2, d_arena, d_r2, d_slots, slot_total, &slot_used, fslot);
  if (rc != GDP_OK) return rc;

  /* the Lists, compacted in gap order */
  int64_t *d_count = nullptr, *d_off = nullptr, *words = nullptr;
  gdp_rec_t *d_out = nullptr;
  gdp_result_t *d_res = nullptr;
  unsigned long long *d_used = nullptr;
  SCK(dev_slot(C, D_FSLOT, &d_fslot, 2 * n2));
  SCK(dev_slot(C, D_COUNT, &d_count, n2 + 1));
  SCK(dev_slot(C, D_OFF, &d_off, n2 + 1));
  SCK(dev_slot(C, D_USED, &d_used, 1));
  SCK(dev_slot(C, D_R1, &d_res, n2));
  SCK(host_slot(C, H_WORDS, &words, 2));
  SCK(cudaMemcpyAsync(d_fslot, fslot, 2 * n2 * sizeof(gdp_rec_t *), cudaMemcpyHostToDevice, s));
  SCK(cudaMemsetAsync(d_used, 0, sizeof(unsigned long long), s));
  cdna_count_kernel<<<(int) std::min<int64_t>((n2 + 256) / 256, (int64_t) v.nsm * 8), 256, 0, s>>>(d_gaps, d_as, d_r2,
                                                                                                   n2, d_count);
  gdpi_count_launch(ctx);
  SCK(cudaGetLastError());
  size_t tmp_bytes = 0;
  SCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_count, d_off, (int) (n2 + 1), s));
  char *d_tmp = nullptr;
  SCK(dev_slot(C, D_TMP, &d_tmp, (int64_t) tmp_bytes));
  SCK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_count, d_off, (int) (n2 + 1), s));
  SCK(cudaMemcpyAsync(&words[0], d_off + n2, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  SCK(dev_slot(C, D_OUT, &d_out, std::min(words[0], max_recs)));
  const int gg = (int) std::min<int64_t>((n2 + 7) / 8, (int64_t) v.nsm * 8);
  cdna_gather_kernel<<<gg, 256, 0, s>>>(d_gaps, d_as, d_r2, d_fslot, d_count, d_off, n2, max_recs, d_arena,
                                        v.d_genome, v.d_genomealt, v.genome_len, d_out, d_res, d_used);
  gdpi_count_launch(ctx);
  SCK(cudaGetLastError());
  SCK(cudaMemcpyAsync(r2, d_res, n2 * sizeof(gdp_result_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaMemcpyAsync(&words[1], d_used, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  const int64_t used = (int64_t) words[1];
  if (used > 0) SCK(cudaMemcpyAsync(recs, d_out, used * sizeof(gdp_rec_t), cudaMemcpyDeviceToHost, s));
  for (int64_t k = 0; k < n2; k++) {
    gdp_result_t &res = results[gap2[k]];
    const gdp_result_t &t = r2[k];
    const int32_t score = res.score, precision = res.precision;
    res = t;
    res.score = score;
    res.precision = precision;
    if (t.nrecs == 0) res.rec_offset = 0;
  }
  if (used > 0) SCK(cudaStreamSynchronize(s));
  if (nrecs_used) *nrecs_used = used;
  return GDP_OK;
}
