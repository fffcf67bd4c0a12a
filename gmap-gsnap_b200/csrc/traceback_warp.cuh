/*
 * traceback_warp.cuh -- the traceback with one warp per pair.
 *
 * The walk of Dynprog_traceback_* (src/dynprog_simd.c:9153-9945) is a chain
 * of dependent reads: every step reads the direction of the cell the
 * previous step moved to.  One thread per pair therefore waits one load
 * latency per step, and a long pair's walk of several thousand steps takes
 * milliseconds.  Here the 32 lanes of a warp examine the next 32 cells of
 * the current straight run at once -- lane j the j-th cell along the
 * diagonal, the row of an E walk or the column of an F walk -- and a ballot
 * finds where the run ends.  The steps before that point are independent:
 * each lane builds its own Pair record, and a prefix count over the lanes
 * gives every record its place in push order.  Records, counters, error
 * codes and the rerun fallback are the same as those of traceback_kernel.
 */
#pragma once
#include "traceback.cuh"

#define GDP_FULL_MASK 0xffffffffu

/* Uniform walk state (every lane holds the same values) plus this lane's
   own direction cursor. */
struct WarpTb {
  const gdp_pair_t *p;
  const char *rseq, *ruc, *gseq, *galt;   /* reference-convention pointers (revp: last char) */
  bool revp;
  gdp_rec_t *out;
  int64_t cap;
  int n;
  int score, nmatch, nmismatch, nopen, nindel;
  int err;
  const uint32_t *genome, *genomealt;
  uint64_t genome_base, genome_len;
  const gdp_tables_t *tab;
  int lane;
  unsigned lt;   /* lanes below this one */

  /* Each lane with `want` pushes one record; Pairpool_push drops records
     with a negative coordinate (src/pairpool.c:189-191). */
  __device__ void push_lanes (bool want, int qpos, int gpos, char cdna, char comp, char g, char ga) {
    const bool keep = want && qpos >= 0 && gpos >= 0;
    const unsigned m = __ballot_sync(GDP_FULL_MASK, keep);
    const int idx = n + __popc(m & lt);
    bool over = false;
    if (keep) {
      if (idx < cap) {
        gdp_rec_t r;
        r.querypos = qpos; r.genomepos = gpos;
        r.cdna = cdna; r.comp = comp; r.genome = g; r.genomealt = ga;
        out[idx] = r;
      } else {
        over = true;
      }
    }
    if (__any_sync(GDP_FULL_MASK, over)) err = GDP_ERR_RECS;
    n += __popc(m);
  }
  __device__ void gapholder (int dist) {
    if (n < cap) {
      if (lane == 0) {
        gdp_rec_t r;
        r.querypos = -1; r.genomepos = dist;   /* gap holder: comp '\0' */
        r.cdna = ' '; r.comp = '\0'; r.genome = ' '; r.genomealt = ' ';
        out[n] = r;
      }
    } else {
      err = GDP_ERR_RECS;
    }
    n++;
  }
  /* Pairpool_add_queryskip (src/pairpool.c:980-1010), 32 records per round */
  __device__ void queryskip (int r, int c, int dist) {
    int qc = r - 1, gc = c - 1, step;
    if (revp) { qc = -qc; gc = -gc; step = 1; } else { step = -1; }
    for (int j0 = 0; j0 < dist; j0 += 32) {
      const int j = j0 + lane;
      const bool want = j < dist;
      const int q = qc + j * step;
      push_lanes(want, p->queryoffset + q, p->genomeoffset + gc, want ? rseq[q] : ' ', '-', ' ', ' ');
    }
    score += -3 - dist; nopen += 1; nindel += dist;
  }
  /* Pairpool_add_genomeskip (src/pairpool.c:1067-1180) */
  __device__ void genomeskip (int r, int c, int dist) {
    int qc = r - 1, left = c - dist, right = c - 1, step;
    if (revp) { const int t = left; qc = -qc; left = -right; right = -t; step = 1; } else { step = -1; }
    if (dist < GDP_MICROINTRON) {
      const bool want = lane < dist;
      const int gc = (revp ? left : right) + lane * step;
      char a = ' ', gch = ' ';
      bool miss = false;
      if (want) {
        gch = genomic_char(*p, p->genomeoffset + gc, genome, genomealt, genome_base, genome_len, &a);
        if (gch == 0) { miss = true; gch = 'N'; a = 'N'; }
      }
      if (__any_sync(GDP_FULL_MASK, miss)) err = GDP_ERR_NOGENOME;
      push_lanes(want, p->queryoffset + qc, p->genomeoffset + gc, ' ', '-', gch, a);
      score += -3 - dist; nopen += 1; nindel += dist;
    } else {
      gapholder(dist);
    }
  }
  /* The diagonal steps (r - j, c - j), j < k: one match / ambiguous /
     mismatch Pair each, none where the genome character is '*'. */
  /* The characters of lane j's cell (r - j, c - j) of a diagonal run, read
     before the run's direction words arrive (the two loads overlap). */
  __device__ void diagchars (int r, int c, bool valid, char &c1, char &c1uc, char &c2, char &c2a) const {
    int qc = r - 1 - lane, gc = c - 1 - lane;
    if (revp) { qc = -qc; gc = -gc; }
    c1 = ' '; c1uc = ' '; c2 = '*'; c2a = '*';
    if (valid) { c1 = rseq[qc]; c1uc = ruc[qc]; c2 = gseq[gc]; c2a = galt[gc]; }
  }
  __device__ void diagpairs (int r, int c, int k, char c1, char c1uc, char c2, char c2a) {
    const bool on = lane < k;
    int qc = r - 1 - lane, gc = c - 1 - lane;
    if (revp) { qc = -qc; gc = -gc; }
    if (!on) { c1 = ' '; c1uc = ' '; c2 = '*'; c2a = '*'; }
    const bool pair = on && c2 != '*';
    char comp = ' ';
    bool match = false;
    if (pair) {
      if (c1uc == c2 || c1uc == c2a) { comp = '*'; match = true; }
      else if (tab->cons[p->genestrand][c1uc & 127][c2 & 127] || tab->cons[p->genestrand][c1uc & 127][c2a & 127]) {
        comp = ':'; match = true;
      }
    }
    const int nm = __popc(__ballot_sync(GDP_FULL_MASK, pair && match));
    const int nx = __popc(__ballot_sync(GDP_FULL_MASK, pair && !match));
    score += nm - 3 * nx; nmatch += nm; nmismatch += nx;
    push_lanes(pair, p->queryoffset + qc, p->genomeoffset + gc, c1, comp, c2, c2a);
  }
};

/* One walk, every lane of the warp together. */
__device__ void
tb_walk_warp (const gdp_pair_t &p, DirCursor &dc, WarpTb &T) {
  const int lane = T.lane;
  const bool lower = (p.variant == GDP_LOWER);
  const bool full = (p.variant == GDP_FULL);
  int r = p.tb_r, c = p.tb_c;
#define CELL(cc, rr) (lower ? dc.cell((cc), (rr)) : dc.cell((rr), (cc)))
  /* a full-band cell above the band derives from stale scratch in the reference */
#define ABOVE(cc, rr) (full && (rr) < (cc) - p.uband)
  while (r > 0 && c > 0 && !T.err) {
    /* the diagonal run: lane j looks at (r - j, c - j) */
    const bool valid = (r - lane > 0) && (c - lane > 0);
    char c1, c1uc, c2, c2a;
    T.diagchars(r, c, valid, c1, c1uc, c2, c2a);
    const int code = valid ? CELL(c - lane, r - lane) : -1;
    const bool bad = valid && (code < 0 || ABOVE(c - lane, r - lane));
    const bool gap = valid && !bad && (code & 3);
    const unsigned badm = __ballot_sync(GDP_FULL_MASK, bad);
    const unsigned stop = __ballot_sync(GDP_FULL_MASK, !valid || bad || gap);
    const int k = stop ? __ffs(stop) - 1 : 32;
    if (k > 0) T.diagpairs(r, c, k, c1, c1uc, c2, c2a);
    r -= k; c -= k;
    if (T.err) break;
    if (k == 32 || r <= 0 || c <= 0) continue;
    if ((badm >> k) & 1u) { T.err = GDP_ERR_BAND; break; }
    const int kcode = __shfl_sync(GDP_FULL_MASK, code, k);
    if (!full || !(kcode & 2)) {
      /* E walk (full: nogap HORIZ; upper: any gap; lower: any gap, along
         the rows): while the cell's Egap is not DIAG, post-decrement
         (src/dynprog_simd.c:9174) */
      int dist = 1;
      bool done = false;
      while (!done) {
        const int left = lower ? r : c;            /* coordinate the walk decrements */
        if (full && left <= 0) break;              /* the full walk stops at column 0 */
        const int nv = full ? min(32, left) : 32;
        const bool v = lane < nv;
        int e = -1;
        if (v) e = lower ? dc.cell(c, r - lane) : dc.cell(r, c - lane);
        const bool eb = v && (e < 0 || ABOVE(c - lane, r));
        const bool es = v && !eb && !(e & 4);
        const unsigned bm = __ballot_sync(GDP_FULL_MASK, eb), sm = __ballot_sync(GDP_FULL_MASK, es);
        const unsigned any = bm | sm;
        int adv;
        if (any) {
          const int j = __ffs(any) - 1;
          if ((bm >> j) & 1u) { T.err = GDP_ERR_BAND; break; }
          adv = j + 1; dist += j; done = true;
        } else {
          adv = nv; dist += nv;
        }
        if (lower) r -= adv; else c -= adv;
      }
      if (T.err) break;
      if (lower) T.queryskip(r + dist, c, dist);
      else T.genomeskip(r, c + dist, dist);
    } else {
      /* F walk (full, nogap VERT): while the cell's Fgap is VERT (:9200) */
      int dist = 1;
      bool done = false;
      while (!done && r > 0) {
        const int nv = min(32, r);
        const bool v = lane < nv;
        const int f = v ? dc.cell(r - lane, c) : -1;
        const bool fb = v && (f < 0 || ABOVE(c, r - lane));
        const bool fs = v && !fb && !(f & 8);
        const unsigned bm = __ballot_sync(GDP_FULL_MASK, fb), sm = __ballot_sync(GDP_FULL_MASK, fs);
        const unsigned any = bm | sm;
        if (any) {
          const int j = __ffs(any) - 1;
          if ((bm >> j) & 1u) { T.err = GDP_ERR_BAND; break; }
          r -= j + 1; dist += j; done = true;
        } else {
          r -= nv; dist += nv;
        }
      }
      if (T.err) break;
      T.queryskip(r + dist, c, dist);
    }
  }
  if (!T.err) {
    if (full) {
      if (r == 0 && c == 0) {
      } else if (c == 0) {
        T.queryskip(r, 1, r);
      } else {
        T.genomeskip(1, c, c);
      }
    } else if (lower) {
      if (r != 0) T.queryskip(r, 1, r);
    } else {
      if (c != 0) T.genomeskip(1, c, c);
    }
  }
#undef CELL
#undef ABOVE
}

__global__ void __launch_bounds__(128, 6)
traceback_warp_kernel (TbParams P) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  const int n = *P.count;
  for (int64_t li = warp; li < n; li += nwarps) {
    const int pi = __ldg(P.list + li);
    const gdp_pair_t p = P.pairs[pi];
    gdp_result_t *res = P.res + pi;
    if (res->status != GDP_OK) continue;
    const gdp_meta_t m = P.meta[pi];
    int W = (res->precision == 8) ? 32 : 16;
    WarpTb T;
    T.p = &p;
    T.lane = lane;
    T.lt = (1u << lane) - 1u;
    T.revp = (p.flags & GDP_FLAG_REVP) != 0;
    T.rseq = P.arena + p.rseq; T.ruc = P.arena + p.rseq_uc;
    T.gseq = P.arena + p.gseq; T.galt = P.arena + p.gseq_alt;
    if (T.revp) {
      T.rseq += p.rlength - 1; T.ruc += p.rlength - 1;
      T.gseq += p.glength - 1; T.galt += p.glength - 1;
    }
    T.out = P.recs + P.rec_off[pi];
    T.cap = (int64_t) p.rlength + p.glength + 2;
    T.genome = P.genome; T.genomealt = P.genomealt ? P.genomealt : P.genome;
    T.genome_base = P.genome_base;
    T.genome_len = P.genome_len;
    T.tab = P.tab;
    int precision = res->precision, rerun = res->rerun, score = res->score;
    for (int attempt = 0; attempt < 2; attempt++) {
      DirCursor dc;
      dc.init(p, W, P.dirs + (W == 16 ? m.dir16 : m.dir8));
      T.n = 0; T.score = T.nmatch = T.nmismatch = T.nopen = T.nindel = 0; T.err = 0;
      tb_walk_warp(p, dc, T);
      /* An 8-bit walk that leaves the cells its fill wrote has no defined
         result; a rerun pair then takes its 16-bit fill and traceback. */
      if (T.err == GDP_ERR_BAND && W == 32 && m.dir16 >= 0) {
        W = 16;
        precision = 16;
        rerun = 1;
        score = m.final16;
        continue;
      }
      break;
    }
    __syncwarp();
    if (lane == 0) {
      res->precision = precision;
      res->rerun = rerun;
      res->score = score;
      res->tb_score = T.score;
      res->nmatches = T.nmatch;
      res->nmismatches = T.nmismatch;
      res->nopens = T.nopen;
      res->nindels = T.nindel;
      res->nrecs = T.n;
      res->rec_offset = P.rec_off[pi];
      if (T.err) res->status = T.err;
    }
  }
}
