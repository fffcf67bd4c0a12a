/*
 * traceback.cuh -- device traceback, one thread per pair.
 *
 * Walks the packed direction words from (tb_r, tb_c) exactly as
 * Dynprog_traceback_{8,16}[_upper|_lower] do (src/dynprog_simd.c:9153-9945)
 * and writes the Pair records the reference would push through
 * Pairpool_push / Pairpool_add_queryskip / Pairpool_add_genomeskip /
 * Pairpool_push_gapholder (src/pairpool.c:179-257, :374, :980-1010,
 * :1067-1179), in push order, plus the traceback score and counts
 * (scores of src/scores.h:4-9: MATCH +1, MISMATCH -3, open -3, indel -1).
 * Genome characters of short genome skips come from the resident genome in
 * genomecomp form, as get_genomic_nt reads them through Genome_get_char
 * (src/pairpool.c:1015-1063, src/genome.c:9723-9792, :11003-11017).
 *
 * A walk that reaches a cell the fill never wrote -- where the reference
 * reads stale scratch, so the result is undefined -- stops with status
 * GDP_ERR_BAND instead of reading garbage.
 */
#pragma once
#include "gdp_internal.h"
#include "genome_chars.cuh"

struct TbParams {
  const gdp_pair_t *pairs;
  const char *arena;
  const int32_t *list;
  const int32_t *count;
  const uint32_t *dirs;
  const gdp_meta_t *meta;
  gdp_result_t *res;
  gdp_rec_t *recs;
  const int64_t *rec_off;
  const uint32_t *genome, *genomealt;   /* genomecomp blocks, may be NULL */
  uint64_t genome_base;                  /* absolute position of the blocks' first nt */
  uint64_t genome_len;
  const gdp_tables_t *tab;
};

/* Direction-word cursor over one pair's block-column layout. */
struct DirCursor {
  gdp_geom_t g;
  const uint32_t *base;
  int b;            /* current block index */
  int64_t boff;     /* word offset of block b */
  int y0, y1;       /* sweep of block b */

  __device__ void init (const gdp_pair_t &p, int W, const uint32_t *dirs) {
    gdp_geom_of(&p, W, &g);
    base = dirs;
    b = 0;
    boff = 0;
    gdp_block_sweep(&g, 0, &y0, &y1);
  }
  __device__ void seek (int nb) {
    while (b < nb) {
      boff += gdp_block_words(&g, b * g.W);
      b++;
      gdp_block_sweep(&g, b * g.W, &y0, &y1);
    }
    while (b > nb) {
      b--;
      boff -= gdp_block_words(&g, b * g.W);
      gdp_block_sweep(&g, b * g.W, &y0, &y1);
    }
  }
  /* 4-bit code of lane x, swept column y: bit0 nogap HORIZ, bit1 nogap
     VERT, bit2 Egap != DIAG, bit3 Fgap VERT; -1 if the cell was not swept. */
  __device__ int cell (int x, int y) {
    if (x < 0 || y < 0 || x > g.X) return -1;
    const int nb = x / g.W;
    if (nb != b) seek(nb);
    if (y < y0 || y > y1) return -1;
    const int lane = x - b * g.W;
    const uint32_t w = __ldg(base + boff + (int64_t) (y - y0) * (g.W / 8) + gdp_dir_word(g.W, lane));
    const int sh = gdp_dir_bit(g.W, lane);
    return (int) (((w >> sh) & 1u) | (((w >> (8 + sh)) & 1u) << 1) |
                  (((w >> (16 + sh)) & 1u) << 2) | (((w >> (24 + sh)) & 1u) << 3));
  }
};


/*
 * Genome windows of the pairs flagged GDP_FLAG_GWINDOW, read from the
 * resident genome into the arena at gseq (and gseq_alt when it differs):
 * window character j is the genome character at genomic coordinate
 * genomeoffset + j (revp: genomeoffset - (glength - 1) + j), the positions
 * the traceback's genome skips address (GDP_XFLAG_SEGMENT: as the single
 * gap's genome segment holds them).  One block per pair.
 */
__global__ void __launch_bounds__(256)
window_kernel (const gdp_pair_t *pairs, const int32_t *status, int64_t n, char *arena, const uint32_t *genome,
               const uint32_t *genomealt, uint64_t genome_len) {
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    const gdp_pair_t p = pairs[i];
    if (!(p.flags & GDP_FLAG_GWINDOW) || status[i] != GDP_OK) continue;
    const int gl = p.glength;
    const int g0 = (p.flags & GDP_FLAG_REVP) ? p.genomeoffset - (gl - 1) : p.genomeoffset;
    char *w = arena + p.gseq, *wa = arena + p.gseq_alt;
    const bool same = (p.gseq_alt == p.gseq);
    const bool segment = (p.xflags & (GDP_XFLAG_SEGMENT | GDP_XFLAG_SEGMENT_REV)) != 0;
    for (int j = threadIdx.x; j < gl; j += blockDim.x) {
      char a, c;
      if (segment) {
        c = segment_char(p, g0 + j, genome, genomealt, genome_len, &a);
      } else {
        c = genomic_char(p, g0 + j, genome, genomealt, 0, genome_len, &a);
        if (c == 0) { c = 'N'; a = 'N'; }
      }
      w[j] = c;
      if (!same) wa[j] = a;
    }
  }
}

struct TbState {
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

  __device__ void push (int qpos, int gpos, char cdna, char comp, char g, char ga) {
    if (qpos < 0 || gpos < 0) return;   /* Pairpool_push drops these (:189-191) */
    if (n < cap) {
      gdp_rec_t r;
      r.querypos = qpos; r.genomepos = gpos;
      r.cdna = cdna; r.comp = comp; r.genome = g; r.genomealt = ga;
      out[n] = r;
    } else {
      err = GDP_ERR_RECS;
    }
    n++;
  }
  __device__ void gapholder (int dist) {
    if (n < cap) {
      gdp_rec_t r;
      r.querypos = -1; r.genomepos = dist;   /* gap holder: comp '\0' */
      r.cdna = ' '; r.comp = '\0'; r.genome = ' '; r.genomealt = ' ';
      out[n] = r;
    } else {
      err = GDP_ERR_RECS;
    }
    n++;
  }
  /* get_genomic_nt (src/pairpool.c:1015-1063) */
  __device__ char genomic_nt (char *alt, int gp) {
    const char c = genomic_char(*p, gp, genome, genomealt, genome_base, genome_len, alt);
    if (c == 0) { err = GDP_ERR_NOGENOME; *alt = 'N'; return 'N'; }
    return c;
  }
  __device__ void queryskip (int r, int c, int dist) {
    int qc = r - 1, gc = c - 1, step;
    if (revp) { qc = -qc; gc = -gc; step = 1; } else { step = -1; }
    for (int j = 0; j < dist; j++) {
      push(p->queryoffset + qc, p->genomeoffset + gc, rseq[qc], '-', ' ', ' ');
      qc += step;
    }
    score += -3 - dist; nopen += 1; nindel += dist;
  }
  __device__ void genomeskip (int r, int c, int dist) {
    int qc = r - 1, left = c - dist, right = c - 1, step;
    if (revp) { const int t = left; qc = -qc; left = -right; right = -t; step = 1; } else { step = -1; }
    if (dist < GDP_MICROINTRON) {
      int gc = revp ? left : right;
      for (int j = 0; j < dist; j++) {
        char a;
        const char gch = genomic_nt(&a, p->genomeoffset + gc);
        push(p->queryoffset + qc, p->genomeoffset + gc, ' ', '-', gch, a);
        gc += step;
      }
      score += -3 - dist; nopen += 1; nindel += dist;
    } else {
      gapholder(dist);
    }
  }
  __device__ void diagpair (int r, int c) {
    int qc = r - 1, gc = c - 1;
    if (revp) { qc = -qc; gc = -gc; }
    const char c1 = rseq[qc], c1uc = ruc[qc], c2 = gseq[gc], c2a = galt[gc];
    if (c2 == '*') return;
    if (c1uc == c2 || c1uc == c2a) {
      score += 1; nmatch += 1;
      push(p->queryoffset + qc, p->genomeoffset + gc, c1, '*', c2, c2a);
    } else if (tab->cons[p->genestrand][c1uc & 127][c2 & 127] || tab->cons[p->genestrand][c1uc & 127][c2a & 127]) {
      score += 1; nmatch += 1;
      push(p->queryoffset + qc, p->genomeoffset + gc, c1, ':', c2, c2a);
    } else {
      score += -3; nmismatch += 1;
      push(p->queryoffset + qc, p->genomeoffset + gc, c1, ' ', c2, c2a);
    }
  }
};

/* One traceback walk over the direction words behind `dc`. */
__device__ void
tb_walk (const gdp_pair_t &p, DirCursor &dc, TbState &T) {
  int r = p.tb_r, c = p.tb_c;
  const bool lower = (p.variant == GDP_LOWER);
  /* (x, y) of cell (c, r): lanes are rows except in the lower fill */
#define CELL(cc, rr) (lower ? dc.cell((cc), (rr)) : dc.cell((rr), (cc)))
  /* a full-band cell above the band derives from stale scratch in the reference */
#define ABOVE(cc, rr) (p.variant == GDP_FULL && (rr) < (cc) - p.uband)
  if (p.variant == GDP_FULL) {
    while (r > 0 && c > 0 && !T.err) {
      const int code = CELL(c, r);
      if (code < 0 || ABOVE(c, r)) { T.err = GDP_ERR_BAND; break; }
      const int dir = (code & 2) ? -2 : (code & 1) ? -1 : 0;
      if (dir == -1) {
        int dist = 1;
        while (c > 0) {
          const int e = CELL(c, r);
          if (e < 0 || ABOVE(c, r)) { T.err = GDP_ERR_BAND; break; }
          c--;
          if (!(e & 4)) break;
          dist++;
        }
        if (T.err) break;
        T.genomeskip(r, c + dist, dist);
      } else if (dir == -2) {
        int dist = 1;
        while (r > 0) {
          const int f = CELL(c, r);
          if (f < 0 || ABOVE(c, r)) { T.err = GDP_ERR_BAND; break; }
          r--;
          if (!(f & 8)) break;
          dist++;
        }
        if (T.err) break;
        T.queryskip(r + dist, c, dist);
      } else {
        T.diagpair(r, c);
        r--; c--;
      }
    }
    if (!T.err) {
      if (r == 0 && c == 0) {
      } else if (c == 0) {
        T.queryskip(r, 1, r);
      } else {
        T.genomeskip(1, c, c);
      }
    }
  } else if (p.variant == GDP_UPPER) {
    while (r > 0 && c > 0 && !T.err) {
      const int code = CELL(c, r);
      if (code < 0) { T.err = GDP_ERR_BAND; break; }
      if (code & 3) {
        int dist = 1;
        for (;;) {
          const int e = CELL(c, r);
          if (e < 0) { T.err = GDP_ERR_BAND; break; }
          c--;
          if (!(e & 4)) break;
          dist++;
        }
        if (T.err) break;
        T.genomeskip(r, c + dist, dist);
      } else {
        T.diagpair(r, c);
        r--; c--;
      }
    }
    if (!T.err && c != 0) T.genomeskip(1, c, c);
  } else {
    while (r > 0 && c > 0 && !T.err) {
      const int code = CELL(c, r);
      if (code < 0) { T.err = GDP_ERR_BAND; break; }
      if (code & 3) {
        int dist = 1;
        for (;;) {
          const int e = CELL(c, r);
          if (e < 0) { T.err = GDP_ERR_BAND; break; }
          r--;
          if (!(e & 4)) break;
          dist++;
        }
        if (T.err) break;
        T.queryskip(r + dist, c, dist);
      } else {
        T.diagpair(r, c);
        r--; c--;
      }
    }
    if (!T.err && r != 0) T.queryskip(r, 1, r);
  }
#undef CELL
#undef ABOVE
}

__global__ void __launch_bounds__(128)
traceback_kernel (TbParams P) {
  const int64_t nthreads = (int64_t) gridDim.x * blockDim.x;
  const int n = *P.count;
  for (int64_t li = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; li < n; li += nthreads) {
    const int pi = __ldg(P.list + li);
    const gdp_pair_t p = P.pairs[pi];
    gdp_result_t *res = P.res + pi;
    if (res->status != GDP_OK) continue;
    const gdp_meta_t m = P.meta[pi];
    int W = (res->precision == 8) ? 32 : 16;
    TbState T;
    T.p = &p;
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
    for (int attempt = 0; attempt < 2; attempt++) {
      DirCursor dc;
      dc.init(p, W, P.dirs + (W == 16 ? m.dir16 : m.dir8));
      T.n = 0; T.score = T.nmatch = T.nmismatch = T.nopen = T.nindel = 0; T.err = 0;
      tb_walk(p, dc, T);
      /* An 8-bit walk that leaves the cells its fill wrote has no defined
         result; a rerun pair then takes its 16-bit fill and traceback. */
      if (T.err == GDP_ERR_BAND && W == 32 && m.dir16 >= 0) {
        W = 16;
        res->precision = 16;
        res->rerun = 1;
        res->score = m.final16;
        continue;
      }
      break;
    }
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
