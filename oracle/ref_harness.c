/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Plain-C wrappers around the reference's own compiled dynamic-programming
 * functions (src/dynprog_simd.c, src/dynprog.c, src/pairpool.c, built from
 * the reference sources by oracle/Makefile into oracle/_ref/).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm use
 * this library; the product never links it.
 *
 * What it provides:
 *   - ref_init(mode): Dynprog_init (src/dynprog.c:1007-1196).
 *   - ref_set_genome(): the synthetic Genome_T the tracebacks read through
 *     Genome_get_char for genome skips (src/pairpool.c:1015-1063).
 *   - ref_align(): one fill (Dynprog_simd_{8,16}[_upper|_lower],
 *     src/dynprog_simd.c:2986, :4303, :5339, :6561, :7713, :8585) plus an
 *     optional traceback (src/dynprog_simd.c:9153-9945), dumping the
 *     in-band scores and directions over the reference's own compare domain
 *     (src/dynprog_simd.c:1044-1051, :1089-1096, :1134-1141) and the Pair
 *     list as flat records in push order.
 *   - ref_bench(): the CPU baseline -- the same fills and tracebacks over a
 *     batch of pairs, one pthread per requested core, each thread with its
 *     own Dynprog_T and Pairpool_T (as gmap.c:4907-4911 does per worker).
 *
 * Genome_get_char is not part of the six linked reference files; the stub
 * below decodes the reference's genomecomp block format (three uint32 per
 * 32 nt: high = nt 16..31, low = nt 0..15, 2 bits each; flags = 1 bit per nt
 * meaning 'N'), restating uncompress_one_char and Genome_get_char
 * (src/genome.c:9723-9763, :9766-9792, :11003-11017).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>

#include "dynprog.h"
#include "dynprog_simd.h"
#include "pairpool.h"
#include "pairdef.h"
#include "list.h"
#include "genome.h"

#include "gdp.h"   /* gdp_pair_t, gdp_rec_t: the batch formats shared with the product */

/* ------------------------------------------------------------------ */
/* Synthetic genome behind Genome_get_char                             */
/* ------------------------------------------------------------------ */

static struct Genome_T genome_main, genome_alt;
static int genome_set = 0;

void
ref_set_genome (const uint32_t *blocks, const uint32_t *altblocks, uint64_t genomelength) {
  memset(&genome_main, 0, sizeof(genome_main));
  memset(&genome_alt, 0, sizeof(genome_alt));
  genome_main.blocks = (Genomecomp_T *) blocks;
  genome_main.genomelength = (Univcoord_T) genomelength;
  genome_alt.blocks = (Genomecomp_T *) (altblocks ? altblocks : blocks);
  genome_alt.genomelength = (Univcoord_T) genomelength;
  genome_set = 1;
}

Genome_T ref_genome_main (void) { return &genome_main; }
Genome_T ref_genome_alt (void) { return &genome_alt; }

static const char ACGT[4] = {'A', 'C', 'G', 'T'};

static char
decode_nt (const Genomecomp_T *blocks, Univcoord_T pos, int honour_flags) {
  Univcoord_T ptr = pos / 32U * 3;
  int bit = (int) (pos % 32);
  if (honour_flags && (blocks[ptr + 2] & (1U << bit))) {
    return 'N';
  } else if (bit < 16) {
    return ACGT[(blocks[ptr + 1] >> (2 * bit)) & 3U];
  } else {
    return ACGT[(blocks[ptr] >> (2 * bit - 32)) & 3U];
  }
}

char
Genome_get_char (char *charalt, Genome_T genome, Genome_T genomealt, Univcoord_T left) {
  char c = decode_nt(genome->blocks, left, 1);
  if (c == 'N') {
    *charalt = c;
  } else {
    *charalt = decode_nt(genomealt->blocks, left, 0);
  }
  return c;
}

/* ------------------------------------------------------------------ */
/* Per-thread reference state                                          */
/* ------------------------------------------------------------------ */

typedef struct {
  Dynprog_T one;       /* full-band fills (doublep = false) */
  Dynprog_T two;       /* upper/lower fills (doublep = true) */
  int cap_r, cap_g;
  Pairpool_T pool;
} refstate_t;

static void
refstate_ensure (refstate_t *st, int rlength, int glength) {
  int R, G;
  if (st->one != NULL && rlength <= st->cap_r && glength <= st->cap_g) {
    return;
  }
  if (st->one) Dynprog_free(&st->one);
  if (st->two) Dynprog_free(&st->two);
  R = rlength > st->cap_r ? rlength : st->cap_r;
  G = glength > st->cap_g ? glength : st->cap_g;
  if (G < R) G = R;
  /* Dynprog_new: max_rlength = maxlookback + maxpeelback,
     max_glength = max_rlength + extraquerygap + max(extras) (src/dynprog.c:606-626) */
  st->one = Dynprog_new(R, G - R, 0, 0, 0, /*doublep*/false);
  st->two = Dynprog_new(R, G - R, 0, 0, 0, /*doublep*/true);
  st->cap_r = st->one->max_rlength;
  st->cap_g = st->one->max_glength;
  if (st->pool == NULL) st->pool = Pairpool_new();
}

static void
refstate_free (refstate_t *st) {
  if (st->one) Dynprog_free(&st->one);
  if (st->two) Dynprog_free(&st->two);
  if (st->pool) Pairpool_free(&st->pool);
}

static refstate_t main_state;
static int inited = 0;
static int inited_mode = 0;

void
ref_init (int mode) {
  if (inited) {
    Dynprog_term((Mode_T) inited_mode);
  }
  Dynprog_init((Mode_T) mode);
  inited = 1;
  inited_mode = mode;
}

int
ref_use8p_size (int mismatchtype) {
  return use8p_size[mismatchtype];
}

int
ref_pairdistance (int mismatchtype, int c1, int c2) {
  return pairdistance_array[mismatchtype][c1][c2];
}

int
ref_consistent (int genestrand, int c1, int c2) {
  return consistent_array[genestrand][c1][c2] ? 1 : 0;
}

/* ------------------------------------------------------------------ */
/* One fill (+ traceback)                                              */
/* ------------------------------------------------------------------ */

typedef struct {
  void **matrix;   /* Score8_T** or Score16_T** */
  void **nogap, **Egap, **Fgap;
  int prec, variant;
} fillout_t;

static void
run_fill (refstate_t *st, const gdp_pair_t *p, const char *arena, fillout_t *o) {
  char *rseq = (char *) arena + p->rseq;
  char *gseq = (char *) arena + p->gseq;
  char *galt = (char *) arena + p->gseq_alt;
  int revp = (p->flags & GDP_FLAG_REVP) != 0;
  int late = (p->flags & GDP_FLAG_JUMP_LATE) != 0;
  if (revp) {
    /* the reference indexes backwards from the last character: seq[1-r] */
    rseq += p->rlength - 1;
    gseq += p->glength - 1;
    galt += p->glength - 1;
  }
  refstate_ensure(st, p->rlength, p->glength);
  o->prec = p->precision;
  o->variant = p->variant;
  o->Fgap = NULL;
  if (p->precision == 8) {
    Direction8_T **n = NULL, **e = NULL, **f = NULL;
    if (p->variant == GDP_FULL) {
      o->matrix = (void **) Dynprog_simd_8(&n, &e, &f, st->one, rseq, gseq, galt, p->rlength, p->glength,
                                           (Mismatchtype_T) p->mismatchtype, p->open, p->extend,
                                           p->lband, p->uband, late, revp);
    } else if (p->variant == GDP_UPPER) {
      o->matrix = (void **) Dynprog_simd_8_upper(&n, &e, st->two, rseq, gseq, galt, p->rlength, p->glength,
                                                 (Mismatchtype_T) p->mismatchtype, p->open, p->extend,
                                                 p->uband, late, revp);
    } else {
      o->matrix = (void **) Dynprog_simd_8_lower(&n, &e, st->two, rseq, gseq, galt, p->rlength, p->glength,
                                                 (Mismatchtype_T) p->mismatchtype, p->open, p->extend,
                                                 p->lband, late, revp);
    }
    o->nogap = (void **) n; o->Egap = (void **) e; o->Fgap = (void **) f;
  } else {
    Direction16_T **n = NULL, **e = NULL, **f = NULL;
    if (p->variant == GDP_FULL) {
      o->matrix = (void **) Dynprog_simd_16(&n, &e, &f, st->one, rseq, gseq, galt, p->rlength, p->glength,
                                            (Mismatchtype_T) p->mismatchtype, p->open, p->extend,
                                            p->lband, p->uband, late, revp);
    } else if (p->variant == GDP_UPPER) {
      o->matrix = (void **) Dynprog_simd_16_upper(&n, &e, st->two, rseq, gseq, galt, p->rlength, p->glength,
                                                  (Mismatchtype_T) p->mismatchtype, p->open, p->extend,
                                                  p->uband, late, revp);
    } else {
      o->matrix = (void **) Dynprog_simd_16_lower(&n, &e, st->two, rseq, gseq, galt, p->rlength, p->glength,
                                                  (Mismatchtype_T) p->mismatchtype, p->open, p->extend,
                                                  p->lband, late, revp);
    }
    o->nogap = (void **) n; o->Egap = (void **) e; o->Fgap = (void **) f;
  }
}

static int
get_cell (void **m, int prec, int i, int j) {
  if (m == NULL) return 0;
  if (prec == 8) return ((Score8_T **) m)[i][j];
  return ((Score16_T **) m)[i][j];
}

/* Row range of the compare domain for column c (src/dynprog_simd.c:1044-1051,
   :1089-1096, :1134-1141). */
static void
domain_rows (const gdp_pair_t *p, int c, int *lo, int *hi) {
  if (p->variant == GDP_FULL) {
    *lo = c - p->uband; *hi = c + p->lband;
  } else if (p->variant == GDP_UPPER) {
    *lo = c - p->uband; *hi = c;
  } else {
    *lo = c; *hi = c + p->lband;
  }
  if (*lo < 1) *lo = 1;
  if (*hi > p->rlength) *hi = p->rlength;
}

static int
run_traceback (refstate_t *st, const gdp_pair_t *p, const char *arena, fillout_t *o,
               int *stats, gdp_rec_t *recs, int max_recs) {
  char *rseq = (char *) arena + p->rseq;
  char *ruc = (char *) arena + p->rseq_uc;
  char *gseq = (char *) arena + p->gseq;
  char *galt = (char *) arena + p->gseq_alt;
  int revp = (p->flags & GDP_FLAG_REVP) != 0;
  int score = 0, nmatches = 0, nmismatches = 0, nopens = 0, nindels = 0;
  int r = p->tb_r, c = p->tb_c;
  List_T pairs = NULL, q;
  int n, k;
  if (revp) {
    rseq += p->rlength - 1;
    ruc += p->rlength - 1;
    gseq += p->glength - 1;
    galt += p->glength - 1;
  }
  Pairpool_reset(st->pool);
  if (p->precision == 8) {
    if (p->variant == GDP_FULL) {
      pairs = Dynprog_traceback_8(NULL, &score, &nmatches, &nmismatches, &nopens, &nindels,
                                  (Direction8_T **) o->nogap, (Direction8_T **) o->Egap, (Direction8_T **) o->Fgap,
                                  r, c, rseq, ruc, gseq, galt, p->queryoffset, p->genomeoffset,
                                  &genome_main, &genome_alt, st->pool, revp,
                                  p->chroffset, p->chrhigh, p->watsonp, p->genestrand, p->dynprogindex);
    } else if (p->variant == GDP_UPPER) {
      pairs = Dynprog_traceback_8_upper(NULL, &score, &nmatches, &nmismatches, &nopens, &nindels,
                                        (Direction8_T **) o->nogap, (Direction8_T **) o->Egap,
                                        r, c, rseq, ruc, gseq, galt, p->queryoffset, p->genomeoffset,
                                        &genome_main, &genome_alt, st->pool, revp,
                                        p->chroffset, p->chrhigh, p->watsonp, p->genestrand, p->dynprogindex);
    } else {
      pairs = Dynprog_traceback_8_lower(NULL, &score, &nmatches, &nmismatches, &nopens, &nindels,
                                        (Direction8_T **) o->nogap, (Direction8_T **) o->Egap,
                                        r, c, rseq, ruc, gseq, galt, p->queryoffset, p->genomeoffset,
                                        st->pool, p->genestrand, revp, p->dynprogindex);
    }
  } else {
    if (p->variant == GDP_FULL) {
      pairs = Dynprog_traceback_16(NULL, &score, &nmatches, &nmismatches, &nopens, &nindels,
                                   (Direction16_T **) o->nogap, (Direction16_T **) o->Egap, (Direction16_T **) o->Fgap,
                                   r, c, rseq, ruc, gseq, galt, p->queryoffset, p->genomeoffset,
                                   &genome_main, &genome_alt, st->pool, revp,
                                   p->chroffset, p->chrhigh, p->watsonp, p->genestrand, p->dynprogindex);
    } else if (p->variant == GDP_UPPER) {
      pairs = Dynprog_traceback_16_upper(NULL, &score, &nmatches, &nmismatches, &nopens, &nindels,
                                         (Direction16_T **) o->nogap, (Direction16_T **) o->Egap,
                                         r, c, rseq, ruc, gseq, galt, p->queryoffset, p->genomeoffset,
                                         &genome_main, &genome_alt, st->pool, revp,
                                         p->chroffset, p->chrhigh, p->watsonp, p->genestrand, p->dynprogindex);
    } else {
      pairs = Dynprog_traceback_16_lower(NULL, &score, &nmatches, &nmismatches, &nopens, &nindels,
                                         (Direction16_T **) o->nogap, (Direction16_T **) o->Egap,
                                         r, c, rseq, ruc, gseq, galt, p->queryoffset, p->genomeoffset,
                                         st->pool, p->genestrand, revp, p->dynprogindex);
    }
  }
  n = 0;
  for (q = pairs; q != NULL; q = q->rest) n++;
  if (stats) {
    stats[0] = score; stats[1] = nmatches; stats[2] = nmismatches;
    stats[3] = nopens; stats[4] = nindels; stats[5] = n;
  }
  if (recs != NULL) {
    /* The list is in reverse push order (each push prepends); store push order. */
    k = n - 1;
    for (q = pairs; q != NULL; q = q->rest, k--) {
      Pair_T pr = (Pair_T) q->first;
      if (k < max_recs) {
        gdp_rec_t *d = &recs[k];
        if (pr->gapp) {
          /* a gap holder: comp '\0', genomepos = the skipped genome length */
          d->querypos = pr->querypos;
          d->genomepos = pr->genomejump;
          d->cdna = pr->cdna;
          d->comp = '\0';
        } else {
          d->querypos = pr->querypos;
          d->genomepos = (int32_t) pr->genomepos;
          d->cdna = pr->cdna;
          d->comp = pr->comp;
        }
        d->genome = pr->genome;
        d->genomealt = pr->genomealt;
      }
    }
  }
  return n;
}

/*
 * One pair: fill, dump the compare domain densely in (c, r) order
 * (out[c * (rlength + 1) + r]; lower variants transposed from [r][c]), and
 * optionally trace back from (tb_r, tb_c).  Cells outside the domain are
 * left untouched.  Returns the number of Pair records of the traceback
 * (0 when no traceback was asked for).
 */
int
ref_align (const gdp_pair_t *p, const char *arena,
           int16_t *H, int8_t *dN, int8_t *dE, int8_t *dF, int32_t *final_score,
           int32_t *tb_stats, gdp_rec_t *recs, int max_recs) {
  fillout_t o;
  int c, r, lo, hi, n = 0, R = p->rlength + 1;
  if (!inited) ref_init(0);
  run_fill(&main_state, p, arena, &o);
  for (c = 1; c <= p->glength; c++) {
    domain_rows(p, c, &lo, &hi);
    for (r = lo; r <= hi; r++) {
      int i = (p->variant == GDP_LOWER) ? r : c;
      int j = (p->variant == GDP_LOWER) ? c : r;
      size_t at = (size_t) c * R + r;
      if (H) H[at] = (int16_t) get_cell(o.matrix, o.prec, i, j);
      if (dN) dN[at] = (int8_t) get_cell(o.nogap, o.prec, i, j);
      if (dE) dE[at] = (int8_t) get_cell(o.Egap, o.prec, i, j);
      if (dF) dF[at] = (int8_t) (o.Fgap ? get_cell(o.Fgap, o.prec, i, j) : 0);
    }
  }
  if (final_score) {
    if (p->variant == GDP_LOWER) {
      *final_score = get_cell(o.matrix, o.prec, p->rlength, p->glength);
    } else {
      *final_score = get_cell(o.matrix, o.prec, p->glength, p->rlength);
    }
  }
  if (p->flags & GDP_FLAG_TRACEBACK) {
    n = run_traceback(&main_state, p, arena, &o, tb_stats, recs, max_recs);
  }
  return n;
}

/* ------------------------------------------------------------------ */
/* CPU baseline: the reference over a batch, one pthread per core      */
/* ------------------------------------------------------------------ */

typedef struct {
  const gdp_pair_t *pairs;
  const char *arena;
  const int8_t *kept;
  int64_t npairs;
  int tid, nthreads;
  int64_t checksum;
  int32_t *out;      /* ref_outputs: 8 words per pair, else NULL */
} benchjob_t;

/* 32-bit digest of n Pair records in push order: the sum over records k
   of (w0 * 0x9E3779B1 + w1 * 0x85EBCA77 + w2 * 0xC2B2AE3D + 1) * (2k + 1),
   w0..w2 the record's three words (the benchmark computes the same digest
   of the device's records). */
static uint32_t
rec_digest (const gdp_rec_t *recs, int n) {
  uint32_t d = 0;
  int k;
  for (k = 0; k < n; k++) {
    uint32_t w[3];
    memcpy(w, &recs[k], sizeof(w));
    d += (w[0] * 0x9E3779B1u + w[1] * 0x85EBCA77u + w[2] * 0xC2B2AE3Du + 1u) * (uint32_t) (2 * k + 1);
  }
  return d;
}

static void *
bench_worker (void *arg) {
  benchjob_t *job = (benchjob_t *) arg;
  refstate_t st;
  int64_t i, sum = 0;
  gdp_rec_t *recs = NULL;
  int cap = 0;
  memset(&st, 0, sizeof(st));
  for (i = job->tid; i < job->npairs; i += job->nthreads) {
    const gdp_pair_t *p = &job->pairs[i];
    gdp_pair_t q;
    fillout_t o;
    int stats[6] = {0, 0, 0, 0, 0, 0};
    int fs;
    uint32_t dig = 0;
    if (p->precision == 8 && (p->flags & GDP_FLAG_RERUN16)) {
      /* only the kept precision runs */
      q = *p;
      q.precision = job->kept ? job->kept[i] : 16;
      p = &q;
    }
    run_fill(&st, p, job->arena, &o);
    if (p->variant == GDP_LOWER) {
      fs = get_cell(o.matrix, o.prec, p->rlength, p->glength);
    } else {
      fs = get_cell(o.matrix, o.prec, p->glength, p->rlength);
    }
    sum += fs;
    if (p->flags & GDP_FLAG_TRACEBACK) {
      if (job->out) {
        const int need = p->rlength + p->glength + 8;
        int n;
        if (need > cap) {
          free(recs);
          cap = 2 * need;
          recs = (gdp_rec_t *) malloc((size_t) cap * sizeof(gdp_rec_t));
        }
        n = run_traceback(&st, p, job->arena, &o, stats, recs, cap);
        dig = rec_digest(recs, n < cap ? n : cap);
      } else {
        run_traceback(&st, p, job->arena, &o, stats, NULL, 0);
      }
      sum += stats[0];
    }
    if (job->out) {
      int32_t *w = job->out + 8 * i;
      w[0] = fs;
      memcpy(w + 1, stats, sizeof(stats));
      w[7] = (int32_t) dig;
    }
  }
  free(recs);
  refstate_free(&st);
  job->checksum = sum;
  return NULL;
}

/* Runs every pair once across nthreads threads; returns wall seconds and
   writes a checksum of final and traceback scores.  An 8-bit pair flagged
   RERUN16 runs at the precision kept[i] only (16 when kept is NULL): the
   least work that gives the rerun contract's outputs, and never an 8-bit
   traceback that would read unwritten scratch. */
static double
run_bench (const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads,
           int64_t *checksum, const int8_t *kept, int32_t *out) {
  pthread_t *th;
  benchjob_t *jobs;
  struct timespec t0, t1;
  int t;
  int64_t sum = 0;
  if (!inited) ref_init(0);
  if (nthreads < 1) nthreads = 1;
  th = (pthread_t *) calloc(nthreads, sizeof(pthread_t));
  jobs = (benchjob_t *) calloc(nthreads, sizeof(benchjob_t));
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (t = 0; t < nthreads; t++) {
    jobs[t].pairs = pairs; jobs[t].arena = arena; jobs[t].npairs = npairs; jobs[t].kept = kept;
    jobs[t].tid = t; jobs[t].nthreads = nthreads; jobs[t].out = out;
    pthread_create(&th[t], NULL, bench_worker, &jobs[t]);
  }
  for (t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    sum += jobs[t].checksum;
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  free(th);
  free(jobs);
  if (checksum) *checksum = sum;
  return (double) (t1.tv_sec - t0.tv_sec) + 1e-9 * (double) (t1.tv_nsec - t0.tv_nsec);
}

double
ref_bench (const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads,
           int64_t *checksum, const int8_t *kept) {
  return run_bench(pairs, arena, npairs, nthreads, checksum, kept, NULL);
}

/* The same run, keeping per pair 8 words: the final score, the traceback
   score, nmatches, nmismatches, nopens, nindels, the record count and the
   records' digest (rec_digest; 0 without a traceback).  Returns wall
   seconds. */
double
ref_outputs (const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads, const int8_t *kept,
             int32_t *out) {
  return run_bench(pairs, arena, npairs, nthreads, NULL, kept, out);
}
