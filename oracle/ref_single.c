/*
 * ref_single.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Runs the reference's own Dynprog_single_gap (src/dynprog_single.c:428-675,
 * compiled from the reference sources into oracle/_ref/ by oracle/Makefile)
 * over a batch of gaps, for the parity tests of gdp_single_gap_batch.
 *
 * src/dynprog_single.c reads its genome segment through
 * Genome_get_segment_right / _left (src/genome.c:11022-11120), which are not
 * among the linked reference files; they are restated below over the
 * harness's synthetic genome (ref_set_genome, genomecomp blocks): positions
 * at or above chrhigh (right) or below chroffset (left) read '*', the N
 * flags of the genome read 'N' in both segments, the alternate segment
 * decodes the alternate genome, and revcomp reverses and complements.
 * The same file's microexon searches reference BoyerMoore_nt and the
 * Maxent_hr_* splice-site models; the single gap never calls them, so they
 * are stubs that abort.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>

#include "dynprog.h"
#include "dynprog_single.h"
#include "pairpool.h"
#include "pairdef.h"
#include "list.h"
#include "genome.h"

#include "gdp.h"

void BoyerMoore_nt (void) { fprintf(stderr, "ref_single: BoyerMoore_nt is not linked\n"); abort(); }
void Maxent_hr_donor_prob (void) { fprintf(stderr, "ref_single: Maxent_hr is not linked\n"); abort(); }
void Maxent_hr_acceptor_prob (void) { fprintf(stderr, "ref_single: Maxent_hr is not linked\n"); abort(); }
void Maxent_hr_antidonor_prob (void) { fprintf(stderr, "ref_single: Maxent_hr is not linked\n"); abort(); }
void Maxent_hr_antiacceptor_prob (void) { fprintf(stderr, "ref_single: Maxent_hr is not linked\n"); abort(); }

/* the harness's synthetic genome (ref_harness.c) */
extern Genome_T ref_genome_main (void);
extern Genome_T ref_genome_alt (void);

static const char NT[4] = {'A', 'C', 'G', 'T'};

static char
nt_at (const Genomecomp_T *blocks, const Genomecomp_T *flagblocks, Univcoord_T pos) {
  const Genomecomp_T *b = blocks + pos / 32U * 3;
  const int bit = (int) (pos % 32U);
  if (flagblocks[pos / 32U * 3 + 2] & (1U << bit)) return 'N';
  return NT[(bit < 16 ? b[1] >> (2 * bit) : b[0] >> (2 * bit - 32)) & 3U];
}

static char
compl_nt (char c) {
  switch (c) {
  case 'A': return 'T';
  case 'C': return 'G';
  case 'G': return 'C';
  case 'T': return 'A';
  default: return c;   /* 'N' and '*' are their own complements */
  }
}

static void
reverse_complement (char *s, Chrpos_T length) {
  Chrpos_T i;
  for (i = 0; i < length / 2; i++) {
    char a = compl_nt(s[i]);
    s[i] = compl_nt(s[length - 1 - i]);
    s[length - 1 - i] = a;
  }
  if (length % 2 == 1) s[length / 2] = compl_nt(s[length / 2]);
}

/* segment[i] = the genome at first + i, '*' where first + i lies outside
   [lo_ok, hi_ok).  Positions are signed: the left segment of a window that
   starts before coordinate 0 (right < length) reads '*' there, as the
   reference's out_of_bounds count does. */
static void
fill_segment (char *segment, char *segmentalt, Genome_T genome, Genome_T genomealt, int64_t first,
              Chrpos_T length, int64_t lo_ok, int64_t hi_ok, bool revcomp) {
  Chrpos_T i;
  for (i = 0; i < length; i++) {
    const int64_t pos = first + (int64_t) i;
    if (pos < lo_ok || pos >= hi_ok) {
      segment[i] = segmentalt[i] = '*';
    } else {
      segment[i] = nt_at(genome->blocks, genome->blocks, (Univcoord_T) pos);
      segmentalt[i] = nt_at(genomealt->blocks, genome->blocks, (Univcoord_T) pos);
    }
  }
  segment[length] = segmentalt[length] = '\0';
  if (revcomp) {
    reverse_complement(segment, length);
    reverse_complement(segmentalt, length);
  }
}

void
Genome_get_segment_right (char *segment, char *segmentalt, Genome_T genome, Genome_T genomealt,
                          Univcoord_T left, Chrpos_T length, Univcoord_T chrhigh, bool revcomp) {
  if (length == 0) { segment[0] = segmentalt[0] = '\0'; return; }
  fill_segment(segment, segmentalt, genome, genomealt, (int64_t) left, length, 0, (int64_t) chrhigh, revcomp);
}

void
Genome_get_segment_left (char *segment, char *segmentalt, Genome_T genome, Genome_T genomealt,
                         Univcoord_T right, Chrpos_T length, Univcoord_T chroffset, bool revcomp) {
  if (length == 0) { segment[0] = segmentalt[0] = '\0'; return; }
  fill_segment(segment, segmentalt, genome, genomealt, (int64_t) right - (int64_t) length, length,
               (int64_t) chroffset, INT64_MAX, revcomp);
}

static Dynprog_T single_dynprog = NULL;
static Pairpool_T single_pool = NULL;

/* A Dynprog_T for the single gaps (Dynprog_new, src/dynprog.c:606-626);
   its max_rlength / max_glength come back for the gaps' range checks. */
void
ref_single_init (int maxlookback, int extraquerygap, int *max_rlength, int *max_glength) {
  if (single_dynprog) Dynprog_free(&single_dynprog);
  if (single_pool == NULL) single_pool = Pairpool_new();
  single_dynprog = Dynprog_new(maxlookback, extraquerygap, 0, 0, 0, /*doublep*/false);
  *max_rlength = single_dynprog->max_rlength;
  *max_glength = single_dynprog->max_glength;
}

void
ref_single_setup (int user_open, int user_extend, int user_dynprog_p) {
  Dynprog_single_setup(user_open, user_extend, user_dynprog_p != 0, /*homopolymerp*/false);
}

/*
 * Dynprog_single_gap per gap.  stats[8*i ..]: traceback_score, nmatches,
 * nmismatches, nopens, nindels, number of pairs, 1 when the List is NULL,
 * dynprogindex after the call.  Records: the returned List head first, gap
 * i's at rec_off[i] (gap holders: comp '\0', genomepos = genomejump).
 */
int64_t
ref_single_gap_batch (const gdp_single_gap_t *gaps, int n, const char *arena, int32_t *stats, gdp_rec_t *recs,
                      int64_t max_recs, int64_t *rec_off) {
  int64_t used = 0;
  int i;
  for (i = 0; i < n; i++) {
    const gdp_single_gap_t *g = &gaps[i];
    int dpi = g->dynprogindex, score = 0, nmatches = 0, nmismatches = 0, nopens = 0, nindels = 0, k = 0;
    List_T pairs, q;
    Pairpool_reset(single_pool);
    pairs = Dynprog_single_gap(&dpi, &score, &nmatches, &nmismatches, &nopens, &nindels, single_dynprog,
                               (char *) arena + g->rseq, (char *) arena + g->rseq_uc, g->rlength, g->glength,
                               g->roffset, g->goffset, (Univcoord_T) g->chroffset, (Univcoord_T) g->chrhigh,
                               g->watsonp != 0, g->genestrand, g->jump_late_p != 0, ref_genome_main(),
                               ref_genome_alt(), single_pool, g->extraband_single, g->widebandp != 0,
                               g->defect_rate);
    rec_off[i] = used;
    for (q = pairs; q != NULL; q = q->rest, k++) {
      Pair_T pr = (Pair_T) q->first;
      if (used + k < max_recs) {
        gdp_rec_t *d = &recs[used + k];
        d->querypos = pr->querypos;
        d->genomepos = pr->gapp ? pr->genomejump : (int32_t) pr->genomepos;
        d->cdna = pr->cdna;
        d->comp = pr->gapp ? '\0' : pr->comp;
        d->genome = pr->genome;
        d->genomealt = pr->genomealt;
      }
    }
    stats[8 * i + 0] = score;
    stats[8 * i + 1] = nmatches;
    stats[8 * i + 2] = nmismatches;
    stats[8 * i + 3] = nopens;
    stats[8 * i + 4] = nindels;
    stats[8 * i + 5] = k;
    stats[8 * i + 6] = pairs == NULL;
    stats[8 * i + 7] = dpi;
    used += k;
  }
  return used;
}

/* ------------------------------------------------------------------ */
/* CPU baseline: Dynprog_single_gap over a batch, one pthread per core   */
/* ------------------------------------------------------------------ */

typedef struct {
  const gdp_single_gap_t *gaps;
  const char *arena;
  int n, tid, nthreads, maxlookback, extraquerygap;
  int64_t checksum;
} singlejob_t;

static void *
single_worker (void *arg) {
  singlejob_t *j = (singlejob_t *) arg;
  /* each thread owns its Dynprog_T and Pairpool_T, as each GMAP worker
     thread does (src/gmap.c:4907-4911) */
  Dynprog_T dp = Dynprog_new(j->maxlookback, j->extraquerygap, 0, 0, 0, /*doublep*/false);
  Pairpool_T pool = Pairpool_new();
  int64_t sum = 0;
  int i;
  for (i = j->tid; i < j->n; i += j->nthreads) {
    const gdp_single_gap_t *g = &j->gaps[i];
    int dpi = g->dynprogindex, score = 0, nmatches = 0, nmismatches = 0, nopens = 0, nindels = 0;
    List_T pairs;
    Pairpool_reset(pool);
    pairs = Dynprog_single_gap(&dpi, &score, &nmatches, &nmismatches, &nopens, &nindels, dp,
                               (char *) j->arena + g->rseq, (char *) j->arena + g->rseq_uc, g->rlength,
                               g->glength, g->roffset, g->goffset, (Univcoord_T) g->chroffset,
                               (Univcoord_T) g->chrhigh, g->watsonp != 0, g->genestrand, g->jump_late_p != 0,
                               ref_genome_main(), ref_genome_alt(), pool, g->extraband_single,
                               g->widebandp != 0, g->defect_rate);
    sum += score + List_length(pairs);
  }
  Pairpool_free(&pool);
  Dynprog_free(&dp);
  j->checksum = sum;
  return NULL;
}

/* Dynprog_single_gap for every gap once, on nthreads threads (static
   round-robin); returns wall seconds and a checksum of the traceback
   scores and list lengths.  The user penalties of ref_single_setup
   apply. */
double
ref_single_gap_bench (const gdp_single_gap_t *gaps, int n, const char *arena, int nthreads, int maxlookback,
                      int extraquerygap, int64_t *checksum) {
  pthread_t *th;
  singlejob_t *jobs;
  struct timespec t0, t1;
  int64_t sum = 0;
  int t;
  if (nthreads < 1) nthreads = 1;
  th = (pthread_t *) calloc(nthreads, sizeof(pthread_t));
  jobs = (singlejob_t *) calloc(nthreads, sizeof(singlejob_t));
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (t = 0; t < nthreads; t++) {
    jobs[t].gaps = gaps; jobs[t].arena = arena; jobs[t].n = n; jobs[t].tid = t; jobs[t].nthreads = nthreads;
    jobs[t].maxlookback = maxlookback; jobs[t].extraquerygap = extraquerygap;
    pthread_create(&th[t], NULL, single_worker, &jobs[t]);
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
