/*
 * ref_end.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Runs the reference's own Dynprog_end5_gap and Dynprog_end3_gap
 * (src/dynprog_end.c:1293-1650, :1923-2245, compiled from the reference
 * sources into oracle/_ref/ by oracle/Makefile) over a batch of end gaps,
 * for the parity tests of gdp_end_gap_batch.  Their genome segments come
 * from the Genome_get_segment_right / _left restatement of ref_single.c over
 * the harness's synthetic genome.
 *
 * src/dynprog_end.c also holds the splice-junction and known-splice end
 * solvers, which reference Pair_protect_end5/3, Splicetrie_solve_end5/3 and
 * Genome_fill_buffer_blocks_noterm; the two end-gap solvers never call
 * them, so they are stubs that abort.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>

#include "dynprog.h"
#include "dynprog_end.h"
#include "pairpool.h"
#include "pairdef.h"
#include "list.h"
#include "genome.h"
#include "pair.h"

#include "gdp.h"

List_T Pair_protect_end5 (List_T pairs) {
  (void) pairs;
  fprintf(stderr, "ref_end: Pair_protect_end5 is not linked\n");
  abort();
}
List_T Pair_protect_end3 (List_T pairs) {
  (void) pairs;
  fprintf(stderr, "ref_end: Pair_protect_end3 is not linked\n");
  abort();
}
void Splicetrie_solve_end5 (void) { fprintf(stderr, "ref_end: Splicetrie_solve_end5 is not linked\n"); abort(); }
void Splicetrie_solve_end3 (void) { fprintf(stderr, "ref_end: Splicetrie_solve_end3 is not linked\n"); abort(); }
void Genome_fill_buffer_blocks_noterm (Genome_T genome, Genome_T genomealt, Univcoord_T left, Chrpos_T length,
                                       char *gbuffer1, char *gbuffer2) {
  (void) genome; (void) genomealt; (void) left; (void) length; (void) gbuffer1; (void) gbuffer2;
  fprintf(stderr, "ref_end: Genome_fill_buffer_blocks_noterm is not linked\n");
  abort();
}

/* the harness's synthetic genome (ref_harness.c) */
extern Genome_T ref_genome_main (void);
extern Genome_T ref_genome_alt (void);

static Dynprog_T end_dynprog = NULL;
static Pairpool_T end_pool = NULL;

/* A Dynprog_T for the end gaps (Dynprog_new, src/dynprog.c:606-626); its
   max_rlength / max_glength come back for the gaps' length cuts. */
void
ref_end_init (int maxlookback, int extraquerygap, int *max_rlength, int *max_glength) {
  if (end_dynprog) Dynprog_free(&end_dynprog);
  if (end_pool == NULL) end_pool = Pairpool_new();
  end_dynprog = Dynprog_new(maxlookback, extraquerygap, 0, 0, 0, /*doublep*/true);
  *max_rlength = end_dynprog->max_rlength;
  *max_glength = end_dynprog->max_glength;
}

void
ref_end_setup (int user_open, int user_extend, int user_dynprog_p) {
  Dynprog_end_setup(NULL, NULL, NULL, 0, NULL, NULL, NULL, NULL, user_open, user_extend, user_dynprog_p != 0);
}

/*
 * Dynprog_end5_gap / Dynprog_end3_gap per gap.  stats[8*i ..]:
 * traceback_score, nmatches, nmismatches, nopens, nindels, number of pairs,
 * 1 when the List is NULL, dynprogindex after the call.  Records: the
 * returned List head first, gap i's at rec_off[i] (gap holders: comp '\0',
 * genomepos = genomejump).
 */
int64_t
ref_end_gap_batch (const gdp_end_gap_t *gaps, int n, const char *arena, int32_t *stats, gdp_rec_t *recs,
                   int64_t max_recs, int64_t *rec_off) {
  int64_t used = 0;
  int i;
  for (i = 0; i < n; i++) {
    const gdp_end_gap_t *g = &gaps[i];
    int dpi = g->dynprogindex, score = 0, nmatches = 0, nmismatches = 0, nopens = 0, nindels = 0, k = 0;
    List_T pairs, q;
    Pairpool_reset(end_pool);
    if (g->end == 5) {
      pairs = Dynprog_end5_gap(&dpi, &score, &nmatches, &nmismatches, &nopens, &nindels, end_dynprog,
                               (char *) arena + g->rseq, (char *) arena + g->rseq_uc, g->rlength, g->glength,
                               g->roffset, g->goffset, (Univcoord_T) g->chroffset, (Univcoord_T) g->chrhigh,
                               g->watsonp != 0, g->genestrand, g->jump_late_p != 0, ref_genome_main(),
                               ref_genome_alt(), end_pool, g->extraband_end, g->defect_rate,
                               (Endalign_T) g->endalign, g->require_pos_score_p != 0);
    } else {
      pairs = Dynprog_end3_gap(&dpi, &score, &nmatches, &nmismatches, &nopens, &nindels, end_dynprog,
                               (char *) arena + g->rseq, (char *) arena + g->rseq_uc, g->rlength, g->glength,
                               g->roffset, g->goffset, (Univcoord_T) g->chroffset, (Univcoord_T) g->chrhigh,
                               g->watsonp != 0, g->genestrand, g->jump_late_p != 0, ref_genome_main(),
                               ref_genome_alt(), end_pool, g->extraband_end, g->defect_rate,
                               (Endalign_T) g->endalign, g->require_pos_score_p != 0);
    }
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
/* CPU baseline: the end-gap solvers over a batch, one pthread per core */
/* ------------------------------------------------------------------ */

typedef struct {
  const gdp_end_gap_t *gaps;
  const char *arena;
  int n, tid, nthreads, maxlookback, extraquerygap;
  int64_t checksum;
} endjob_t;

static void *
end_worker (void *arg) {
  endjob_t *j = (endjob_t *) arg;
  /* each thread owns its Dynprog_T and Pairpool_T, as each GMAP worker
     thread does */
  Dynprog_T dp = Dynprog_new(j->maxlookback, j->extraquerygap, 0, 0, 0, /*doublep*/true);
  Pairpool_T pool = Pairpool_new();
  int64_t sum = 0;
  int i;
  for (i = j->tid; i < j->n; i += j->nthreads) {
    const gdp_end_gap_t *g = &j->gaps[i];
    int dpi = g->dynprogindex, score = 0, nmatches = 0, nmismatches = 0, nopens = 0, nindels = 0;
    List_T pairs;
    Pairpool_reset(pool);
    if (g->end == 5) {
      pairs = Dynprog_end5_gap(&dpi, &score, &nmatches, &nmismatches, &nopens, &nindels, dp,
                               (char *) j->arena + g->rseq, (char *) j->arena + g->rseq_uc, g->rlength,
                               g->glength, g->roffset, g->goffset, (Univcoord_T) g->chroffset,
                               (Univcoord_T) g->chrhigh, g->watsonp != 0, g->genestrand, g->jump_late_p != 0,
                               ref_genome_main(), ref_genome_alt(), pool, g->extraband_end, g->defect_rate,
                               (Endalign_T) g->endalign, g->require_pos_score_p != 0);
    } else {
      pairs = Dynprog_end3_gap(&dpi, &score, &nmatches, &nmismatches, &nopens, &nindels, dp,
                               (char *) j->arena + g->rseq, (char *) j->arena + g->rseq_uc, g->rlength,
                               g->glength, g->roffset, g->goffset, (Univcoord_T) g->chroffset,
                               (Univcoord_T) g->chrhigh, g->watsonp != 0, g->genestrand, g->jump_late_p != 0,
                               ref_genome_main(), ref_genome_alt(), pool, g->extraband_end, g->defect_rate,
                               (Endalign_T) g->endalign, g->require_pos_score_p != 0);
    }
    sum += score + List_length(pairs);
  }
  Pairpool_free(&pool);
  Dynprog_free(&dp);
  j->checksum = sum;
  return NULL;
}

/* The end-gap solver of every gap once, on nthreads threads (static
   round-robin); returns wall seconds and a checksum of the traceback
   scores and list lengths.  The user penalties of ref_end_setup apply. */
double
ref_end_gap_bench (const gdp_end_gap_t *gaps, int n, const char *arena, int nthreads, int maxlookback,
                   int extraquerygap, int64_t *checksum) {
  pthread_t *th;
  endjob_t *jobs;
  struct timespec t0, t1;
  int64_t sum = 0;
  int t;
  if (nthreads < 1) nthreads = 1;
  th = (pthread_t *) calloc(nthreads, sizeof(pthread_t));
  jobs = (endjob_t *) calloc(nthreads, sizeof(endjob_t));
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (t = 0; t < nthreads; t++) {
    jobs[t].gaps = gaps; jobs[t].arena = arena; jobs[t].n = n; jobs[t].tid = t; jobs[t].nthreads = nthreads;
    jobs[t].maxlookback = maxlookback; jobs[t].extraquerygap = extraquerygap;
    pthread_create(&th[t], NULL, end_worker, &jobs[t]);
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
