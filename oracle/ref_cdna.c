/*
 * ref_cdna.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Runs the reference's own Dynprog_cdna_gap (src/dynprog_cdna.c:786-1290,
 * compiled from the reference sources into oracle/_ref/ by oracle/Makefile)
 * over a batch of cDNA gaps, for the parity tests of gdp_cdna_gap_batch.
 * Its genome segments come from the Genome_get_segment_right / _left
 * restatement of ref_single.c over the harness's synthetic genome.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>

#include "dynprog.h"
#include "dynprog_cdna.h"
#include "pairpool.h"
#include "pairdef.h"
#include "list.h"
#include "genome.h"

#include "gdp.h"

/* the harness's synthetic genome (ref_harness.c) */
extern Genome_T ref_genome_main (void);
extern Genome_T ref_genome_alt (void);

static Dynprog_T cdna_dynprogL = NULL, cdna_dynprogR = NULL;
static Pairpool_T cdna_pool = NULL;

/* Two Dynprog_T for the gaps' left and right fills (Dynprog_new,
   src/dynprog.c:606-626); their max_rlength / max_glength come back for
   the gaps' length checks. */
void
ref_cdna_init (int maxlookback, int extraquerygap, int *max_rlength, int *max_glength) {
  if (cdna_dynprogL) Dynprog_free(&cdna_dynprogL);
  if (cdna_dynprogR) Dynprog_free(&cdna_dynprogR);
  if (cdna_pool == NULL) cdna_pool = Pairpool_new();
  cdna_dynprogL = Dynprog_new(maxlookback, extraquerygap, 0, 0, 0, /*doublep*/true);
  cdna_dynprogR = Dynprog_new(maxlookback, extraquerygap, 0, 0, 0, /*doublep*/true);
  *max_rlength = cdna_dynprogL->max_rlength;
  *max_glength = cdna_dynprogL->max_glength;
}

/*
 * Dynprog_cdna_gap per gap.  stats[8*i ..]: traceback_score, incompletep,
 * 0, 0, 0, number of pairs, 1 when the List is NULL, dynprogindex after
 * the call.  Records: the returned List head first, gap i's at rec_off[i]
 * (gap holders: comp '\0', querypos = -1 - queryjump, genomepos =
 * genomejump).
 */
int64_t
ref_cdna_gap_batch (const gdp_cdna_gap_t *gaps, int n, const char *arena, int32_t *stats, gdp_rec_t *recs,
                    int64_t max_recs, int64_t *rec_off) {
  int64_t used = 0;
  int i;
  for (i = 0; i < n; i++) {
    const gdp_cdna_gap_t *g = &gaps[i];
    int dpi = g->dynprogindex, score = 0, k = 0;
    bool incomplete = false;
    List_T pairs, q;
    char *rs = (char *) arena + g->rseq, *ru = (char *) arena + g->rseq_uc;
    const int to_r = g->rev_roffsetR - g->roffsetL;
    Pairpool_reset(cdna_pool);
    pairs = Dynprog_cdna_gap(&dpi, &score, &incomplete, cdna_dynprogL, cdna_dynprogR, rs, ru, rs + to_r, ru + to_r,
                             g->rlengthL, g->rlengthR, g->glength, g->roffsetL, g->rev_roffsetR, g->goffset,
                             (Univcoord_T) g->chroffset, (Univcoord_T) g->chrhigh, g->watsonp != 0, g->genestrand,
                             g->jump_late_p != 0, ref_genome_main(), ref_genome_alt(), cdna_pool,
                             g->extraband_paired, g->defect_rate);
    rec_off[i] = used;
    for (q = pairs; q != NULL; q = q->rest, k++) {
      Pair_T pr = (Pair_T) q->first;
      if (used + k < max_recs) {
        gdp_rec_t *d = &recs[used + k];
        d->querypos = pr->gapp ? -1 - pr->queryjump : pr->querypos;
        d->genomepos = pr->gapp ? pr->genomejump : (int32_t) pr->genomepos;
        d->cdna = pr->gapp ? ' ' : pr->cdna;
        d->comp = pr->gapp ? '\0' : pr->comp;
        d->genome = pr->gapp ? ' ' : pr->genome;
        d->genomealt = pr->gapp ? ' ' : pr->genomealt;
      }
    }
    stats[8 * i + 0] = score;
    stats[8 * i + 1] = incomplete ? 1 : 0;
    stats[8 * i + 2] = stats[8 * i + 3] = stats[8 * i + 4] = 0;
    stats[8 * i + 5] = k;
    stats[8 * i + 6] = pairs == NULL;
    stats[8 * i + 7] = dpi;
    used += k;
  }
  return used;
}

/* ------------------------------------------------------------------ */
/* CPU baseline: Dynprog_cdna_gap over a batch, one pthread per core    */
/* ------------------------------------------------------------------ */

typedef struct {
  const gdp_cdna_gap_t *gaps;
  const char *arena;
  int n, tid, nthreads, maxlookback, extraquerygap;
  int64_t checksum;
} cdnajob_t;

static void *
cdna_worker (void *arg) {
  cdnajob_t *j = (cdnajob_t *) arg;
  /* each thread owns its Dynprog_T pair and Pairpool_T, as each GMAP
     worker thread does */
  Dynprog_T dl = Dynprog_new(j->maxlookback, j->extraquerygap, 0, 0, 0, /*doublep*/true);
  Dynprog_T dr = Dynprog_new(j->maxlookback, j->extraquerygap, 0, 0, 0, /*doublep*/true);
  Pairpool_T pool = Pairpool_new();
  int64_t sum = 0;
  int i;
  for (i = j->tid; i < j->n; i += j->nthreads) {
    const gdp_cdna_gap_t *g = &j->gaps[i];
    int dpi = g->dynprogindex, score = 0;
    bool incomplete = false;
    List_T pairs;
    char *rs = (char *) j->arena + g->rseq, *ru = (char *) j->arena + g->rseq_uc;
    const int to_r = g->rev_roffsetR - g->roffsetL;
    Pairpool_reset(pool);
    pairs = Dynprog_cdna_gap(&dpi, &score, &incomplete, dl, dr, rs, ru, rs + to_r, ru + to_r, g->rlengthL,
                             g->rlengthR, g->glength, g->roffsetL, g->rev_roffsetR, g->goffset,
                             (Univcoord_T) g->chroffset, (Univcoord_T) g->chrhigh, g->watsonp != 0, g->genestrand,
                             g->jump_late_p != 0, ref_genome_main(), ref_genome_alt(), pool, g->extraband_paired,
                             g->defect_rate);
    sum += score + List_length(pairs);
  }
  Pairpool_free(&pool);
  Dynprog_free(&dr);
  Dynprog_free(&dl);
  j->checksum = sum;
  return NULL;
}

/* Dynprog_cdna_gap for every gap once, on nthreads threads (static
   round-robin); returns wall seconds and a checksum of the traceback
   scores and list lengths. */
double
ref_cdna_gap_bench (const gdp_cdna_gap_t *gaps, int n, const char *arena, int nthreads, int maxlookback,
                    int extraquerygap, int64_t *checksum) {
  pthread_t *th;
  cdnajob_t *jobs;
  struct timespec t0, t1;
  int64_t sum = 0;
  int t;
  if (nthreads < 1) nthreads = 1;
  th = (pthread_t *) calloc(nthreads, sizeof(pthread_t));
  jobs = (cdnajob_t *) calloc(nthreads, sizeof(cdnajob_t));
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (t = 0; t < nthreads; t++) {
    jobs[t].gaps = gaps; jobs[t].arena = arena; jobs[t].n = n; jobs[t].tid = t; jobs[t].nthreads = nthreads;
    jobs[t].maxlookback = maxlookback; jobs[t].extraquerygap = extraquerygap;
    pthread_create(&th[t], NULL, cdna_worker, &jobs[t]);
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
