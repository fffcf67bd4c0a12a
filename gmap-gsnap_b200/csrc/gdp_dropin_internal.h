/* Internal interfaces between the runtime (runtime.cu) and its host layers:
   the reference-signature entry points (dropin.cu) and the single-gap
   batch (single_gap.cu).  Not part of the C ABI. */
#ifndef GDP_DROPIN_INTERNAL_H
#define GDP_DROPIN_INTERNAL_H
#include <vector>
#include <cuda_runtime.h>
#include "gdp_internal.h"

struct gdpi_fill;

/* A reusable single-pair fill: its device and host buffers only grow. */
gdpi_fill *gdpi_fill_new(void);
/* Fills one pair on the device and keeps its device state for a later
   traceback; the host receives the pair's direction words and the scores of
   every swept cell.  Blocks until the results are on the host. */
int gdpi_fill_run(gdp_ctx *ctx, gdpi_fill *f, const gdp_pair_t *p, const char *arena, int64_t arena_bytes);
const uint32_t *gdpi_fill_words(const gdpi_fill *f);
const int16_t *gdpi_fill_scores(const gdpi_fill *f);
int gdpi_fill_width(const gdpi_fill *f);       /* 16 or 32 (the kept precision's block height) */
int64_t gdpi_fill_base(const gdpi_fill *f);    /* first word of the pair in gdpi_fill_words */
const gdp_result_t *gdpi_fill_result(const gdpi_fill *f);
const gdp_pair_t *gdpi_fill_pair(const gdpi_fill *f);

/* Traces back the retained fill from p->tb_r, p->tb_c on the device; the
   genome window (genomecomp blocks starting at absolute position gbase,
   glen nt) serves short genome skips. */
int gdpi_traceback_one(gdp_ctx *ctx, gdpi_fill *f, const gdp_pair_t *p, const char *arena, int64_t arena_bytes,
                       const uint32_t *gblocks, const uint32_t *galtblocks, uint64_t gbase, uint64_t glen,
                       gdp_result_t *res, std::vector<gdp_rec_t> *recs);
void gdpi_fill_free(gdpi_fill *f);
int gdpi_set_tables(gdp_ctx *ctx, const gdp_tables_t *t);

/* The gap solvers' state in a context (single_gap.cu, end_gap.cu): the
   user penalties of Dynprog_single_setup and Dynprog_end_setup, and the
   single gap's working memory, kept between calls: grow-only device
   buffers, pinned host staging and one plan whose buffers are reused. */
struct gdp_plan;
struct gdpi_single_cfg {
  int user_open = 0, user_extend = 0;
  bool user_p = false;   /* user_dynprog_p */
  int end_open = 0, end_extend = 0;
  bool end_user_p = false;   /* Dynprog_end_setup's user_dynprog_p */
  static constexpr int NBUF = 24;
  void *dbuf[NBUF] = {};
  size_t dcap[NBUF] = {};
  void *hbuf[NBUF] = {};
  size_t hcap[NBUF] = {};
  gdp_plan *plan = nullptr;
  gdp_plan *dump_plan = nullptr;   /* plans whose fills also dump their scores (cdna_gap.cu) */
};
/* Plans pairs[0..n) into *plan (created on first use; its host and device
   buffers only grow) and uploads the plan on the context stream. */
int gdpi_plan_reuse(gdp_ctx *ctx, gdp_plan **plan, const gdp_pair_t *pairs, int64_t n);
/* As gdpi_plan_reuse, and the plan's fills also write the score of every
   swept cell, in the direction words' block-column layout (the score of
   lane l of the word-column at word offset w is at w * 8 + l); after
   gdp_plan_execute, gdpi_plan_scores and gdpi_plan_meta (each pair's word
   offsets, dir16 / dir8) point at them on the device until the plan's next
   use.  The plan must not be used for pairs that need no scores: its fills
   keep dumping. */
int gdpi_plan_reuse_dump(gdp_ctx *ctx, gdp_plan **plan, const gdp_pair_t *pairs, int64_t n);
const int16_t *gdpi_plan_scores(const gdp_plan *plan);
const gdp_meta_t *gdpi_plan_meta(const gdp_plan *plan);
void gdpi_single_release(gdpi_single_cfg *c);
struct gdpi_view {
  int device;
  cudaStream_t stream;
  const gdp_tables_t *d_tab;
  const uint32_t *d_genome, *d_genomealt;   /* d_genomealt == d_genome without an alternate genome */
  bool has_alt;
  uint64_t genome_len;
  int64_t budget;                           /* direction bytes per plan */
  int nsm;
  gdpi_single_cfg *single;
};
int gdpi_view_of(gdp_ctx *ctx, gdpi_view *v);
void gdpi_count_launch(gdp_ctx *ctx);
int gdpi_fail(gdp_ctx *ctx, const char *what, cudaError_t e);
#endif
