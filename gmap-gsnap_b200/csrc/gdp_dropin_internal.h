/* Internal single-pair interface between the runtime (runtime.cu) and the
   reference-signature entry points (dropin.cu).  Not part of the C ABI. */
#ifndef GDP_DROPIN_INTERNAL_H
#define GDP_DROPIN_INTERNAL_H
#include <vector>
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
#endif
