/* gdp_oracle.h -- TEST INFRASTRUCTURE ONLY: the CPU restatement of the
   reference's dynamic-programming fills and tracebacks (gdp_oracle.c).
   Same entry points as oracle/ref_harness.c with the prefix orc_. */
#ifndef GDP_ORACLE_H
#define GDP_ORACLE_H
#include <stdint.h>
#include "gdp.h"

void orc_init(int mode);
int orc_pairdistance(int mismatchtype, int c1, int c2);
int orc_consistent(int genestrand, int c1, int c2);
void orc_set_genome(const uint32_t *blocks, const uint32_t *altblocks, uint64_t genomelength);
int orc_align(const gdp_pair_t *p, const char *arena,
              int16_t *H, int8_t *dN, int8_t *dE, int8_t *dF, int32_t *final_score,
              int32_t *tb_stats, gdp_rec_t *recs, int max_recs);
int orc_last_tb_outside(void);
int orc_last_tb_stale(void);
double orc_bench(const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads,
                 int64_t *checksum, const int8_t *kept);
void orc_kept_precision(const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads,
                        int8_t *kept);
#endif
