/*
 * gdp_internal.h -- data shared by the host runtime and the CUDA kernels.
 *
 * Direction storage ("block-column words").  The reference fills a matrix
 * in blocks of W lanes (W = 16 for 16-bit, 32 for 8-bit AVX2 lanes,
 * src/dynprog.h:127-132), sweeping for each block a range of columns
 * (src/dynprog_simd.c:3216-3256, :4484, :5558, :6762-6802, :7872, :8776).
 * Its traceback can read any cell such a sweep wrote -- including the
 * below-band cells of a block (src/dynprog_simd.c:9174 walks one column
 * past the band edge) -- so the device keeps every swept cell: for block b
 * and swept column y, W/8 consecutive uint32 words with
 *     bits  0..7   nogap == HORIZ   (set by the vector step)
 *     bits  8..15  nogap == VERT    (set by the F loop; overrides HORIZ)
 *     bits 16..23  Egap  != DIAG
 *     bits 24..31  Fgap  == VERT
 * 4 bits per cell.  Which word and which bit of each byte hold lane i
 * (gdp_dir_word, gdp_dir_bit): for W = 16, word i % 2, bit i / 2 (the
 * even lanes in word 0, the odd lanes in word 1, as the packed two-lane
 * fill produces them); for W = 32, word i / 8, bit i % 8.  Blocks are
 * stored one after another; block b starts at the sum of the sizes of
 * blocks 0..b-1.  "Lanes" are query rows for the full and upper fills and
 * genome columns for the lower fill (which the reference computes
 * transposed, src/dynprog_simd.c:8545-8558).
 */
#ifndef GDP_INTERNAL_H
#define GDP_INTERNAL_H

#include <stdint.h>
#include "gdp.h"

#ifdef __CUDACC__
#define GDP_HD __host__ __device__ __forceinline__
#else
#define GDP_HD static inline
#endif

#define GDP_NEGINT (-32768)   /* NEG_INFINITY_INT (src/dynprog.h:176) */
#define GDP_MICROINTRON 9     /* MICROINTRON_LENGTH (src/pairpool.c:18) */

/* Word (of the W/8 words of a block column) and bit (of each byte) of
   lane `lane`'s direction bits. */
GDP_HD int gdp_dir_word (int W, int lane) { return W == 16 ? (lane & 1) : (lane >> 3); }
GDP_HD int gdp_dir_bit (int W, int lane) { return W == 16 ? (lane >> 1) : (lane & 7); }

/* Substitution and consistency tables, built on the host as Dynprog_init
   does (src/dynprog.c:1007-1196) and copied to the device. */
typedef struct gdp_tables {
  int16_t pd[4][128][128];      /* pairdistance_array[mismatchtype][c1][c2] */
  uint8_t cons[3][128][128];    /* consistent_array[genestrand][c1][c2] */
  int8_t nt2int[128];           /* nt_to_int_array: A/C/G/T -> 0..3, else 4 */
  /* Packed 5-class profiles: bytes 0..4 = score against classes A,C,G,T,N. */
  uint32_t profq_lo[4][128], profq_hi[4][128];   /* pd[mt][q][ACGTN[k]]   (query lanes) */
  uint32_t profg_lo[4][128], profg_hi[4][128];   /* pd[mt][ACGTN[k]][g]   (genome lanes) */
} gdp_tables_t;

#ifdef __cplusplus
extern "C"
#endif
void gdp_build_tables(gdp_tables_t *t, int mode);
#ifdef __cplusplus
extern "C"
#endif
void gdp_tables_derive(gdp_tables_t *t);   /* class profiles from pd */
#ifdef __cplusplus
extern "C"
#endif
void gdp_workload_genomecomp(const char *genome, int64_t n, uint32_t *blocks);   /* workload.c */

/* Geometry of a pair in lane/sweep terms. */
typedef struct gdp_geom {
  int W;          /* block height: 16 (16-bit) or 32 (8-bit) */
  int X, Y;       /* lane dimension length, swept dimension length */
  int lband, uband;
  int band_hi;    /* how far beyond a block's last lane the sweep runs */
  int variant;
} gdp_geom_t;

GDP_HD void
gdp_geom_of (const gdp_pair_t *p, int W, gdp_geom_t *g) {
  g->W = W;
  g->variant = p->variant;
  g->lband = p->lband;
  g->uband = p->uband;
  if (p->variant == GDP_LOWER) {
    g->X = p->glength; g->Y = p->rlength; g->band_hi = p->lband;
  } else {
    g->X = p->rlength; g->Y = p->glength; g->band_hi = p->uband;
  }
}

/* First and last swept column of block xlo (possibly y1 < y0: nothing swept). */
GDP_HD void
gdp_block_sweep (const gdp_geom_t *g, int xlo, int *y0, int *y1) {
  int xhi = xlo + g->W - 1;
  if (xhi > g->X) xhi = g->X;
  if (g->variant == GDP_FULL) {
    *y0 = xlo - g->lband;
    if (*y0 < 0) *y0 = 0;
  } else {
    *y0 = xlo;
  }
  *y1 = xhi + g->band_hi;
  if (*y1 > g->Y) *y1 = g->Y;
}

GDP_HD int64_t
gdp_block_words (const gdp_geom_t *g, int xlo) {
  int y0, y1;
  gdp_block_sweep(g, xlo, &y0, &y1);
  return (y1 >= y0) ? (int64_t) (y1 - y0 + 1) * (g->W / 8) : 0;
}

/* Direction words of a whole pair at block height W. */
GDP_HD int64_t
gdp_pair_words (const gdp_pair_t *p, int W) {
  gdp_geom_t g;
  int64_t total = 0;
  int xlo;
  gdp_geom_of(p, W, &g);
  for (xlo = 0; xlo <= g.X; xlo += W) total += gdp_block_words(&g, xlo);
  return total;
}

/* Per-pair device metadata written by the planner. */
typedef struct gdp_meta {
  int64_t dir16;      /* word offset of the 16-bit layout (-1: none) */
  int64_t dir8;       /* word offset of the 8-bit layout (-1: none) */
  int32_t maxh16;     /* rerun pairs: >= 127 iff an in-band 16-bit score reached 127 */
  int32_t status8;    /* 8-bit pass: 0 = kept, 1 = overflowed (use 16-bit) */
  int32_t final8;     /* 8-bit final score */
  int32_t final16;    /* 16-bit final score (rerun pairs) */
} gdp_meta_t;

#endif
