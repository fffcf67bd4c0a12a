/*
 * genome_chars.cuh -- genome characters on the device, from the resident
 * genome in the reference's genomecomp format (three uint32 per 32 nt:
 * high, low, N-flags; src/genome.c:9723-9792).
 */
#pragma once
#include "gdp_internal.h"

__device__ __forceinline__ char
gnt_decode (const uint32_t *b, uint32_t pos, bool flags) {
  const uint32_t ptr = pos / 32u * 3u;
  const int bit = (int) (pos % 32u);
  if (flags && (__ldg(b + ptr + 2) & (1u << bit))) return 'N';
  const uint32_t w = (bit < 16) ? __ldg(b + ptr + 1) : __ldg(b + ptr);
  const int code = (int) ((w >> ((bit < 16) ? 2 * bit : 2 * bit - 32)) & 3u);
  return "ACGT"[code];
}

__device__ __forceinline__ char
gnt_compl (char c) {
  return c == 'A' ? 'T' : c == 'C' ? 'G' : c == 'G' ? 'C' : c == 'T' ? 'A' : c;
}

/*
 * Genome character at genomic coordinate gp of a pair, as get_genomic_nt
 * reads it (src/pairpool.c:1015-1063): chroffset + gp on the plus strand,
 * the complement of chrhigh - gp on the minus strand, '*' outside
 * [chroffset, chrhigh); 32-bit unsigned coordinates.  `genome` holds
 * genomecomp blocks starting at absolute position `base` and covering `len`
 * nt.  Returns 0 when the position lies outside those blocks.
 */
__device__ __forceinline__ char
genomic_char (const gdp_pair_t &p, int gp, const uint32_t *genome, const uint32_t *genomealt, uint64_t base,
              uint64_t len, char *alt) {
  const uint32_t pos = p.watsonp ? p.chroffset + (uint32_t) gp : p.chrhigh - (uint32_t) gp;
  if (pos < p.chroffset || pos >= p.chrhigh) { *alt = '*'; return '*'; }
  if (genome == nullptr || pos < base || pos - base >= len) { *alt = 'N'; return 0; }
  const uint32_t rp = (uint32_t) (pos - base);
  const char c = gnt_decode(genome, rp, true);
  const char ca = (c == 'N') ? c : gnt_decode(genomealt, rp, false);
  if (p.watsonp) { *alt = ca; return c; }
  *alt = gnt_compl(ca);
  return gnt_compl(c);
}

/*
 * The character Dynprog_single_gap's gsequence holds for genomic coordinate
 * gp (GDP_XFLAG_SEGMENT): Genome_get_segment_right on the plus strand ('*'
 * at and above chrhigh), the reverse complement of Genome_get_segment_left
 * on the minus strand ('*' below chroffset), src/genome.c:11022-11120; with
 * GDP_XFLAG_SEGMENT_REV the mirrored segment Dynprog_end5_gap reads
 * (segment_left on the plus strand, '*' below chroffset; the reverse
 * complement of segment_right on the minus strand, '*' at and above
 * chrhigh).  The positions it reads must be resident (the planner checks).
 */
__device__ __forceinline__ char
segment_char (const gdp_pair_t &p, int gp, const uint32_t *genome, const uint32_t *genomealt, uint64_t len,
              char *alt) {
  const int64_t pos = p.watsonp ? (int64_t) p.chroffset + gp : (int64_t) p.chrhigh - gp;
  const bool rev = (p.xflags & GDP_XFLAG_SEGMENT_REV) != 0;
  const bool below = pos < (int64_t) p.chroffset, above = pos >= (int64_t) p.chrhigh;
  if (p.watsonp ? (rev ? below : above) : (rev ? above : below)) { *alt = '*'; return '*'; }
  if (genome == nullptr || pos < 0 || (uint64_t) pos >= len) { *alt = 'N'; return 'N'; }
  const uint32_t rp = (uint32_t) pos;
  const char c = gnt_decode(genome, rp, true);
  const char ca = (c == 'N') ? c : gnt_decode(genomealt, rp, false);
  if (p.watsonp) { *alt = ca; return c; }
  *alt = gnt_compl(ca);
  return gnt_compl(c);
}
