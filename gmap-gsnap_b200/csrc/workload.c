/*
 * workload.c -- seeded synthetic alignment workloads for tests and
 * benchmarks (not on the alignment path).
 *
 * No public dataset is named for this path, so every benchmark input is
 * synthetic: a uniform-ACGT random genome (xoshiro256** seeded), reads drawn
 * from random genome positions, and genome windows derived from them with
 * substitutions and indels.  Shapes follow the workload definitions:
 *   short   rlength U{75..300}, lband/uband U{3..30}, 3% subs, 1% indels,
 *           5% random non-matching windows (8-bit with 16-bit rerun)
 *   fixed   rlength 150, glength 160, lband = uband = 10, 2% subs,
 *           0.5% indels of length U{1..3} (16-bit)
 *   long    rlength U{1000..10000}, lband/uband U{50..200}, 3% subs,
 *           1% indels (16-bit)
 *   cdna    rlength log-U[200, 5000], glength = rlength * U(1.0, 1.5),
 *           1% subs, 2% indels of geometric length (mean 4); an upper fill
 *           with uband = glength - rlength + 14 (src/dynprog.c:1246-1261
 *           wideband with extraband_paired = 14, src/gmap.c:292) traced back
 *           from (rlength, glength), followed by the lower fill of the same
 *           sequences with lband = 14 and no traceback, as a cDNA gap fills
 *           both halves (src/dynprog_cdna.c:944-1098); the lower fill takes
 *           the next slot of the batch
 * Gap penalties default to HIGHQ open -8 / extend -3 (src/dynprog.h:61-65).
 * Draws alternate the tie rule: even draws jump late, odd draws jump early
 * (jump_late_p), so both fills of every kind are exercised.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "gdp.h"

typedef struct { uint64_t s[4]; } rng_t;

static inline uint64_t rotl (uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t
rng_next (rng_t *r) {
  uint64_t *s = r->s;
  uint64_t result = rotl(s[1] * 5, 7) * 9;
  uint64_t t = s[1] << 17;
  s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
  s[2] ^= t; s[3] = rotl(s[3], 45);
  return result;
}

static void
rng_seed (rng_t *r, uint64_t seed) {
  /* splitmix64 expansion */
  int i;
  for (i = 0; i < 4; i++) {
    uint64_t z = (seed += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    r->s[i] = z ^ (z >> 31);
  }
}

static inline double rng_unif (rng_t *r) { return (double) (rng_next(r) >> 11) * 0x1.0p-53; }
static inline int rng_int (rng_t *r, int lo, int hi) {  /* inclusive */
  return lo + (int) (rng_next(r) % (uint64_t) (hi - lo + 1));
}

static const char NT[4] = {'A', 'C', 'G', 'T'};

/* Fills `genome` (length n) with uniform ACGT. */
void
gdp_workload_genome (uint64_t seed, char *genome, int64_t n) {
  rng_t r;
  int64_t i;
  rng_seed(&r, seed);
  for (i = 0; i + 32 <= n; i += 32) {
    uint64_t x = rng_next(&r);
    int k;
    for (k = 0; k < 32; k++) { genome[i + k] = NT[x & 3]; x >>= 2; }
  }
  for (; i < n; i++) genome[i] = NT[rng_next(&r) & 3];
}

/*
 * Encodes a character genome into the reference's genomecomp blocks
 * (src/genome.c:9723-9763): for each 32-nt word three uint32 {high, low,
 * flags}; nt k (0..15) in bits 2k of low, nt 16+k in bits 2k of high, and
 * flag bit k set (character 'N') for anything that is not A/C/G/T.
 * `blocks` must hold 3 * ceil(n / 32) words.
 */
void
gdp_workload_genomecomp (const char *genome, int64_t n, uint32_t *blocks) {
  int64_t w, nwords = (n + 31) / 32;
  for (w = 0; w < nwords; w++) {
    uint32_t high = 0, low = 0, flags = 0;
    int k;
    for (k = 0; k < 32; k++) {
      int64_t i = w * 32 + k;
      int code = 0, isn = 0;
      if (i < n) {
        switch (genome[i]) {
        case 'A': case 'a': code = 0; break;
        case 'C': case 'c': code = 1; break;
        case 'G': case 'g': code = 2; break;
        case 'T': case 't': code = 3; break;
        default: isn = 1; code = 0;
        }
      }
      if (k < 16) low |= (uint32_t) code << (2 * k);
      else high |= (uint32_t) code << (2 * (k - 16));
      if (isn) flags |= 1U << k;
    }
    blocks[3 * w] = high;
    blocks[3 * w + 1] = low;
    blocks[3 * w + 2] = flags;
  }
}

/* Workload kinds */
enum { WL_FIXED = 1, WL_SHORT = 2, WL_CDNA = 3, WL_LONG = 5 };

typedef struct {
  double sub, indel;      /* per-base rates */
  int geom_mean;          /* >0: indel length geometric with this mean, else U{1..3} */
} mut_t;

/* Copies src (n) into dst with mutations; returns the output length (<= cap). */
static int
mutate (rng_t *r, const char *src, int n, char *dst, int cap, const mut_t *m) {
  int i = 0, o = 0;
  while (i < n && o < cap) {
    double u = rng_unif(r);
    if (u < m->indel) {
      int len;
      if (m->geom_mean > 0) {
        double p = 1.0 / m->geom_mean;
        len = 1;
        while (rng_unif(r) > p && len < 64) len++;
      } else {
        len = rng_int(r, 1, 3);
      }
      if (rng_next(r) & 1) {
        int k;
        for (k = 0; k < len && o < cap; k++) dst[o++] = NT[rng_next(r) & 3];  /* insertion */
      } else {
        i += len;  /* deletion */
      }
    } else if (u < m->indel + m->sub) {
      char c = src[i++];
      char d;
      do { d = NT[rng_next(r) & 3]; } while (d == c);
      dst[o++] = d;
    } else {
      dst[o++] = src[i++];
    }
  }
  return o;
}

static void
upcase (const char *src, char *dst, int n) {
  int i;
  for (i = 0; i < n; i++) {
    char c = src[i];
    dst[i] = (c >= 'a' && c <= 'z') ? (char) (c - 32) : c;
  }
}

/*
 * Appends one pair of the given kind to (pairs, arena).  The genome window
 * is taken from `genome` (length glen_total) and its alternate equals it.
 * Returns the arena bytes used by the pair, or -1 if it does not fit.
 */
static int64_t
make_pair (rng_t *r, int kind, const char *genome, int64_t glen_total,
           gdp_pair_t *p, char *arena, int64_t off, int64_t cap) {
  int rlength, glength, lband = 0, uband = 0, variant = GDP_FULL, prec = 16, flags;
  int64_t pos;
  mut_t m;
  char *q, *quc, *w;
  int random_window = 0;
  memset(p, 0, sizeof(*p));
  flags = GDP_FLAG_JUMP_LATE | GDP_FLAG_TRACEBACK;
  switch (kind) {
  case WL_FIXED:
    rlength = 150; lband = uband = 10; m.sub = 0.02; m.indel = 0.005; m.geom_mean = 0;
    break;
  case WL_SHORT:
    rlength = rng_int(r, 75, 300); lband = rng_int(r, 3, 30); uband = rng_int(r, 3, 30);
    m.sub = 0.03; m.indel = 0.01; m.geom_mean = 0; prec = 8; flags |= GDP_FLAG_RERUN16;
    random_window = rng_unif(r) < 0.05;
    break;
  case WL_LONG:
    rlength = rng_int(r, 1000, 10000); lband = rng_int(r, 50, 200); uband = rng_int(r, 50, 200);
    m.sub = 0.03; m.indel = 0.01; m.geom_mean = 0;
    break;
  case WL_CDNA:
  default:
    rlength = (int) floor(exp(log(200.0) + rng_unif(r) * (log(5000.0) - log(200.0))));
    m.sub = 0.01; m.indel = 0.02; m.geom_mean = 4; variant = GDP_UPPER;
    break;
  }
  if (kind == WL_CDNA) {
    glength = (int) floor(rlength * (1.0 + 0.5 * rng_unif(r)));
    if (glength < rlength) glength = rlength;
    uband = glength - rlength + 14;
    lband = 14;
  } else if (kind == WL_FIXED) {
    glength = rlength + 10;
  } else {
    glength = rlength;  /* adjusted below from the mutated read */
  }
  if (off + rlength * 2 + glength + 4096 > cap) return -1;
  q = arena + off;
  pos = (int64_t) (rng_next(r) % (uint64_t) (glen_total - 2 * (glength + 512)));
  if (kind == WL_FIXED) {
    /* read = genome[pos, pos+150); window = mutated read padded/truncated to 160 */
    char tmp[512];
    int n;
    memcpy(q, genome + pos, rlength);
    n = mutate(r, q, rlength, tmp, 400, &m);
    w = q + 2 * rlength;
    if (n >= glength) {
      memcpy(w, tmp, glength);
    } else {
      memcpy(w, tmp, n);
      memcpy(w + n, genome + pos + rlength, glength - n);
    }
  } else if (kind == WL_CDNA) {
    /* window = genome[pos, pos+g); read = window minus an intron-like
       block of (g - r) bases, then mutated */
    char *tmp = (char *) malloc((size_t) glength + 64);
    int skip = glength - rlength, at, n, k;
    w = q + 2 * rlength + 64;
    memcpy(w, genome + pos, glength);
    at = skip > 0 ? rng_int(r, 0, rlength) : 0;
    n = 0;
    for (k = 0; k < glength; k++) {
      if (k >= at && k < at + skip) continue;
      tmp[n++] = w[k];
    }
    n = mutate(r, tmp, n, q, rlength + 64, &m);
    free(tmp);
    if (n > rlength) n = rlength;
    while (n < rlength) q[n++] = NT[rng_next(r) & 3];
    uband = glength - rlength + 14;
  } else {
    /* read from the genome; window = mutated read, g = its length clamped
       into [r - lband, r + uband] and filled from the flanking genome */
    char *tmp = (char *) malloc((size_t) rlength * 2 + 128);
    int n;
    memcpy(q, genome + pos, rlength);
    w = q + 2 * rlength + 64;
    if (random_window) {
      int64_t p2 = (int64_t) (rng_next(r) % (uint64_t) (glen_total - 2 * (rlength + 512)));
      n = rlength + rng_int(r, -lband, uband);
      memcpy(tmp, genome + p2, n);
    } else {
      n = mutate(r, q, rlength, tmp, rlength * 2 + 64, &m);
    }
    {
      int want = n;
      if (want < rlength - lband) want = rlength - lband;
      if (want > rlength + uband) want = rlength + uband;
      if (want < 1) want = 1;
      if (want > n) memcpy(tmp + n, genome + pos + rlength, want - n);   /* pad from the flank */
      n = want;
    }
    glength = n;
    memcpy(w, tmp, glength);
    free(tmp);
  }
  quc = q + rlength;
  upcase(q, quc, rlength);
  p->rseq = off;
  p->rseq_uc = off + rlength;
  p->gseq = (int64_t) (w - arena);
  p->gseq_alt = p->gseq;
  p->rlength = rlength;
  p->glength = glength;
  p->lband = lband;
  p->uband = uband;
  p->variant = (int8_t) variant;
  p->precision = (int8_t) prec;
  p->mismatchtype = GDP_HIGHQ;
  p->flags = (int8_t) flags;
  p->open = -8;
  p->extend = -3;
  p->tb_r = rlength;
  p->tb_c = glength;
  p->queryoffset = 0;
  p->genomeoffset = (int32_t) pos;
  p->chroffset = 0;
  p->chrhigh = (uint32_t) glen_total;
  p->watsonp = 1;
  p->genestrand = 0;
  p->dynprogindex = 1;
  return (int64_t) (w - arena) + glength - off;
}

/*
 * One pair whose genome window is a slice of the genome, for callers that
 * keep the genome resident on the device (GDP_FLAG_GWINDOW): the window is
 * genome[pos, pos + glength), written to the arena as well, and the read is
 * its mutated copy, its length clamped so that (rlength, glength) stays in
 * the band.  Same length, band and mutation distributions as make_pair.
 */
static int64_t
make_pair_resident (rng_t *r, int kind, const char *genome, int64_t glen_total,
                    gdp_pair_t *p, char *arena, int64_t off, int64_t cap) {
  int glength, rlength, lband, uband, prec = 16, flags, n, lo, hi;
  int random_window = 0;
  int64_t pos, used;
  mut_t m;
  char *w, *q, *tmp;
  if (kind == WL_CDNA) {
    /* its window is already a genome slice */
    used = make_pair(r, kind, genome, glen_total, p, arena, off, cap);
    if (used >= 0) p->flags = (int8_t) (p->flags | GDP_FLAG_GWINDOW);
    return used;
  }
  memset(p, 0, sizeof(*p));
  flags = GDP_FLAG_JUMP_LATE | GDP_FLAG_TRACEBACK | GDP_FLAG_GWINDOW;
  switch (kind) {
  case WL_FIXED:
    glength = 160; lband = uband = 10; m.sub = 0.02; m.indel = 0.005; m.geom_mean = 0;
    break;
  case WL_SHORT:
    glength = rng_int(r, 75, 300); lband = rng_int(r, 3, 30); uband = rng_int(r, 3, 30);
    m.sub = 0.03; m.indel = 0.01; m.geom_mean = 0; prec = 8; flags |= GDP_FLAG_RERUN16;
    random_window = rng_unif(r) < 0.05;
    break;
  case WL_LONG:
  default:
    glength = rng_int(r, 1000, 10000); lband = rng_int(r, 50, 200); uband = rng_int(r, 50, 200);
    m.sub = 0.03; m.indel = 0.01; m.geom_mean = 0;
    break;
  }
  /* the read length range that keeps (rlength, glength) in the band */
  lo = glength - uband; hi = glength + lband;
  if (kind == WL_FIXED) lo = hi = 150;
  if (lo < 1) lo = 1;
  if (off + (int64_t) glength + 2 * (int64_t) hi + 4096 > cap) return -1;
  pos = (int64_t) (rng_next(r) % (uint64_t) (glen_total - 2 * (glength + hi + 512)));
  w = arena + off;
  memcpy(w, genome + pos, glength);
  q = w + glength + 64;
  tmp = (char *) malloc((size_t) hi * 2 + (size_t) glength * 2 + 128);
  if (random_window) {
    int64_t p2 = (int64_t) (rng_next(r) % (uint64_t) (glen_total - 2 * (hi + 512)));
    n = rng_int(r, lo, hi);
    memcpy(tmp, genome + p2, n);
  } else {
    n = mutate(r, w, glength, tmp, hi + 64, &m);
  }
  if (n > hi) n = hi;
  if (n < lo) {
    memcpy(tmp + n, genome + pos + glength, lo - n);   /* continue into the flank */
    n = lo;
  }
  rlength = n;
  memcpy(q, tmp, rlength);
  free(tmp);
  upcase(q, q + rlength, rlength);
  p->rseq = (int64_t) (q - arena);
  p->rseq_uc = p->rseq + rlength;
  p->gseq = off;
  p->gseq_alt = off;
  p->rlength = rlength;
  p->glength = glength;
  p->lband = lband;
  p->uband = uband;
  p->variant = GDP_FULL;
  p->precision = (int8_t) prec;
  p->mismatchtype = GDP_HIGHQ;
  p->flags = (int8_t) flags;
  p->open = -8;
  p->extend = -3;
  p->tb_r = rlength;
  p->tb_c = glength;
  p->genomeoffset = (int32_t) pos;
  p->chroffset = 0;
  p->chrhigh = (uint32_t) glen_total;
  p->watsonp = 1;
  p->dynprogindex = 1;
  return (int64_t) (q - arena) + 2 * rlength - off;
}

/*
 * Completes draw `draw` whose first fill is pairs[i]: odd draws jump early;
 * a cDNA draw appends the lower fill of the same sequences (lband 14, no
 * traceback) in the next slot when there is one.  Returns the index of the
 * draw's last fill.
 */
static int64_t
finish_draw (gdp_pair_t *pairs, int64_t i, int64_t npairs, int kind, int64_t draw) {
  if (draw & 1) pairs[i].flags = (int8_t) (pairs[i].flags & ~GDP_FLAG_JUMP_LATE);
  if (kind == WL_CDNA && i + 1 < npairs) {
    gdp_pair_t *lo = &pairs[i + 1];
    *lo = pairs[i];
    lo->variant = GDP_LOWER;
    lo->lband = 14;
    lo->uband = 0;
    lo->flags = (int8_t) (lo->flags & ~GDP_FLAG_TRACEBACK);
    return i + 1;
  }
  return i;
}

/*
 * Like gdp_workload_pairs, with every genome window a slice of `genome`
 * and flagged GDP_FLAG_GWINDOW (genomeoffset = the slice's first position,
 * chroffset 0, chrhigh genome_length, plus strand).  The window bytes are
 * also written to the arena, so the same pairs without the flag are an
 * equivalent host-window batch.
 */
int64_t
gdp_workload_resident_pairs (int kind, uint64_t seed, const char *genome, int64_t genome_length,
                             int64_t npairs, gdp_pair_t *pairs, char *arena, int64_t arena_cap,
                             int64_t *arena_used) {
  rng_t r;
  int64_t i, off = 0, draw = 0;
  rng_seed(&r, seed);
  for (i = 0; i < npairs; i++) {
    int k = kind;
    int64_t used;
    if (kind == 4) {
      double u = rng_unif(&r);
      k = (u < 0.70) ? WL_SHORT : (u < 0.95) ? WL_LONG : WL_CDNA;
    }
    used = make_pair_resident(&r, k, genome, genome_length, &pairs[i], arena, off, arena_cap);
    if (used < 0) break;
    off += (used + 15) & ~(int64_t) 15;
    i = finish_draw(pairs, i, npairs, k, draw++);
  }
  if (arena_used) *arena_used = off;
  return i;
}

/*
 * Generates npairs pairs.  kind: 1 fixed-150, 2 short, 3 cdna, 5 long,
 * 4 = the mixed batch (70% short / 25% long / 5% cdna).  Returns the number
 * of pairs generated (fewer if the arena is full); *arena_used gets the
 * arena bytes consumed.
 */
int64_t
gdp_workload_pairs (int kind, uint64_t seed, const char *genome, int64_t genome_length,
                    int64_t npairs, gdp_pair_t *pairs, char *arena, int64_t arena_cap,
                    int64_t *arena_used) {
  rng_t r;
  int64_t i, off = 0, draw = 0;
  rng_seed(&r, seed);
  for (i = 0; i < npairs; i++) {
    int k = kind;
    int64_t used;
    if (kind == 4) {
      double u = rng_unif(&r);
      k = (u < 0.70) ? WL_SHORT : (u < 0.95) ? WL_LONG : WL_CDNA;
    }
    used = make_pair(&r, k, genome, genome_length, &pairs[i], arena, off, arena_cap);
    if (used < 0) break;
    off += (used + 15) & ~(int64_t) 15;
    i = finish_draw(pairs, i, npairs, k, draw++);
  }
  if (arena_used) *arena_used = off;
  return i;
}

/* In-band cell count of one pair over the reference's compare domain
   (src/dynprog_simd.c:1044-1051, :1089-1096, :1134-1141). */
int64_t
gdp_pair_cells (const gdp_pair_t *p) {
  int64_t total = 0;
  int c;
  for (c = 1; c <= p->glength; c++) {
    int lo, hi;
    if (p->variant == GDP_FULL) { lo = c - p->uband; hi = c + p->lband; }
    else if (p->variant == GDP_UPPER) { lo = c - p->uband; hi = c; }
    else { lo = c; hi = c + p->lband; }
    if (lo < 1) lo = 1;
    if (hi > p->rlength) hi = p->rlength;
    if (hi >= lo) total += hi - lo + 1;
  }
  return total;
}
