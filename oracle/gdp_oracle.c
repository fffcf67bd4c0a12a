/*
 * gdp_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C restatement of the reference's banded affine-gap fills and
 * tracebacks (src/dynprog_simd.c) used as an independent checker for the
 * CUDA kernels.  It is pinned against the reference's own compiled
 * functions (oracle/_ref/libgdpref.so) by tests/test_oracle.py.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU baseline load it.
 *
 * The reference fills a matrix in blocks of W rows (W = 16 for 16-bit, 32
 * for 8-bit AVX2 lanes; SIMD_NSHORTS/SIMD_NCHARS, src/dynprog.h:127-132),
 * sweeping for each block the columns [rlo - lband, rhigh + uband]
 * (src/dynprog_simd.c:3216-3256, :6762-6802).  Cells of a block that lie
 * outside the band are computed too and feed the in-band E values, so the
 * restatement reproduces the block structure exactly instead of a plain
 * banded recurrence.  Per cell (x = lane / query row, y = swept column):
 *
 *   T1 = sat(H[y-1][x] + open);  dirE = E[y-1][x] >= T1 (late) | > (early)
 *   E  = sat(max(E[y-1][x], T1) + extend)                (:6862-6875)
 *   Hv = sat(H[y-1][x-1] + max(prof[g], prof[g_alt]))     (:6880-6900)
 *   dirN = HORIZ if E >= Hv (late) | > (early); H = max(Hv, E)  (:6904-6913)
 *   full band only: bottom cell x = y + lband takes Hv with DIAG dirs
 *   (:6926-6945), then the scalar F loop over the in-band rows with the top
 *   cell special case and the int-valued FF carry (:6950-6999).
 *   upper/lower: E clamped to -inf on and below (above) the diagonal via
 *   E_mask (:7921, :7943) and DIAG directions on the diagonal (:7966-7969).
 * sat() saturates to the lane type (int8 or int16), as _mm256_adds_epi8/16.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>
#include <ctype.h>
#include "gdp_oracle.h"

#define NEGINT (-32768)     /* NEG_INFINITY_INT, src/dynprog.h:176 */
#define DIAG 0
#define HORIZ (-1)
#define VERT (-2)

/* ------------------------------------------------------------------ */
/* Tables (src/dynprog.c:1007-1196)                                    */
/* ------------------------------------------------------------------ */

static int16_t pd_tab[4][128][128];       /* pairdistance_array */
static uint8_t cons_tab[3][128][128];     /* consistent_array */
static int nt_to_int[128];
static int tables_mode = -1;

static void
set_pair (int A, int B, int score, int mode, int oneway, int genestrand) {
  int a = tolower(A), b = tolower(B), i;
  int pairs[4][2] = {{a, b}, {a, B}, {A, b}, {A, B}};
  int k;
  for (k = 0; k < 4; k++) {
    int x = pairs[k][0], y = pairs[k][1];
    if (oneway) {
      cons_tab[genestrand][x][y] = 1;
    } else if (mode == 0 || mode == 1 || mode == 3 || mode == 5) {
      cons_tab[0][x][y] = 1; cons_tab[0][y][x] = 1;
    } else {
      cons_tab[1][x][y] = 1; cons_tab[1][y][x] = 1;
      cons_tab[2][x][y] = 1; cons_tab[2][y][x] = 1;
    }
    for (i = 0; i < 4; i++) {
      pd_tab[i][x][y] = (int16_t) score;
      if (!oneway) pd_tab[i][y][x] = (int16_t) score;
    }
  }
}

void
orc_init (int mode) {
  static const int mism[4] = {-3, -2, -1, -5};  /* MISMATCH_HIGHQ/MEDQ/LOWQ/ENDQ */
  int c1, c2, i, c;
  memset(pd_tab, 0, sizeof(pd_tab));
  memset(cons_tab, 0, sizeof(cons_tab));
  for (i = 0; i < 128; i++) nt_to_int[i] = 4;
  nt_to_int['A'] = nt_to_int['a'] = 0;
  nt_to_int['C'] = nt_to_int['c'] = 1;
  nt_to_int['G'] = nt_to_int['g'] = 2;
  nt_to_int['T'] = nt_to_int['t'] = 3;
  /* mismatch default over 'A'..'z' x 'A'..'y' (the inner bound is exclusive) */
  for (c1 = 'A'; c1 <= 'z'; c1++)
    for (c2 = 'A'; c2 < 'z'; c2++)
      for (i = 0; i < 4; i++) pd_tab[i][c1][c2] = (int16_t) mism[i];
  for (c = 'A'; c < 'Z'; c++) set_pair(c, c, 3, mode, 0, 0);
  set_pair('U', 'T', 3, mode, 0, 0);
  {
    static const char half[][2] = {{'R','A'},{'R','G'},{'Y','T'},{'Y','C'},{'W','A'},{'W','T'},
                                   {'S','G'},{'S','C'},{'M','A'},{'M','C'},{'K','G'},{'K','T'}};
    static const char amb[][2] = {{'H','A'},{'H','T'},{'H','C'},{'B','G'},{'B','C'},{'B','T'},
                                  {'V','G'},{'V','A'},{'V','C'},{'D','G'},{'D','A'},{'D','T'},
                                  {'N','T'},{'N','C'},{'N','A'},{'N','G'},
                                  {'X','T'},{'X','C'},{'X','A'},{'X','G'},{'N','N'},{'X','X'}};
    for (i = 0; i < (int) (sizeof(half) / 2); i++) set_pair(half[i][0], half[i][1], 1, mode, 0, 0);
    for (i = 0; i < (int) (sizeof(amb) / 2); i++) set_pair(amb[i][0], amb[i][1], 3, mode, 0, 0);
  }
  switch (mode) {
  case 1: set_pair('T', 'C', 3, mode, 1, 0); break;                             /* CMET_STRANDED */
  case 2: set_pair('T', 'C', 3, mode, 1, 1); set_pair('A', 'G', 3, mode, 1, 2); break;
  case 3: set_pair('G', 'A', 3, mode, 1, 0); break;                             /* ATOI_STRANDED */
  case 4: set_pair('G', 'A', 3, mode, 1, 1); set_pair('C', 'T', 3, mode, 1, 2); break;
  case 5: set_pair('C', 'T', 3, mode, 1, 0); break;                             /* TTOC_STRANDED */
  case 6: set_pair('C', 'T', 3, mode, 1, 1); set_pair('G', 'A', 3, mode, 1, 2); break;
  default: break;
  }
  tables_mode = mode;
}

int orc_pairdistance (int mt, int c1, int c2) { return pd_tab[mt][c1 & 127][c2 & 127]; }
int orc_consistent (int gs, int c1, int c2) { return cons_tab[gs][c1 & 127][c2 & 127]; }

/* ------------------------------------------------------------------ */
/* Genome (genomecomp blocks, src/genome.c:9723-9792, :11003-11017)    */
/* ------------------------------------------------------------------ */

static const uint32_t *gblocks = NULL, *galtblocks = NULL;

void
orc_set_genome (const uint32_t *blocks, const uint32_t *altblocks, uint64_t len) {
  (void) len;
  gblocks = blocks;
  galtblocks = altblocks ? altblocks : blocks;
}

static char
decode_nt (const uint32_t *b, uint32_t pos, int flags) {
  static const char ACGT[4] = {'A', 'C', 'G', 'T'};
  uint32_t ptr = pos / 32U * 3;
  int bit = (int) (pos % 32);
  if (flags && (b[ptr + 2] & (1U << bit))) return 'N';
  if (bit < 16) return ACGT[(b[ptr + 1] >> (2 * bit)) & 3U];
  return ACGT[(b[ptr] >> (2 * bit - 32)) & 3U];
}

static char
genome_char (char *alt, uint32_t pos) {
  char c = decode_nt(gblocks, pos, 1);
  *alt = (c == 'N') ? c : decode_nt(galtblocks, pos, 0);
  return c;
}

static char
compl_nt (char c) {
  switch (c) {
  case 'A': return 'T'; case 'C': return 'G'; case 'G': return 'C'; case 'T': return 'A';
  default: return c;  /* 'N' */
  }
}

/* get_genomic_nt (src/pairpool.c:1015-1063); Univcoord_T is 32-bit unsigned */
static char
genomic_nt (char *alt, int genomicpos, uint32_t chroffset, uint32_t chrhigh, int watsonp) {
  uint32_t pos;
  char c2, c2a;
  if (watsonp) {
    pos = chroffset + (uint32_t) genomicpos;
    if (pos < chroffset || pos >= chrhigh) { *alt = '*'; return '*'; }
    return genome_char(alt, pos);
  }
  pos = chrhigh - (uint32_t) genomicpos;
  if (pos < chroffset || pos >= chrhigh) { *alt = '*'; return '*'; }
  c2 = genome_char(&c2a, pos);
  *alt = compl_nt(c2a);
  return compl_nt(c2);
}

/* ------------------------------------------------------------------ */
/* Fill                                                                */
/* ------------------------------------------------------------------ */

typedef struct {
  int variant, W, lo, hi;
  int X, Y;            /* lane dimension length, swept dimension length */
  int xstride;         /* X rounded up: ((X + W) / W) * W */
  int32_t *M;          /* scores [y * xstride + x] (values in lane range) */
  int8_t *dN, *dE, *dF;
  uint8_t *wr;         /* 1 where this fill wrote dN/dE (the swept region) */
} grid_t;

static inline int sat (int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int imax (int a, int b) { return a > b ? a : b; }

/* Character of a sequence at 1-based position i, honouring revp (seq[1-i]
   from the last character) */
static inline int
seqchar (const char *base, int len, int i, int revp) {
  return (unsigned char) (revp ? base[len - i] : base[i - 1]) & 127;
}

static void
fill (const gdp_pair_t *p, const char *arena, grid_t *G) {
  const char *rseq = arena + p->rseq, *gseq = arena + p->gseq, *galt = arena + p->gseq_alt;
  int revp = (p->flags & GDP_FLAG_REVP) != 0, late = (p->flags & GDP_FLAG_JUMP_LATE) != 0;
  int variant = p->variant, W = (p->precision == 8) ? 32 : 16;
  int lo = (p->precision == 8) ? -128 : -32768, hi = (p->precision == 8) ? 127 : 32767;
  int NEG = lo, open = p->open, extend = p->extend, mt = p->mismatchtype;
  int X = (variant == GDP_LOWER) ? p->glength : p->rlength;
  int Y = (variant == GDP_LOWER) ? p->rlength : p->glength;
  int band_hi = (variant == GDP_LOWER) ? p->lband : p->uband;   /* sweep beyond the block */
  int xstride = ((X + W) / W) * W;
  int *V;             /* per-lane profile: V[x * 5 + k] */
  int *ycls, *ycls_alt;
  int *FF;
  int32_t *Hp, *Ep, *Hn, *En;
  int xlo, i, y;
  static const char ACGTN[5] = {'A', 'C', 'G', 'T', 'N'};

  G->variant = variant; G->W = W; G->lo = lo; G->hi = hi; G->X = X; G->Y = Y; G->xstride = xstride;
  G->M = (int32_t *) calloc((size_t) (Y + 1) * xstride, sizeof(int32_t));
  G->dN = (int8_t *) calloc((size_t) (Y + 1) * xstride, 1);
  G->dE = (int8_t *) calloc((size_t) (Y + 1) * xstride, 1);
  G->dF = (int8_t *) calloc((size_t) (Y + 1) * xstride, 1);   /* Fgap starts DIAG (:2203-2218) */
  G->wr = (uint8_t *) calloc((size_t) (Y + 1) * xstride, 1);

  V = (int *) calloc((size_t) xstride * 5, sizeof(int));
  ycls = (int *) calloc((size_t) Y + 1, sizeof(int));
  ycls_alt = (int *) calloc((size_t) Y + 1, sizeof(int));
  FF = (int *) calloc((size_t) Y + 1, sizeof(int));
  Hp = (int32_t *) malloc(W * sizeof(int32_t)); Ep = (int32_t *) malloc(W * sizeof(int32_t));
  Hn = (int32_t *) malloc(W * sizeof(int32_t)); En = (int32_t *) malloc(W * sizeof(int32_t));

  if (variant != GDP_LOWER) {
    /* query profile (:6700-6725): lane x scores against genome classes */
    for (i = 0; i < 5; i++) V[0 * 5 + i] = pd_tab[mt]['N'][(int) ACGTN[i]];
    for (i = 1; i <= X; i++) {
      int q = seqchar(rseq, p->rlength, i, revp), k;
      for (k = 0; k < 5; k++) V[i * 5 + k] = pd_tab[mt][q][(int) ACGTN[k]];
    }
    for (y = 1; y <= Y; y++) {
      ycls[y] = nt_to_int[seqchar(gseq, p->glength, y, revp)];
      ycls_alt[y] = nt_to_int[seqchar(galt, p->glength, y, revp)];
    }
    ycls[0] = ycls_alt[0] = 4;
  } else {
    /* genome profile (:8690-8720): lane x = genome column, max(g, g_alt) folded in */
    int k;
    /* column 0 scores against 'N' in the 16-bit fill (:8689), but against
       character code 4 in the 8-bit fill (:5459, na2 = 4), which the table
       leaves at 0 */
    int col0 = (p->precision == 8) ? 4 : 'N';
    for (k = 0; k < 5; k++) V[0 * 5 + k] = pd_tab[mt][(int) ACGTN[k]][col0];
    for (i = 1; i <= X; i++) {
      int g = seqchar(gseq, p->glength, i, revp), ga = seqchar(galt, p->glength, i, revp);
      for (k = 0; k < 5; k++) V[i * 5 + k] = imax(pd_tab[mt][(int) ACGTN[k]][g], pd_tab[mt][(int) ACGTN[k]][ga]);
    }
    for (y = 1; y <= Y; y++) ycls[y] = ycls_alt[y] = nt_to_int[seqchar(rseq, p->rlength, y, revp)];
    ycls[0] = ycls_alt[0] = 4;
  }

  for (xlo = 0; xlo <= X; xlo += W) {
    int xhi = (xlo + W - 1 > X) ? X : xlo + W - 1;
    int y0, y1;
    if (variant == GDP_FULL) {
      y0 = (xlo - p->lband < 0) ? 0 : xlo - p->lband;
    } else {
      y0 = xlo;
    }
    y1 = xhi + band_hi;
    if (y1 > Y) y1 = Y;
    for (i = 0; i < W; i++) { Hp[i] = NEG - open; Ep[i] = late ? NEG : NEG + 1; }

    for (y = y0; y <= y1; y++) {
      int32_t *Mcol = G->M + (size_t) y * xstride;
      int8_t *nN = G->dN + (size_t) y * xstride, *nE = G->dE + (size_t) y * xstride;
      int8_t *nF = G->dF + (size_t) y * xstride;
      int diag0;
      if (variant == GDP_FULL) {
        if (y == 0) diag0 = (xlo == 0) ? 0 : NEG;
        else diag0 = (xlo == 0) ? NEG : G->M[(size_t) (y - 1) * xstride + xlo - 1];
      } else {
        if (y == 0) diag0 = 0;
        else if (xlo == 0) diag0 = NEG;
        else diag0 = G->M[(size_t) (y - 1) * xstride + xlo - 1];
      }
      for (i = 0; i < W; i++) {
        int x = xlo + i;
        int Eold = Ep[i], T1, E, diag, ps, Hv, dirE, dirN;
        int masked = (variant != GDP_FULL) && (x >= y);
        if (masked) Eold = NEG;
        T1 = sat(Hp[i] + open, lo, hi);
        dirE = late ? (Eold >= T1) : (Eold > T1);
        E = sat(imax(Eold, T1) + extend, lo, hi);
        if (masked) E = NEG;
        diag = (i == 0) ? diag0 : Hp[i - 1];
        if (x > X) {
          ps = 0;   /* lanes past the end read uninitialised profile memory in the reference; never used */
        } else if (variant == GDP_FULL && y == 0) {
          ps = (x == 0) ? 0 : NEG;    /* pairscores_col0 (:6668-6678) */
        } else {
          ps = imax(V[x * 5 + ycls[y]], V[x * 5 + ycls_alt[y]]);
        }
        Hv = sat(diag + ps, lo, hi);
        dirN = late ? (E >= Hv) : (E > Hv);
        Hn[i] = imax(Hv, E);
        En[i] = E;
        Mcol[x] = Hn[i];
        G->wr[(size_t) y * xstride + x] = 1;
        nE[x] = (int8_t) (dirE ? HORIZ : DIAG);
        nN[x] = (int8_t) (dirN ? HORIZ : DIAG);
        if (variant == GDP_FULL && x == y + p->lband && y > 0 && x <= xhi) {
          /* bottom band cell: diagonal only, DIAG directions (:6926-6945) */
          Hn[i] = Hv;
          Mcol[x] = Hv;
          nE[x] = DIAG;
          nN[x] = DIAG;
        }
      }
      if (variant != GDP_FULL) {
        if (xhi >= y) { nE[y] = DIAG; nN[y] = DIAG; }   /* diagonal fix (:7966-7969) */
      } else {
        /* F loop (:6916-7000) */
        int rlo_calc = (xlo > y - p->uband) ? xlo : y - p->uband;
        int rhigh_calc = (xhi < y + p->lband) ? xhi : y + p->lband;
        int cgap, last, r, s;
        if (xlo == 0 || y >= xlo + p->uband) {
          cgap = NEGINT; last = NEGINT;
        } else {
          cgap = FF[y]; last = Mcol[rlo_calc - 1];
        }
        r = rlo_calc;
        if (r == y - p->uband) {
          cgap = last + open + extend;
          last = Mcol[r];
          r++;
        }
        for (; r <= rhigh_calc; r++) {
          s = last + open;
          if (late ? (cgap >= s) : (cgap > s)) { cgap += extend; nF[r] = VERT; }
          else { cgap = s + extend; }
          last = Mcol[r];
          if (late ? (cgap >= last) : (cgap > last)) {
            last = cgap;
            Mcol[r] = (cgap < NEG) ? NEG : cgap;
            nN[r] = VERT;
          }
        }
        FF[y] = cgap;
        for (i = 0; i < W; i++) Hn[i] = Mcol[xlo + i];   /* reload after the F loop */
      }
      for (i = 0; i < W; i++) { Hp[i] = Hn[i]; Ep[i] = En[i]; }
    }
  }
  free(V); free(ycls); free(ycls_alt); free(FF); free(Hp); free(Ep); free(Hn); free(En);
}

static void
grid_free (grid_t *G) {
  free(G->M); free(G->dN); free(G->dE); free(G->dF); free(G->wr);
}

/* cell (c, r) in reference indexing: full/upper [c][r], lower [r][c] */
static inline size_t
gidx (const grid_t *G, int c, int r) {
  return (G->variant == GDP_LOWER) ? (size_t) r * G->xstride + c : (size_t) c * G->xstride + r;
}

/* ------------------------------------------------------------------ */
/* Traceback (src/dynprog_simd.c:9153-9945, src/pairpool.c)            */
/* ------------------------------------------------------------------ */

typedef struct {
  gdp_rec_t *recs;
  int n, cap;
  int dpi;
} pool_t;

static void
push (pool_t *P, int querypos, int genomepos, char cdna, char comp, char g, char galt) {
  if (querypos < 0 || genomepos < 0) return;   /* Pairpool_push (:189-191) */
  if (P->recs && P->n < P->cap) {
    gdp_rec_t *d = &P->recs[P->n];
    d->querypos = querypos; d->genomepos = genomepos;
    d->cdna = cdna; d->comp = comp; d->genome = g; d->genomealt = galt;
  }
  P->n++;
}

static void
push_gapholder (pool_t *P, int dist) {
  if (P->recs && P->n < P->cap) {
    gdp_rec_t *d = &P->recs[P->n];
    d->querypos = -1; d->genomepos = dist;   /* gap holder: comp '\0' */
    d->cdna = ' '; d->comp = '\0'; d->genome = ' '; d->genomealt = ' ';
  }
  P->n++;
}

typedef struct {
  const char *rseq, *ruc, *gseq, *galt;   /* revp-adjusted pointers (reference convention) */
  const gdp_pair_t *p;
  int revp;
} tbin_t;

/* Pairpool_add_queryskip (src/pairpool.c:980-1010) */
static void
add_queryskip (pool_t *P, const tbin_t *T, int r, int c, int dist) {
  int qc = r - 1, gc = c - 1, step, j;
  if (T->revp) { qc = -qc; gc = -gc; step = +1; } else { step = -1; }
  for (j = 0; j < dist; j++) {
    push(P, T->p->queryoffset + qc, T->p->genomeoffset + gc, T->rseq[qc], '-', ' ', ' ');
    qc += step;
  }
}

/* Pairpool_add_genomeskip (src/pairpool.c:1067-1179); returns add_dashes_p */
static int
add_genomeskip (pool_t *P, const tbin_t *T, int r, int c, int dist) {
  int qc = r - 1, left = c - dist, right = c - 1, step, j, gc;
  if (T->revp) { int t = left; qc = -qc; left = -right; right = -t; step = +1; } else { step = -1; }
  if (dist < 9) {
    gc = T->revp ? left : right;
    for (j = 0; j < dist; j++) {
      char a, g = genomic_nt(&a, T->p->genomeoffset + gc, T->p->chroffset, T->p->chrhigh, T->p->watsonp);
      push(P, T->p->queryoffset + qc, T->p->genomeoffset + gc, ' ', '-', g, a);
      gc += step;
    }
    return 1;
  }
  push_gapholder(P, dist);
  return 0;
}

static void
diag_pair (pool_t *P, const tbin_t *T, int r, int c, int *st) {
  int qc = r - 1, gc = c - 1;
  char c1, c1uc, c2, c2a;
  if (T->revp) { qc = -qc; gc = -gc; }
  c1 = T->rseq[qc]; c1uc = T->ruc[qc]; c2 = T->gseq[gc]; c2a = T->galt[gc];
  if (c2 == '*') return;
  if (c1uc == c2 || c1uc == c2a) {
    st[0] += 1; st[1] += 1;
    push(P, T->p->queryoffset + qc, T->p->genomeoffset + gc, c1, '*', c2, c2a);
  } else if (cons_tab[T->p->genestrand][c1uc & 127][c2 & 127] || cons_tab[T->p->genestrand][c1uc & 127][c2a & 127]) {
    st[0] += 1; st[1] += 1;
    push(P, T->p->queryoffset + qc, T->p->genomeoffset + gc, c1, ':', c2, c2a);
  } else {
    st[0] += -3; st[2] += 1;
    push(P, T->p->queryoffset + qc, T->p->genomeoffset + gc, c1, ' ', c2, c2a);
  }
}

/* stats: score, nmatches, nmismatches, nopens, nindels, nrecs */
/* Direction reads of the last traceback outside the compare domain
   (tb_outside), and reads of cells this fill never wrote (tb_stale): the
   reference reads stale scratch there, so such a traceback has no defined
   result.  Fgap is cleared by every full-band fill (:2203-2218), so only
   nogap/Egap reads can be stale. */
static __thread int tb_outside = 0, tb_stale = 0;
int orc_last_tb_outside (void) { return tb_outside; }
int orc_last_tb_stale (void) { return tb_stale; }

static int
in_domain (const gdp_pair_t *p, int c, int r) {
  int lo, hi;
  if (c < 1 || r < 1 || c > p->glength || r > p->rlength) return 0;
  if (p->variant == GDP_FULL) { lo = c - p->uband; hi = c + p->lband; }
  else if (p->variant == GDP_UPPER) { lo = c - p->uband; hi = c; }
  else { lo = c; hi = c + p->lband; }
  return r >= lo && r <= hi;
}

static inline int
tbread (const gdp_pair_t *p, const grid_t *G, const int8_t *plane, int c, int r) {
  size_t at;
  tb_outside += !in_domain(p, c, r);
  if (c < 0 || r < 0 || (p->variant == GDP_LOWER ? (r > G->Y || c >= G->xstride) : (c > G->Y || r >= G->xstride))) {
    tb_stale++;
    return 0;
  }
  at = gidx(G, c, r);
  if (plane != G->dF && !G->wr[at]) tb_stale++;
  /* Full band: a cell above the band was computed from the previous block's
     row at a column that block never swept (the reference's X_prev read of
     matrix[c-1][rlo-1], src/dynprog_simd.c:6838), i.e. from stale scratch. */
  if (p->variant == GDP_FULL && r < c - p->uband) tb_stale++;
  return plane[at];
}
#define TBREAD(plane, c, r) tbread(p, G, G->plane, (c), (r))

static int
traceback (const gdp_pair_t *p, const char *arena, const grid_t *G, int *st, gdp_rec_t *recs, int cap) {
  pool_t P;
  tbin_t T;
  int r = p->tb_r, c = p->tb_c, dist;
  P.recs = recs; P.n = 0; P.cap = cap; P.dpi = p->dynprogindex;
  T.p = p; T.revp = (p->flags & GDP_FLAG_REVP) != 0;
  T.rseq = arena + p->rseq; T.ruc = arena + p->rseq_uc; T.gseq = arena + p->gseq; T.galt = arena + p->gseq_alt;
  if (T.revp) {
    T.rseq += p->rlength - 1; T.ruc += p->rlength - 1; T.gseq += p->glength - 1; T.galt += p->glength - 1;
  }
  memset(st, 0, 6 * sizeof(int));
  tb_outside = 0;
  tb_stale = 0;
  if (p->variant == GDP_FULL) {
    while (r > 0 && c > 0) {
      int dir = TBREAD(dN, c, r);
      if (dir == HORIZ) {
        dist = 1;
        while (c > 0) { int d = TBREAD(dE, c, r); c--; if (d == DIAG) break; dist++; }
        if (add_genomeskip(&P, &T, r, c + dist, dist)) { st[0] += -3 - dist; st[3] += 1; st[4] += dist; }
      } else if (dir == VERT) {
        dist = 1;
        while (r > 0) { int d = TBREAD(dF, c, r); r--; if (d == DIAG) break; dist++; }
        add_queryskip(&P, &T, r + dist, c, dist);
        st[0] += -3 - dist; st[3] += 1; st[4] += dist;
      } else if (dir == DIAG) {
        diag_pair(&P, &T, r, c, st);
        r--; c--;
      } else {
        return -1;   /* the reference aborts ("Bad dir") */
      }
    }
    if (r == 0 && c == 0) {
    } else if (c == 0) {
      dist = r;
      add_queryskip(&P, &T, r, 1, dist);
      st[0] += -3 - dist; st[3] += 1; st[4] += dist;
    } else {
      dist = c;
      if (add_genomeskip(&P, &T, 1, c, dist)) { st[0] += -3 - dist; st[3] += 1; st[4] += dist; }
    }
  } else if (p->variant == GDP_UPPER) {
    while (r > 0 && c > 0) {
      if (TBREAD(dN, c, r) != DIAG) {
        dist = 1;
        for (;;) {
          int d;
          if (c < 0) return -1;
          d = TBREAD(dE, c, r); c--;
          if (d == DIAG) break;
          dist++;
        }
        if (add_genomeskip(&P, &T, r, c + dist, dist)) { st[0] += -3 - dist; st[3] += 1; st[4] += dist; }
      } else {
        diag_pair(&P, &T, r, c, st);
        r--; c--;
      }
    }
    if (c != 0) {
      dist = c;
      if (add_genomeskip(&P, &T, 1, c, dist)) { st[0] += -3 - dist; st[3] += 1; st[4] += dist; }
    }
  } else {
    while (r > 0 && c > 0) {
      if (TBREAD(dN, c, r) != DIAG) {
        dist = 1;
        for (;;) {
          int d;
          if (r < 0) return -1;
          d = TBREAD(dE, c, r); r--;
          if (d == DIAG) break;
          dist++;
        }
        add_queryskip(&P, &T, r + dist, c, dist);
        st[0] += -3 - dist; st[3] += 1; st[4] += dist;
      } else {
        diag_pair(&P, &T, r, c, st);
        r--; c--;
      }
    }
    if (r != 0) {
      dist = r;
      add_queryskip(&P, &T, r, 1, dist);
      st[0] += -3 - dist; st[3] += 1; st[4] += dist;
    }
  }
  st[5] = P.n;
  return P.n;
}

/* ------------------------------------------------------------------ */
/* Entry points (same interface as oracle/ref_harness.c)               */
/* ------------------------------------------------------------------ */

int
orc_align (const gdp_pair_t *p, const char *arena,
           int16_t *H, int8_t *dN, int8_t *dE, int8_t *dF, int32_t *final_score,
           int32_t *tb_stats, gdp_rec_t *recs, int max_recs) {
  grid_t G;
  int c, r, n = 0, R = p->rlength + 1;
  if (tables_mode < 0) orc_init(0);
  fill(p, arena, &G);
  for (c = 1; c <= p->glength; c++) {
    int lo, hi;
    if (p->variant == GDP_FULL) { lo = c - p->uband; hi = c + p->lband; }
    else if (p->variant == GDP_UPPER) { lo = c - p->uband; hi = c; }
    else { lo = c; hi = c + p->lband; }
    if (lo < 1) lo = 1;
    if (hi > p->rlength) hi = p->rlength;
    for (r = lo; r <= hi; r++) {
      size_t at = (size_t) c * R + r, g = gidx(&G, c, r);
      if (H) H[at] = (int16_t) G.M[g];
      if (dN) dN[at] = G.dN[g];
      if (dE) dE[at] = G.dE[g];
      if (dF) dF[at] = G.dF[g];
    }
  }
  if (final_score) *final_score = G.M[gidx(&G, p->glength, p->rlength)];
  if (p->flags & GDP_FLAG_TRACEBACK) {
    int st[6];
    n = traceback(p, arena, &G, st, recs, max_recs);
    if (tb_stats) memcpy(tb_stats, st, sizeof(st));
  }
  grid_free(&G);
  return n;
}

/* The precision whose outputs the rerun contract keeps for pair p
   (GDP_FLAG_RERUN16 on an 8-bit pair): 8 unless the 8-bit fill reaches 127
   inside the compare domain, ends at or below -98, or (with a traceback)
   its 8-bit traceback reads a cell the 8-bit fill never wrote. */
static int
kept_precision (const gdp_pair_t *p, const char *arena) {
  gdp_pair_t q = *p;
  grid_t G;
  int c, r, keep = 8;
  if (p->precision != 8 || !(p->flags & GDP_FLAG_RERUN16)) return p->precision;
  q.flags &= ~GDP_FLAG_RERUN16;
  fill(&q, arena, &G);
  for (c = 1; c <= q.glength && keep == 8; c++) {
    int lo, hi;
    if (q.variant == GDP_FULL) { lo = c - q.uband; hi = c + q.lband; }
    else if (q.variant == GDP_UPPER) { lo = c - q.uband; hi = c; }
    else { lo = c; hi = c + q.lband; }
    if (lo < 1) lo = 1;
    if (hi > q.rlength) hi = q.rlength;
    for (r = lo; r <= hi; r++)
      if (G.M[gidx(&G, c, r)] >= 127) { keep = 16; break; }
  }
  if (keep == 8 && G.M[gidx(&G, q.glength, q.rlength)] <= -98) keep = 16;
  if (keep == 8 && (q.flags & GDP_FLAG_TRACEBACK)) {
    int st[6];
    traceback(&q, arena, &G, st, NULL, 0);
    if (tb_stale) keep = 16;
  }
  grid_free(&G);
  return keep;
}

typedef struct {
  const gdp_pair_t *pairs; const char *arena; int64_t n; int tid, nt; int64_t sum;
  const int8_t *kept_in;
  int8_t *kept_out;
  int32_t *out;      /* orc_outputs: 8 words per pair, else NULL */
} job_t;

/* 32-bit digest of n Pair records in push order, as the reference harness
   and the benchmark compute it: the sum over records k of (w0 *
   0x9E3779B1 + w1 * 0x85EBCA77 + w2 * 0xC2B2AE3D + 1) * (2k + 1). */
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
worker (void *arg) {
  job_t *j = (job_t *) arg;
  int64_t i;
  gdp_rec_t *recs = NULL;
  int cap = 0;
  for (i = j->tid; i < j->n; i += j->nt) {
    const gdp_pair_t *p = &j->pairs[i];
    gdp_pair_t q;
    int32_t fs = 0, st[6] = {0};
    int n = 0;
    if (j->kept_out) {
      j->kept_out[i] = (int8_t) kept_precision(p, j->arena);
      continue;
    }
    if (p->precision == 8 && (p->flags & GDP_FLAG_RERUN16)) {
      /* only the kept precision runs */
      q = *p;
      q.flags &= ~GDP_FLAG_RERUN16;
      q.precision = j->kept_in ? j->kept_in[i] : 16;
      p = &q;
    }
    if (j->out && (p->flags & GDP_FLAG_TRACEBACK) && p->rlength + p->glength + 8 > cap) {
      free(recs);
      cap = 2 * (p->rlength + p->glength + 8);
      recs = (gdp_rec_t *) malloc((size_t) cap * sizeof(gdp_rec_t));
    }
    n = orc_align(p, j->arena, NULL, NULL, NULL, NULL, &fs, st, j->out ? recs : NULL, j->out ? cap : 0);
    j->sum += fs + st[0];
    if (j->out) {
      int32_t *w = j->out + 8 * i;
      w[0] = fs;
      memcpy(w + 1, st, sizeof(st));
      w[7] = (p->flags & GDP_FLAG_TRACEBACK) ? (int32_t) rec_digest(recs, n < cap ? n : cap) : 0;
    }
  }
  free(recs);
  return NULL;
}

static double
run_jobs (const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads, int64_t *checksum,
          const int8_t *kept_in, int8_t *kept_out, int32_t *out) {
  pthread_t *th;
  job_t *jobs;
  struct timespec t0, t1;
  int t;
  int64_t sum = 0;
  if (tables_mode < 0) orc_init(0);
  if (nthreads < 1) nthreads = 1;
  th = (pthread_t *) calloc(nthreads, sizeof(pthread_t));
  jobs = (job_t *) calloc(nthreads, sizeof(job_t));
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (t = 0; t < nthreads; t++) {
    jobs[t].pairs = pairs; jobs[t].arena = arena; jobs[t].n = npairs; jobs[t].tid = t;
    jobs[t].nt = nthreads; jobs[t].sum = 0; jobs[t].kept_in = kept_in; jobs[t].kept_out = kept_out;
    jobs[t].out = out;
    pthread_create(&th[t], NULL, worker, &jobs[t]);
  }
  for (t = 0; t < nthreads; t++) { pthread_join(th[t], NULL); sum += jobs[t].sum; }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  free(th);
  free(jobs);
  if (checksum) *checksum = sum;
  return (double) (t1.tv_sec - t0.tv_sec) + 1e-9 * (double) (t1.tv_nsec - t0.tv_nsec);
}

/* Every pair once across nthreads threads (fill, and traceback when asked);
   returns wall seconds.  An 8-bit pair flagged RERUN16 runs at the
   precision kept[i] only (16 when kept is NULL): the least work that gives
   the rerun contract's outputs. */
double
orc_bench (const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads, int64_t *checksum,
           const int8_t *kept) {
  return run_jobs(pairs, arena, npairs, nthreads, checksum, kept, NULL, NULL);
}

/* The same run, keeping per pair 8 words: the final score, the traceback
   score, nmatches, nmismatches, nopens, nindels, the record count and the
   records' digest (rec_digest; 0 without a traceback). */
double
orc_outputs (const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads, const int8_t *kept,
             int32_t *out) {
  return run_jobs(pairs, arena, npairs, nthreads, NULL, kept, NULL, out);
}

/* kept[i] = the precision the rerun contract keeps for pair i, computed on
   nthreads threads. */
void
orc_kept_precision (const gdp_pair_t *pairs, const char *arena, int64_t npairs, int nthreads, int8_t *kept) {
  run_jobs(pairs, arena, npairs, nthreads, NULL, NULL, kept, NULL);
}
