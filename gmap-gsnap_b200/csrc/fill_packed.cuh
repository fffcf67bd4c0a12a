/*
 * fill_packed.cuh -- the 16-bit full-band fill on packed two-lane words.
 *
 * The same block sweep as block_column (src/dynprog_simd.c:6760-7000, the
 * jump-late copy, and :7009-7250, the jump-early one), with the 16 lanes of
 * a block held as 8 words of two 16-bit halves (lane 2k in the low half of
 * word k, lane 2k + 1 in the high half) and every step done by the 16x2
 * integer instructions of sm_90 and later (add.s16x2, max.s16x2,
 * min.u16x2), two lanes per instruction.
 *
 * Exactness.  The reference saturates its int16 lanes (_mm256_adds_epi16,
 * :6862-6913); add.s16x2 wraps.  Every value here is kept as value + OFF,
 * so that the reference's floor -32768 becomes NEG = OFF - 32768 and a
 * saturating add of a non-positive penalty, max(a + b, -32768), becomes
 * max(a + b, NEG) with no wrap: the most negative value an add can form is
 * NEG - 381 (a score at the floor plus open + extend, both at least -127,
 * plus one more extend in the F chain), far above -32768.  The top end
 * never saturates: every score is a path score from the matrix corner, at
 * most (min(r, c) + 1) times the largest table entry, and the planner sends
 * only pairs whose (min(rlength, glength) + 16) times that entry stays
 * below 32767 - OFF here (FillParams::packed_len; the 16 covers the lanes
 * of a last block beyond the matrix).  So every add, max and comparison
 * gives the reference's result, shifted by OFF.
 *
 * The F loop (:6950-7000) is a max-plus chain down the lanes,
 * F(i) = max(F(i-1), H(i-1) + open) + extend with H(i-1) taken after its
 * own F step; since open <= 0 this is F(i) = max(F(i-1) + extend,
 * Hpre(i-1) + open + extend) with Hpre the score before the F step, which
 * runs two lanes per word step.  The top band cell restarts the chain with
 * F = NEG_INFINITY + open + extend (:6962-6974): lanes above it are masked
 * out of the chain and the chain is entered so that it holds exactly that
 * value at the top lane.
 *
 * Directions.  Each tie rule compares a with b through m = max(a, b),
 * which the step computes anyway: jump late takes a on a >= b, that is
 * m == a; jump early only on a > b, that is m != b.  min.u16x2(m ^ x, 1)
 * turns the equality of each half into 0 or 1, and one multiply-add moves
 * the two lanes' bits into place: bit k of byte 0 (byte 2) for lane 2k
 * (2k + 1).  Jump late accumulates the negations and flips them at the end
 * of the column.  The result is the W = 16 layout of gdp_internal.h.
 *
 * Bodies.  A steady column (every lane inside the band) needs no lane
 * masks; the general body handles the band edges with per-word masks built
 * from the lane index; the half body skips lanes 0-7 once the top band lane
 * is 8 or more (they never feed an in-band cell again); the bottom-half
 * body skips lanes 8-15 while the bottom band lane is 7 or less, where that
 * is exact (below).  Every body is one
 * run of straight-line code over the eight words (edges are masks, not
 * branches), so the compiler interleaves the words' independent steps:
 * per-word skip branches, tried and measured, split the column into basic
 * blocks and made the kernel a third slower.
 */
#pragma once
#include "gdp_internal.h"

namespace gdp_pk {

constexpr int OFF = 4096;                  /* offset of every value */
constexpr int NEG = -32768 + OFF;          /* the int16 floor (and NEG_INFINITY_INT) */
constexpr uint32_t LOW2 = 0x80008000u;     /* -32768 in both halves: below every value */

__device__ __forceinline__ uint32_t pk (int lo, int hi) { return ((uint32_t) lo & 0xffffu) | ((uint32_t) hi << 16); }
__device__ __forceinline__ uint32_t bc (int v) { return pk(v, v); }
__device__ __forceinline__ int lo16 (uint32_t x) { return (int) (int16_t) (x & 0xffffu); }
__device__ __forceinline__ int hi16 (uint32_t x) { return (int) (int16_t) (x >> 16); }
__device__ __forceinline__ uint32_t add2 (uint32_t a, uint32_t b) {
  uint32_t r;
  asm("add.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t max2 (uint32_t a, uint32_t b) {
  uint32_t r;
  asm("max.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t min2 (uint32_t a, uint32_t b) {
  uint32_t r;
  asm("min.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
/* 1 in each half where a and b differ, else 0 */
__device__ __forceinline__ uint32_t ne01 (uint32_t a, uint32_t b) {
  uint32_t r;
  asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a ^ b), "r"(0x00010001u));
  return r;
}
__device__ __forceinline__ uint32_t addmax (uint32_t a, uint32_t b, uint32_t c) { return __viaddmax_s16x2(a, b, c); }
__device__ __forceinline__ uint32_t prmt (uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
  return r;
}
/* 0xffff in each half whose signed value is negative */
__device__ __forceinline__ uint32_t negmask (uint32_t x) { return prmt(x, x, 0xBB99u); }
/* (x & ~m) | (LOW2 & m): the masked halves become -32768 */
__device__ __forceinline__ uint32_t lowwhere (uint32_t x, uint32_t m) { return (x & ~m) | (LOW2 & m); }
/* lane indices of word k, and their negations */
__device__ __forceinline__ constexpr uint32_t lanes2 (int k) { return (uint32_t) (2 * k) | ((uint32_t) (2 * k + 1) << 16); }
__device__ __forceinline__ constexpr uint32_t neglanes2 (int k) {
  return ((uint32_t) (-2 * k) & 0xffffu) | ((uint32_t) (-2 * k - 1) << 16);
}
/* 0 in each half equal to 0, else 1 (halves read unsigned) */
__device__ __forceinline__ uint32_t nz01 (uint32_t x) {
  uint32_t r;
  asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(0x00010001u));
  return r;
}
/* Bits of the lanes lo..hi in the accumulator layout: lane 2j at bit j,
   lane 2j + 1 at bit 16 + j (0 when the range is empty); no branches, so
   the column stays one run of straight-line code. */
__device__ __forceinline__ uint32_t lanes_acc (int lo, int hi) {
  lo = max(lo, 0);
  hi = min(hi, 15);
  const int e0 = (lo + 1) >> 1, e1 = hi >> 1, o0 = lo >> 1, o1 = (hi - 1) >> 1;
  const uint32_t even = (0xffu << min(e0, 8)) & (0xffu >> min(max(7 - e1, 0), 8));
  const uint32_t odd = (0xffu << min(o0, 8)) & (0xffu >> min(max(7 - o1, 0), 8));
  return (even & 0xffu) | ((odd & 0xffu) << 16);
}
/* PRMT selector: sign-extended byte `a` of lane 2k (first source) and of
   lane 2k + 1 (second source), as a 16x2 word */
__device__ __forceinline__ constexpr uint32_t sel_class (int a) {
  return (uint32_t) a | ((uint32_t) (a | 8) << 4) | ((uint32_t) (4 + a) << 8) | ((uint32_t) ((4 + a) | 8) << 12);
}
/* the same for class N, whose bytes of lanes 2k, 2k + 1 sit in one word */
__device__ __forceinline__ constexpr uint32_t sel_n (int k) {
  return (uint32_t) ((2 * k) & 3) | ((uint32_t) (((2 * k) & 3) | 8) << 4) | ((uint32_t) ((2 * k + 1) & 3) << 8) |
         ((uint32_t) (((2 * k + 1) & 3) | 8) << 12);
}

}  // namespace gdp_pk

/* The lanes of one block in packed form: profiles as block_start lays them
   out (bytes 0-3 of plo = classes A, C, G, T; the class-N byte of lane i is
   byte i % 4 of phi4[i / 4]), and the (H, E) state of the last swept
   column, each word two lanes, every value + OFF. */
struct PBlock {
  int xlo, last, y0, y1;
  uint32_t plo[16], phi4[4];
  uint32_t H[8], E[8];
};

template <bool LATE>
__device__ __forceinline__ void
pblock_start (PBlock &B, const PairView &v, const gdp_tables_t *tab, int xlo) {
  using namespace gdp_pk;
  B.xlo = xlo;
  const int xhi = min(xlo + 15, v.g.X);
  B.last = xhi - xlo;
  gdp_block_sweep(&v.g, xlo, &B.y0, &B.y1);
#pragma unroll
  for (int j = 0; j < 4; j++) B.phi4[j] = 0;
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const int x = xlo + i;
    /* row 0 and the lanes past the last row take the 'N' row, as in block_start */
    const int q = (x == 0) ? 'N' : (x <= v.llen ? seqch(v.lseq, v.llen, x, v.revp) : 'N');
    B.plo[i] = __ldg(&tab->profq_lo[v.mt][q]);
    const uint32_t hi = __ldg(&tab->profq_hi[v.mt][q]);
    B.phi4[i >> 2] |= (hi & 0xffu) << (8 * (i & 3));
  }
  /* the reference's per-block start: H = NEG_INFINITY - open, E = NEG_INFINITY
     (late) or NEG_INFINITY + 1 (early) (:6783-6799, :7038-7055) */
  const uint32_t h0 = bc(NEG - v.open), e0 = bc(LATE ? NEG : NEG + 1);
#pragma unroll
  for (int k = 0; k < 8; k++) { B.H[k] = h0; B.E[k] = e0; }
}

/* Column class scores of words K0..7: max(score(ka), score(kb)) per lane. */
template <int K0, int K1>
__device__ __forceinline__ void
pcol_scores (const PBlock &B, int ka, int kb, uint32_t ps[8]) {
  using namespace gdp_pk;
  if (ka < 4) {
    const uint32_t s = sel_class(ka);
#pragma unroll
    for (int k = K0; k < K1; k++) ps[k] = prmt(B.plo[2 * k], B.plo[2 * k + 1], s);
  } else {
#pragma unroll
    for (int k = K0; k < K1; k++) ps[k] = prmt(B.phi4[k >> 1], B.phi4[k >> 1], sel_n(k));
  }
  if (kb != ka) {
    if (kb < 4) {
      const uint32_t s = sel_class(kb);
#pragma unroll
      for (int k = K0; k < K1; k++) ps[k] = max2(ps[k], prmt(B.plo[2 * k], B.plo[2 * k + 1], s));
    } else {
#pragma unroll
      for (int k = K0; k < K1; k++) ps[k] = max2(ps[k], prmt(B.phi4[k >> 1], B.phi4[k >> 1], sel_n(k)));
    }
  }
}

/*
 * One swept column y of a full-band block, lanes 2 K0 .. 2 K1 - 1.
 * GEN = false: a steady column (no band edge inside the block: the top
 * band lane is above lane 0 and the bottom one below lane 15, y >= 1, a
 * full block).  GEN = true: any column, with the band edges of
 * block_column: the bottom cell (H from the diagonal only, DIAG
 * directions, :6926-6945), the top cell (F chain restart, :6962-6974), F
 * only on the lanes between them, column 0 (pairscores_col0, :6668-6678).
 * K0 = 4 (the half body): lanes 0-7 lie above the band for good and are
 * skipped (GEN, top lane >= 8).  K1 = 4 (the bottom-half body): lanes
 * 8-15 lie below the band and are skipped (GEN, bottom lane <= 7, not the
 * last column); they keep the block's start values until a general column
 * takes them up again.  Bodies specialised further by band edge (top edge
 * only, bottom edge only) left out the masks of the other edge but made
 * the kernel 17 % slower: six bodies overflow the instruction cache.
 *
 * Why skipping lanes below the band is exact where pair_fill_packed uses
 * it.  The reference computes them, and their values enter the band only
 * as the E of a lane that has just become the bottom cell: the bottom cell
 * ignores its E (H from the diagonal and F, Egap DIAG), and the next column
 * takes max(E, H_bottom + open).  A below-band value is a score of the
 * block's start values (H = NEG_INFINITY - open) plus at most 15 table
 * entries, so it is at most NEG - open + 15 mx, in the reference and here
 * alike.  Every in-band H off column 0 is at least the score of the path
 * from the corner along the main diagonal and then straight along a row
 * or a column (E and F only add to H), that is at least
 * mn min(r, c) + open + extend |r - c| with mn the most negative table
 * entry; a bottom cell has |r - c| = lband.  Where that bound plus open
 * lies above NEG - open + 15 mx (the pair's test in pair_fill_packed) and
 * the block's sweep starts right of column 0 (whose cells are
 * NEG_INFINITY), max(E, H_bottom + open) is H_bottom + open whichever
 * below-band values E came from, and so are its tie-rule direction bits:
 * every in-band score and direction is the reference's.  Only the
 * direction bits and the carries of the skipped below-band cells differ,
 * and nothing reads them (a traceback stops at the bottom cell's DIAG
 * Egap; the next block reads carries from its own sweep's first column
 * on, where lane 15 is in the band).
 *
 *   diag    H[y-1][xlo-1] + OFF (or the row-0 value);
 *   Hc, Fc  H[y][xlo-1] and the F carry of the block above, + OFF.
 * Writes the column's two direction words and, with hd, its 16 scores.
 * Returns the carry for the block below: the last lane's H and its F, packed.
 * With `track`, the in-band scores of the column go into vmax.
 */
template <bool LATE, bool GEN, int K0, int K1 = 8>
__device__ __forceinline__ uint32_t
pcol (PBlock &B, const PairView &v, int y, int diag, int Hc, int Fc, int ka, int kb, uint32_t *dcol,
      int16_t *hd, uint32_t &vmax, bool track, const uint32_t *s_pre) {
  using namespace gdp_pk;
  static_assert(K0 == 0 || GEN, "the half body handles band edges");
  static_assert(K1 == 8 || (GEN && K0 == 0), "the bottom-half body handles band edges");
  const uint32_t open2 = bc(v.open), ext2 = bc(v.ext), oe2 = bc(v.oe), neg2 = bc(NEG);
  const int xlo = B.xlo, last = B.last;
  const int rel = y - xlo;
  const int t = rel - v.uband;       /* top band lane */
  const int bt = rel + v.lband;      /* bottom band lane */
  const bool col0 = GEN && (y == 0);
  const bool hasbot = GEN && y > 0 && bt >= 0 && bt <= last;
  const int s = max(t + 1, 0);       /* first F lane */
  const int fhi = min(bt, last);     /* last F lane */
  const bool cut_hi = GEN && fhi < 15;
  const bool cut_lo = GEN && t >= 1;

  uint32_t ps[8];
  pcol_scores<K0, K1>(B, ka, kb, ps);

  /* E and H steps (:6862-6913); accE / accN collect the Egap / HORIZ bits
     (jump late: their negations) */
  uint32_t accN = 0, accE = 0;
  uint32_t prev = (K0 == 0) ? ((uint32_t) diag << 16) : B.H[K0 - 1];
  const uint32_t negbt2 = bc(-bt);
#pragma unroll
  for (int k = K0; k < K1; k++) {
    const uint32_t Hold = B.H[k], Eold = B.E[k];
    const uint32_t T1 = addmax(Hold, open2, neg2);
    const uint32_t m = max2(Eold, T1);
    accE = ne01(m, LATE ? Eold : T1) * (1u << k) + accE;
    const uint32_t Ee = addmax(m, ext2, neg2);
    const uint32_t dg = prmt(prev, Hold, 0x5432u);    /* (H[2k-1], H[2k]) of the last column */
    prev = Hold;
    uint32_t Hv = addmax(dg, ps[k], neg2);
    if (col0) Hv = (k == 0 && xlo == 0) ? pk(lo16(dg), NEG) : neg2;
    uint32_t Eh = Ee;
    /* the bottom band cell takes the diagonal alone: its E is kept but
       does not enter its H */
    if (hasbot) Eh = min2(Ee, 0x80008000u - nz01(add2(lanes2(k), negbt2)));
    const uint32_t Hp = max2(Eh, Hv);
    accN = ne01(Hp, LATE ? Eh : Hv) * (1u << k) + accN;
    B.H[k] = Hp;
    B.E[k] = Ee;
  }

  /* F chain (:6950-7000), entered with F(0) */
  int Fin;
  uint32_t pF0 = 0;   /* F direction of lane 0 */
  if (t < 0) {
    const int Fp = (xlo == 0) ? NEG : Fc, Hp0 = (xlo == 0) ? NEG : Hc;
    const int a = Hp0 + v.open;
    pF0 = LATE ? (Fp >= a) : (Fp > a);
    Fin = max(Fp, a) + v.ext;
  } else {
    /* the top cell at lane t: the chain holds NEG_INFINITY + open + extend
       there, the lanes above it masked out */
    Fin = NEG + v.oe - t * v.ext;
  }
  uint32_t accV = 0, accFj = 0;
  uint32_t PP = bc(Fin + 2 * K0 * v.ext);     /* (F(2k), F(2k)) */
  const uint32_t c01 = pk(0, v.ext);
  const uint32_t negt2 = bc(-t), fhi2 = bc(fhi);
  uint32_t Flast = 0;
#pragma unroll
  for (int k = K0; k < K1; k++) {
    const uint32_t Hpre = B.H[k];
    uint32_t Hoe = add2(Hpre, oe2);
    if (cut_lo) Hoe = lowwhere(Hoe, negmask(add2(lanes2(k), negt2)));    /* lanes above the top cell */
    const uint32_t Z = prmt(Hoe, LOW2, 0x1054u);                           /* (LOW, Hoe(2k)) */
    const uint32_t Wf = addmax(PP, c01, Z);                                /* (F(2k), F(2k+1)) */
    const uint32_t V = addmax(Wf, ext2, Hoe);                              /* high half: F(2k+2) */
    const uint32_t Y = prmt(Wf, V, 0x7632u);                               /* (F(2k+1), F(2k+2)) */
    /* Fgap of lanes 2k+1 and 2k+2 (lane 2k+1 at bit k, lane 2k+2 at bit
       16 + k): jump late, F(i) == F(i-1) + extend; jump early,
       F(i) != Hpre(i-1) + open + extend */
    accFj = ne01(Y, LATE ? add2(Wf, ext2) : Hoe) * (1u << k) + accFj;
    PP = prmt(V, V, 0x3232u);
    uint32_t Fm = Wf;
    if (cut_hi) Fm = lowwhere(Fm, negmask(add2(fhi2, neglanes2(k))));     /* lanes below the last F lane */
    const uint32_t Hn = max2(Hpre, Fm);
    accV = ne01(Hn, LATE ? Fm : Hpre) * (1u << (8 + k)) + accV;
    B.H[k] = Hn;
    if (k == 7) Flast = Wf;
  }

  /* the direction words (W = 16 layout of gdp_internal.h) */
  const uint32_t comp = lanes_acc(2 * K0, 2 * K1 - 1);         /* lanes computed */
  /* lanes with an F step: s_pre[i] = lanes_acc(0, i - 1), so lanes lo..hi
     are s_pre[hi + 1] & ~s_pre[lo] (0 <= lo <= 16, -1 <= hi <= 15) */
  const uint32_t frange = s_pre[fhi + 1] & ~s_pre[max(s, 2 * K0)];
  uint32_t nb = LATE ? (accN ^ comp) : accN;
  uint32_t vb = LATE ? (accV ^ (comp << 8)) : accV;
  uint32_t eb = LATE ? (accE ^ comp) : accE;
  uint32_t fj = accFj;
  if (LATE) fj ^= (((1u << K1) - 1u) & ~((1u << K0) - 1u)) * 0x10001u;
  const uint32_t odd = fj & 0xffu;                              /* lanes 2k+1 */
  const uint32_t even = ((fj >> 16) << 1) & 0xfeu;              /* lanes 2k+2 */
  uint32_t fb = (even | (odd << 16)) & ~1u;
  if (!LATE && v.open == 0) fb = 0;   /* jump early with open 0: F never beats H + open */
  fb |= (s == 0) ? pF0 : 0u;
  nb = (nb & comp) | (vb & (frange << 8));
  eb = (eb & comp) | ((fb & frange) << 8);
  if (hasbot) eb &= ~(s_pre[bt + 1] & ~s_pre[bt]);
  *reinterpret_cast<uint2 *>(dcol) = make_uint2(prmt(nb, eb, 0x5410u), prmt(nb, eb, 0x7632u));

  if (track) {
#pragma unroll
    for (int k = K0; k < K1; k++) {
      uint32_t h = B.H[k];
      if (cut_lo) h = lowwhere(h, negmask(add2(lanes2(k), negt2)));
      if (cut_hi) h = lowwhere(h, negmask(add2(fhi2, neglanes2(k))));
      vmax = max2(vmax, h);
    }
  }
  if (hd != nullptr) {
    uint32_t *h32 = reinterpret_cast<uint32_t *>(hd);
#pragma unroll
    for (int k = 0; k < 8; k++) h32[k] = add2(B.H[k], bc(-OFF));
  }
  return pk(hi16(B.H[7]), hi16(Flast));
}

/*
 * One pair of a full-band 16-bit fill on packed lanes: MODE 0 a plain
 * fill, MODE 1 the 16-bit pass of a rerun pair (it also records whether an
 * in-band score reaches PairView::lim).  The block sweep and the next
 * column's prefetch are those of fill_thread_kernel; the carry from a
 * block to the next is one word, the last lane's H and F (+ OFF).  Every
 * pair of a launch of this kernel is packed, so the per-slot scratch is
 * addressed in words: half the bytes of the int2 carries.
 */
template <bool LATE, int MODE>
__device__ __forceinline__ void
pair_fill_packed (const FillParams &P, int pi, gdp_meta_t *mp, const PairView &v, const int8_t *s_nt2int,
                  const uint32_t *s_pre, int64_t slot) {
  using namespace gdp_pk;
  static_assert(MODE == 0 || MODE == 1, "plain fills and the 16-bit pass of rerun pairs");
  uint32_t *dir = P.dirs + mp->dir16;
  uint32_t *sc = reinterpret_cast<uint32_t *>(P.scratch) + slot;
  const int64_t scs = P.nslots;
  int final_score = -32768;
  uint32_t vmax = LOW2;
  /* the pair's bound for skipping lanes below the band (pcol): every
     bottom cell, at least mn min(r, c) + open + extend lband, plus open
     lies above NEG_INFINITY - open + 15 mx; no dump asked for */
  const bool skip_ok = P.hdump == nullptr &&
                       P.tab_mn * min(v.g.X, v.g.Y) + 3 * v.open + v.ext * v.lband - 15 * P.tab_mx > -32768 + 64;
  for (int xlo = 0; xlo <= v.g.X; xlo += 16) {
    PBlock B;
    pblock_start<LATE>(B, v, P.tab, xlo);
    if (B.y1 < B.y0) continue;
    /* ... and the block's sweep starts right of column 0 */
    const bool skip_bot = skip_ok && B.y0 >= 1;
    /* a 16-bit pass that has already seen an in-band score at the limit
       has decided the rerun: no further tracking */
    const bool need_track = MODE == 1 && max(lo16(vmax), hi16(vmax)) < v.lim + OFF;
    int bot_prev = NEG;   /* H[y-1][xlo-1] from the block above */
    if (xlo > 0 && B.y0 > 0) bot_prev = lo16(sc[(int64_t) (B.y0 - 1) * scs]);
    int ka, kb;
    column_classes<GDP_FULL>(v, s_nt2int, B.y0, ka, kb);
    uint32_t above = pk(NEG, NEG);
    if (xlo > 0) above = sc[(int64_t) B.y0 * scs];
    /* column y + 1's genome characters and carry, loaded one column before
       they are classified / used (two columns ahead of their use) */
    int ra = 'N', rb = 'N';
    uint32_t above1 = pk(NEG, NEG);
    if (B.y0 + 1 <= B.y1) {
      ra = seqch(v.sseq, v.slen, B.y0 + 1, v.revp);
      rb = seqch(v.salt, v.slen, B.y0 + 1, v.revp);
      if (xlo > 0) above1 = sc[(int64_t) (B.y0 + 1) * scs];
    }
    uint32_t *dcol = dir;
    /* the block's steady columns: no band edge inside the block */
    const int ys0 = max(xlo + 16 - v.lband, 1), ys1 = (B.last == 15) ? xlo + v.uband - 1 : -1;
    for (int y = B.y0; y <= B.y1; y++) {
      /* column y + 1 from the characters loaded last column, and the
         loads for column y + 2 */
      const int ka2 = s_nt2int[ra], kb2 = s_nt2int[rb];
      const uint32_t above2 = above1;
      if (y + 2 <= B.y1) {
        ra = seqch(v.sseq, v.slen, y + 2, v.revp);
        rb = seqch(v.salt, v.slen, y + 2, v.revp);
        if (xlo > 0) above1 = sc[(int64_t) (y + 2) * scs];
      }
      int diag;
      if (y == 0) diag = (xlo == 0) ? OFF : NEG;   /* the corner scores 0 */
      else diag = (xlo == 0) ? NEG : bot_prev;
      bot_prev = lo16(above);
      int16_t *hd = (P.hdump != nullptr) ? P.hdump + (dcol - P.dirs) * 8 : nullptr;
      const bool track = need_track && y >= 1 && y >= v.reach_from && xlo + B.last >= v.reach_from;
      const int t = y - xlo - v.uband;
      uint32_t out;
      if (y >= ys0 && y <= ys1)
        out = pcol<LATE, false, 0>(B, v, y, diag, lo16(above), hi16(above), ka, kb, dcol, hd, vmax, track, s_pre);
      else if (y >= 1 && t >= 8 && y != v.g.Y)
        out = pcol<LATE, true, 4>(B, v, y, diag, lo16(above), hi16(above), ka, kb, dcol, hd, vmax, track, s_pre);
      else if (skip_bot && y - xlo + v.lband <= 7 && y != v.g.Y)
        out = pcol<LATE, true, 0, 4>(B, v, y, diag, lo16(above), hi16(above), ka, kb, dcol, nullptr, vmax, track, s_pre);
      else
        out = pcol<LATE, true, 0>(B, v, y, diag, lo16(above), hi16(above), ka, kb, dcol, hd, vmax, track, s_pre);
      sc[(int64_t) y * scs] = out;
      if (y == v.g.Y) {
        const int L = v.g.X - xlo;
        if (L >= 0 && L <= B.last) {
          /* word L / 2 through all-ones / zero masks the compiler cannot
             turn into a runtime array index (which would put the block's
             words in local memory for the whole sweep) */
          uint32_t w = 0;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            uint32_t m;
            asm("{.reg .pred p; setp.eq.s32 p, %1, %2; selp.b32 %0, -1, 0, p;}" : "=r"(m) : "r"(k), "r"(L >> 1));
            w |= B.H[k] & m;
          }
          final_score = ((L & 1) ? hi16(w) : lo16(w)) - OFF;
        }
      }
      dcol += 2;
      ka = ka2; kb = kb2; above = above2;
    }
    dir = dcol;
  }
  const bool reached = MODE == 1 && max(lo16(vmax), hi16(vmax)) >= v.lim + OFF;
  fill_finish<16, MODE>(P, pi, mp, v.g, reached, final_score);
}

#ifndef GDP_PACKED_MINB
#define GDP_PACKED_MINB 4
#endif

/*
 * The packed fill of one thread-per-pair kind of full-band 16-bit pairs:
 * every pair of the list with min(rlength, glength) <= FillParams::
 * packed_len; fill_thread_kernel takes the others.
 */
template <bool LATE, int MODE>
__global__ void __launch_bounds__(128, GDP_PACKED_MINB)
fill_packed_kernel (FillParams P) {
  __shared__ int8_t s_nt2int[128];
  __shared__ uint32_t s_pre[17];   /* lanes_acc(0, i - 1): the lane-range masks of pcol */
  for (int i = threadIdx.x; i < 128; i += blockDim.x) s_nt2int[i] = P.tab->nt2int[i];
  if (threadIdx.x < 17) s_pre[threadIdx.x] = gdp_pk::lanes_acc(0, (int) threadIdx.x - 1);
  __syncthreads();
  const int64_t slot = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *P.count;
  for (int64_t li = slot; li < n; li += P.nslots) {
    const int pi = __ldg(P.list + li);
    if (pi < 0) continue;   /* padding: warps hold pairs of one band width */
    const gdp_pair_t p = P.pairs[pi];
    if (min(p.rlength, p.glength) > P.packed_len) continue;
    PairView v;
    pair_view<16, GDP_FULL>(p, P.arena, v);
    v.reach_from = (int) ((P.reach_from4 >> (8 * (v.mt & 3))) & 255u);
    v.endmode = 0;
    pair_fill_packed<LATE, MODE>(P, pi, P.meta + pi, v, s_nt2int, s_pre, slot);
  }
}

/* The longest min(rlength, glength) the packed fill takes under tables t:
   (min + 16) times the largest entry must stay below 32767 - OFF, and the
   most negative entry above -200 (no add below the offset floor wraps). */
static inline int
gdp_packed_len_of (const gdp_tables_t *t) {
  int lim = 1 << 30;
  for (int mt = 0; mt < 4; mt++) {
    int mx = -32768, mn = 32767;
    for (int a = 0; a < 128; a++)
      for (int b = 0; b < 128; b++) {
        mx = mx > t->pd[mt][a][b] ? mx : t->pd[mt][a][b];
        mn = mn < t->pd[mt][a][b] ? mn : t->pd[mt][a][b];
      }
    int len = (mx <= 0) ? (1 << 30) : (32767 - gdp_pk::OFF) / mx - 16;
    if (mn < -200 || mx > 127) len = -1;
    lim = lim < len ? lim : len;
  }
  return lim;
}
