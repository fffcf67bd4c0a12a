/*
 * fill_thread.cuh -- one-thread-per-pair fill kernels for sm_100a.
 *
 * Each thread runs one alignment pair through exactly the block sweep of
 * the reference (src/dynprog_simd.c): blocks of W lanes (W = 16 for the
 * 16-bit fills, 32 for the 8-bit fills), each block swept over its column
 * range, every lane of a block computed for every swept column (including
 * the lanes outside the band, whose values reach the in-band E values),
 * then for the full band the scalar F loop over the in-band lanes.  A
 * block's W lane states (H, E) and their query profiles live in registers;
 * the only state that crosses blocks -- the last lane's final H and the F
 * carry FF (src/dynprog_simd.c:6999) -- goes through a per-thread scratch
 * column in global memory, interleaved across threads so a warp's accesses
 * coalesce.
 *
 * Saturating int8/int16 lane arithmetic is done in int32 with explicit
 * clamps (the F chain is plain int, as in the reference).  Directions are
 * packed to 4 bits per cell (see gdp_internal.h) and written as W/8 words
 * per block column.
 */
#pragma once
#include "gdp_internal.h"

#define GDP_SEL(k) ((uint32_t) (k) | ((uint32_t) ((k) | 8) << 4) | ((uint32_t) ((k) | 8) << 8) | ((uint32_t) ((k) | 8) << 12))

/* Sign-extended byte `sel` of {hi:lo} (PTX prmt, default mode). */
__device__ __forceinline__ int
prof_byte (uint32_t lo, uint32_t hi, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
  return (int) r;
}

/* Signed byte-wise max of two packed profiles (lower fill folds g, g_alt). */
__device__ __forceinline__ uint32_t
bytemax (uint32_t a, uint32_t b) {
  uint32_t r = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int x = (int) (int8_t) (a >> (8 * k)), y = (int) (int8_t) (b >> (8 * k));
    r |= (uint32_t) (uint8_t) (x > y ? x : y) << (8 * k);
  }
  return r;
}

/* Character at 1-based position i of a sequence, honouring revp. */
__device__ __forceinline__ int
seqch (const char *base, int len, int i, bool revp) {
  return (int) (uint8_t) __ldg(base + (revp ? len - i : i - 1)) & 127;
}

struct FillParams {
  const gdp_pair_t *pairs;
  const char *arena;
  const int32_t *list;     /* pair indices of this group */
  const int32_t *count;    /* device: number of entries in list */
  uint32_t *dirs;          /* direction words */
  int16_t *hdump;          /* debug (may be NULL): score of every swept cell, 8 per direction word */
  gdp_meta_t *meta;
  gdp_result_t *res;
  int2 *scratch;           /* [y * nslots + slot] = (H of the block's last lane, FF) */
  int64_t nslots;
  int scratch_rows;        /* columns available per slot */
  const gdp_tables_t *tab;
  /* Byte k: for mismatch type k, the smallest row and column index at which
     an in-band score can reach 127 (at most 255).  Every score is the score
     of a path from the matrix corner, whose own score is at most one table
     entry (upper and lower fills), so H(r, c) <= (min(r, c) + 1) times the
     table's largest entry.  The in-band 127 checks (MODE != 0) skip cells
     below it; 0 checks every cell. */
  uint32_t reach_from4;
  /* Byte k: for mismatch type k, how far a 16-bit lower-fill score can lie
     above the 8-bit one at the same cell.  The reference's 8-bit lower
     fill scores its corner against character code 4 (src/dynprog_simd.c:
     5459), the 16-bit one against 'N' (:8689), so the 16-bit scores of
     paths from the corner are that much higher; elsewhere every operation
     is monotone and the 8-bit scores are never the lower ones.  A 16-bit
     pass (MODE 1) of a lower fill proves the 8-bit overflow only from
     127 + this slack. */
  uint32_t lower_slack4;
  /* Full-band 16-bit pairs (plain fills and the 16-bit pass of rerun
     pairs) with min(rlength, glength) at most this run the packed two-lane
     fill (fill_packed_kernel, launched first for such a kind); the one-lane-
     per-register fill_thread_kernel skips them and takes the others (every
     pair when this is below 0). */
  int packed_len;
  /* the smallest (at most 0) and the largest (at least 0) entry of the
     substitution tables over every mismatch type (fill_packed_kernel's
     bound for skipping lanes below the band) */
  int tab_mn, tab_mx;
};

/* Lanes lo..hi (0 <= lo <= hi <= 31) as a bit mask. */
__device__ __forceinline__ uint32_t
lane_range (int lo, int hi) {
  const uint32_t upto = (hi >= 31) ? 0xffffffffu : ((1u << (hi + 1)) - 1u);
  return upto & ~((1u << lo) - 1u);
}

/* max(a, b) and the tie rule of the reference: jump late takes a on a >= b,
   jump early only on a > b. */
template <bool LATE>
__device__ __forceinline__ int
tie_max (int a, int b, bool &a_wins) {
  if (LATE) return __vibmax_s32(a, b, &a_wins);
  bool q;
  const int m = __vibmax_s32(b, a, &q);
  a_wins = !q;
  return m;
}

/* Per-pair constants of a fill at block height W. */
struct PairView {
  gdp_geom_t g;
  bool revp;
  int open, ext, oe, mt, lband, uband;
  int dlo, dhi;                  /* in-band lanes of column y: y - dhi <= x <= y + dlo */
  int reach_from;                /* FillParams::reach_from of the pair's mismatch type */
  int lim;                       /* an in-band score at or above this proves the 8-bit overflow */
  int endmode;                   /* 0, or 1 (GDP_FLAG_ENDPOINT), or 2 (GDP_FLAG_ENDPOINT_QEND) */
  const char *lseq, *lalt, *sseq, *salt;
  int llen, slen;
};

template <int W, int VARIANT>
__device__ __forceinline__ void
pair_view (const gdp_pair_t &p, const char *arena, PairView &v) {
  gdp_geom_of(&p, W, &v.g);
  v.revp = (p.flags & GDP_FLAG_REVP) != 0;
  v.open = p.open; v.ext = p.extend; v.oe = p.open + p.extend;
  v.mt = p.mismatchtype;
  v.lband = p.lband; v.uband = p.uband;
  v.dlo = (VARIANT == GDP_FULL) ? p.lband : 0;
  v.dhi = (VARIANT == GDP_FULL) ? p.uband : (VARIANT == GDP_UPPER ? p.uband : p.lband);
  v.lim = 127;
  v.lseq = arena + (VARIANT == GDP_LOWER ? p.gseq : p.rseq);
  v.lalt = arena + (VARIANT == GDP_LOWER ? p.gseq_alt : p.rseq);
  v.llen = (VARIANT == GDP_LOWER) ? p.glength : p.rlength;
  v.sseq = arena + (VARIANT == GDP_LOWER ? p.rseq : p.gseq);
  v.salt = arena + (VARIANT == GDP_LOWER ? p.rseq : p.gseq_alt);
  v.slen = (VARIANT == GDP_LOWER) ? p.rlength : p.glength;
}

/* One half of the end-gap endpoint search (GDP_FLAG_ENDPOINT*;
   find_best_endpoint_{8,16}, src/dynprog_end.c:143-294, and
   find_best_endpoint_to_queryend_indels_{8,16}, :358-508).  The reference
   scans cells in row-then-column order and keeps the first best cell with
   a score above the start (jump early) or the last one from the start up
   (jump late).  That winner is the best score with the smallest (early) or
   largest (late) (row, column) among the cells that pass, so the fill can
   offer its cells in any order. */
struct EndBest {
  int score, r, c;
  bool found;
};

template <bool LATE>
__device__ __forceinline__ void
end_offer (EndBest &b, int h, int r, int c, int start) {
  if (LATE ? (h < start) : (h <= start)) return;
  bool better;
  if (!b.found || h > b.score) better = true;
  else if (h < b.score) better = false;
  else if (LATE) better = (r > b.r) || (r == b.r && c > b.c);
  else better = (r < b.r) || (r == b.r && c < b.c);
  if (better) { b.score = h; b.r = r; b.c = c; b.found = true; }
}

/* Offers the cells of swept column y of block xlo to the search: upper
   fills their cells with c >= r (lanes are rows), lower fills their cells
   with c < r (lanes are genome columns); the last-row search takes row
   rlength only.  H holds the column's final scores. */
template <int W, int VARIANT, bool LATE, class BlockT>
__device__ __forceinline__ void
end_column (EndBest &b, const BlockT &B, const PairView &v, int y, int start) {
  const int xlo = B.xlo, last = B.last;
  if (y < 1) return;
  int lo, hi;
  if (VARIANT == GDP_UPPER) {
    lo = max(1, y - v.uband) - xlo;
    hi = min(y, v.g.X) - xlo;
    if (v.endmode == 2) lo = max(lo, v.g.X - xlo), hi = min(hi, v.g.X - xlo);
  } else {
    if (v.endmode == 2 && y != v.g.Y) return;
    lo = max(1, y - v.lband) - xlo;
    hi = min(y - 1, v.g.X) - xlo;
  }
  lo = max(lo, 0);
  hi = min(hi, last);
  if (lo > hi) return;
  /* The column's own winner first: its cells share the column y, and the
     lane order is the scan order among them (upper: rows; lower: genome
     columns of one row), so the first lane with the column maximum (jump
     early) or the last (jump late) is the one to offer. */
  int cm = INT_MIN, ci = -1;
#pragma unroll
  for (int i = 0; i < W; i++) {
    const int h = B.H[i];
    const bool take = (i >= lo) & (i <= hi) & (LATE ? (h >= cm) : (h > cm));
    cm = take ? h : cm;
    ci = take ? i : ci;
  }
  if (VARIANT == GDP_UPPER) end_offer<LATE>(b, cm, xlo + ci, y, start);
  else end_offer<LATE>(b, cm, y, xlo + ci, start);
}

/* Classes (0..4) of swept column y for the two genome strings (lower: the
   query class twice). */
template <int VARIANT>
__device__ __forceinline__ void
column_classes (const PairView &v, const int8_t *nt2int, int y, int &ka, int &kb) {
  if (VARIANT == GDP_LOWER) {
    ka = kb = (y == 0) ? 4 : nt2int[seqch(v.sseq, v.slen, y, v.revp)];
  } else if (y == 0) {
    ka = kb = 4;
  } else {
    ka = nt2int[seqch(v.sseq, v.slen, y, v.revp)];
    kb = nt2int[seqch(v.salt, v.slen, y, v.revp)];
  }
}

/* The W lanes of one block: profiles and the (H, E) state of the last
   swept column.  Fully unrolled loops keep the arrays in registers. */
template <int W>
struct Block {
  int xlo, xhi, last, y0, y1;
  uint32_t plo[W], phi4[W / 4];
  int H[W], E[W];
};

/* Loads the lane profiles of block xlo and resets its state to the
   reference's per-block start: H = NEG - open, E = NEG (late) / NEG + 1
   (early) (src/dynprog_simd.c:6783-6799, :7038-7055). */
template <int W, int VARIANT, bool LATE>
__device__ __forceinline__ void
block_start (Block<W> &B, const PairView &v, const gdp_tables_t *tab, int xlo) {
  constexpr int LO = (W == 32) ? -128 : -32768;
  B.xlo = xlo;
  B.xhi = min(xlo + W - 1, v.g.X);
  B.last = B.xhi - xlo;
  gdp_block_sweep(&v.g, xlo, &B.y0, &B.y1);
  /* bytes 0..3 of plo = scores against classes A,C,G,T; the class-N score
     of lane i is byte (i & 3) of phi4[i >> 2] */
#pragma unroll
  for (int j = 0; j < W / 4; j++) B.phi4[j] = 0;
#pragma unroll
  for (int i = 0; i < W; i++) {
    const int x = xlo + i;
    uint32_t lo, hi;
    if (VARIANT != GDP_LOWER) {
      const int q = (x == 0) ? 'N' : (x <= v.llen ? seqch(v.lseq, v.llen, x, v.revp) : 'N');
      lo = __ldg(&tab->profq_lo[v.mt][q]);
      hi = __ldg(&tab->profq_hi[v.mt][q]);
    } else if (x == 0) {
      /* 16-bit: column 0 scores against 'N' (:8689); 8-bit: against code 4 (:5459) */
      const int c0 = (W == 32) ? 4 : 'N';
      lo = __ldg(&tab->profg_lo[v.mt][c0]);
      hi = __ldg(&tab->profg_hi[v.mt][c0]);
    } else if (x <= v.llen) {
      const int a = seqch(v.lseq, v.llen, x, v.revp), b = seqch(v.lalt, v.llen, x, v.revp);
      lo = bytemax(__ldg(&tab->profg_lo[v.mt][a]), __ldg(&tab->profg_lo[v.mt][b]));
      hi = bytemax(__ldg(&tab->profg_hi[v.mt][a]), __ldg(&tab->profg_hi[v.mt][b]));
    } else {
      lo = 0; hi = 0;
    }
    B.plo[i] = lo;
    B.phi4[i >> 2] |= (hi & 0xffu) << (8 * (i & 3));
    B.H[i] = LO - v.open;
    B.E[i] = LATE ? LO : LO + 1;
  }
}

/*
 * One swept column y of a block: the vector step (E, then H from the
 * diagonal; src/dynprog_simd.c:6862-6913), the bottom-cell fix
 * (:6926-6945) or the upper/lower E mask and diagonal fix (:7921-7969),
 * and for the full band the F loop over the in-band lanes with the top-cell
 * special case (:6950-7000).  Band geometry is reduced to lane masks that
 * are uniform over the column.
 *
 *   diag   H[y-1][xlo-1] of the block above (final), or the reference's
 *          row/column-0 values;
 *   above  (H[y][xlo-1], FF[y]) of the block above.
 * Writes the column's direction words to dcol (and scores to hd when not
 * NULL).  Returns (H of the last lane, F carry) for the block below.
 *
 * LS > 0 (full band only): lanes 0 .. LS-1 lie above the band's top lane
 * and are skipped.  Such lanes have left the band for good: their H feeds
 * only the diagonal of the lane below at the next column, which is above
 * the band too, and their E only their own row, so no in-band cell reads
 * them again.  Their scores keep the values of the last column computed
 * and their direction bits are 0; a traceback reaching such a cell stops
 * with GDP_ERR_BAND by position (the reference reads stale scratch there).
 * The caller takes this body only when the column's top lane is at least
 * LS, the column is not the last one, and no score dump is asked for.
 */
template <int W, int VARIANT, bool LATE, int MODE, int LS = 0>
__device__ __forceinline__ int2
block_column (Block<W> &B, const PairView &v, int y, int diag, int2 above, int ka, int kb,
              uint32_t *dcol, int16_t *hd, bool &reached, int &final_score) {
  static_assert(LS == 0 || VARIANT == GDP_FULL, "lanes above the band exist in full-band fills");
  constexpr int LO = (W == 32) ? -128 : -32768;
  constexpr int HI = (W == 32) ? 127 : 32767;
  constexpr int WORDS = W / 8;
  const int open = v.open, ext = v.ext;
  const int xlo = B.xlo, last = B.last;
  const bool col0 = (VARIANT == GDP_FULL) && (y == 0);
  /* PRMT selectors; class N (4) reads byte 4 + (i & 3) of {phi4, plo} */
  uint32_t sA[4], sB[4];
  {
    const uint32_t dA = (ka == 4) ? 0x1111u : 0u, dB = (kb == 4) ? 0x1111u : 0u;
    sA[0] = GDP_SEL(ka); sB[0] = GDP_SEL(kb);
#pragma unroll
    for (int k = 1; k < 4; k++) { sA[k] = sA[k - 1] + dA; sB[k] = sB[k - 1] + dB; }
  }
  /* lane masks of this column */
  const int rel = y - xlo;                       /* lane index of x == y */
  uint32_t fmask = 0, topmask = 0, botmask = 0, emask = 0, dmask = 0;
  if (VARIANT == GDP_FULL) {
    const int t = rel - v.uband, bt = rel + v.lband;  /* top and bottom lanes */
    const int flo = max(0, t + 1), fhi = min(bt, last);
    if (fhi >= flo) fmask = lane_range(flo, fhi);
    if (t >= 0 && t <= last) topmask = 1u << t;
    if (y > 0 && bt >= 0 && bt <= last) botmask = 1u << bt;
  } else {
    if (rel <= W - 1) emask = lane_range(max(rel, 0), W - 1);
    if (rel >= 0 && rel <= last) dmask = 1u << rel;
  }
  uint32_t w[WORDS];
#pragma unroll
  for (int j = 0; j < WORDS; j++) w[j] = 0;

  if (LS > 0) diag = B.H[LS - 1];   /* the skipped lane above: its last computed score */
#pragma unroll
  for (int i = LS; i < W; i++) {
    const uint32_t bit = 1u << i;
    const int Hold = B.H[i];
    int Eold = B.E[i];
    if (VARIANT != GDP_FULL && (emask & bit)) Eold = LO;
    const int T1 = __viaddmax_s32(Hold, open, LO);
    bool pE;
    const int m = tie_max<LATE>(Eold, T1, pE);
    int Ee = __viaddmax_s32(m, ext, LO);
    if (VARIANT != GDP_FULL && (emask & bit)) Ee = LO;
    int ps;
    if (VARIANT == GDP_FULL && col0) {
      ps = (xlo + i == 0) ? 0 : LO;     /* pairscores_col0 (:6668-6678) */
    } else if (VARIANT == GDP_LOWER) {
      ps = prof_byte(B.plo[i], B.phi4[i >> 2], sA[i & 3]);
    } else {
      ps = max(prof_byte(B.plo[i], B.phi4[i >> 2], sA[i & 3]), prof_byte(B.plo[i], B.phi4[i >> 2], sB[i & 3]));
    }
    const int Hv = min(__viaddmax_s32(diag, ps, LO), HI);
    diag = Hold;
    bool pN;
    int Hn = tie_max<LATE>(Ee, Hv, pN);
    if (VARIANT == GDP_FULL) {
      if (botmask & bit) { Hn = Hv; pE = false; pN = false; }
    } else {
      if (dmask & bit) { pE = false; pN = false; }
    }
    B.H[i] = Hn;
    B.E[i] = Ee;
    if (pE) w[gdp_dir_word(W, i)] |= 1u << (16 + gdp_dir_bit(W, i));
    if (pN) w[gdp_dir_word(W, i)] |= 1u << gdp_dir_bit(W, i);
  }
  int2 out;
  if (VARIANT == GDP_FULL) {
    int Fp, Hp;
    if (xlo == 0 || y >= xlo + v.uband) { Fp = GDP_NEGINT; Hp = GDP_NEGINT; }
    else { Fp = above.y; Hp = above.x; }
#pragma unroll
    for (int i = LS; i < W; i++) {
      const uint32_t bit = 1u << i;
      if (topmask & bit) {
        Fp = GDP_NEGINT + v.oe;
        Hp = B.H[i];
      } else if (fmask & bit) {
        bool pF, pV;
        const int F = tie_max<LATE>(Fp, Hp + open, pF) + ext;
        const int Hn = tie_max<LATE>(F, B.H[i], pV);
        B.H[i] = Hn;
        Hp = Hn;
        Fp = F;
        if (pF) w[gdp_dir_word(W, i)] |= 1u << (24 + gdp_dir_bit(W, i));
        if (pV) w[gdp_dir_word(W, i)] |= 1u << (8 + gdp_dir_bit(W, i));
      }
    }
    out = make_int2(B.H[W - 1], Fp);
  } else {
    out = make_int2(B.H[W - 1], 0);
  }
  if (MODE != 0 && !reached && y >= 1 && y >= v.reach_from && xlo + last >= v.reach_from) {
    const int dl = max(rel - v.dhi, (xlo == 0) ? 1 : 0), dh = min(rel + v.dlo, last);
    if (dh >= dl) {
      const uint32_t dom = lane_range(max(dl, 0), dh);
#pragma unroll
      for (int i = LS; i < W; i++)
        if ((dom & (1u << i)) && B.H[i] >= v.lim) reached = true;
    }
  }
  if (y == v.g.Y && v.g.X - xlo >= 0 && v.g.X - xlo < W) {
    /* lane X - xlo through all-ones / zero masks the compiler cannot turn
       into a runtime array index (which would keep B.H in local memory) */
    const int L = v.g.X - xlo;
    int fs = 0;
#pragma unroll
    for (int i = 0; i < W; i++) {
      int m;
      asm("{.reg .pred p; setp.eq.s32 p, %1, %2; selp.b32 %0, -1, 0, p;}" : "=r"(m) : "r"(i), "r"(L));
      fs |= B.H[i] & m;
    }
    final_score = fs;
  }
  if (hd != nullptr) {
#pragma unroll
    for (int i = 0; i < W; i++) hd[i] = (int16_t) B.H[i];
  }
  if (WORDS == 2) {
    *reinterpret_cast<uint2 *>(dcol) = make_uint2(w[0], w[1]);
  } else {
    *reinterpret_cast<uint4 *>(dcol) = make_uint4(w[0], w[1], w[WORDS > 2 ? 2 : 0], w[WORDS > 3 ? 3 : 0]);
  }
  return out;
}

/* Writes the per-pair outcome of a fill (see MODE). */
template <int W, int MODE>
__device__ __forceinline__ void
fill_finish (const FillParams &P, int pi, gdp_meta_t *mp, const gdp_geom_t &g, bool reached, int final_score,
             const EndBest *eb = nullptr) {
  int y0l, y1l;
  gdp_block_sweep(&g, (g.X / W) * W, &y0l, &y1l);
  /* the final cell was filled: swept, and for the full band not above the
     band's top (the lanes above the band are not kept once they leave it) */
  const bool swept = (g.Y >= y0l && g.Y <= y1l) && !(g.variant == GDP_FULL && g.Y - g.X > g.uband);
  if (!swept) final_score = (W == 32) ? -128 : -32768;
  if (MODE == 1) {
    mp->maxh16 = reached ? 127 : -32768;   /* >= 127 iff an in-band 16-bit score reached 127 */
    mp->final16 = final_score;
  }
  if (MODE == 2) {
    /* the result takes the 8-bit outcome after both passes
       (apply_rerun8_kernel): the two may run at the same time */
    const bool overflow = reached || final_score <= -128 + 30;
    mp->status8 = overflow ? 1 : 0;
    mp->final8 = final_score;
  } else {
    gdp_result_t *r = P.res + pi;
    r->score = final_score;
    r->precision = W == 16 ? 16 : 8;
    r->rerun = (MODE == 1) ? 1 : 0;
    /* only a traceback from the final cell needs it: an end-gap half, or
       the lower fill of a gap with glength > rlength (a cDNA gap's lower
       half), holds none and keeps GDP_OK with score NEG_INFINITY, the
       cell the reference leaves unwritten.  A traceback from another cell
       (an end gap's best cell) checks its own cells as it walks. */
    const gdp_pair_t &pp = P.pairs[pi];
    if (!swept && eb == nullptr && (pp.flags & GDP_FLAG_TRACEBACK) && pp.tb_r == pp.rlength &&
        pp.tb_c == pp.glength)
      r->status = GDP_ERR_BAND;
    if (eb != nullptr) {
      r->end_score = eb->score;
      r->end_r = eb->r;
      r->end_c = eb->c;
      r->end_found = eb->found ? 1 : 0;
    }
  }
}

/*
 * A steady column: every lane of a full block lies inside the band.  For
 * the full fill that means no top and no bottom band cell in the block
 * (lane 0 below the top edge, lane W-1 above the bottom edge); for the
 * upper and lower fills, the diagonal has passed the block (no E mask, no
 * diagonal fix).  Those columns need none of the lane masks of
 * block_column, and in the bands of long pairs they are most of the work.
 * The result equals block_column's for the same column.  `vmax` collects
 * the in-band scores (MODE != 0) when `track` says that the column and the
 * block can hold a score of 127 (FillParams::reach_from).
 */
template <int W, int VARIANT, bool LATE, int MODE>
__device__ __forceinline__ int2
block_column_steady (Block<W> &B, const PairView &v, int diag, int2 above, int ka, int kb, uint32_t *dcol,
                     int &vmax, bool track) {
  constexpr int LO = (W == 32) ? -128 : -32768;
  constexpr int HI = (W == 32) ? 127 : 32767;
  constexpr int WORDS = W / 8;
  const int open = v.open, ext = v.ext;
  uint32_t sA[4], sB[4];
  {
    const uint32_t dA = (ka == 4) ? 0x1111u : 0u, dB = (kb == 4) ? 0x1111u : 0u;
    sA[0] = GDP_SEL(ka); sB[0] = GDP_SEL(kb);
#pragma unroll
    for (int k = 1; k < 4; k++) { sA[k] = sA[k - 1] + dA; sB[k] = sB[k - 1] + dB; }
  }
  uint32_t w[WORDS];
#pragma unroll
  for (int j = 0; j < WORDS; j++) w[j] = 0;
#pragma unroll
  for (int i = 0; i < W; i++) {
    const int Hold = B.H[i];
    const int T1 = __viaddmax_s32(Hold, open, LO);
    bool pE;
    const int m = tie_max<LATE>(B.E[i], T1, pE);
    const int Ee = __viaddmax_s32(m, ext, LO);
    int ps;
    if (VARIANT == GDP_LOWER) {
      ps = prof_byte(B.plo[i], B.phi4[i >> 2], sA[i & 3]);
    } else {
      ps = max(prof_byte(B.plo[i], B.phi4[i >> 2], sA[i & 3]), prof_byte(B.plo[i], B.phi4[i >> 2], sB[i & 3]));
    }
    const int Hv = min(__viaddmax_s32(diag, ps, LO), HI);
    diag = Hold;
    bool pN;
    B.H[i] = tie_max<LATE>(Ee, Hv, pN);
    B.E[i] = Ee;
    if (pE) w[gdp_dir_word(W, i)] |= 1u << (16 + gdp_dir_bit(W, i));
    if (pN) w[gdp_dir_word(W, i)] |= 1u << gdp_dir_bit(W, i);
  }
  int2 out;
  if (VARIANT == GDP_FULL) {
    int Fp = GDP_NEGINT, Hp = GDP_NEGINT;
    if (B.xlo > 0) { Fp = above.y; Hp = above.x; }
#pragma unroll
    for (int i = 0; i < W; i++) {
      bool pF, pV;
      const int F = tie_max<LATE>(Fp, Hp + open, pF) + ext;
      const int Hn = tie_max<LATE>(F, B.H[i], pV);
      B.H[i] = Hn;
      Hp = Hn;
      Fp = F;
      if (pF) w[gdp_dir_word(W, i)] |= 1u << (24 + gdp_dir_bit(W, i));
      if (pV) w[gdp_dir_word(W, i)] |= 1u << (8 + gdp_dir_bit(W, i));
    }
    out = make_int2(B.H[W - 1], Fp);
  } else {
    out = make_int2(B.H[W - 1], 0);
  }
  if (MODE != 0 && track) {
#pragma unroll
    for (int i = 0; i < W; i++) vmax = max(vmax, B.H[i]);
  }
  if (WORDS == 2) {
    *reinterpret_cast<uint2 *>(dcol) = make_uint2(w[0], w[1]);
  } else {
    *reinterpret_cast<uint4 *>(dcol) = make_uint4(w[0], w[1], w[WORDS > 2 ? 2 : 0], w[WORDS > 3 ? 3 : 0]);
  }
  return out;
}

/* Whether column y of the full block at xlo is steady (see
   block_column_steady).  For the upper and lower fills with an in-band
   score check (MODE != 0) the column must also hold no lane above the band,
   so that every lane's score counts. */
template <int W, int VARIANT, int MODE>
__device__ __forceinline__ bool
column_steady (const PairView &v, int xlo, int y) {
  const int rel = y - xlo;
  if (VARIANT == GDP_FULL) return rel < v.uband && rel + v.lband > W - 1;
  return rel > W - 1 && (MODE == 0 || rel <= v.g.band_hi);
}

/* Steady columns take block_column_steady in the one-thread-per-pair
   16-bit fills (GDP_STEADY) and 8-bit fills (GDP_STEADY8); 0 switches it
   off. */
#ifndef GDP_STEADY
#define GDP_STEADY 1
#endif
#ifndef GDP_STEADY8
#define GDP_STEADY8 0
#endif

#ifndef GDP_FILL_MINB
#define GDP_FILL_MINB 4
#endif
/* resident blocks of 128 threads per SM the 8-bit fills are built for */
#ifndef GDP_FILL_MINB8
#define GDP_FILL_MINB8 3
#endif

#include "fill_packed.cuh"

/* MODE: 0 plain fill, 1 = 16-bit fill of a rerun pair (records whether an
   in-band score reaches 127), 2 = 8-bit pass of a rerun pair (skipped when
   the 16-bit pass proved an overflow; stops at the first in-band 127).
   One thread per pair; the next column's characters and carry are fetched
   one column ahead. */
template <int W, int VARIANT, bool LATE, int MODE>
__global__ void __launch_bounds__(128, (W == 16) ? GDP_FILL_MINB : GDP_FILL_MINB8)
fill_thread_kernel (FillParams P) {
  constexpr int LO = (W == 32) ? -128 : -32768;
  /* lanes skipped in full-band columns whose top half left the band */
  constexpr int HALF = (VARIANT == GDP_FULL && W == 16) ? W / 2 : 0;
  constexpr int WORDS = W / 8;
  __shared__ int8_t s_nt2int[128];
  for (int i = threadIdx.x; i < 128; i += blockDim.x) s_nt2int[i] = P.tab->nt2int[i];
  __syncthreads();

  const int64_t slot = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *P.count;
  for (int64_t li = slot; li < n; li += P.nslots) {
    const int pi = __ldg(P.list + li);
    if (pi < 0) continue;   /* padding: warps hold pairs of one band width */
    const gdp_pair_t p = P.pairs[pi];
    gdp_meta_t *mp = P.meta + pi;
    if (MODE == 2 && mp->maxh16 >= 127) {
      mp->status8 = 1;   /* the 16-bit scores reach 127, so the 8-bit fill overflows */
      continue;
    }
    PairView v;
    pair_view<W, VARIANT>(p, P.arena, v);
    v.reach_from = (int) ((P.reach_from4 >> (8 * (v.mt & 3))) & 255u);
    if (MODE == 1 && VARIANT == GDP_LOWER) v.lim += (int) ((P.lower_slack4 >> (8 * (v.mt & 3))) & 255u);
    v.endmode = (VARIANT == GDP_FULL) ? 0 : (p.flags & GDP_FLAG_ENDPOINT) ? 1 : (p.flags & GDP_FLAG_ENDPOINT_QEND) ? 2 : 0;
    if constexpr (W == 16 && VARIANT == GDP_FULL && MODE != 2) {
      if (min(p.rlength, p.glength) <= P.packed_len) continue;   /* fill_packed_kernel's */
    }
    EndBest eb;
    eb.score = 0; eb.r = 0; eb.c = 0; eb.found = false;
    const int end_start = (v.endmode == 2) ? LO : 0;
    uint32_t *dir = P.dirs + ((W == 16) ? mp->dir16 : mp->dir8);
    int2 *sc = P.scratch + slot;
    const int64_t scs = P.nslots;
    int final_score = LO;
    bool reached = false;
    int vmax = LO;   /* in-band scores of the steady columns */

    for (int xlo = 0; xlo <= v.g.X; xlo += W) {
      Block<W> B;
      block_start<W, VARIANT, LATE>(B, v, P.tab, xlo);
      if (B.y1 < B.y0) continue;
      int bot_prev = LO;   /* H[y-1][xlo-1] from the block above */
      if (xlo > 0 && B.y0 > 0) bot_prev = sc[(int64_t) (B.y0 - 1) * scs].x;
      /* fetch column y0's inputs */
      int ka, kb;
      column_classes<VARIANT>(v, s_nt2int, B.y0, ka, kb);
      int2 above = make_int2(LO, GDP_NEGINT);
      if (xlo > 0) above = sc[(int64_t) B.y0 * scs];
      uint32_t *dcol = dir;
      for (int y = B.y0; y <= B.y1; y++) {
        /* prefetch column y + 1 */
        int ka2 = 0, kb2 = 0;
        int2 above2 = make_int2(LO, GDP_NEGINT);
        if (y < B.y1) {
          column_classes<VARIANT>(v, s_nt2int, y + 1, ka2, kb2);
          if (xlo > 0) above2 = sc[(int64_t) (y + 1) * scs];
        }
        int diag;
        if (y == 0) diag = (VARIANT == GDP_FULL) ? (xlo == 0 ? 0 : LO) : 0;
        else diag = (xlo == 0) ? LO : bot_prev;
        bot_prev = above.x;
        int16_t *hd = (P.hdump != nullptr) ? P.hdump + (dcol - P.dirs) * 8 : nullptr;
        int2 out;
        if constexpr ((W == 16 && MODE != 2 && GDP_STEADY) || (W == 32 && GDP_STEADY8)) {
          if (hd == nullptr && B.last == W - 1 && y >= 1 && y != v.g.Y && column_steady<W, VARIANT, MODE>(v, xlo, y)) {
            out = block_column_steady<W, VARIANT, LATE, MODE>(B, v, diag, above, ka, kb, dcol, vmax,
                                                              y >= v.reach_from && xlo + W - 1 >= v.reach_from);
            if (MODE == 2 && vmax >= 127) reached = true;
          } else if (HALF > 0 && hd == nullptr && y != v.g.Y && y - xlo - v.uband >= HALF) {
            /* the top half of the block has left the band */
            out = block_column<W, VARIANT, LATE, MODE, HALF>(B, v, y, diag, above, ka, kb, dcol, hd, reached,
                                                             final_score);
          } else
            out = block_column<W, VARIANT, LATE, MODE>(B, v, y, diag, above, ka, kb, dcol, hd, reached,
                                                       final_score);
        } else {
          out = block_column<W, VARIANT, LATE, MODE>(B, v, y, diag, above, ka, kb, dcol, hd, reached, final_score);
        }
        sc[(int64_t) y * scs] = out;
        if (VARIANT != GDP_FULL && v.endmode != 0) end_column<W, VARIANT, LATE>(eb, B, v, y, end_start);
        dcol += WORDS;
        ka = ka2; kb = kb2; above = above2;
        if (MODE == 2 && reached) break;
      }
      dir = dcol;
      if (MODE == 2 && reached) break;
    }
    if (vmax >= v.lim) reached = true;
    if (v.endmode == 2 && !eb.found) {
      /* the last-row search starts at (rlength, 0) */
      eb.score = LO;
      eb.r = (VARIANT == GDP_UPPER) ? v.g.X : v.g.Y;
    }
    fill_finish<W, MODE>(P, pi, mp, v.g, reached, final_score, v.endmode != 0 ? &eb : nullptr);
  }
}

/*
 * One group of K lanes (K = 4 .. 32; 32 / K pairs per warp) per pair: long
 * 16-bit pairs (plain fills), and the 8-bit pass of rerun pairs (W = 32,
 * MODE 2), whose few pairs would leave most of the device idle with one
 * thread each.  Lane l of a group owns the blocks b = l,
 * l + K, l + 2K, ... and processes column y of block b at step t = y + b:
 * block b needs the final column y (F carry, last lane H) and column y - 1
 * (diagonal) of block b - 1, which the previous lane of the group produced
 * one and two steps earlier, so one rotation shuffle inside the group per
 * step carries them.  A lane's next block starts after its previous one
 * ends as long as a block sweeps fewer than (W + 1) K - 16 columns; the planner
 * picks the smallest K that allows the pair's sweep, so lanes idle between
 * blocks for at most a few steps.  Each lane runs block_column, the same
 * column step as the one-thread-per-pair kernel.
 */
template <int VARIANT, bool LATE, int K, int W = 16, int MODE = 0>
__global__ void __launch_bounds__(128, (W == 16) ? 4 : 2)
fill_warp_kernel (FillParams P) {
  constexpr int WORDS = W / 8, LO = (W == 32) ? -128 : -32768, G = 32 / K;
  static_assert(K == 4 || K == 8 || K == 16 || K == 32, "group sizes divide the warp");
  static_assert(MODE == 0 || (MODE == 2 && W == 32), "plain fills, or the 8-bit pass of rerun pairs");
  __shared__ int8_t s_nt2int[128];
  for (int i = threadIdx.x; i < 128; i += blockDim.x) s_nt2int[i] = P.tab->nt2int[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, glane = lane & (K - 1), group = lane / K;
  const int prev = group * K + ((glane + K - 1) & (K - 1));   /* previous lane of the group */
  const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t) gridDim.x * blockDim.x) >> 5;
  const int n = *P.count;
  /* every lane of the warp stays in both loops: the shuffles need all 32 */
  for (int64_t base = warp * G; base < n; base += nwarps * G) {
    const int64_t li = base + group;
    const bool valid = li < n;
    const int pi = valid ? __ldg(P.list + li) : -1;
    gdp_pair_t p;
    if (valid) {
      p = P.pairs[pi];
    } else {
      memset(&p, 0, sizeof(p));
      p.rlength = p.glength = 1;
    }
    gdp_meta_t *mp = valid ? P.meta + pi : nullptr;
    PairView v;
    pair_view<W, VARIANT>(p, P.arena, v);
    v.reach_from = (int) ((P.reach_from4 >> (8 * (v.mt & 3))) & 255u);
    uint32_t *dir = valid ? P.dirs + ((W == 16) ? mp->dir16 : mp->dir8) : nullptr;
    /* blocks that sweep something: 0 .. nb - 1 */
    int nb = 0, tend = -1;
    if (valid) {
      nb = v.g.X / W + 1;
      while (nb > 0) {
        int a0, a1;
        gdp_block_sweep(&v.g, (nb - 1) * W, &a0, &a1);
        if (a1 >= a0) break;
        nb--;
      }
      if (nb > 0) {
        int a0, a1;
        gdp_block_sweep(&v.g, (nb - 1) * W, &a0, &a1);
        tend = a1 + nb - 1;
      }
    }
    int tmax = tend;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tmax = max(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
    /* this lane's first block and its word offset */
    int b = glane;
    int64_t boff = 0;
    for (int k = 0; k < b && k < nb; k++) boff += gdp_block_words(&v.g, k * W);
    Block<W> B;
    bool started = false;
    int final_score = LO;
    bool reached = false;
    int2 mine = make_int2(LO, GDP_NEGINT);   /* this lane's output of the last step */
    int bot_prev = LO;                         /* H[y-1][xlo-1] received a step ago */
    for (int t = 0; t <= tmax; t++) {
      /* (H, F) of block b - 1 at column t - b, produced by the previous lane */
      const int rx = __shfl_sync(0xffffffffu, mine.x, prev);
      const int ry = __shfl_sync(0xffffffffu, mine.y, prev);
      if (b < nb) {
        if (!started) {
          block_start<W, VARIANT, LATE>(B, v, P.tab, b * W);
          started = true;
        }
        const int y = t - b;
        if (y >= B.y0 && y <= B.y1) {
          int ka, kb;
          column_classes<VARIANT>(v, s_nt2int, y, ka, kb);
          const int2 above = (b > 0) ? make_int2(rx, ry) : make_int2(LO, GDP_NEGINT);
          int diag;
          if (y == 0) diag = (VARIANT == GDP_FULL) ? (b == 0 ? 0 : LO) : 0;
          else diag = (b == 0) ? LO : bot_prev;
          uint32_t *dcol = dir + boff + (int64_t) (y - B.y0) * WORDS;
          int16_t *hd = (P.hdump != nullptr) ? P.hdump + (dcol - P.dirs) * 8 : nullptr;
          mine = block_column<W, VARIANT, LATE, MODE>(B, v, y, diag, above, ka, kb, dcol, hd, reached,
                                                      final_score);
          if (y == B.y1) {
            /* move to block b + K */
            for (int k = b; k < b + K && k < nb; k++) boff += gdp_block_words(&v.g, k * W);
            b += K;
            started = false;
          }
        }
      }
      bot_prev = rx;
    }
    /* the lane that owned the final cell's block reports its score; the
       8-bit pass also needs whether any lane saw an in-band 127 */
    const int fs = __shfl_sync(0xffffffffu, final_score, group * K + ((v.g.X / W) & (K - 1)));
    const unsigned gmask = (K == 32) ? 0xffffffffu : (((1u << K) - 1u) << (group * K));
    const bool any_reached = (__ballot_sync(0xffffffffu, reached) & gmask) != 0;
    if (valid && glane == 0) fill_finish<W, MODE>(P, pi, mp, v.g, any_reached, fs);
  }
}

/*
 * One CTA of NW warps per pair for 16-bit plain fills whose blocks sweep
 * too many columns for one warp (wide bands: cDNA gap fills, long reads
 * with wide bands).  Same schedule as fill_warp_kernel over 32 * NW lanes:
 * lane L owns blocks L, L + 32 NW, ... and processes column y of block b at
 * step t = y + b.  Inside a warp the hand-off from block b - 1 is a
 * shuffle; across warps the last lane of each warp leaves its output in a
 * double-buffered shared slot, and one barrier per step orders it.
 */
template <int VARIANT, bool LATE, int NW>
__global__ void __launch_bounds__(NW * 32)
fill_cta_kernel (FillParams P) {
  constexpr int W = 16, WORDS = 2, LO = -32768, NL = NW * 32;
  __shared__ int8_t s_nt2int[128];
  __shared__ int2 s_hand[2][NW];
  for (int i = threadIdx.x; i < 128; i += blockDim.x) s_nt2int[i] = P.tab->nt2int[i];
  __syncthreads();
  const int L = threadIdx.x, lane = L & 31, wid = L >> 5;
  const int n = *P.count;
  for (int64_t li = blockIdx.x; li < n; li += gridDim.x) {
    const int pi = __ldg(P.list + li);
    const gdp_pair_t p = P.pairs[pi];
    gdp_meta_t *mp = P.meta + pi;
    PairView v;
    pair_view<W, VARIANT>(p, P.arena, v);
    v.reach_from = (int) ((P.reach_from4 >> (8 * (v.mt & 3))) & 255u);
    uint32_t *dir = P.dirs + mp->dir16;
    int nb = v.g.X / W + 1;
    while (nb > 0) {
      int a0, a1;
      gdp_block_sweep(&v.g, (nb - 1) * W, &a0, &a1);
      if (a1 >= a0) break;
      nb--;
    }
    int tend = -1;
    if (nb > 0) {
      int a0, a1;
      gdp_block_sweep(&v.g, (nb - 1) * W, &a0, &a1);
      tend = a1 + nb - 1;
    }
    int b = L;
    int64_t boff = 0;
    for (int k = 0; k < b && k < nb; k++) boff += gdp_block_words(&v.g, k * W);
    Block<W> B;
    bool started = false, reached = false;
    int final_score = LO;
    int2 mine = make_int2(LO, GDP_NEGINT);
    int bot_prev = LO;
    if (L < NW) s_hand[1][L] = make_int2(LO, GDP_NEGINT);
    __syncthreads();
    for (int t = 0; t <= tend; t++) {
      /* (H, F) of block b - 1 at column t - b from the previous lane */
      int rx = __shfl_sync(0xffffffffu, mine.x, (lane + 31) & 31);
      int ry = __shfl_sync(0xffffffffu, mine.y, (lane + 31) & 31);
      if (lane == 0) {
        const int2 h = s_hand[(t + 1) & 1][(wid + NW - 1) % NW];
        rx = h.x;
        ry = h.y;
      }
      if (b < nb) {
        if (!started) {
          block_start<W, VARIANT, LATE>(B, v, P.tab, b * W);
          started = true;
        }
        const int y = t - b;
        if (y >= B.y0 && y <= B.y1) {
          int ka, kb;
          column_classes<VARIANT>(v, s_nt2int, y, ka, kb);
          const int2 above = (b > 0) ? make_int2(rx, ry) : make_int2(LO, GDP_NEGINT);
          int diag;
          if (y == 0) diag = (VARIANT == GDP_FULL) ? (b == 0 ? 0 : LO) : 0;
          else diag = (b == 0) ? LO : bot_prev;
          uint32_t *dcol = dir + boff + (int64_t) (y - B.y0) * WORDS;
          int16_t *hd = (P.hdump != nullptr) ? P.hdump + (dcol - P.dirs) * 8 : nullptr;
          mine = block_column<W, VARIANT, LATE, 0>(B, v, y, diag, above, ka, kb, dcol, hd, reached,
                                                   final_score);
          if (y == B.y1) {
            for (int k = b; k < b + NL && k < nb; k++) boff += gdp_block_words(&v.g, k * W);
            b += NL;
            started = false;
          }
        }
      }
      bot_prev = rx;
      if (lane == 31) s_hand[t & 1][wid] = mine;
      __syncthreads();
    }
    if (L == ((v.g.X / W) % NL)) fill_finish<W, 0>(P, pi, mp, v.g, false, final_score);
    __syncthreads();
  }
}

/* After both passes of the rerun pairs in `list`: a pair whose 16-bit
   scores stayed below 127 and whose 8-bit fill did not overflow keeps the
   8-bit outcome (score, precision 8, no rerun); the others keep the 16-bit
   outcome the 16-bit pass wrote. */
static __global__ void
apply_rerun8_kernel (const int32_t *list, const int32_t *count, const gdp_meta_t *meta, gdp_result_t *res) {
  const int n = *count;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int pi = list[i];
    if (pi < 0) continue;
    const gdp_meta_t m = meta[pi];
    if (m.maxh16 < 127 && m.status8 == 0) {
      res[pi].score = m.final8;
      res[pi].precision = 8;
      res[pi].rerun = 0;
    }
  }
}

/* The rerun pairs whose 16-bit in-band maximum stays below 127: only those
   need the 8-bit pass (the others provably overflow in 8 bits). */
struct NeedsPass8 {
  const gdp_meta_t *meta;
  __device__ __forceinline__ bool operator() (const int32_t &pi) const {
    return pi >= 0 && meta[pi].maxh16 < 127;
  }
};
