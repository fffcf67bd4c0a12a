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

/* MODE: 0 plain fill, 1 = 16-bit fill of a rerun pair (records whether an
   in-band score reaches 127), 2 = 8-bit pass of a rerun pair (skipped when
   the 16-bit pass proved an overflow; stops at the first in-band 127).

   Per block column the band geometry is reduced to a few lane masks that
   are uniform over the column: the lanes of the F loop, the top cell
   (src/dynprog_simd.c:6962-6974), the bottom cell (:6926-6945), the lanes
   whose E is clamped (upper/lower E_mask, :7921, :7943) and the diagonal
   cell (:7966-7969).  The lane loop is fully unrolled, so each mask test is
   a test of a constant bit. */
#ifndef GDP_FILL_MINB
#define GDP_FILL_MINB 1
#endif

template <int W, int VARIANT, bool LATE, int MODE>
__global__ void __launch_bounds__(128, (W == 16) ? GDP_FILL_MINB : 1)
fill_thread_kernel (FillParams P) {
  constexpr int LO = (W == 32) ? -128 : -32768;
  constexpr int HI = (W == 32) ? 127 : 32767;
  constexpr int WORDS = W / 8;
  __shared__ int8_t s_nt2int[128];
  for (int i = threadIdx.x; i < 128; i += blockDim.x) s_nt2int[i] = P.tab->nt2int[i];
  __syncthreads();

  const int64_t slot = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *P.count;
  for (int64_t li = slot; li < n; li += P.nslots) {
    const int pi = __ldg(P.list + li);
    const gdp_pair_t p = P.pairs[pi];
    gdp_meta_t *mp = P.meta + pi;
    if (MODE == 2 && mp->maxh16 >= 127) {
      mp->status8 = 1;   /* the 16-bit scores reach 127, so the 8-bit fill overflows */
      continue;
    }
    gdp_geom_t g;
    gdp_geom_of(&p, W, &g);
    const bool revp = (p.flags & GDP_FLAG_REVP) != 0;
    const int open = p.open, ext = p.extend, oe = p.open + p.extend;
    const int mt = p.mismatchtype;
    const int lband = p.lband, uband = p.uband;
    const char *lseq = P.arena + (VARIANT == GDP_LOWER ? p.gseq : p.rseq);
    const char *lalt = P.arena + (VARIANT == GDP_LOWER ? p.gseq_alt : p.rseq);
    const int llen = (VARIANT == GDP_LOWER) ? p.glength : p.rlength;
    const char *sseq = P.arena + (VARIANT == GDP_LOWER ? p.rseq : p.gseq);
    const char *salt = P.arena + (VARIANT == GDP_LOWER ? p.rseq : p.gseq_alt);
    const int slen = (VARIANT == GDP_LOWER) ? p.rlength : p.glength;
    /* domain band of the lane index relative to y: lanes x with y - dhi <= x <= y + dlo */
    const int dlo = (VARIANT == GDP_FULL) ? lband : 0;
    const int dhi = (VARIANT == GDP_FULL) ? uband : (VARIANT == GDP_UPPER ? uband : lband);
    uint32_t *dir = P.dirs + ((W == 16) ? mp->dir16 : mp->dir8);
    int2 *sc = P.scratch + slot;
    const int64_t scs = P.nslots;
    int final_score = LO;
    bool reached = false;     /* an in-band score reached 127 */

    for (int xlo = 0; xlo <= g.X; xlo += W) {
      const int xhi = min(xlo + W - 1, g.X);
      const int last = xhi - xlo;
      int y0, y1;
      gdp_block_sweep(&g, xlo, &y0, &y1);
      if (y1 < y0) continue;

      /* lane profiles: bytes 0..3 of plo = scores against classes A,C,G,T;
         the class-N score of lane i is byte (i & 3) of phi4[i >> 2] */
      uint32_t plo[W], phi4[W / 4];
#pragma unroll
      for (int j = 0; j < W / 4; j++) phi4[j] = 0;
#pragma unroll
      for (int i = 0; i < W; i++) {
        const int x = xlo + i;
        uint32_t lo, hi;
        if (VARIANT != GDP_LOWER) {
          const int q = (x == 0) ? 'N' : (x <= llen ? seqch(lseq, llen, x, revp) : 'N');
          lo = __ldg(&P.tab->profq_lo[mt][q]);
          hi = __ldg(&P.tab->profq_hi[mt][q]);
        } else if (x == 0) {
          /* 16-bit: column 0 scores against 'N' (:8689); 8-bit: against code 4 (:5459) */
          const int c0 = (W == 32) ? 4 : 'N';
          lo = __ldg(&P.tab->profg_lo[mt][c0]);
          hi = __ldg(&P.tab->profg_hi[mt][c0]);
        } else if (x <= llen) {
          const int a = seqch(lseq, llen, x, revp), b = seqch(lalt, llen, x, revp);
          lo = bytemax(__ldg(&P.tab->profg_lo[mt][a]), __ldg(&P.tab->profg_lo[mt][b]));
          hi = bytemax(__ldg(&P.tab->profg_hi[mt][a]), __ldg(&P.tab->profg_hi[mt][b]));
        } else {
          lo = 0; hi = 0;
        }
        plo[i] = lo;
        phi4[i >> 2] |= (hi & 0xffu) << (8 * (i & 3));
      }
      int H[W], E[W];
#pragma unroll
      for (int i = 0; i < W; i++) { H[i] = LO - open; E[i] = LATE ? LO : LO + 1; }
      int bot_prev = LO;   /* H[y-1][xlo-1] from the block above */
      if (xlo > 0 && y0 > 0) bot_prev = sc[(int64_t) (y0 - 1) * scs].x;
      uint32_t *dcol = dir;

      for (int y = y0; y <= y1; y++) {
        /* swept-column classes -> PRMT selectors; class N (4) reads the
           packed byte (i & 3) of phi4, i.e. byte 4 + (i & 3) of {phi4, plo} */
        int ka, kb;
        if (VARIANT == GDP_LOWER) {
          ka = kb = (y == 0) ? 4 : s_nt2int[seqch(sseq, slen, y, revp)];
        } else if (y == 0) {
          ka = kb = 4;
        } else {
          ka = s_nt2int[seqch(sseq, slen, y, revp)];
          kb = s_nt2int[seqch(salt, slen, y, revp)];
        }
        const bool col0 = (VARIANT == GDP_FULL) && (y == 0);
        uint32_t sA[4], sB[4];
        {
          const uint32_t dA = (ka == 4) ? 0x1111u : 0u, dB = (kb == 4) ? 0x1111u : 0u;
          sA[0] = GDP_SEL(ka); sB[0] = GDP_SEL(kb);
#pragma unroll
          for (int k = 1; k < 4; k++) { sA[k] = sA[k - 1] + dA; sB[k] = sB[k - 1] + dB; }
        }
        int2 above = make_int2(LO, GDP_NEGINT);
        if (xlo > 0) above = sc[(int64_t) y * scs];
        int diag;
        if (y == 0) diag = (VARIANT == GDP_FULL) ? (xlo == 0 ? 0 : LO) : 0;
        else diag = (xlo == 0) ? LO : bot_prev;
        bot_prev = above.x;

        /* lane masks of this column */
        const int rel = y - xlo;                       /* lane index of x == y */
        uint32_t fmask = 0, topmask = 0, botmask = 0, emask = 0, dmask = 0;
        if (VARIANT == GDP_FULL) {
          const int t = rel - uband, bt = rel + lband;  /* top and bottom lanes */
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

        /* vector step (E, then H from the diagonal), :6862-6913 */
#pragma unroll
        for (int i = 0; i < W; i++) {
          const uint32_t bit = 1u << i;
          const int Hold = H[i];
          int Eold = E[i];
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
            ps = prof_byte(plo[i], phi4[i >> 2], sA[i & 3]);
          } else {
            ps = max(prof_byte(plo[i], phi4[i >> 2], sA[i & 3]), prof_byte(plo[i], phi4[i >> 2], sB[i & 3]));
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
          H[i] = Hn;
          E[i] = Ee;
          if (pE) w[i >> 3] |= 1u << (16 + (i & 7));
          if (pN) w[i >> 3] |= 1u << (i & 7);
        }
        if (VARIANT == GDP_FULL) {
          /* F loop over the in-band lanes (:6916-7000) */
          int Fp, Hp;
          if (xlo == 0 || y >= xlo + uband) { Fp = GDP_NEGINT; Hp = GDP_NEGINT; }
          else { Fp = above.y; Hp = above.x; }
#pragma unroll
          for (int i = 0; i < W; i++) {
            const uint32_t bit = 1u << i;
            if (topmask & bit) {
              Fp = GDP_NEGINT + oe;
              Hp = H[i];
            } else if (fmask & bit) {
              bool pF, pV;
              const int F = tie_max<LATE>(Fp, Hp + open, pF) + ext;
              const int Hn = tie_max<LATE>(F, H[i], pV);
              H[i] = Hn;
              Hp = Hn;
              Fp = F;
              if (pF) w[i >> 3] |= 1u << (24 + (i & 7));
              if (pV) w[i >> 3] |= 1u << (8 + (i & 7));
            }
          }
          sc[(int64_t) y * scs] = make_int2(H[W - 1], Fp);
        } else {
          sc[(int64_t) y * scs] = make_int2(H[W - 1], 0);
        }
        if (MODE != 0 && !reached && y >= 1) {
          /* in-band lanes: y - dhi <= x <= y + dlo, x >= 1 */
          const int dl = max(rel - dhi, (xlo == 0) ? 1 : 0), dh = min(rel + dlo, last);
          if (dh >= dl) {
            const uint32_t dom = lane_range(max(dl, 0), dh);
#pragma unroll
            for (int i = 0; i < W; i++)
              if ((dom & (1u << i)) && H[i] >= 127) reached = true;
          }
        }
        if (y == g.Y) {
#pragma unroll
          for (int i = 0; i < W; i++) if (xlo + i == g.X) final_score = H[i];
        }
        if (P.hdump != nullptr) {
          int16_t *hd = P.hdump + (dcol - P.dirs) * 8;
#pragma unroll
          for (int i = 0; i < W; i++) hd[i] = (int16_t) H[i];
        }
        if (WORDS == 2) {
          *reinterpret_cast<uint2 *>(dcol) = make_uint2(w[0], w[1]);
        } else {
          *reinterpret_cast<uint4 *>(dcol) = make_uint4(w[0], w[1], w[WORDS > 2 ? 2 : 0], w[WORDS > 3 ? 3 : 0]);
        }
        dcol += WORDS;
        if (MODE == 2 && reached) break;
      }
      dir = dcol;
      if (MODE == 2 && reached) break;
    }

    /* the final cell must have been swept */
    int y0l, y1l;
    gdp_block_sweep(&g, (g.X / W) * W, &y0l, &y1l);
    const bool swept = (g.Y >= y0l && g.Y <= y1l);
    if (MODE == 1) {
      mp->maxh16 = reached ? 127 : -32768;   /* >= 127 iff an in-band 16-bit score reached 127 */
      mp->final16 = final_score;
    }
    if (MODE == 2) {
      const bool overflow = reached || final_score <= -128 + 30;
      mp->status8 = overflow ? 1 : 0;
      mp->final8 = final_score;
      if (!overflow) {
        P.res[pi].score = final_score;
        P.res[pi].precision = 8;
        P.res[pi].rerun = 0;
      }
    } else {
      gdp_result_t *r = P.res + pi;
      r->score = final_score;
      r->precision = W == 16 ? 16 : 8;
      r->rerun = (MODE == 1) ? 1 : 0;
      if (!swept) r->status = GDP_ERR_BAND;
    }
  }
}

/* Keeps the rerun pairs whose 16-bit in-band maximum stays below 127: only
   those need the 8-bit pass (the others provably overflow in 8 bits). */
static __global__ void
compact_rerun_kernel (const int32_t *list, const int32_t *count, const gdp_meta_t *meta,
                      int32_t *out, int32_t *out_count) {
  const int n = *count;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int pi = list[i];
    const bool need = meta[pi].maxh16 < 127;
    const unsigned mask = __ballot_sync(__activemask(), need);
    const int lane = threadIdx.x & 31;
    int base = 0;
    const int leader = __ffs(mask) - 1;
    if (mask && lane == leader) base = atomicAdd(out_count, __popc(mask));
    base = __shfl_sync(__activemask(), base, leader < 0 ? 0 : leader);
    if (need) out[base + __popc(mask & ((1u << lane) - 1))] = pi;
  }
}
