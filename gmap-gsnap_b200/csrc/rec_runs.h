/*
 * rec_runs.h -- the record-run transport of gdp_align_batch: a pair's
 * traceback records leave the device as a byte stream and the host rebuilds
 * the exact gdp_rec_t bytes.  Internal.
 *
 * Most records follow from the one before and from the pair's sequences: a
 * diagonal step moves querypos and genomepos by one in the walk's direction
 * (down, or up for revp) and takes the query, genome and alternate-genome
 * characters at the new positions, with one of the comparison characters
 * '*', ':' or ' '; a step of a query skip moves querypos alone and carries
 * '-' with blank genome characters; the first diagonal record after a skip
 * moves only one of the two positions.  Such a record is one token: its
 * move and its comparison character.  Everything else -- a pair's first
 * record, gap holders, genome skips (whose characters come from the
 * resident genome, not the arena), and any record the prediction does not
 * reproduce -- travels whole.
 *
 * Stream of one pair, byte by byte:
 *   0xFF          escape: the next 12 bytes are the record as it is;
 *   (t << 4) | 12 token t (0..11) c + 1 times, c the next byte (1..256);
 *   (r << 4) | t  token t (0..11) r + 1 times (1..16).
 * Token t: move t >> 2 (0: both positions step, 1: querypos steps, 2:
 * genomepos steps), kind t & 3 (0 '*', 1 ':', 2 ' ' with the three
 * characters from the sequences; 3 a query-skip record: query character,
 * '-', blanks).
 *
 * The encoder accepts a token only when rec_predict rebuilds the record
 * byte for byte, and the decoder calls the same function, so the host's
 * records equal the device's whatever the pair.  Pairs whose genome window
 * the device wrote (GDP_FLAG_GWINDOW) travel whole: the host arena does
 * not hold their window.
 */
#pragma once
#include <stdint.h>
#include <string.h>
#include "gdp.h"

#ifdef __CUDACC__
#define GDP_HD __host__ __device__ __forceinline__
#else
#define GDP_HD inline
#endif

/* a 32-bit word of a record, which may alias the record's fields */
typedef uint32_t __attribute__((__may_alias__)) run_word;

enum { RUN_ESCAPE = 0xFF, RUN_TOKENS = 12, RUN_LONG = 12, RUN_SHORT_REPEAT = 16, RUN_MAX_REPEAT = 256 };

/* Writes token t repeated reps times (1..RUN_MAX_REPEAT) at out[len] when
   out is not NULL; returns the bytes it takes. */
GDP_HD int
run_put (uint8_t *out, int64_t len, int t, int reps) {
  if (reps <= RUN_SHORT_REPEAT) {
    if (out) out[len] = (uint8_t) (((reps - 1) << 4) | t);
    return 1;
  }
  if (out) {
    out[len] = (uint8_t) ((t << 4) | RUN_LONG);
    out[len + 1] = (uint8_t) (reps - 1);
  }
  return 2;
}

/* The sequences of one pair, as forward arena bytes. */
struct RunSeqs {
  const char *rseq, *gseq, *galt;
  int32_t rlength, glength, queryoffset, genomeoffset;
  int32_t step;        /* -1, or +1 for revp: the direction positions move in */
  int32_t revp;
};

GDP_HD RunSeqs
run_seqs (const gdp_pair_t &p, const char *arena) {
  RunSeqs s;
  s.rseq = arena + p.rseq;
  s.gseq = arena + p.gseq;
  s.galt = arena + p.gseq_alt;
  s.rlength = p.rlength;
  s.glength = p.glength;
  s.queryoffset = p.queryoffset;
  s.genomeoffset = p.genomeoffset;
  s.revp = (p.flags & GDP_FLAG_REVP) != 0;
  s.step = s.revp ? 1 : -1;
  return s;
}

/* Arena index of the character the traceback reads for position pos
   (offset off, length len): the reference indexes seq[c] forward, or
   seq[-c] back from the last character for revp; -1 outside. */
GDP_HD int32_t
run_index (int32_t pos, int32_t off, int32_t len, int32_t revp) {
  const int32_t c = pos - off;
  const int32_t i = revp ? len - 1 + c : c;
  return (i >= 0 && i < len) ? i : -1;
}

/* The record token t predicts after `prev`; false when the positions leave
   the sequences. */
GDP_HD bool
rec_predict (const RunSeqs &s, const gdp_rec_t &prev, int t, gdp_rec_t *out) {
  const int move = t >> 2, kind = t & 3;
  const int32_t q = prev.querypos + (move != 2 ? s.step : 0);
  const int32_t g = prev.genomepos + (move != 1 ? s.step : 0);
  const int32_t qi = run_index(q, s.queryoffset, s.rlength, s.revp);
  if (qi < 0) return false;
  out->querypos = q;
  out->genomepos = g;
  out->cdna = s.rseq[qi];
  if (kind == 3) {
    out->comp = '-';
    out->genome = ' ';
    out->genomealt = ' ';
    return true;
  }
  const int32_t gi = run_index(g, s.genomeoffset, s.glength, s.revp);
  if (gi < 0) return false;
  out->comp = kind == 0 ? '*' : kind == 1 ? ':' : ' ';
  out->genome = s.gseq[gi];
  out->genomealt = s.galt[gi];
  return true;
}

GDP_HD bool
rec_equal (const gdp_rec_t &a, const gdp_rec_t &b) {
  return a.querypos == b.querypos && a.genomepos == b.genomepos && a.cdna == b.cdna && a.comp == b.comp &&
         a.genome == b.genome && a.genomealt == b.genomealt;
}

/* The one token that can rebuild rec after prev, or -1. */
GDP_HD int
rec_token (const RunSeqs &s, const gdp_rec_t &prev, const gdp_rec_t &rec) {
  const int32_t dq = rec.querypos - prev.querypos, dg = rec.genomepos - prev.genomepos;
  int move;
  if (dq == s.step && dg == s.step) move = 0;
  else if (dq == s.step && dg == 0) move = 1;
  else if (dq == 0 && dg == s.step) move = 2;
  else return -1;
  int kind;
  switch (rec.comp) {
    case '*': kind = 0; break;
    case ':': kind = 1; break;
    case ' ': kind = 2; break;
    case '-': kind = 3; break;
    default: return -1;
  }
  const int t = move * 4 + kind;
  gdp_rec_t p;
  if (!rec_predict(s, prev, t, &p) || !rec_equal(p, rec)) return -1;
  return t;
}

/*
 * Encodes n records; writes the stream to out when out is not NULL and
 * returns its length in bytes.  `whole` sends every record as it is.
 */
GDP_HD int64_t
rec_encode (const RunSeqs &s, const gdp_rec_t *recs, int n, bool whole, uint8_t *out) {
  int64_t len = 0;
  int pend = -1, reps = 0;
  gdp_rec_t prev;
  memset(&prev, 0, sizeof(prev));
  for (int k = 0; k < n; k++) {
    const gdp_rec_t rec = recs[k];
    const int t = (k == 0 || whole) ? -1 : rec_token(s, prev, rec);
    if (t >= 0 && t == pend && reps < RUN_MAX_REPEAT) {
      reps++;
    } else {
      if (pend >= 0) len += run_put(out, len, pend, reps);
      pend = -1;
      reps = 0;
      if (t >= 0) {
        pend = t;
        reps = 1;
      } else {
        if (out) {
          out[len] = RUN_ESCAPE;
          memcpy(out + len + 1, &rec, sizeof(gdp_rec_t));
        }
        len += 1 + (int64_t) sizeof(gdp_rec_t);
      }
    }
    prev = rec;
  }
  if (pend >= 0) len += run_put(out, len, pend, reps);
  return len;
}

/* Rebuilds n records from a stream of len bytes; false when the stream is
   malformed or ends early. */
GDP_HD bool
rec_decode (const RunSeqs &s, const uint8_t *in, int64_t len, gdp_rec_t *recs, int n) {
  int64_t at = 0;
  int k = 0;
  gdp_rec_t prev;
  memset(&prev, 0, sizeof(prev));
  while (k < n) {
    if (at >= len) return false;
    const uint8_t b = in[at++];
    if (b == RUN_ESCAPE) {
      if (at + (int64_t) sizeof(gdp_rec_t) > len) return false;
      memcpy(&prev, in + at, sizeof(gdp_rec_t));
      at += sizeof(gdp_rec_t);
      recs[k++] = prev;
      continue;
    }
    int t = b & 15, reps = (b >> 4) + 1;
    if (t == RUN_LONG) {
      if (at >= len) return false;
      t = b >> 4;
      reps = in[at++] + 1;
    }
    if (t >= RUN_TOKENS || k + reps > n) return false;
    /* rec_predict reps times: positions move by (dq, dg) a step, and so do
       their arena indices; they are monotonic, so the first and the last
       step bound the whole run */
    const int move = t >> 2, kind = t & 3;
    const int32_t dq = move != 2 ? s.step : 0, dg = move != 1 ? s.step : 0;
    int32_t qi = run_index(prev.querypos + dq, s.queryoffset, s.rlength, s.revp);
    if (qi < 0 || run_index(prev.querypos + reps * dq, s.queryoffset, s.rlength, s.revp) < 0) return false;
    gdp_rec_t x;
    x.querypos = prev.querypos;
    x.genomepos = prev.genomepos;
    if (kind == 3) {
      x.comp = '-';
      x.genome = ' ';
      x.genomealt = ' ';
      for (int r = 0; r < reps; r++, qi += dq) {
        x.querypos += dq;
        x.genomepos += dg;
        x.cdna = s.rseq[qi];
        recs[k++] = x;
      }
    } else {
      int32_t gi = run_index(prev.genomepos + dg, s.genomeoffset, s.glength, s.revp);
      if (gi < 0 || run_index(prev.genomepos + reps * dg, s.genomeoffset, s.glength, s.revp) < 0) return false;
      x.comp = kind == 0 ? '*' : kind == 1 ? ':' : ' ';
      /* the records as 32-bit words: two positions, then the four
         characters (cdna, comp, genome, genomealt in memory order) */
      const uint32_t cmp = (uint32_t) (uint8_t) x.comp << 8;
      run_word *w = reinterpret_cast<run_word *>(recs + k);
      const uint8_t *rq = reinterpret_cast<const uint8_t *>(s.rseq) + qi;
      const uint8_t *gg = reinterpret_cast<const uint8_t *>(s.gseq) + gi;
      const uint8_t *ga = reinterpret_cast<const uint8_t *>(s.galt) + gi;
      uint32_t qp = (uint32_t) x.querypos, gp = (uint32_t) x.genomepos;
      for (int r = 0; r < reps; r++, w += 3) {
        qp += (uint32_t) dq;
        gp += (uint32_t) dg;
        w[0] = qp;
        w[1] = gp;
        w[2] = (uint32_t) rq[r * dq] | cmp | (uint32_t) gg[r * dg] << 16 | (uint32_t) ga[r * dg] << 24;
      }
      k += reps;
      x.querypos = (int32_t) qp;
      x.genomepos = (int32_t) gp;
      x.cdna = (char) rq[(reps - 1) * dq];
      x.genome = (char) gg[(reps - 1) * dg];
      x.genomealt = (char) ga[(reps - 1) * dg];
    }
    prev = x;
  }
  return at == len;
}
