/*
 * dropin.cu -- the twelve entry points of src/dynprog_simd.h with the
 * reference's own signatures (include/gdp_dynprog_simd.h).
 *
 * A fill runs one pair through the device fill kernels (the batch runtime
 * with a one-pair plan), then writes the scores and the three direction
 * planes of every swept cell into the caller's Dynprog_T spaces, laid out
 * as the reference's aligned_*_alloc helpers lay them out
 * (src/dynprog_simd.c:2158-2283).  The device fill stays resident, keyed by
 * the direction space it was expanded into; the matching traceback walks
 * it on the device and replays the walk's Pair records through the
 * caller's Pairpool_push / Pairpool_push_gapholder, exactly as
 * Pairpool_add_genomeskip / Pairpool_add_queryskip push them
 * (src/pairpool.c:1067-1180).
 *
 * GMAP's symbols (Pairpool_push, Pairpool_push_gapholder, Genome_get_char,
 * pairdistance_array, consistent_array, nt_to_int_array) are weak
 * references, resolved at load time when the library is linked into GMAP,
 * else looked up in the process's global scope at first use; the library
 * therefore also loads in processes without them (its batch ABI needs
 * none).
 */
#include <dlfcn.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <cuda_runtime.h>

#include "gdp_dynprog_simd.h"
#include "gdp_internal.h"
#include "gdp_dropin_internal.h"

typedef List_T (*push_fn)(List_T, Pairpool_T, int, int, char, char, char, char, int);
typedef List_T (*gapholder_fn)(List_T, Pairpool_T, int, int, void *, void *, gdp_bool_t);
typedef char (*getchar_fn)(char *, Genome_T, Genome_T, Univcoord_T);

extern "C" {
List_T Pairpool_push(List_T, Pairpool_T, int, int, char, char, char, char, int) __attribute__((weak));
List_T Pairpool_push_gapholder(List_T, Pairpool_T, int, int, void *, void *, gdp_bool_t) __attribute__((weak));
char Genome_get_char(char *, Genome_T, Genome_T, Univcoord_T) __attribute__((weak));
extern short **pairdistance_array[4] __attribute__((weak));
extern unsigned char **consistent_array[3] __attribute__((weak));
extern int *nt_to_int_array __attribute__((weak));
}

#define DIR_DIAG 0
#define DIR_HORIZ (-1)
#define DIR_VERT (-2)

namespace {

[[noreturn]] void
die (const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fputs("libgdp: ", stderr);
  vfprintf(stderr, fmt, ap);
  fputc('\n', stderr);
  va_end(ap);
  abort();
}

struct GmapSyms {
  push_fn push = nullptr;
  gapholder_fn gapholder = nullptr;
  getchar_fn getchar = nullptr;
  short ***pd = nullptr;            /* &pairdistance_array[0] */
  unsigned char ***cons = nullptr;  /* &consistent_array[0] */
  int **nt2int = nullptr;           /* &nt_to_int_array */
};

const GmapSyms &
gmap_syms () {
  static const GmapSyms s = [] {
    GmapSyms g;
    g.push = Pairpool_push ? &Pairpool_push : (push_fn) dlsym(RTLD_DEFAULT, "Pairpool_push");
    g.gapholder = Pairpool_push_gapholder ? &Pairpool_push_gapholder
                                          : (gapholder_fn) dlsym(RTLD_DEFAULT, "Pairpool_push_gapholder");
    g.getchar = Genome_get_char ? &Genome_get_char : (getchar_fn) dlsym(RTLD_DEFAULT, "Genome_get_char");
    g.pd = &pairdistance_array[0] ? &pairdistance_array[0] : (short ***) dlsym(RTLD_DEFAULT, "pairdistance_array");
    g.cons = &consistent_array[0] ? &consistent_array[0]
                                  : (unsigned char ***) dlsym(RTLD_DEFAULT, "consistent_array");
    g.nt2int = &nt_to_int_array ? &nt_to_int_array : (int **) dlsym(RTLD_DEFAULT, "nt_to_int_array");
    return g;
  }();
  return s;
}

int
env_int (const char *name, int dflt) {
  const char *v = getenv(name);
  return (v && *v) ? atoi(v) : dflt;
}

/* The fill most recently expanded into one direction space. */
struct SpaceFill {
  const void *key = nullptr;   /* the space's nogap column-pointer array */
  const void *col0 = nullptr;  /* its column 0 as that fill set it */
  int precision = 0, variant = -1;
  uint64_t used = 0;
  gdpi_fill *f = nullptr;
};

constexpr int NSPACES = 16;    /* direction spaces remembered per thread */

struct DropinThread {
  gdp_ctx *ctx = nullptr;
  SpaceFill space[NSPACES];
  uint64_t clock = 0;
  bool warned_band = false;
  std::vector<char> arena;
  std::vector<char> gwin, gwinalt;
  std::vector<uint32_t> gblk, galtblk;
  std::vector<gdp_rec_t> recs;

  ~DropinThread () { release(); }

  void release () {
    for (SpaceFill &s : space) {
      if (s.f) gdpi_fill_free(s.f);
      s = SpaceFill();
    }
    if (ctx) gdp_ctx_destroy(ctx);
    ctx = nullptr;
  }

  /* The entry of `key`, or the least recently used one, reset for it. */
  SpaceFill &claim (const void *key) {
    SpaceFill *best = &space[0];
    for (SpaceFill &s : space) {
      if (s.key == key) { best = &s; break; }
      if (s.used < best->used) best = &s;
    }
    best->key = key;
    best->used = ++clock;
    if (!best->f) best->f = gdpi_fill_new();
    return *best;
  }

  SpaceFill *find (const void *key) {
    for (SpaceFill &s : space)
      if (s.key == key && s.f) { s.used = ++clock; return &s; }
    return nullptr;
  }
};

thread_local DropinThread t_state;

/* The calling thread's context, created at its first call.  GMAP's own
   tables are used when the process has run Dynprog_init. */
gdp_ctx *
thread_ctx () {
  DropinThread &t = t_state;
  if (t.ctx) return t.ctx;
  const int device = env_int("GDP_DEVICE", 0), mode = env_int("GDP_MODE", 0);
  gdp_ctx *ctx = nullptr;
  int rc = gdp_ctx_create(&ctx, device, mode, 0);
  if (rc != GDP_OK) die("cannot create a context on device %d (status %d)", device, rc);
  const GmapSyms &g = gmap_syms();
  if (g.pd && g.pd[0] && g.nt2int && *g.nt2int) {
    std::vector<gdp_tables_t> tab(1);
    gdp_tables_t *tb = tab.data();
    gdp_build_tables(tb, mode);
    for (int mt = 0; mt < 4; mt++)
      for (int a = 0; a < 128; a++)
        for (int b = 0; b < 128; b++) tb->pd[mt][a][b] = g.pd[mt][a][b];
    for (int gs = 0; gs < 3; gs++) {
      if (g.cons == nullptr || g.cons[gs] == nullptr) {
        memset(tb->cons[gs], 0, sizeof(tb->cons[gs]));
        continue;
      }
      for (int a = 0; a < 128; a++)
        for (int b = 0; b < 128; b++) tb->cons[gs][a][b] = g.cons[gs][a][b] ? 1 : 0;
    }
    for (int a = 0; a < 128; a++) tb->nt2int[a] = (int8_t) (*g.nt2int)[a];
    gdp_tables_derive(tb);
    rc = gdpi_set_tables(ctx, tb);
    if (rc != GDP_OK) die("cannot upload the substitution tables: %s", gdp_last_error(ctx));
  }
  t.ctx = ctx;
  return ctx;
}

/* The planes of one fill in the caller's Dynprog_T. */
struct Planes {
  void **mptrs, *mspace;
  void **nptrs, *nspace;
  void **eptrs, *espace;
  void **fptrs, *fspace;   /* full fill only */
};

Planes
planes_of (Dynprog_T self, int variant) {
  Planes P;
  if (variant == GDP_FULL) {
    P.mptrs = self->aligned.one.matrix_ptrs; P.mspace = self->aligned.one.matrix_space;
    P.nptrs = self->aligned.one.directions_ptrs_0; P.nspace = self->aligned.one.directions_space_0;
    P.eptrs = self->aligned.one.directions_ptrs_1; P.espace = self->aligned.one.directions_space_1;
    P.fptrs = self->aligned.one.directions_ptrs_2; P.fspace = self->aligned.one.directions_space_2;
  } else if (variant == GDP_UPPER) {
    P.mptrs = self->aligned.two.upper_matrix_ptrs; P.mspace = self->aligned.two.upper_matrix_space;
    P.nptrs = self->aligned.two.upper_directions_ptrs_0; P.nspace = self->aligned.two.upper_directions_space_0;
    P.eptrs = self->aligned.two.upper_directions_ptrs_1; P.espace = self->aligned.two.upper_directions_space_1;
    P.fptrs = nullptr; P.fspace = nullptr;
  } else {
    P.mptrs = self->aligned.two.lower_matrix_ptrs; P.mspace = self->aligned.two.lower_matrix_space;
    P.nptrs = self->aligned.two.lower_directions_ptrs_0; P.nspace = self->aligned.two.lower_directions_space_0;
    P.eptrs = self->aligned.two.lower_directions_ptrs_1; P.espace = self->aligned.two.lower_directions_space_1;
    P.fptrs = nullptr; P.fspace = nullptr;
  }
  return P;
}

/* Column pointers as aligned_score*_alloc sets them: Y + 1 columns of
   `stride` cells. */
template <typename S>
S **
lay_out (void **ptrs, void *space, int Y, int stride) {
  S **m = (S **) ptrs;
  S *p = (S *) space;
  for (int y = 0; y <= Y; y++) m[y] = p + (size_t) y * stride;
  return m;
}

/* The sequences of one pair, first character first, as one arena:
   query, upper-case query, genome window, alternate window. */
void
stage_arena (std::vector<char> &arena, gdp_pair_t &p, const char *rseq, const char *ruc, const char *gseq,
             const char *galt, bool revp) {
  const int rl = p.rlength, gl = p.glength;
  if (revp) {
    rseq -= rl - 1;
    ruc -= rl - 1;
    gseq -= gl - 1;
    galt -= gl - 1;
  }
  arena.resize((size_t) 2 * rl + 2 * gl + 16);
  char *a = arena.data();
  memcpy(a, rseq, rl);
  memcpy(a + rl, ruc, rl);
  memcpy(a + 2 * rl, gseq, gl);
  memcpy(a + 2 * rl + gl, galt, gl);
  p.rseq = 0;
  p.rseq_uc = rl;
  p.gseq = 2 * rl;
  p.gseq_alt = 2 * rl + gl;
}

template <typename S>
S **
fill_entry (const char *name, int precision, int variant, S ***dirN, S ***dirE, S ***dirF, Dynprog_T self,
            char *rseq, char *gseq, char *galt, int rlength, int glength, int mismatchtype, int open,
            int extend, int lband, int uband, gdp_bool_t jump_late_p, gdp_bool_t revp) {
  DropinThread &t = t_state;
  gdp_ctx *ctx = thread_ctx();
  if (self == nullptr) die("%s: no Dynprog_T", name);
  if (rlength <= 0 || glength <= 0 || rlength > self->max_rlength || glength > self->max_glength)
    die("%s: rlength %d / glength %d outside 1..%d / 1..%d of the Dynprog_T", name, rlength, glength,
        self->max_rlength, self->max_glength);
  const int W = (precision == 8) ? 32 : 16;
  const int X = (variant == GDP_LOWER) ? glength : rlength;
  const int Y = (variant == GDP_LOWER) ? rlength : glength;
  const int stride = (X + W) / W * W;
  const Planes P = planes_of(self, variant);

  gdp_pair_t p;
  memset(&p, 0, sizeof(p));
  p.rlength = rlength;
  p.glength = glength;
  p.lband = (variant == GDP_UPPER) ? 0 : lband;
  p.uband = (variant == GDP_LOWER) ? 0 : uband;
  p.variant = (int8_t) variant;
  p.precision = (int8_t) precision;
  p.mismatchtype = (int8_t) mismatchtype;
  p.flags = (int8_t) ((jump_late_p ? GDP_FLAG_JUMP_LATE : 0) | (revp ? GDP_FLAG_REVP : 0));
  p.open = (int16_t) open;
  p.extend = (int16_t) extend;
  p.tb_r = rlength;
  p.tb_c = glength;
  stage_arena(t.arena, p, rseq, rseq, gseq, galt, revp != 0);

  SpaceFill &sf = t.claim(P.nptrs);
  sf.precision = 0;   /* unusable until the fill below succeeds */
  int rc = gdpi_fill_run(ctx, sf.f, &p, t.arena.data(), (int64_t) t.arena.size());
  if (rc != GDP_OK) die("%s: device fill failed (status %d): %s", name, rc, gdp_last_error(ctx));
  const gdp_result_t &res = *gdpi_fill_result(sf.f);
  if (res.status != GDP_OK)
    die("%s: pair rejected (status %d; rlength %d glength %d lband %d uband %d open %d extend %d)", name,
        res.status, rlength, glength, lband, uband, open, extend);

  S **H = lay_out<S>(P.mptrs, P.mspace, Y, stride);
  S **N = lay_out<S>(P.nptrs, P.nspace, Y, stride);
  S **E = lay_out<S>(P.eptrs, P.espace, Y, stride);
  S **F = nullptr;
  if (P.fptrs) {
    F = lay_out<S>(P.fptrs, P.fspace, Y, stride);
    memset(P.fspace, 0, (size_t) (Y + 1) * stride * sizeof(S));
  }

  /* expand the block-column words of every swept cell */
  gdp_geom_t g;
  gdp_geom_of(&p, W, &g);
  const int64_t base = gdpi_fill_base(sf.f);
  const uint32_t *words = gdpi_fill_words(sf.f) + base;
  const int16_t *scores = gdpi_fill_scores(sf.f) + base * 8;
  int64_t boff = 0;
  for (int xlo = 0; xlo <= X; xlo += W) {
    int y0, y1;
    gdp_block_sweep(&g, xlo, &y0, &y1);
    for (int y = y0; y <= y1; y++) {
      const int64_t col = boff + (int64_t) (y - y0) * (W / 8);
      S *h = H[y] + xlo, *n = N[y] + xlo, *e = E[y] + xlo, *f = F ? F[y] + xlo : nullptr;
      const int16_t *sc = scores + col * 8;   /* the column's scores, lane by lane */
      for (int lane = 0; lane < W; lane++) {
        const uint32_t w = words[col + gdp_dir_word(W, lane)];
        const int i = gdp_dir_bit(W, lane);
        h[lane] = (S) sc[lane];
        n[lane] = (S) (((w >> (8 + i)) & 1) ? DIR_VERT : ((w >> i) & 1) ? DIR_HORIZ : DIR_DIAG);
        e[lane] = (S) (((w >> (16 + i)) & 1) ? DIR_HORIZ : DIR_DIAG);
        if (f) f[lane] = (S) (((w >> (24 + i)) & 1) ? DIR_VERT : DIR_DIAG);
      }
    }
    boff += gdp_block_words(&g, xlo);
  }

  sf.precision = precision;
  sf.variant = variant;
  sf.col0 = N[0];
  *dirN = N;
  *dirE = E;
  if (dirF) *dirF = F;
  return H;
}

/* Genome characters of every position a short genome skip of this
   traceback can read (get_genomic_nt, src/pairpool.c:1015-1063), fetched
   through the caller's Genome_get_char and packed as genomecomp blocks. */
void
stage_genome_window (DropinThread &t, const gdp_pair_t &p, Genome_T genome, Genome_T genomealt,
                     uint64_t *gbase, uint64_t *glen) {
  *gbase = 0;
  *glen = 0;
  const getchar_fn getch = gmap_syms().getchar;
  if (genome == nullptr || getch == nullptr) return;
  const bool revp = (p.flags & GDP_FLAG_REVP) != 0;
  const int gl = p.glength;
  uint64_t lo = UINT64_MAX, hi = 0;
  /* genome skips address coordinates c - dist .. c - 1; the E walk that
     reaches column 0 leaves them one past the window (src/dynprog_simd.c:9174),
     so a margin of two on either side covers every reachable position */
  for (int k = -2; k < gl + 2; k++) {
    const int gp = p.genomeoffset + (revp ? -k : k);
    const uint32_t pos = p.watsonp ? p.chroffset + (uint32_t) gp : p.chrhigh - (uint32_t) gp;
    if (pos < p.chroffset || pos >= p.chrhigh) continue;
    lo = std::min<uint64_t>(lo, pos);
    hi = std::max<uint64_t>(hi, pos);
  }
  if (lo > hi) return;
  if (hi - lo > (uint64_t) gl + 64) die("traceback: genome positions of one window wrap around");
  const uint64_t b = lo & ~(uint64_t) 31;
  const uint64_t n = hi - b + 1;
  const size_t nblk = (size_t) (n + 31) / 32;
  t.gwin.assign(nblk * 32, 'A');
  t.gwinalt.assign(nblk * 32, 'A');
  for (uint64_t pos = lo; pos <= hi; pos++) {
    char alt = 'N';
    const char c = getch(&alt, genome, genomealt ? genomealt : genome, (Univcoord_T) pos);
    t.gwin[pos - b] = c;
    t.gwinalt[pos - b] = (c == 'N') ? 'A' : alt;
  }
  t.gblk.assign(nblk * 3, 0);
  t.galtblk.assign(nblk * 3, 0);
  gdp_workload_genomecomp(t.gwin.data(), (int64_t) (nblk * 32), t.gblk.data());
  gdp_workload_genomecomp(t.gwinalt.data(), (int64_t) (nblk * 32), t.galtblk.data());
  *gbase = b;
  *glen = n;
}

template <typename S>
List_T
traceback_entry (const char *name, int precision, int variant, List_T pairs, int *traceback_score,
                 int *nmatches, int *nmismatches, int *nopens, int *nindels, S **dirN, int r, int c,
                 char *rseq, char *ruc, char *gseq, char *galt, int queryoffset, int genomeoffset,
                 Genome_T genome, Genome_T genomealt, Pairpool_T pool, gdp_bool_t revp, Univcoord_T chroffset,
                 Univcoord_T chrhigh, gdp_bool_t watsonp, int genestrand, int dynprogindex) {
  DropinThread &t = t_state;
  gdp_ctx *ctx = thread_ctx();
  const GmapSyms &syms = gmap_syms();
  if (syms.push == nullptr || syms.gapholder == nullptr)
    die("%s: Pairpool_push / Pairpool_push_gapholder are not defined in this process", name);
  SpaceFill *sf = t.find(dirN);
  if (sf == nullptr || sf->precision != precision || sf->variant != variant || dirN[0] != sf->col0)
    die("%s: the direction planes are not those of this thread's latest %d-bit fill of that space", name,
        precision);
  gdp_pair_t p = *gdpi_fill_pair(sf->f);
  if (r < 0 || c < 0 || r > p.rlength || c > p.glength)
    die("%s: start (%d, %d) outside the filled %d x %d matrix", name, r, c, p.rlength, p.glength);
  p.flags = (int8_t) ((p.flags & GDP_FLAG_JUMP_LATE) | (revp ? GDP_FLAG_REVP : 0) | GDP_FLAG_TRACEBACK);
  p.tb_r = r;
  p.tb_c = c;
  p.queryoffset = queryoffset;
  p.genomeoffset = genomeoffset;
  p.chroffset = (uint32_t) chroffset;
  p.chrhigh = (uint32_t) chrhigh;
  p.watsonp = (int8_t) (watsonp ? 1 : 0);
  p.genestrand = (int8_t) genestrand;
  p.dynprogindex = dynprogindex;
  stage_arena(t.arena, p, rseq, ruc, gseq, galt, revp != 0);
  uint64_t gbase = 0, glen = 0;
  if (variant != GDP_LOWER) stage_genome_window(t, p, genome, genomealt, &gbase, &glen);

  gdp_result_t res;
  const int rc = gdpi_traceback_one(ctx, sf->f, &p, t.arena.data(), (int64_t) t.arena.size(),
                                    glen ? t.gblk.data() : nullptr, glen ? t.galtblk.data() : nullptr, gbase,
                                    glen, &res, &t.recs);
  if (rc != GDP_OK) die("%s: device traceback failed (status %d): %s", name, rc, gdp_last_error(ctx));
  if (res.status == GDP_ERR_NOGENOME)
    die("%s: a short genome skip needs the genome, and none was given", name);
  if (res.status == GDP_ERR_BAND && !t.warned_band) {
    /* The reference's walk reads cells its fill never wrote: its result is
       that of uninitialised memory.  The walk up to that point is kept. */
    fprintf(stderr, "libgdp: %s: the traceback left the filled cells at a band edge; "
                    "its Pair list stops there\n", name);
    t.warned_band = true;
  } else if (res.status != GDP_OK && res.status != GDP_ERR_BAND) {
    die("%s: traceback status %d", name, res.status);
  }
  const int64_t nrecs = std::min<int64_t>(res.nrecs, (int64_t) t.recs.size());
  for (int64_t k = 0; k < nrecs; k++) {
    const gdp_rec_t &x = t.recs[k];
    if (x.comp == '\0')   /* gap holder: genomepos holds the skipped genome length */
      pairs = syms.gapholder(pairs, pool, 0, x.genomepos, nullptr, nullptr, 0);
    else
      pairs = syms.push(pairs, pool, x.querypos, x.genomepos, x.cdna, x.comp, x.genome, x.genomealt,
                        dynprogindex);
  }
  *traceback_score += res.tb_score;
  *nmatches += res.nmatches;
  *nmismatches += res.nmismatches;
  *nopens += res.nopens;
  *nindels += res.nindels;
  return pairs;
}

}  // namespace

/* ------------------------------------------------------------------ */
/* src/dynprog_simd.h:17-77                                            */
/* ------------------------------------------------------------------ */

extern "C" Score8_T **
Dynprog_simd_8 (Direction8_T ***directions_nogap, Direction8_T ***directions_Egap,
                Direction8_T ***directions_Fgap, Dynprog_T dynprog, char *rsequence, char *gsequence,
                char *gsequence_alt, int rlength, int glength, Mismatchtype_T mismatchtype, int open, int extend,
                int lband, int uband, gdp_bool_t jump_late_p, gdp_bool_t revp) {
  return fill_entry<Score8_T>("Dynprog_simd_8", 8, GDP_FULL, directions_nogap, directions_Egap, directions_Fgap,
                              dynprog, rsequence, gsequence, gsequence_alt, rlength, glength, mismatchtype, open,
                              extend, lband, uband, jump_late_p, revp);
}

extern "C" Score8_T **
Dynprog_simd_8_upper (Direction8_T ***directions_nogap, Direction8_T ***directions_Egap, Dynprog_T dynprog,
                      char *rsequence, char *gsequence, char *gsequence_alt, int rlength, int glength,
                      Mismatchtype_T mismatchtype, int open, int extend, int uband, gdp_bool_t jump_late_p,
                      gdp_bool_t revp) {
  return fill_entry<Score8_T>("Dynprog_simd_8_upper", 8, GDP_UPPER, directions_nogap, directions_Egap, nullptr,
                              dynprog, rsequence, gsequence, gsequence_alt, rlength, glength, mismatchtype, open,
                              extend, 0, uband, jump_late_p, revp);
}

extern "C" Score8_T **
Dynprog_simd_8_lower (Direction8_T ***directions_nogap, Direction8_T ***directions_Egap, Dynprog_T dynprog,
                      char *rsequence, char *gsequence, char *gsequence_alt, int rlength, int glength,
                      Mismatchtype_T mismatchtype, int open, int extend, int lband, gdp_bool_t jump_late_p,
                      gdp_bool_t revp) {
  return fill_entry<Score8_T>("Dynprog_simd_8_lower", 8, GDP_LOWER, directions_nogap, directions_Egap, nullptr,
                              dynprog, rsequence, gsequence, gsequence_alt, rlength, glength, mismatchtype, open,
                              extend, lband, 0, jump_late_p, revp);
}

extern "C" Score16_T **
Dynprog_simd_16 (Direction16_T ***directions_nogap, Direction16_T ***directions_Egap,
                 Direction16_T ***directions_Fgap, Dynprog_T dynprog, char *rsequence, char *gsequence,
                 char *gsequence_alt, int rlength, int glength, Mismatchtype_T mismatchtype, int open, int extend,
                 int lband, int uband, gdp_bool_t jump_late_p, gdp_bool_t revp) {
  return fill_entry<Score16_T>("Dynprog_simd_16", 16, GDP_FULL, directions_nogap, directions_Egap,
                               directions_Fgap, dynprog, rsequence, gsequence, gsequence_alt, rlength, glength,
                               mismatchtype, open, extend, lband, uband, jump_late_p, revp);
}

extern "C" Score16_T **
Dynprog_simd_16_upper (Direction16_T ***directions_nogap, Direction16_T ***directions_Egap, Dynprog_T dynprog,
                       char *rsequence, char *gsequence, char *gsequence_alt, int rlength, int glength,
                       Mismatchtype_T mismatchtype, int open, int extend, int uband, gdp_bool_t jump_late_p,
                       gdp_bool_t revp) {
  return fill_entry<Score16_T>("Dynprog_simd_16_upper", 16, GDP_UPPER, directions_nogap, directions_Egap, nullptr,
                               dynprog, rsequence, gsequence, gsequence_alt, rlength, glength, mismatchtype, open,
                               extend, 0, uband, jump_late_p, revp);
}

extern "C" Score16_T **
Dynprog_simd_16_lower (Direction16_T ***directions_nogap, Direction16_T ***directions_Egap, Dynprog_T dynprog,
                       char *rsequence, char *gsequence, char *gsequence_alt, int rlength, int glength,
                       Mismatchtype_T mismatchtype, int open, int extend, int lband, gdp_bool_t jump_late_p,
                       gdp_bool_t revp) {
  return fill_entry<Score16_T>("Dynprog_simd_16_lower", 16, GDP_LOWER, directions_nogap, directions_Egap, nullptr,
                               dynprog, rsequence, gsequence, gsequence_alt, rlength, glength, mismatchtype, open,
                               extend, lband, 0, jump_late_p, revp);
}

/* ------------------------------------------------------------------ */
/* src/dynprog_simd.h:79-126                                           */
/* ------------------------------------------------------------------ */

extern "C" List_T
Dynprog_traceback_8 (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens,
                     int *nindels, Direction8_T **directions_nogap, Direction8_T **directions_Egap,
                     Direction8_T **directions_Fgap, int r, int c, char *rsequence, char *rsequenceuc,
                     char *gsequence, char *gsequence_alt, int queryoffset, int genomeoffset, Genome_T genome,
                     Genome_T genomealt, Pairpool_T pairpool, gdp_bool_t revp, Univcoord_T chroffset,
                     Univcoord_T chrhigh, gdp_bool_t watsonp, int genestrand, int dynprogindex) {
  (void) directions_Egap; (void) directions_Fgap;
  return traceback_entry<Direction8_T>("Dynprog_traceback_8", 8, GDP_FULL, pairs, traceback_score, nmatches,
                                       nmismatches, nopens, nindels, directions_nogap, r, c, rsequence,
                                       rsequenceuc, gsequence, gsequence_alt, queryoffset, genomeoffset, genome,
                                       genomealt, pairpool, revp, chroffset, chrhigh, watsonp, genestrand,
                                       dynprogindex);
}

extern "C" List_T
Dynprog_traceback_8_upper (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens,
                           int *nindels, Direction8_T **directions_nogap, Direction8_T **directions_Egap, int r,
                           int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                           int queryoffset, int genomeoffset, Genome_T genome, Genome_T genomealt,
                           Pairpool_T pairpool, gdp_bool_t revp, Univcoord_T chroffset, Univcoord_T chrhigh,
                           gdp_bool_t watsonp, int genestrand, int dynprogindex) {
  (void) directions_Egap;
  return traceback_entry<Direction8_T>("Dynprog_traceback_8_upper", 8, GDP_UPPER, pairs, traceback_score,
                                       nmatches, nmismatches, nopens, nindels, directions_nogap, r, c, rsequence,
                                       rsequenceuc, gsequence, gsequence_alt, queryoffset, genomeoffset, genome,
                                       genomealt, pairpool, revp, chroffset, chrhigh, watsonp, genestrand,
                                       dynprogindex);
}

extern "C" List_T
Dynprog_traceback_8_lower (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens,
                           int *nindels, Direction8_T **directions_nogap, Direction8_T **directions_Egap, int r,
                           int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                           int queryoffset, int genomeoffset, Pairpool_T pairpool, int genestrand,
                           gdp_bool_t revp, int dynprogindex) {
  (void) directions_Egap;
  return traceback_entry<Direction8_T>("Dynprog_traceback_8_lower", 8, GDP_LOWER, pairs, traceback_score,
                                       nmatches, nmismatches, nopens, nindels, directions_nogap, r, c, rsequence,
                                       rsequenceuc, gsequence, gsequence_alt, queryoffset, genomeoffset, nullptr,
                                       nullptr, pairpool, revp, 0, 0, 1, genestrand, dynprogindex);
}

extern "C" List_T
Dynprog_traceback_16 (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens,
                      int *nindels, Direction16_T **directions_nogap, Direction16_T **directions_Egap,
                      Direction16_T **directions_Fgap, int r, int c, char *rsequence, char *rsequenceuc,
                      char *gsequence, char *gsequence_alt, int queryoffset, int genomeoffset, Genome_T genome,
                      Genome_T genomealt, Pairpool_T pairpool, gdp_bool_t revp, Univcoord_T chroffset,
                      Univcoord_T chrhigh, gdp_bool_t watsonp, int genestrand, int dynprogindex) {
  (void) directions_Egap; (void) directions_Fgap;
  return traceback_entry<Direction16_T>("Dynprog_traceback_16", 16, GDP_FULL, pairs, traceback_score, nmatches,
                                        nmismatches, nopens, nindels, directions_nogap, r, c, rsequence,
                                        rsequenceuc, gsequence, gsequence_alt, queryoffset, genomeoffset, genome,
                                        genomealt, pairpool, revp, chroffset, chrhigh, watsonp, genestrand,
                                        dynprogindex);
}

extern "C" List_T
Dynprog_traceback_16_upper (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens,
                            int *nindels, Direction16_T **directions_nogap, Direction16_T **directions_Egap, int r,
                            int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                            int queryoffset, int genomeoffset, Genome_T genome, Genome_T genomealt,
                            Pairpool_T pairpool, gdp_bool_t revp, Univcoord_T chroffset, Univcoord_T chrhigh,
                            gdp_bool_t watsonp, int genestrand, int dynprogindex) {
  (void) directions_Egap;
  return traceback_entry<Direction16_T>("Dynprog_traceback_16_upper", 16, GDP_UPPER, pairs, traceback_score,
                                        nmatches, nmismatches, nopens, nindels, directions_nogap, r, c, rsequence,
                                        rsequenceuc, gsequence, gsequence_alt, queryoffset, genomeoffset, genome,
                                        genomealt, pairpool, revp, chroffset, chrhigh, watsonp, genestrand,
                                        dynprogindex);
}

extern "C" List_T
Dynprog_traceback_16_lower (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens,
                            int *nindels, Direction16_T **directions_nogap, Direction16_T **directions_Egap, int r,
                            int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                            int queryoffset, int genomeoffset, Pairpool_T pairpool, int genestrand,
                            gdp_bool_t revp, int dynprogindex) {
  (void) directions_Egap;
  return traceback_entry<Direction16_T>("Dynprog_traceback_16_lower", 16, GDP_LOWER, pairs, traceback_score,
                                        nmatches, nmismatches, nopens, nindels, directions_nogap, r, c, rsequence,
                                        rsequenceuc, gsequence, gsequence_alt, queryoffset, genomeoffset, nullptr,
                                        nullptr, pairpool, revp, 0, 0, 1, genestrand, dynprogindex);
}

extern "C" void
gdp_dropin_release_thread (void) {
  t_state.release();
}
