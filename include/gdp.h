/*
 * gdp.h -- C ABI of the B200 banded affine-gap dynamic-programming library
 * (libgdp.so), a drop-in for the fills and tracebacks of GMAP's
 * src/dynprog_simd.c.
 *
 * Two layers are exported:
 *
 *  1. The batch API below (gdp_*): plain pointers and sizes, one call per
 *     batch of independent alignment pairs.  Each pair carries exactly the
 *     arguments of the reference entry point it replaces:
 *       Dynprog_simd_8 / Dynprog_simd_16           (src/dynprog_simd.h:16-26, :46-55)
 *       Dynprog_simd_8_upper / _16_upper           (src/dynprog_simd.h:27-35, :56-64)
 *       Dynprog_simd_8_lower / _16_lower           (src/dynprog_simd.h:37-45, :66-74)
 *       Dynprog_traceback_8 / _16                  (src/dynprog_simd.h:76-83, :102-109)
 *       Dynprog_traceback_8_upper / _16_upper      (src/dynprog_simd.h:85-92, :111-118)
 *       Dynprog_traceback_8_lower / _16_lower      (src/dynprog_simd.h:94-100, :120-125)
 *     rsequence/gsequence/gsequence_alt, rlength/glength, lband/uband,
 *     mismatchtype, open/extend, jump_late_p, revp, and for the traceback
 *     (r, c), rsequenceuc, queryoffset, genomeoffset, chroffset, chrhigh,
 *     watsonp, genestrand, dynprogindex keep the reference's meaning.
 *
 *  2. The twelve reference-signature entry points themselves, declared in
 *     gdp_dynprog_simd.h, implemented on top of the batch API.
 *
 * All arithmetic is integer and bit-exact with the reference's AVX2 build:
 * the final score, every in-band score and E/F/nogap direction, and the
 * traceback Pair list.
 */
#ifndef GDP_H
#define GDP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Variants: which reference fill a pair runs. */
enum {
  GDP_FULL = 0,   /* Dynprog_simd_{8,16}: band lband below, uband above the diagonal */
  GDP_UPPER = 1,  /* Dynprog_simd_{8,16}_upper: r <= c <= r + uband, horizontal gaps only */
  GDP_LOWER = 2   /* Dynprog_simd_{8,16}_lower: c <= r <= c + lband, vertical gaps only */
};

/* gdp_pair_t.flags */
enum {
  GDP_FLAG_JUMP_LATE = 1,   /* jump_late_p */
  GDP_FLAG_REVP = 2,        /* revp: sequences are read backwards from their last character */
  GDP_FLAG_TRACEBACK = 4,   /* run Dynprog_traceback_* from (tb_r, tb_c) */
  GDP_FLAG_RERUN16 = 8,     /* precision 8: rerun in 16-bit when the 8-bit fill overflows */
  GDP_FLAG_GWINDOW = 16,    /* the genome window comes from the resident genome (see below) */
  GDP_FLAG_ENDPOINT = 32,   /* end-gap endpoint search over the band (see below) */
  GDP_FLAG_ENDPOINT_QEND = 64  /* the same over the last query row only */
};

/* Mismatch types (src/dynprog.h:53) */
enum { GDP_HIGHQ = 0, GDP_MEDQ = 1, GDP_LOWQ = 2, GDP_ENDQ = 3 };

/* Per-pair and per-call status codes */
enum {
  GDP_OK = 0,
  GDP_ERR_LEN = 1,       /* rlength/glength <= 0 or above the library maximum */
  GDP_ERR_BAND = 2,      /* negative band, or the traceback start lies outside the filled band */
  GDP_ERR_PARAM = 3,     /* bad variant / precision / mismatchtype / open / extend */
  GDP_ERR_BUDGET = 4,    /* the pair's direction storage exceeds the context budget */
  GDP_ERR_TIMEOUT = 5,   /* a bounded device wait gave up */
  GDP_ERR_CUDA = 6,      /* a CUDA call failed */
  GDP_ERR_RECS = 7,      /* traceback record buffer too small */
  GDP_ERR_NOGENOME = 8   /* genome characters are needed beyond the resident genome (or none is loaded) */
};

/*
 * One alignment pair.  Sequence fields are byte offsets into the caller's
 * sequence arena.  Every sequence is stored forward in memory; with
 * GDP_FLAG_REVP the reference's convention (a pointer to the last character,
 * indexed seq[1-r]) is applied by the library.
 *
 * GDP_FLAG_GWINDOW: the device writes the genome window itself, from the
 * genome made resident by gdp_set_genome, into the arena at gseq (and at
 * gseq_alt from the alternate genome, when gseq_alt != gseq), before the
 * fill; the caller only reserves those glength bytes.  Window character j
 * is the character the traceback reads for genomic coordinate
 * genomeoffset + j (revp: genomeoffset - (glength - 1) + j): chroffset + gp
 * on the plus strand, the complement of chrhigh - gp on the minus strand,
 * '*' outside [chroffset, chrhigh) (get_genomic_nt, src/pairpool.c:1015).
 * A window that reaches past the resident genome gets GDP_ERR_NOGENOME.
 *
 * GDP_FLAG_ENDPOINT / GDP_FLAG_ENDPOINT_QEND (upper and lower fills, no
 * GDP_FLAG_RERUN16): the fill also runs its half of the reference's
 * end-gap endpoint search over the scores it computes.  Dynprog_end5_gap
 * and Dynprog_end3_gap fill the upper and the lower matrix of one gap and
 * scan both (src/dynprog_end.c:1415-1534): find_best_endpoint_{8,16}
 * (:143-294) takes the best cell of the band, rows 1..rlength, with a score
 * above 0 (jump early: the first such best cell in row-then-column order;
 * jump late: the last, from score 0 up); find_best_endpoint_to_queryend_
 * indels_{8,16} (:358-508) does the same on row rlength alone, from the
 * most negative score.  The upper fill scans its cells with c >= r, the
 * lower fill its cells with c < r, so one gap is two pairs (an upper and a
 * lower pair with the same sequences and flags); the result's end_score,
 * end_r and end_c hold each half's best, and gdp_endpoint_combine merges
 * the two halves into the reference's finalscore, bestr and bestc.  A
 * half whose final cell (rlength, glength) lies outside its triangle keeps
 * GDP_OK (its score is then NEG_INFINITY_8/16: the cell is not computed).
 */
typedef struct gdp_pair {
  int64_t rseq;          /* rsequence, rlength bytes */
  int64_t rseq_uc;       /* rsequenceuc (upper-case query), used by the traceback */
  int64_t gseq;          /* gsequence, glength bytes */
  int64_t gseq_alt;      /* gsequence_alt, glength bytes (may equal gseq) */
  int32_t rlength, glength;
  int32_t lband, uband;  /* FULL uses both; UPPER uses uband; LOWER uses lband */
  int8_t variant;        /* GDP_FULL / GDP_UPPER / GDP_LOWER */
  int8_t precision;      /* 8 or 16 */
  int8_t mismatchtype;   /* GDP_HIGHQ.. */
  int8_t flags;          /* GDP_FLAG_* */
  int16_t open, extend;  /* gap penalties, each in [-127, 0] */
  int32_t tb_r, tb_c;    /* traceback start (normally rlength, glength) */
  int32_t queryoffset, genomeoffset;
  uint32_t chroffset, chrhigh;
  int8_t watsonp, genestrand;
  int16_t xflags;        /* GDP_XFLAG_* (0 for the reference's fills and tracebacks) */
  int32_t dynprogindex;
} gdp_pair_t;

/* gdp_pair_t.xflags */
enum {
  /* GDP_FLAG_GWINDOW windows as Dynprog_single_gap reads its gsequence:
     Genome_get_segment_right on the plus strand (positions from
     chroffset + genomeoffset, '*' at and above chrhigh) and the reverse
     complement of Genome_get_segment_left on the minus strand (positions
     down from chrhigh - genomeoffset, '*' below chroffset), src/genome.c:
     11022-11120.  The two differ from get_genomic_nt only on the minus
     strand at genomic coordinate 0, which reads position chrhigh. */
  GDP_XFLAG_SEGMENT = 1,
  /* the mirrored segment, as Dynprog_end5_gap reads its rev_gsequence:
     Genome_get_segment_left on the plus strand ('*' below chroffset) and
     the reverse complement of Genome_get_segment_right on the minus strand
     ('*' at and above chrhigh) */
  GDP_XFLAG_SEGMENT_REV = 2
};

/*
 * One traceback Pair record, 12 bytes: the fields of the reference's struct
 * Pair_T (src/pairdef.h:10-50) that Dynprog_traceback_* sets.  Records of a
 * pair are stored in push order: the first record is the one the reference
 * pushes first (nearest the traceback start).  Pairpool_push records
 * (src/pairpool.c:169) carry querypos, genomepos and the four characters;
 * their dynprogindex is the pair's and their genomejump 0.  A gap holder
 * (Pairpool_push_gapholder, src/pairpool.c:374; the reference's Pair has
 * querypos = genomepos = -1, blank characters and genomejump = the skipped
 * genome length) is the record with comp == '\0': querypos = -1, genomepos =
 * the skipped genome length, cdna = genome = genomealt = ' '.  No pushed
 * record has comp == '\0' (comp is one of the reference's comparison
 * characters).
 */
typedef struct gdp_rec {
  int32_t querypos;
  int32_t genomepos;     /* gap holder: the skipped genome length */
  char cdna, comp, genome, genomealt;   /* gap holder: comp == '\0' */
} gdp_rec_t;

/* Per-pair result. */
typedef struct gdp_result {
  int32_t status;        /* GDP_OK or GDP_ERR_* */
  int32_t score;         /* matrix[glength][rlength] (lower: matrix[rlength][glength]); NEG_INFINITY_8/16
                            when that cell lies outside the band of a fill without traceback */
  int32_t precision;     /* 8 or 16: the precision whose outputs were kept */
  int32_t rerun;         /* 1 if an 8-bit fill overflowed and was rerun in 16 bits */
  int32_t tb_score, nmatches, nmismatches, nopens, nindels;  /* traceback totals */
  int32_t nrecs;         /* number of Pair records */
  int64_t rec_offset;    /* index of the first record in the record buffer */
  int32_t end_score, end_r, end_c;  /* GDP_FLAG_ENDPOINT*: this half's best cell (else 0) */
  int32_t end_found;     /* 1 if a cell of this half passed the search's threshold */
} gdp_result_t;

/*
 * Merges the endpoint-search halves of one end gap (the upper and the lower
 * pair's results, GDP_FLAG_ENDPOINT or GDP_FLAG_ENDPOINT_QEND, the same
 * jump_late_p) into the reference's finalscore, bestr and bestc
 * (find_best_endpoint_{8,16}, src/dynprog_end.c:143-294, and
 * find_best_endpoint_to_queryend_indels_{8,16}, :358-508).  `qend` selects
 * the last-row search, `precision` its starting score (NEG_INFINITY_8 or
 * _16) and `rlength` its default row.  Returns GDP_OK.
 */
int gdp_endpoint_combine(const gdp_result_t *upper, const gdp_result_t *lower, int jump_late, int qend,
                         int precision, int rlength, int *finalscore, int *bestr, int *bestc);

/*
 * The record-run codec: the records of one pair (push order) as a byte
 * stream, one byte for most records -- each follows from the record before
 * it and the pair's sequences in `arena` -- and 13 bytes for the others.
 * gdp_runs_encode returns the stream's length (out may be NULL to size
 * it), or -GDP_ERR_PARAM; gdp_runs_decode rebuilds the records byte for
 * byte from the same pair and arena (GDP_ERR_PARAM for a malformed
 * stream).  Pairs with GDP_FLAG_GWINDOW encode every record whole.
 * gdp_align_batch uses the same codec to bring records to the host.
 */
int64_t gdp_runs_encode(const gdp_pair_t *pair, const char *arena, const gdp_rec_t *recs, int32_t nrecs,
                        uint8_t *out);
int gdp_runs_decode(const gdp_pair_t *pair, const char *arena, const uint8_t *in, int64_t len, gdp_rec_t *recs,
                    int32_t nrecs);

typedef struct gdp_ctx gdp_ctx;

/* Library version string. */
const char *gdp_version(void);

/*
 * Creates a context on CUDA device `device`.  `mode` is the reference's
 * Mode_T (src/mode.h:4; 0 = STANDARD) and selects the substitution and
 * consistency tables built as Dynprog_init does (src/dynprog.c:1007-1196).
 * `dir_budget_bytes` bounds the device memory used for direction matrices
 * per wave of gdp_align_batch (0 = 40 GB): a wave ends before its pairs'
 * direction words would pass it (a pair larger than the budget runs in a
 * wave of its own).
 */
int gdp_ctx_create(gdp_ctx **ctx, int device, int mode, int64_t dir_budget_bytes);
void gdp_ctx_destroy(gdp_ctx *ctx);

/*
 * Makes a genome resident on the device, in the reference's genomecomp
 * format (three uint32 per 32 nt: high, low, N-flags; src/genome.c:9723).
 * `altblocks` may be NULL (then the alternate genome equals the genome).
 * Tracebacks read genome characters for short genome skips from it, as
 * Pairpool_add_genomeskip does through Genome_get_char.
 */
int gdp_set_genome(gdp_ctx *ctx, const uint32_t *blocks, const uint32_t *altblocks,
                   uint64_t genomelength);

/*
 * Aligns a batch end to end: host arena and pairs in, host results and
 * traceback records out.  Returns GDP_OK when every pair was processed
 * (per-pair failures are reported in results[i].status).  `recs` may be
 * NULL when no pair asks for a traceback.
 */
int gdp_align_batch(gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t npairs,
                    const char *arena, int64_t arena_bytes,
                    gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs,
                    int64_t *nrecs_used);

/*
 * gdp_align_batch over several contexts, typically one per GPU (contexts
 * on one GPU also work).  The pairs split into contiguous shards of about
 * equal band cells, one per context, each aligned by gdp_align_batch from
 * its own host thread: pairs are independent, so no data crosses between
 * devices, and each shard copies only its own part of the arena.  Every
 * context needs the genome set.  Results come back in pair order.  Shard
 * k's records start at the record slots of the pairs before it (a
 * traceback pair has rlength + glength + 2 slots), so records are in pair
 * order with gaps between shards: read pair i's records at
 * results[i].rec_offset (counted from recs), results[i].nrecs of them.
 * `max_recs` must hold the slots of every traceback pair (else
 * GDP_ERR_RECS before any work); *nrecs_used is the end of the last
 * shard's records.  Returns the first failing shard's status.  The
 * reference has no counterpart (it aligns one pair per call, on the
 * calling thread).
 */
int gdp_align_batch_multi(gdp_ctx *const *ctxs, int nctx, const gdp_pair_t *pairs, int64_t npairs,
                          const char *arena, int64_t arena_bytes,
                          gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs,
                          int64_t *nrecs_used);

/*
 * Plans for device-resident batches.  gdp_plan_create inspects the pairs
 * (host copy) once: it validates them, bins them by fill kind and work,
 * and lays out the device direction storage and the traceback record
 * slots.  gdp_plan_execute then enqueues the fills and tracebacks on the
 * context's stream for device-resident pairs / arena / results / records
 * (device pointers, same contents as planned) without synchronising the
 * host.  Record slots: pair i may write up to rlength + glength + 2
 * records starting at gdp_plan_rec_offset(plan, i).
 */
typedef struct gdp_plan gdp_plan;
int gdp_plan_create(gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t npairs, gdp_plan **plan);
int gdp_plan_execute(gdp_ctx *ctx, gdp_plan *plan, const gdp_pair_t *d_pairs, const char *d_arena,
                     gdp_result_t *d_results, gdp_rec_t *d_recs);
int64_t gdp_plan_total_recs(const gdp_plan *plan);
int64_t gdp_plan_rec_offset(const gdp_plan *plan, int64_t i);
int64_t gdp_plan_dir_bytes(const gdp_plan *plan);
void gdp_plan_destroy(gdp_plan *plan);

/*
 * With on != 0, gdp_plan_execute runs the plan's launches as one CUDA
 * graph: the first call with a given set of device pointers runs the plan
 * and captures its launches; later calls with the same pointers launch the
 * graph.  Calls with profiling enabled run without the graph.
 */
int gdp_plan_use_graph(gdp_plan *plan, int on);

/*
 * Routing parameters of a context (they take effect in later plans):
 *   "warp_min_x"     pairs with at least this many lanes (query rows; lower:
 *                    genome columns) go to the lane-group / one-CTA fills
 *   "warp_max_sweep" widest block sweep a lane group of 32 takes; wider
 *                    sweeps go one CTA per pair
 *   "group_slack"    a group of K lanes takes sweeps up to 17 K - slack
 *   "tb_warp"        1: tracebacks with one warp per pair, 0: one thread
 *   "check_groups"   1: the 8-bit pass of rerun pairs on lane groups,
 *                    0: one thread per pair, except ...
 *   "check_min_x"    ... pairs with at least this many lanes, whose 8-bit
 *                    pass goes to lane groups all the same
 *   "wave_pairs"     pairs per wave of gdp_align_batch
 *   "first_wave_pairs" pairs of its first wave (0: wave_pairs / 2, at least
 *                    16,384); each next wave holds twice the one before,
 *                    up to wave_pairs
 *   "wave_priority"  stream priority of a batch's first wave, 0 the highest
 *                    (later waves step down from it); the serving loop
 *                    runs its long-request batches below its short ones
 *   "grid_blocks_per_sm" at most this many blocks per SM in the fill and
 *                    traceback grids (0: no limit); the serving loop's long
 *                    batches keep to part of each SM, so that short batches
 *                    find block slots free
 *   "record_runs"    how gdp_align_batch's records leave the device: 0
 *                    (default) as 12-byte records; 1 as runs -- one byte
 *                    for most records, which follow from the one before and
 *                    the pair's sequences -- rebuilt byte for byte on host
 *                    threads (a sixteenth of the PCIe bytes, for hosts
 *                    whose PCIe is the bottleneck); 2 the waves from
 *                    "runs_from_wave" (default 5) on as runs, the earlier
 *                    ones plain
 * gdp_ctx_get_param also reads "last_d2h_bytes": the bytes the last
 * gdp_align_batch copied from the device to the host.
 * gdp_autotune times plan executions of a sample batch (device-resident
 * copies, the caller's pairs and arena) under candidate values of the first
 * six, one parameter at a time, and keeps the fastest; *best_ms gets the
 * sample's device time with the chosen values.  Results never depend on
 * these parameters.
 */
int gdp_ctx_set_param(gdp_ctx *ctx, const char *name, int64_t value);
int gdp_ctx_get_param(gdp_ctx *ctx, const char *name, int64_t *value);
int gdp_autotune(gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t npairs, const char *arena, int64_t arena_bytes,
                 double *best_ms);

/* Waits for the context's stream. */
int gdp_sync(gdp_ctx *ctx);

/*
 * Parity/debug entry: fills every pair and expands its in-band scores and
 * directions into dense (glength+1) x (rlength+1) arrays in (c, r) order
 * (out[c * (rlength+1) + r], lower variants transposed), covering the
 * reference's compare domain (src/dynprog_simd.c:1044-1051, :1089-1096,
 * :1134-1141).  Directions use the reference's codes: DIAG 0, HORIZ -1,
 * VERT -2.  dense_offsets[i] is pair i's first element in the dense arrays.
 * With H == NULL no scores are dumped, and the fills run exactly as a
 * production batch does (the same column bodies for every column); the
 * directions are then decoded from the production direction words.
 */
int gdp_fill_dump(gdp_ctx *ctx, const gdp_pair_t *pairs, int64_t npairs,
                  const char *arena, int64_t arena_bytes, const int64_t *dense_offsets,
                  int16_t *H, int8_t *dN, int8_t *dE, int8_t *dF, gdp_result_t *results);

/*
 * Host-only: fills caller arrays with the tables a context built for
 * `mode`: pd[4][128][128] (pairdistance_array), cons[3][128][128]
 * (consistent_array), nt2int[128] (nt_to_int_array).  Any may be NULL.
 */
int gdp_debug_tables(int mode, int16_t *pd, uint8_t *cons, int8_t *nt2int);

/* The context's CUDA stream (a cudaStream_t), for callers that time or
   order work against it. */
void *gdp_ctx_stream(gdp_ctx *ctx);

/*
 * Per-kernel timing.  While enabled, every kernel launch of the context is
 * bracketed by CUDA events on its stream.  gdp_profile_read(ctx, id, ...)
 * returns, for kernel id 0..127 (the fill kinds first, then the traceback,
 * result initialisation, integer-rate probe, rerun-list compaction, record
 * compaction and window extraction; unused ids have an empty name), its
 * name, total device milliseconds and launch count since the last reset.
 * While enabled, a plan's kernels run one after another on the context's
 * stream (without it, the jump-late fills run beside the jump-early ones
 * on a side stream), so that each launch's events time it alone.
 */
int gdp_profile_enable(gdp_ctx *ctx, int on);
int gdp_profile_read(gdp_ctx *ctx, int id, char *name, int name_cap, double *ms, int64_t *launches);
int gdp_profile_reset(gdp_ctx *ctx);

/* Integer issue rate of the device (32-bit lane-ops per second), measured
   with an ALU/FMA-pipe probe kernel: the denominator of the fill roofline. */
double gdp_measure_int_peak(gdp_ctx *ctx);

/*
 * No counterpart in the reference: a fill for callers that cannot allocate
 * device memory (code running inside another framework's memory pool, a
 * host that forbids allocation on its hot path, or a caller that owns all
 * of its buffers).  It runs the 16-bit full-band fill (Dynprog_simd_16
 * semantics) for device-resident pairs and arena, with no context, and
 * allocates nothing: its working memory is a fixed file-scope device array
 * of about 36 MB, held on each GPU that loads the library until exit.
 *
 *   npairs <= 65,536 per call, every pair full band and precision 16,
 *   glength <= 1,023; otherwise the call returns GDP_ERR_LEN (too many
 *   pairs) or the pair gets GDP_ERR_PARAM / GDP_ERR_LEN.  Only the flags
 *   GDP_FLAG_JUMP_LATE and GDP_FLAG_REVP are taken (no traceback, rerun,
 *   genome window or endpoint search): a pair with any other flag gets
 *   GDP_ERR_PARAM.  A pair whose rseq, gseq or gseq_alt bytes do not lie
 *   inside the arena's first arena_bytes gets GDP_ERR_LEN and is not read.
 *
 * Outputs: d_results[i] (status, score, precision) and pair i's direction
 * words (the library's block-column layout), written to d_dirs (8-byte
 * aligned) starting at word d_results[i].rec_offset.  A pair whose words do not fit into
 * dir_words_cap gets GDP_ERR_BUDGET.  Work is enqueued on `stream` (a
 * cudaStream_t; NULL for the legacy stream).
 *
 * The first call on a device sets up that device (it takes the array
 * addresses, uploads the tables for `mode` and waits for the upload), so it
 * should come before any stream capture; later calls must use the same
 * mode.  All calls share the array: calls that overlap on the GPU race and
 * must be ordered by the caller.  The call restores the calling thread's
 * current device before it returns, and neither fails on nor clears a CUDA
 * error that the caller's earlier work left pending.
 */
int gdp_fill16_noalloc(int device, int mode, const gdp_pair_t *d_pairs, int64_t npairs, const char *d_arena,
                       int64_t arena_bytes, uint32_t *d_dirs, int64_t dir_words_cap, gdp_result_t *d_results,
                       void *stream);

/*
 * Serving loop (continuous batching).  A server owns `nworkers` contexts
 * on `device` (tables of `mode`), each holding the resident genome (may be
 * NULL).  Requests of one or more pairs are submitted from any thread and
 * admitted while the direction-matrix memory of the admitted, unfinished
 * requests stays within `dir_budget_bytes` (0: 40 GB).
 *
 * Size classes.  A request is short (class 0) when none of its pairs has
 * a query or genome stretch longer than `short_max_length` (default 512
 * bases), else long (class 1): a lone pair's time on the device follows
 * its longest stretch (the fill's column steps run one after another).
 * Each class has its own arrival-
 * order queue, and a batch holds requests of one class only, so a short
 * request never waits for a long one in its batch.  With two or more
 * workers, the first `short_workers` (default: three in four, at least one
 * and at most all but one) take short
 * batches only; the others take long batches and, when no long request is
 * admissible, short ones.  Short batches compute on the highest stream
 * priority, long batches on the lowest.  A worker takes every admissible
 * waiting request of its class (up to `max_batch_pairs` pairs; 0: 131,072)
 * as one batch.  gdp_server_set_classes changes the threshold and the
 * split before the first submission.  Results do not depend on the
 * batching.
 *
 * gdp_server_submit copies the request and returns its id (>= 0), or
 * -GDP_ERR_* when it is malformed; a request larger than the budget
 * completes at once with GDP_ERR_BUDGET.  gdp_server_wait blocks until the
 * request is done and copies its results (rec_offset relative to `recs`),
 * records and latency (submit to results on the host, in ms).
 *
 * gdp_server_drive is a load generator: `nrequests` single-pair requests,
 * request k being pool[k % npool] (offsets into `arena`), submitted from the
 * calling thread at Poisson arrival times of `rate` requests per second.
 * It returns when all are done, with each request's latency, optionally its
 * result (results_out may be NULL; records are not kept), and the elapsed
 * time from the first arrival to the last completion.
 */
typedef struct gdp_server gdp_server;
int gdp_server_create(int device, int mode, int nworkers, int64_t dir_budget_bytes, int64_t max_batch_pairs,
                      const uint32_t *genome_blocks, const uint32_t *alt_blocks, uint64_t genome_length,
                      gdp_server **server);
int64_t gdp_server_submit(gdp_server *server, const gdp_pair_t *pairs, int64_t npairs, const char *arena,
                          int64_t arena_bytes);
int gdp_server_wait(gdp_server *server, int64_t id, gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs,
                    int64_t *nrecs, double *latency_ms);
int gdp_server_drive(gdp_server *server, const gdp_pair_t *pool, int64_t npool, const char *arena,
                     int64_t nrequests, double rate, uint64_t seed, gdp_result_t *results_out,
                     double *latency_ms, double *elapsed_s);
int gdp_server_stats(gdp_server *server, int64_t *batches, int64_t *pairs, int64_t *max_batch_pairs,
                     int64_t *peak_reserved_bytes, double *busy_s);
int gdp_server_set_classes(gdp_server *server, int64_t short_max_length, int short_workers);
/* The size class (0 short, 1 long) of a request of these pairs, or -GDP_ERR_PARAM. */
int gdp_server_class_of(gdp_server *server, const gdp_pair_t *pairs, int64_t npairs);
/* Batches and pairs run per class (arrays of 2). */
int gdp_server_class_stats(gdp_server *server, int64_t *batches, int64_t *pairs);
void gdp_server_destroy(gdp_server *server);

/*
 * Dynprog_single_gap (src/dynprog_single.c:428-675) for a batch of gaps:
 * the single-gap step of GMAP's stage 3 (src/stage3.c:9117), which fills
 * the gap between two aligned blocks and traces it back.  Per gap, as the
 * reference does:
 *   - rlength <= 0, glength <= 0, or either above max_rlength / max_glength
 *     (the caller's Dynprog_T sizes): no pairs, traceback score
 *     NEG_INFINITY_32 (-32768), counts 0 (path GDP_SINGLE_NULL);
 *   - the genome segment is read from the resident genome (gdp_set_genome)
 *     as Genome_get_segment_right / _left read it (GDP_XFLAG_SEGMENT);
 *   - glength == rlength: the ungapped diagonal (single_gap_simple, :345)
 *     when it has at most one mismatch and at least one pair (path
 *     GDP_SINGLE_SIMPLE, nopens = nindels = 0);
 *   - otherwise Dynprog_compute_bands(extraband_single, widebandp), the
 *     8-bit fill and traceback when rlength and glength are both below
 *     use8p_size[mismatchtype] (41 HIGHQ, 63 MEDQ, 127 LOWQ), else the
 *     16-bit ones, from (rlength, glength) (path GDP_SINGLE_DP).
 * mismatchtype, open and extend follow defect_rate (DEFECT_HIGHQ 0.003,
 * DEFECT_MEDQ 0.014) or gdp_single_setup's user penalties.
 *
 * results[i]: status, score (matrix[glength][rlength] of the DP path, else
 * 0), precision (8 or 16 for the DP path, else 0), the traceback totals
 * and the gap's records at rec_offset in `recs`.  Records come in the order
 * of the List the reference returns, head first (the DP path's push order
 * after its List_reverse; the simple path from its last query position
 * down).  path[i] (may be NULL) gets the path taken.  The caller advances
 * its dynprogindex by one per gap, as the reference does.  When the
 * records do not fit into max_recs, the first gap whose records pass it and
 * every later gap with records get GDP_ERR_RECS (and no records).
 * The context keeps the call's working memory for the next call, so calls
 * on one context must not overlap (one context per thread, or the gap
 * queue below).
 */
typedef struct gdp_single_gap {
  int64_t rseq;          /* rsequence (&queryseq_ptr[querydp5]), rlength bytes of the arena */
  int64_t rseq_uc;       /* rsequenceuc (&queryuc_ptr[querydp5]) */
  int32_t rlength, glength;       /* queryjump, genomejump */
  int32_t roffset, goffset;       /* querydp5, genomedp5 */
  uint32_t chroffset, chrhigh;
  int8_t watsonp, genestrand, jump_late_p, widebandp;
  int32_t extraband_single;
  double defect_rate;
  int32_t max_rlength, max_glength;   /* dynprog->max_rlength, dynprog->max_glength */
  int32_t dynprogindex;
  int32_t pad;
} gdp_single_gap_t;

enum { GDP_SINGLE_NULL = 0, GDP_SINGLE_SIMPLE = 1, GDP_SINGLE_DP = 2 };

/* Dynprog_single_setup (src/dynprog_single.c:100): user gap penalties for
   later gdp_single_gap_batch calls on the context.  homopolymerp != 0 is
   rejected (GDP_ERR_PARAM): the reference's homopolymer branch fills with a
   gsequence it never sets (src/dynprog_single.c:524-546). */
int gdp_single_setup(gdp_ctx *ctx, int user_open, int user_extend, int user_dynprog_p, int homopolymerp);

int gdp_single_gap_batch(gdp_ctx *ctx, const gdp_single_gap_t *gaps, int64_t ngaps, const char *arena,
                         int64_t arena_bytes, gdp_result_t *results, int8_t *path, gdp_rec_t *recs,
                         int64_t max_recs, int64_t *nrecs_used);

/*
 * Dynprog_end5_gap / Dynprog_end3_gap (src/dynprog_end.c:1293-1650,
 * :1923-2245) for a batch of end gaps: the alignment of a read end beyond
 * its last aligned block, which GMAP's stage 3 runs for the 5' and 3' ends
 * of every alignment.  Per gap, as the reference does:
 *   - mismatch type ENDQ; open / extend by defect_rate (END_OPEN_* /
 *     END_EXTEND_*: -10/-2 below DEFECT_HIGHQ, -8/-2 below DEFECT_MEDQ,
 *     -6/-2 above) or gdp_end_setup's user penalties;
 *   - rlength <= 0, glength <= 0, or (end 5) goffset < 0: no pairs, score
 *     and counts 0; otherwise rlength and glength are cut to max_rlength /
 *     max_glength (the caller's Dynprog_T sizes);
 *   - the genome segment from the resident genome: end 3 as
 *     Genome_get_segment_right (plus strand, from chroffset + goffset) or
 *     the reverse complement of Genome_get_segment_left (minus strand, down
 *     from chrhigh - goffset); end 5 as Genome_get_segment_left (plus
 *     strand, ending at chroffset + goffset) or the reverse complement of
 *     Genome_get_segment_right (minus strand, from chrhigh - goffset), read
 *     backwards (src/genome.c:11022-11120);
 *   - GDP_QUERYEND_GAP and GDP_BEST_LOCAL: wide bands (Dynprog_compute_bands
 *     with extraband_end), an upper and a lower fill, the best cell of the
 *     band (find_best_endpoint_*); GDP_QUERYEND_INDELS: narrow bands and the
 *     best cell of the last query row (find_best_endpoint_to_queryend_
 *     indels_*); 8-bit fills when rlength or glength is below 24
 *     (use8p_size[ENDQ], the || rule), else 16-bit; end 5 fills backwards
 *     with the tie rule reversed (!jump_late_p), end 3 forwards;
 *   - the traceback from the best cell, through the upper fill when
 *     bestc >= bestr, else the lower; none with require_pos_score_p;
 *   - GDP_QUERYEND_GAP / GDP_BEST_LOCAL: a traceback with nmatches + 1 <
 *     nmismatches returns no pairs and score 0 (the counts stay); otherwise
 *     the pairs come in the order of the reference's returned List (head
 *     first), without its leading indel pairs.
 * GDP_QUERYEND_NOGAPS gaps and gaps with an end other than 5 or 3 get
 * GDP_ERR_PARAM (not built).  results[i]: status, tb_score (the traceback
 * score), the counts, nrecs records at rec_offset in `recs`, precision, and
 * in end_score / end_r / end_c the best cell the search found (all 0 for a
 * gap that ran no search: no pairs by the length checks, or
 * require_pos_score_p).  When the records do not fit into max_recs, the
 * first gap whose records pass it and every later gap with records get
 * GDP_ERR_RECS (and no records).  The reference advances dynprogindex away
 * from zero once per gap that passes the length checks (rlength > 0,
 * glength > 0, end 5 goffset >= 0); the caller does the same.  Queries more
 * than one base longer than their genome stretch (after the cuts) have no
 * defined reference result: its endpoint scan then reads lower-matrix cells
 * beyond glength that no fill wrote; here those cells do not exist.  The
 * fills read rseq: the substitution tables score a lower-case query letter
 * as its upper-case letter, so this equals the reference's fill with
 * rsequenceuc when rseq_uc holds rseq upper-cased.  Calls on one context
 * must not overlap.
 */
typedef struct gdp_end_gap {
  int64_t rseq;          /* the reference's sequence pointer as an arena offset: end 5, rev_rsequence (the
                            query's last character, read backwards); end 3, rsequence (its first) */
  int64_t rseq_uc;       /* rev_rsequenceuc / rsequenceuc, the same way */
  int32_t rlength, glength;
  int32_t roffset, goffset;       /* rev_roffset, rev_goffset (end 5); roffset, goffset (end 3) */
  uint32_t chroffset, chrhigh;
  int8_t end;                     /* 5 or 3 */
  int8_t endalign;                /* GDP_QUERYEND_GAP, GDP_QUERYEND_INDELS, GDP_QUERYEND_NOGAPS, GDP_BEST_LOCAL */
  int8_t watsonp, genestrand, jump_late_p, require_pos_score_p;
  int16_t pad;
  int32_t extraband_end;
  int32_t max_rlength, max_glength;   /* dynprog->max_rlength, dynprog->max_glength */
  int32_t dynprogindex;
  double defect_rate;
} gdp_end_gap_t;

/* Endalign_T (src/dynprog.h:24) */
enum { GDP_QUERYEND_GAP = 0, GDP_QUERYEND_INDELS = 1, GDP_QUERYEND_NOGAPS = 2, GDP_BEST_LOCAL = 3 };

/* Dynprog_end_setup (src/dynprog_end.c:118): user gap penalties for later
   gdp_end_gap_batch calls on the context. */
int gdp_end_setup(gdp_ctx *ctx, int user_open, int user_extend, int user_dynprog_p);

int gdp_end_gap_batch(gdp_ctx *ctx, const gdp_end_gap_t *gaps, int64_t ngaps, const char *arena,
                      int64_t arena_bytes, gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs,
                      int64_t *nrecs_used);

/*
 * Dynprog_cdna_gap (src/dynprog_cdna.c:786-1290) for a batch of gaps: the
 * gap GMAP's stage 3 solves where the read holds more than the genome
 * between two aligned blocks (src/stage3.c:9313).  The query stretch left
 * of the gap (rlengthL bases from roffsetL) and the one right of it
 * (rlengthR bases back from rev_roffsetR) are each aligned against the
 * genome stretch between the blocks (glength bases from goffset), the left
 * one forwards and the right one backwards, and the best bridge between the
 * two is chosen (bridge_cdna_gap_{8,16}_ud).  Per gap, as the reference
 * does:
 *   - glength <= 1: no pairs, dynprogindex unchanged; glength or either
 *     rlength above the Dynprog_T maxima: no pairs, dynprogindex advanced;
 *   - mismatch type by defect_rate (HIGHQ / MEDQ / LOWQ), open -10 and
 *     extend -7 (CDNA_OPEN_* / CDNA_EXTEND_*);
 *   - Dynprog_compute_bands(extraband_paired, wide) for each side; 8-bit
 *     fills when glength < use8p_size or (rlengthL < use8p_size and
 *     rlengthR <= use8p_size), else 16-bit;
 *   - the upper and lower fill of each side (the right side reversed, with
 *     the tie rule reversed), the bridge search over their scores, the right
 *     traceback, then a cDNA insertion (queryjump == genomejump == 9: the
 *     skipped query bases, then the skipped genome bases with '~') or a gap
 *     holder (incomplete), then the left traceback;
 *   - a List of the gap holder alone is returned as no pairs.
 * The query bytes from roffsetL through rev_roffsetR lie contiguously in
 * the arena: rseq / rseq_uc are the arena offsets of query position
 * roffsetL.  results[i]: status, tb_score (both tracebacks' score, the
 * reference's finalscore output), score (the bridge's best score), the
 * counts, precision, nrecs records at rec_offset in `recs` (the returned
 * List, head first; its gap holder has comp '\0', querypos = -1 -
 * queryjump and genomepos = genomejump), and end_found = 1 when the gap
 * was left incomplete (the reference's *incompletep).  A gap whose bridge
 * finds no candidate has no defined reference result and gets
 * GDP_ERR_BAND.  The caller advances its dynprogindex as the reference
 * does.  Calls on one context must not overlap.
 */
typedef struct gdp_cdna_gap {
  int64_t rseq;            /* rsequenceL (&queryseq_ptr[roffsetL]) */
  int64_t rseq_uc;         /* rsequence_ucL */
  int32_t rlengthL, rlengthR, glength;
  int32_t roffsetL, rev_roffsetR, goffset;
  uint32_t chroffset, chrhigh;
  int8_t watsonp, genestrand, jump_late_p, pad8;
  int32_t extraband_paired;
  int32_t max_rlength, max_glength;   /* dynprogL / dynprogR maxima (GMAP sizes both alike) */
  int32_t dynprogindex;
  int32_t pad32;
  double defect_rate;
} gdp_cdna_gap_t;

int gdp_cdna_gap_batch(gdp_ctx *ctx, const gdp_cdna_gap_t *gaps, int64_t ngaps, const char *arena,
                       int64_t arena_bytes, gdp_result_t *results, gdp_rec_t *recs, int64_t max_recs,
                       int64_t *nrecs_used);

/*
 * Stage-3 batching adapter.  GMAP's stage 3 calls Dynprog_single_gap once
 * per gap from each worker thread (src/stage3.c:9117).  A gap queue keeps
 * that call shape -- one gap, its rsequence / rsequenceuc by pointer, a
 * blocking call -- and aligns the gaps of all calling threads together: a
 * worker thread owning a context on `device` (tables of `mode`, the genome
 * resident) runs every waiting gap (up to max_batch, 0: 4,096) as one
 * gdp_single_gap_batch once max_batch gaps wait or the oldest has waited
 * max_wait_us.  gdp_gap_queue_align ignores gap->rseq / rseq_uc, returns
 * when the gap is done, with its result (rec_offset 0), path and records
 * (GDP_ERR_RECS when more than max_recs), and the batch call's return code.
 * Results do not depend on the batching.  gdp_gap_queue_setup is
 * Dynprog_single_setup and must come before the first gdp_gap_queue_align;
 * gdp_gap_queue_destroy must come after the last one has returned.
 */
typedef struct gdp_gap_queue gdp_gap_queue;
int gdp_gap_queue_create(int device, int mode, int64_t max_batch, int64_t max_wait_us,
                         const uint32_t *genome_blocks, const uint32_t *alt_blocks, uint64_t genome_length,
                         gdp_gap_queue **queue);
int gdp_gap_queue_setup(gdp_gap_queue *queue, int user_open, int user_extend, int user_dynprog_p, int homopolymerp);
int gdp_gap_queue_align(gdp_gap_queue *queue, const gdp_single_gap_t *gap, const char *rsequence,
                        const char *rsequenceuc, gdp_result_t *result, int8_t *path, gdp_rec_t *recs,
                        int64_t max_recs, int64_t *nrecs);
int gdp_gap_queue_stats(gdp_gap_queue *queue, int64_t *batches, int64_t *gaps, int64_t *max_batch);
void gdp_gap_queue_destroy(gdp_gap_queue *queue);

/* Kernel launches issued by the context since creation (one per kernel). */
int64_t gdp_launch_count(gdp_ctx *ctx);

/* Last error message of the context (empty when none). */
const char *gdp_last_error(gdp_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
