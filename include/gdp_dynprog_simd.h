/*
 * gdp_dynprog_simd.h -- the reference-signature entry points of libgdp.
 *
 * libgdp exports the twelve functions of GMAP's src/dynprog_simd.h with
 * the reference's exact names, argument lists and return conventions, so
 * that a GMAP build can drop src/dynprog_simd.c and link libgdp instead.
 * The fills run on the GPU (the same kernels as the batch ABI in gdp.h);
 * the tracebacks run on the GPU from the retained device fill and replay
 * their Pair records through the caller's own Pairpool_push /
 * Pairpool_push_gapholder.
 *
 * GMAP's own sources keep including src/dynprog_simd.h, whose declarations
 * these match (the build must not define DEBUG_SIMD or DEBUG_AVX2, which
 * add arguments).  This header serves other C/C++ callers and the library
 * itself.  It declares nothing when GMAP's src/dynprog.h has already been
 * included (its include guard DYNPROG_INCLUDED), so both can coexist in
 * one translation unit.
 *
 * Conventions kept from the reference:
 *   - A fill writes its matrix and direction planes into the Dynprog_T's
 *     aligned spaces, laid out as aligned_score*_alloc does
 *     (src/dynprog_simd.c:2158-2283): column c of the full and upper fills
 *     at space + c * rlength_ceil, lower fills transposed (row r at
 *     space + r * glength_ceil), with rlength_ceil = (rlength + W) / W * W
 *     and W = 32 (8-bit) or 16 (16-bit).  Every swept cell is written,
 *     directions as DIAG 0 / HORIZ -1 / VERT -2; the Fgap plane of the full
 *     fill is cleared first as aligned_directions*_calloc does.
 *   - rsequence / gsequence / gsequence_alt point at the first character,
 *     or at the last one when revp is true (the reference reads seq[1-r]).
 *   - A traceback adds to *traceback_score, *nmatches, *nmismatches,
 *     *nopens and *nindels and returns `pairs` with its records pushed in
 *     the reference's order.
 *
 * Additional rules of this implementation:
 *   - A traceback must receive the direction planes of the latest fill into
 *     the same Dynprog_T space on the same thread (which is how every GMAP
 *     caller uses them); the device keeps that fill until the space is
 *     filled again.  Planes that did not come from such a fill abort the
 *     process with a message, as do arguments the reference would overrun
 *     memory with (lengths above the Dynprog_T's maxima).
 *   - The tables are GMAP's pairdistance_array / consistent_array /
 *     nt_to_int_array when the process defines them (Dynprog_init was
 *     called before the first fill), else those of GDP_MODE (default 0,
 *     STANDARD).  The device is GDP_DEVICE (default 0).  Each calling
 *     thread gets its own CUDA stream and buffers.
 *   - Genome characters of short genome skips come from the caller's
 *     Genome_get_char (src/genome.c:11003), read for the positions the
 *     traceback can reach.
 */
#ifndef GDP_DYNPROG_SIMD_H
#define GDP_DYNPROG_SIMD_H

#ifndef DYNPROG_INCLUDED

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* bool of the reference (src/bool.h): one unsigned byte in C and C++ alike */
typedef unsigned char gdp_bool_t;

typedef char Score8_T;
typedef char Direction8_T;
typedef short Score16_T;
typedef short Direction16_T;
typedef int Mismatchtype_T;          /* HIGHQ 0, MEDQ 1, LOWQ 2, ENDQ 3 (src/dynprog.h:50) */
#ifdef LARGE_GENOMES
typedef uint64_t Univcoord_T;
#else
typedef uint32_t Univcoord_T;        /* src/univcoord.h:100 */
#endif

typedef struct gdp_List_s *List_T;           /* GMAP's List_T (src/list.h) */
typedef struct gdp_Pairpool_s *Pairpool_T;   /* GMAP's Pairpool_T (src/pairpool.h) */
typedef struct gdp_Genome_s *Genome_T;       /* GMAP's Genome_T (src/genome.h) */

/* The Dynprog_T of an SSE2/AVX2 build without DEBUG12 / DEBUG_SIMD /
   DEBUG_AVX2 (src/dynprog.h:175-230). */
struct gdp_Space_single {
  void **matrix_ptrs, *matrix_space;
  void **directions_ptrs_0, *directions_space_0;
  void **directions_ptrs_1, *directions_space_1;
  void **directions_ptrs_2, *directions_space_2;
};

struct gdp_Space_double {
  void **upper_matrix_ptrs, *upper_matrix_space;
  void **upper_directions_ptrs_0, *upper_directions_space_0;
  void **upper_directions_ptrs_1, *upper_directions_space_1;
  void **lower_matrix_ptrs, *lower_matrix_space;
  void **lower_directions_ptrs_0, *lower_directions_space_0;
  void **lower_directions_ptrs_1, *lower_directions_space_1;
};

struct gdp_Dynprog_s {
  int max_rlength;
  int max_glength;
  union {
    struct gdp_Space_single one;
    struct gdp_Space_double two;
  } aligned;
  int nspaces;
};
typedef struct gdp_Dynprog_s *Dynprog_T;

/* Fills: src/dynprog_simd.h:17-77 */
Score8_T **
Dynprog_simd_8 (Direction8_T ***directions_nogap, Direction8_T ***directions_Egap,
                Direction8_T ***directions_Fgap,
                Dynprog_T dynprog, char *rsequence, char *gsequence, char *gsequence_alt,
                int rlength, int glength, Mismatchtype_T mismatchtype, int open, int extend,
                int lband, int uband, gdp_bool_t jump_late_p, gdp_bool_t revp);

Score8_T **
Dynprog_simd_8_upper (Direction8_T ***directions_nogap, Direction8_T ***directions_Egap,
                      Dynprog_T dynprog, char *rsequence, char *gsequence, char *gsequence_alt,
                      int rlength, int glength, Mismatchtype_T mismatchtype, int open, int extend,
                      int uband, gdp_bool_t jump_late_p, gdp_bool_t revp);

Score8_T **
Dynprog_simd_8_lower (Direction8_T ***directions_nogap, Direction8_T ***directions_Egap,
                      Dynprog_T dynprog, char *rsequence, char *gsequence, char *gsequence_alt,
                      int rlength, int glength, Mismatchtype_T mismatchtype, int open, int extend,
                      int lband, gdp_bool_t jump_late_p, gdp_bool_t revp);

Score16_T **
Dynprog_simd_16 (Direction16_T ***directions_nogap, Direction16_T ***directions_Egap,
                 Direction16_T ***directions_Fgap,
                 Dynprog_T dynprog, char *rsequence, char *gsequence, char *gsequence_alt,
                 int rlength, int glength, Mismatchtype_T mismatchtype, int open, int extend,
                 int lband, int uband, gdp_bool_t jump_late_p, gdp_bool_t revp);

Score16_T **
Dynprog_simd_16_upper (Direction16_T ***directions_nogap, Direction16_T ***directions_Egap,
                       Dynprog_T dynprog, char *rsequence, char *gsequence, char *gsequence_alt,
                       int rlength, int glength, Mismatchtype_T mismatchtype, int open, int extend,
                       int uband, gdp_bool_t jump_late_p, gdp_bool_t revp);

Score16_T **
Dynprog_simd_16_lower (Direction16_T ***directions_nogap, Direction16_T ***directions_Egap,
                       Dynprog_T dynprog, char *rsequence, char *gsequence, char *gsequence_alt,
                       int rlength, int glength, Mismatchtype_T mismatchtype, int open, int extend,
                       int lband, gdp_bool_t jump_late_p, gdp_bool_t revp);

/* Tracebacks: src/dynprog_simd.h:79-126 */
List_T
Dynprog_traceback_8 (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens, int *nindels,
                     Direction8_T **directions_nogap, Direction8_T **directions_Egap, Direction8_T **directions_Fgap,
                     int r, int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                     int queryoffset, int genomeoffset, Genome_T genome, Genome_T genomealt,
                     Pairpool_T pairpool, gdp_bool_t revp,
                     Univcoord_T chroffset, Univcoord_T chrhigh, gdp_bool_t watsonp, int genestrand,
                     int dynprogindex);

List_T
Dynprog_traceback_8_upper (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens, int *nindels,
                           Direction8_T **directions_nogap, Direction8_T **directions_Egap,
                           int r, int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                           int queryoffset, int genomeoffset, Genome_T genome, Genome_T genomealt,
                           Pairpool_T pairpool, gdp_bool_t revp,
                           Univcoord_T chroffset, Univcoord_T chrhigh, gdp_bool_t watsonp, int genestrand,
                           int dynprogindex);

List_T
Dynprog_traceback_8_lower (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens, int *nindels,
                           Direction8_T **directions_nogap, Direction8_T **directions_Egap,
                           int r, int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                           int queryoffset, int genomeoffset,
                           Pairpool_T pairpool, int genestrand, gdp_bool_t revp, int dynprogindex);

List_T
Dynprog_traceback_16 (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens, int *nindels,
                      Direction16_T **directions_nogap, Direction16_T **directions_Egap, Direction16_T **directions_Fgap,
                      int r, int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                      int queryoffset, int genomeoffset, Genome_T genome, Genome_T genomealt,
                      Pairpool_T pairpool, gdp_bool_t revp,
                      Univcoord_T chroffset, Univcoord_T chrhigh, gdp_bool_t watsonp, int genestrand,
                      int dynprogindex);

List_T
Dynprog_traceback_16_upper (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens, int *nindels,
                            Direction16_T **directions_nogap, Direction16_T **directions_Egap,
                            int r, int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                            int queryoffset, int genomeoffset, Genome_T genome, Genome_T genomealt,
                            Pairpool_T pairpool, gdp_bool_t revp,
                            Univcoord_T chroffset, Univcoord_T chrhigh, gdp_bool_t watsonp, int genestrand,
                            int dynprogindex);

List_T
Dynprog_traceback_16_lower (List_T pairs, int *traceback_score, int *nmatches, int *nmismatches, int *nopens, int *nindels,
                            Direction16_T **directions_nogap, Direction16_T **directions_Egap,
                            int r, int c, char *rsequence, char *rsequenceuc, char *gsequence, char *gsequence_alt,
                            int queryoffset, int genomeoffset,
                            Pairpool_T pairpool, int genestrand, gdp_bool_t revp, int dynprogindex);

/* Frees the calling thread's device fills, buffers and stream (they are
   also freed when the thread exits).  Not part of the reference. */
void gdp_dropin_release_thread (void);

#ifdef __cplusplus
}
#endif

#endif /* DYNPROG_INCLUDED */
#endif /* GDP_DYNPROG_SIMD_H */
