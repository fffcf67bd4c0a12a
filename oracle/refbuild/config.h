/* Minimal configuration header for compiling the reference's dynamic
 * programming sources (src/dynprog_simd.c, src/dynprog.c, src/pairpool.c,
 * src/mem.c, src/list.c, src/except.c) as the test oracle.  It states the
 * same feature set that the reference's configure script detects on an
 * x86-64 host with AVX2 (src/Makefile.am:305, gmap_avx2_CFLAGS), so the
 * compiled functions are the reference's AVX2 code path.  Test
 * infrastructure only: nothing in the product links it. */
#ifndef GDP_REF_CONFIG_H
#define GDP_REF_CONFIG_H

#define USE_INTEL_INTRINSICS 1
#define HAVE_ALLOCA 1
#define HAVE_ALLOCA_H 1
#define HAVE_INLINE 1
#define HAVE_INTTYPES_H 1
#define HAVE_STDINT_H 1
#define HAVE_STDLIB_H 1
#define HAVE_STRING_H 1
#define HAVE_STRINGS_H 1
#define HAVE_UNISTD_H 1
#define HAVE_SYS_TYPES_H 1
#define HAVE_SYS_STAT_H 1
#define HAVE_MEMCPY 1
#define HAVE_MEMSET 1
#define HAVE_MEMMOVE 1
#define HAVE_BUILTIN_CLZ 1
#define HAVE_BUILTIN_CTZ 1
#define HAVE_BUILTIN_POPCOUNT 1
#define HAVE_PTHREAD 1
#define STDC_HEADERS 1
#define PACKAGE "gmap"
#define VERSION "2026-02-05"

/* SIMD level of the gmap.avx2 build */
#define HAVE_SSE2 1
#define HAVE_SSSE3 1
#define HAVE_SSE4_1 1
#define HAVE_SSE4_2 1
#define HAVE_AVX2 1

#endif
