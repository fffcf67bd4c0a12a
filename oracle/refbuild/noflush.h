/* Force-included (gcc -include) into the reference sources for the
   secondary "no clflush" CPU baseline: the per-column _mm_clflush of the
   fills (e.g. src/dynprog_simd.c:6901) becomes a no-op.  Outputs are
   unchanged; only the timing differs.  Test infrastructure only. */
#include <immintrin.h>
#define _mm_clflush(p) ((void) 0)
