/*
 * noalloc.cu -- the fill for callers that cannot allocate device memory.
 *
 * Some callers of this library cannot call cudaMalloc.  For example:
 *   - code that runs inside another framework's memory pool or a graph
 *     being built on a shared stream, where a device allocation would
 *     synchronise the device or break the caller's memory accounting;
 *   - plugins whose host process forbids allocation on the hot path;
 *   - callers that already own their input and output buffers.
 * gdp_fill16_noalloc serves them.  The caller passes its device inputs and
 * outputs.  The entry point allocates nothing and calls no allocating
 * routine.  It runs the 16-bit full-band fill (the Dynprog_simd_16
 * semantics of the batch API) with its working memory in one file-scope
 * device array, g_noalloc_scratch, of a fixed size:
 *
 *   GDP_NOALLOC_MAX_PAIRS pairs per call (65,536)
 *   glength <= GDP_NOALLOC_MAX_COLS - 1 (1,023)
 *   4,096 concurrent pair slots (32 blocks of 128 threads)
 *   = about 36 MB, held on every GPU that loads the library until the
 *     process exits.
 *
 * The substitution tables live in a second file-scope device array.
 *
 * The first call on a device does the set-up: it takes the device
 * addresses of both arrays with cudaGetSymbolAddress (a host-side symbol
 * name is not a device address), uploads the tables and waits for the
 * upload to land.  That first call should therefore come before any stream
 * capture.  Every call shares the same scratch array and leaves its
 * contents behind.  Calls that overlap on the GPU (on different streams, or
 * from different threads on one device) race on it, so a caller must order
 * its calls.
 *
 * The call leaves the calling thread's current device as it found it, and
 * checks its own launches by their return codes, so a CUDA error left
 * pending by the caller's earlier work neither fails this call nor is
 * cleared by it.
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>

#include "gdp_internal.h"
#include "fill_thread.cuh"

#define GDP_NOALLOC_MAX_PAIRS 65536
#define GDP_NOALLOC_MAX_COLS 1024
#define GDP_NOALLOC_BLOCKS 32
#define GDP_NOALLOC_THREADS 128
#define GDP_NOALLOC_SLOTS (GDP_NOALLOC_BLOCKS * GDP_NOALLOC_THREADS)
#define GDP_NOALLOC_MAX_DEVICES 64

/* byte layout of the scratch array */
#define NA_CARRY_BYTES ((size_t) GDP_NOALLOC_MAX_COLS * GDP_NOALLOC_SLOTS * sizeof(int2))
#define NA_META_OFF NA_CARRY_BYTES
#define NA_META_BYTES ((size_t) GDP_NOALLOC_MAX_PAIRS * sizeof(gdp_meta_t))
#define NA_LIST_OFF (NA_META_OFF + NA_META_BYTES)
#define NA_LIST_BYTES ((size_t) 2 * GDP_NOALLOC_MAX_PAIRS * sizeof(int32_t))
#define NA_COUNT_OFF (NA_LIST_OFF + NA_LIST_BYTES)
#define NA_COUNT_BYTES ((size_t) 256)
#define GDP_NOALLOC_SCRATCH_BYTES (NA_COUNT_OFF + NA_COUNT_BYTES)

static __device__ __align__(256) unsigned char g_noalloc_scratch[GDP_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) gdp_tables_t g_noalloc_tables;

/* Per device: the device addresses of the two arrays and the table mode. */
static std::mutex g_noalloc_mu;
static unsigned char *g_scratch_dev[GDP_NOALLOC_MAX_DEVICES];
static gdp_tables_t *g_tables_dev[GDP_NOALLOC_MAX_DEVICES];
static int g_tables_mode[GDP_NOALLOC_MAX_DEVICES];
static bool g_ready[GDP_NOALLOC_MAX_DEVICES];
static int g_packed_len[GDP_NOALLOC_MAX_DEVICES];
static int g_tab_mn[GDP_NOALLOC_MAX_DEVICES], g_tab_mx[GDP_NOALLOC_MAX_DEVICES];
static gdp_tables_t g_host_tables;   /* host staging for the one-time upload */

/*
 * Validates each pair, gives it a slice of the caller's direction buffer
 * (offset written to results[i].rec_offset), initialises its result and
 * meta, and puts it on the late- or early-tie list.  One block: pairs are
 * walked in chunks with a block-wide scan of their direction words.
 */
__global__ void __launch_bounds__(1024)
noalloc_prep_kernel (const gdp_pair_t *pairs, int64_t n, int64_t arena_bytes, int64_t cap, gdp_result_t *res,
                     gdp_meta_t *meta, int32_t *list_late, int32_t *list_early, int32_t *counts) {
  __shared__ int64_t s_words[1024];
  __shared__ int64_t s_base;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (int64_t start = 0; start < n; start += blockDim.x) {
    const int64_t i = start + threadIdx.x;
    int64_t words = 0;
    int st = GDP_OK;
    gdp_pair_t p;
    if (i < n) {
      p = pairs[i];
      /* the fill reads rsequence, gsequence and gsequence_alt from the
         caller's arena: each must lie inside it before any read */
      const bool in_arena = p.rseq >= 0 && p.rseq + p.rlength <= arena_bytes && p.gseq >= 0 &&
                            p.gseq + p.glength <= arena_bytes && p.gseq_alt >= 0 &&
                            p.gseq_alt + p.glength <= arena_bytes;
      if (p.variant != GDP_FULL || p.precision != 16 || p.mismatchtype < 0 || p.mismatchtype > 3 ||
          p.open < -127 || p.open > 0 || p.extend < -127 || p.extend > 0 ||
          (p.flags & ~(GDP_FLAG_JUMP_LATE | GDP_FLAG_REVP)) != 0 || p.genestrand < 0 || p.genestrand > 2 ||
          (p.xflags & ~GDP_XFLAG_SEGMENT) != 0) {
        /* no traceback, rerun, genome window or endpoint search here */
        st = GDP_ERR_PARAM;
      } else if (p.rlength <= 0 || p.glength <= 0 || p.glength >= GDP_NOALLOC_MAX_COLS ||
                 p.rlength > (1 << 20) || !in_arena) {
        st = GDP_ERR_LEN;
      } else if (p.lband < 0 || p.uband < 0) {
        st = GDP_ERR_BAND;
      } else {
        words = (gdp_pair_words(&p, 16) + 3) & ~(int64_t) 3;
      }
    }
    s_words[threadIdx.x] = words;
    __syncthreads();
    /* inclusive scan over the chunk (Hillis-Steele) */
    for (int off = 1; off < (int) blockDim.x; off <<= 1) {
      const int64_t v = (threadIdx.x >= (unsigned) off) ? s_words[threadIdx.x - off] : 0;
      __syncthreads();
      s_words[threadIdx.x] += v;
      __syncthreads();
    }
    const int64_t first = s_base + s_words[threadIdx.x] - words;
    if (i < n) {
      if (st == GDP_OK && first + words > cap) st = GDP_ERR_BUDGET;
      gdp_result_t r;
      r.status = st;
      r.score = 0;
      r.precision = 16;
      r.rerun = 0;
      r.tb_score = r.nmatches = r.nmismatches = r.nopens = r.nindels = 0;
      r.nrecs = 0;
      r.rec_offset = (st == GDP_OK) ? first : -1;
      res[i] = r;
      gdp_meta_t m;
      m.dir16 = first;
      m.dir8 = -1;
      m.maxh16 = -32768; m.status8 = 0; m.final8 = 0; m.final16 = 0;
      meta[i] = m;
      if (st == GDP_OK) {
        if (p.flags & GDP_FLAG_JUMP_LATE) list_late[atomicAdd(&counts[0], 1)] = (int32_t) i;
        else list_early[atomicAdd(&counts[1], 1)] = (int32_t) i;
      }
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_base += s_words[threadIdx.x];
    __syncthreads();
  }
}

/* Once per device, with that device current: device addresses of the
   file-scope arrays, and the tables for `mode`. */
static int
noalloc_setup (int device, int mode, unsigned char **scratch, gdp_tables_t **tables) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (device < 0 || device >= GDP_NOALLOC_MAX_DEVICES) return GDP_ERR_PARAM;
  if (!g_ready[device]) {
    void *ps = nullptr, *pt = nullptr;
    if (cudaGetSymbolAddress(&ps, g_noalloc_scratch) != cudaSuccess) return GDP_ERR_CUDA;
    if (cudaGetSymbolAddress(&pt, g_noalloc_tables) != cudaSuccess) return GDP_ERR_CUDA;
    gdp_build_tables(&g_host_tables, mode);
    if (cudaMemcpyToSymbol(g_noalloc_tables, &g_host_tables, sizeof(gdp_tables_t)) != cudaSuccess)
      return GDP_ERR_CUDA;
    /* from pageable memory the copy may return before the DMA lands; a
       caller's non-blocking stream would not wait for it */
    if (cudaDeviceSynchronize() != cudaSuccess) return GDP_ERR_CUDA;
    g_packed_len[device] = gdp_packed_len_of(&g_host_tables);
    g_tab_mn[device] = g_tab_mx[device] = 0;
    for (int mt = 0; mt < 4; mt++)
      for (int a = 0; a < 128; a++)
        for (int b = 0; b < 128; b++) {
          g_tab_mn[device] = std::min(g_tab_mn[device], (int) g_host_tables.pd[mt][a][b]);
          g_tab_mx[device] = std::max(g_tab_mx[device], (int) g_host_tables.pd[mt][a][b]);
        }
    g_scratch_dev[device] = (unsigned char *) ps;
    g_tables_dev[device] = (gdp_tables_t *) pt;
    g_tables_mode[device] = mode;
    g_ready[device] = true;
  } else if (g_tables_mode[device] != mode) {
    return GDP_ERR_PARAM;   /* the tables of a device are fixed by its first call */
  }
  *scratch = g_scratch_dev[device];
  *tables = g_tables_dev[device];
  return GDP_OK;
}

/* The launches of one call, on `device` (current). */
static int
noalloc_run (int device, int mode, const gdp_pair_t *d_pairs, int64_t npairs, const char *d_arena,
             int64_t arena_bytes, uint32_t *d_dirs, int64_t dir_words_cap, gdp_result_t *d_results,
             cudaStream_t s) {
  unsigned char *scratch = nullptr;
  gdp_tables_t *tables = nullptr;
  int rc = noalloc_setup(device, mode, &scratch, &tables);
  if (rc != GDP_OK) return rc;
  int2 *carry = (int2 *) scratch;
  gdp_meta_t *meta = (gdp_meta_t *) (scratch + NA_META_OFF);
  int32_t *list_late = (int32_t *) (scratch + NA_LIST_OFF);
  int32_t *list_early = list_late + GDP_NOALLOC_MAX_PAIRS;
  int32_t *counts = (int32_t *) (scratch + NA_COUNT_OFF);
  /* the list counts must start at zero on every call */
  if (cudaMemsetAsync(counts, 0, 2 * sizeof(int32_t), s) != cudaSuccess) return GDP_ERR_CUDA;
  {
    void *args[] = {(void *) &d_pairs, (void *) &npairs, (void *) &arena_bytes, (void *) &dir_words_cap,
                    (void *) &d_results, (void *) &meta, (void *) &list_late, (void *) &list_early,
                    (void *) &counts};
    if (cudaLaunchKernel((const void *) noalloc_prep_kernel, dim3(1), dim3(1024), args, 0, s) != cudaSuccess)
      return GDP_ERR_CUDA;
  }
  FillParams P;
  P.pairs = d_pairs;
  P.arena = d_arena;
  P.dirs = d_dirs;
  P.hdump = nullptr;
  P.meta = meta;
  P.res = d_results;
  P.scratch = carry;
  P.nslots = GDP_NOALLOC_SLOTS;
  P.scratch_rows = GDP_NOALLOC_MAX_COLS;
  P.tab = tables;
  P.reach_from4 = 0;
  P.lower_slack4 = 0;
  P.packed_len = g_packed_len[device];
  P.tab_mn = g_tab_mn[device];
  P.tab_mx = g_tab_mx[device];
  for (int late = 1; late >= 0; late--) {
    P.list = late ? list_late : list_early;
    P.count = counts + (late ? 0 : 1);
    void *args[] = {(void *) &P};
    /* the packed fill takes the pairs within its score range, the
       one-lane-per-register fill the others */
    const void *fns[2] = {late ? (const void *) fill_packed_kernel<true, 0> : (const void *) fill_packed_kernel<false, 0>,
                          late ? (const void *) fill_thread_kernel<16, GDP_FULL, true, 0>
                               : (const void *) fill_thread_kernel<16, GDP_FULL, false, 0>};
    for (int f = (P.packed_len >= 0) ? 0 : 1; f < 2; f++)
      if (cudaLaunchKernel(fns[f], dim3(GDP_NOALLOC_BLOCKS), dim3(GDP_NOALLOC_THREADS), args, 0, s) != cudaSuccess)
        return GDP_ERR_CUDA;
  }
  return GDP_OK;
}

extern "C" int
gdp_fill16_noalloc (int device, int mode, const gdp_pair_t *d_pairs, int64_t npairs, const char *d_arena,
                    int64_t arena_bytes, uint32_t *d_dirs, int64_t dir_words_cap, gdp_result_t *d_results,
                    void *stream) {
  if (npairs < 0 || npairs > GDP_NOALLOC_MAX_PAIRS) return GDP_ERR_LEN;
  if (mode < 0 || mode > 6 || arena_bytes < 0) return GDP_ERR_PARAM;
  if (npairs == 0) return GDP_OK;
  int caller_device = -1;
  if (cudaGetDevice(&caller_device) != cudaSuccess) return GDP_ERR_CUDA;
  if (device != caller_device && cudaSetDevice(device) != cudaSuccess) return GDP_ERR_CUDA;
  const int rc = noalloc_run(device, mode, d_pairs, npairs, d_arena, arena_bytes, d_dirs, dir_words_cap,
                             d_results, (cudaStream_t) stream);
  if (device != caller_device && cudaSetDevice(caller_device) != cudaSuccess) return GDP_ERR_CUDA;
  return rc;
}
