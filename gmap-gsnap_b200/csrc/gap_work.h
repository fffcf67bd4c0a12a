/* gap_work.h -- working memory and host threads of the gap solvers
   (single_gap.cu, end_gap.cu): a context's grow-only device and pinned host
   slots, and a parallel loop over host threads.  Internal. */
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <thread>
#include <vector>
#include "gdp_dropin_internal.h"

namespace {

/* device slot k of the context's gap working memory, at least count T */
template <class T> cudaError_t
dev_slot (gdpi_single_cfg *c, int k, T **p, int64_t count) {
  const size_t need = (size_t) std::max<int64_t>(count, 1) * sizeof(T);
  if (c->dcap[k] < need) {
    if (c->dbuf[k]) cudaFree(c->dbuf[k]);
    c->dbuf[k] = nullptr;
    c->dcap[k] = 0;
    const size_t cap = need + need / 4;
    cudaError_t e = cudaMalloc(&c->dbuf[k], cap);
    if (e != cudaSuccess) return e;
    c->dcap[k] = cap;
  }
  *p = (T *) c->dbuf[k];
  return cudaSuccess;
}

/* pinned host slot k, at least count T */
template <class T> cudaError_t
host_slot (gdpi_single_cfg *c, int k, T **p, int64_t count) {
  const size_t need = (size_t) std::max<int64_t>(count, 1) * sizeof(T);
  if (c->hcap[k] < need) {
    if (c->hbuf[k]) cudaFreeHost(c->hbuf[k]);
    c->hbuf[k] = nullptr;
    c->hcap[k] = 0;
    const size_t cap = need + need / 4;
    cudaError_t e = cudaMallocHost(&c->hbuf[k], cap);
    if (e != cudaSuccess) return e;
    c->hcap[k] = cap;
  }
  *p = (T *) c->hbuf[k];
  return cudaSuccess;
}

/* f(lo, hi) over [0, n) on up to 16 host threads (one below 8,192 items). */
template <class F> void
par_for (int64_t n, F f) {
  const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = (int) std::min<int64_t>(std::min<int64_t>(hw, 16), std::max<int64_t>(1, n / 8192));
  if (nt <= 1) { f((int64_t) 0, n); return; }
  std::vector<std::thread> th;
  const int64_t chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; t++) {
    const int64_t lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo < hi) th.emplace_back([=, &f] { f(lo, hi); });
  }
  for (auto &x : th) x.join();
}

}  // namespace
