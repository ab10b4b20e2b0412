// Error capture, device queries, cache release and the commitment-layer step.
#include <atomic>
#include <cstdarg>
#include <mutex>

#include "merkle.h"
#include "ntt.h"
#include "twiddles.h"
#include "vs_common.cuh"

namespace vs {

static thread_local char g_err[512] = "";
static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return status;
}
void clear_error() { g_err[0] = 0; }

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

}  // namespace vs

using namespace vs;

extern "C" {

const char* vs_last_error(void) { return g_err; }
const char* vs_version(void) { return "vstark-b200 0.1 (sm_100a)"; }
uint64_t vs_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int vs_release_caches(void) {
  clear_error();
  release_zh_tables();
  return release_twiddles();
}

// src/cuda/ffi.rs:165-207 (init_memory_pool / init_memory_pool_greedy): the
// reference keeps 2 GiB (or everything, greedy) cached in the current device's
// default stream-ordered pool so per-proof cudaMallocAsync calls reuse memory.
int vs_init_memory_pool(uint64_t release_threshold_bytes) {
  clear_error();
  int dev = 0;
  VS_CUDA(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  VS_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  VS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &release_threshold_bytes));
  return VS_OK;
}

int vs_commit_columns(const uint32_t* d_cols, uint32_t n_cols, uint32_t log_n, uint32_t blowup, uint32_t* d_lde,
                      uint32_t* d_root, vs_stream_t stream) {
  clear_error();
  cudaStream_t st = (cudaStream_t)stream;
  if (!d_cols || !d_lde || !d_root || !n_cols) return set_error(VS_ERR_INVALID, "vs_commit_columns: bad args");
  const uint64_t n = 1ull << log_n, N = n << blowup;
  VS_TRY(lde_cached(TW_STWO, d_cols, n, d_lde, N, n_cols, log_n, blowup, st));
  return merkle_root(LeafRowPacked{d_lde, N, n_cols}, N, d_root, st, nullptr, merkle_split());
}

}  // extern "C"
