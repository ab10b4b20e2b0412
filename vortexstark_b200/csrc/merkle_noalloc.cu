// Row-packed Merkle root that allocates no device memory.
//
// vs_merkle_root_rowpacked needs scratch for the intermediate subtree roots of
// trees above 1024 leaves and obtains it from the stream-ordered allocator. Some
// callers cannot allocate at that point: a serving process that reserved all of
// HBM up front for its admission budget, a host framework whose own caching
// allocator owns the device memory, or a latency-bound step that must not risk an
// allocation failure or the implicit synchronisation cudaMalloc may cause. For
// them, this variant keeps its scratch in a fixed array compiled into the
// library. The caller still provides the columns and the 8-word root.
#include <mutex>

#include "merkle.h"

namespace vs {

// Largest tree this entry point accepts, and the scratch that tree needs: one
// 8-word subtree root per 1024 leaves plus the next reduction level.
constexpr uint32_t NOALLOC_MAX_LOG_LEAVES = 26;
constexpr uint64_t NOALLOC_SCRATCH_WORDS = ((1ull << (NOALLOC_MAX_LOG_LEAVES - 10)) + 64) * 8;  // 2.1 MB

// Every GPU that loads the library holds this array until the process exits.
// All calls on a device share it and it keeps the last call's contents; calls
// whose work overlaps on the GPU would race on it.
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_SCRATCH_WORDS];

namespace {
std::mutex g_noalloc_mu;
uint32_t* g_noalloc_ptr[64] = {nullptr};

// Device address of the array on the current device. The symbol's name in host
// code is only a host-side handle, so the address is looked up once per device
// (with that device current) and cached.
int noalloc_scratch(uint32_t** out) {
  int dev = 0;
  VS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(VS_ERR_INVALID, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    VS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return VS_OK;
}
}  // namespace

}  // namespace vs

using namespace vs;

// Same result as vs_merkle_root_rowpacked. The first call on a device looks up
// the scratch array's address (cudaGetSymbolAddress); make that first call before
// any stream capture. Trees above 2^26 leaves are rejected.
extern "C" int vs_merkle_root_rowpacked_noalloc(const uint32_t* d_cols, uint64_t stride, uint32_t n_cols,
                                                uint32_t log_leaves, uint32_t* d_root, vs_stream_t st) {
  clear_error();
  if (!d_cols || !d_root) return set_error(VS_ERR_INVALID, "vs_merkle_root_rowpacked_noalloc: null pointer");
  if (log_leaves > NOALLOC_MAX_LOG_LEAVES)
    return set_error(VS_ERR_INVALID,
                     "vs_merkle_root_rowpacked_noalloc: 2^%u leaves exceeds the fixed scratch limit of 2^%u leaves",
                     log_leaves, NOALLOC_MAX_LOG_LEAVES);
  const uint64_t n = 1ull << log_leaves;
  uint32_t* scratch = nullptr;  // trees of at most 1024 leaves need no scratch
  if (merkle_scratch_words(n) > NOALLOC_SCRATCH_WORDS)
    return set_error(VS_ERR_INVALID, "vs_merkle_root_rowpacked_noalloc: scratch for 2^%u leaves exceeds the array",
                     log_leaves);
  if (merkle_scratch_words(n) > 0) VS_TRY(noalloc_scratch(&scratch));
  // With scratch supplied (or not needed) merkle_root performs no allocation.
  return merkle_root(LeafRowPacked{d_cols, stride, n_cols}, n, d_root, (cudaStream_t)st, scratch);
}
