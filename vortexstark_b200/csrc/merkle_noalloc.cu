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
#include <cuda.h>

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
struct NoallocAddr {
  unsigned long long ctx_id = 0;  // context the address belongs to (0: none yet)
  uint32_t* ptr = nullptr;
};
NoallocAddr g_noalloc_addr[64];

// Unique id of the calling thread's current CUDA context (never reused within the
// process, unlike a context handle), through the driver entry points the runtime
// exposes, so the library needs no link against the driver library.
int current_context_id(unsigned long long* id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  static cudaError_t looked_up = cudaSuccess;
  std::call_once(once, [] {
    looked_up = cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, nullptr);
    if (looked_up == cudaSuccess)
      looked_up = cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, nullptr);
  });
  VS_CUDA(looked_up);
  if (!get_current || !get_id) return set_error(VS_ERR_CUDA, "driver context queries unavailable");
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return set_error(VS_ERR_CUDA, "no current CUDA context");
  if (get_id(ctx, id) != CUDA_SUCCESS) return set_error(VS_ERR_CUDA, "cuCtxGetId failed");
  return VS_OK;
}

// Device address of the array in the current device's context. The symbol's name
// in host code is only a host-side handle, so the address is looked up with the
// device current (cudaGetSymbolAddress) and cached per device together with the
// id of the context it was found in. If that context is destroyed and recreated
// (cudaDeviceReset), the library's module is loaded again and the array may move:
// the id changes and the address is looked up again.
int noalloc_scratch(uint32_t** out) {
  int dev = 0;
  VS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(VS_ERR_INVALID, "device ordinal %d out of range", dev);
  unsigned long long ctx = 0;
  if (current_context_id(&ctx) != VS_OK) {  // no context current on this thread yet
    VS_CUDA(cudaSetDevice(dev));             // makes the device's primary context current
    VS_TRY(current_context_id(&ctx));
    clear_error();
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoallocAddr& a = g_noalloc_addr[dev];
  if (!a.ptr || a.ctx_id != ctx) {
    void* p = nullptr;
    VS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    a.ptr = static_cast<uint32_t*>(p);
    a.ctx_id = ctx;
  }
  *out = a.ptr;
  return VS_OK;
}
}  // namespace

}  // namespace vs

using namespace vs;

// Same result as vs_merkle_root_rowpacked. The first call on a device (and the
// first after its context was recreated) looks up the scratch array's address
// (cudaGetSymbolAddress); make that first call before any stream capture. Trees
// above 2^26 leaves are rejected.
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
