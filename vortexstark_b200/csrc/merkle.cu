// Blake2s Merkle commitment: drop-in entry points for cuda/blake2s.cu and
// cuda/merkle_leaves_lifted.cu, and vs_merkle_root_* (root-only commitments).
#include <atomic>
#include <cstring>

#include "merkle.h"
#include "vs_field.cuh"
#include "vs_mem.cuh"

namespace vs {

// Split of the root-only trees: the first reduction level stops at 2^split roots
// per 1024-leaf tile (merkle_root). Set by vs_merkle_split_set / vs_autotune_merkle.
static std::atomic<uint32_t> g_merkle_split{0};
uint32_t merkle_split() { return g_merkle_split.load(std::memory_order_relaxed); }

template <class Leaf>
__global__ void leaf_hash_kernel(Leaf leaf, uint64_t n, uint32_t* __restrict__ out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t h[8];
  leaf(i, h);
  st4(out + 8 * i, make_uint4(h[0], h[1], h[2], h[3]));
  st4(out + 8 * i + 4, make_uint4(h[4], h[5], h[6], h[7]));
}

__global__ void hash_nodes_kernel(const uint32_t* __restrict__ children, uint32_t* __restrict__ parents, uint64_t n) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* c = children + 16 * i;
  const uint4 a = ld4_ro(c), b = ld4_ro(c + 4), d = ld4_ro(c + 8), e = ld4_ro(c + 12);
  uint32_t m[16] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, d.x, d.y, d.z, d.w, e.x, e.y, e.z, e.w};
  uint32_t h[8];
  b2s_init(h);
  b2s_compress(h, m, 64u, true);
  st4(parents + 8 * i, make_uint4(h[0], h[1], h[2], h[3]));
  st4(parents + 8 * i + 4, make_uint4(h[4], h[5], h[6], h[7]));
}

// Parent of each SoA4 leaf pair (blake2s.cu:190-231 semantics).
__global__ void leaves_merge_soa4_kernel(LeafSoa4 leaf, uint64_t n_pairs, uint32_t* __restrict__ parents) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n_pairs) return;
  uint32_t l[8], r[8], h[8];
  leaf(2 * i, l);
  leaf(2 * i + 1, r);
  b2s_node(h, l, r);
  for (int w = 0; w < 8; w++) parents[8 * i + w] = h[w];
}

int launch_hash_nodes(const uint32_t* children, uint32_t* parents, uint64_t n, cudaStream_t st) {
  if (!n) return VS_OK;
  hash_nodes_kernel<<<blocks_for(n, 256), 256, 0, st>>>(children, parents, n);
  VS_LAUNCHED("hash_nodes_kernel");
  return VS_OK;
}

// Lifted leaves (merkle_leaves_lifted.cu:18-98): chunks of up to 16 columns of
// one log size; row index lifted to the tree size; standard multi-block Blake2s
// of all the row's words in chunk order.
struct LeafHashChunk {
  uint32_t col_indices[16];
  uint32_t n_cols;
  uint32_t log_size;
};
__global__ void leaves_lifted_kernel(const uint32_t* const* __restrict__ cols, const LeafHashChunk* __restrict__ sched,
                                     uint32_t n_chunks, uint32_t S, uint32_t* __restrict__ out, uint32_t n_leaves) {
  uint32_t leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n_leaves) return;
  uint32_t total = 0;
  for (uint32_t c = 0; c < n_chunks; c++) total += min(sched[c].n_cols, 16u);
  uint32_t h[8], m[16];
  b2s_init(h);
  uint32_t pos = 0, seen = 0;
  for (uint32_t c = 0; c < n_chunks; c++) {
    const uint32_t L = sched[c].log_size, nc = min(sched[c].n_cols, 16u);
    const uint32_t row = (L == S) ? leaf : (((leaf >> (S - L + 1)) << 1) | (leaf & 1));
    for (uint32_t k = 0; k < nc; k++) {
      m[pos++] = cols[sched[c].col_indices[k]][row];
      seen++;
      if (pos == 16 && seen < total) {
        b2s_compress(h, m, seen * 4u, false);
        pos = 0;
      }
    }
  }
  for (uint32_t w = pos; w < 16; w++) m[w] = 0;
  b2s_compress(h, m, total * 4u, true);
  for (int w = 0; w < 8; w++) out[8 * (uint64_t)leaf + w] = h[w];
}

}  // namespace vs

using namespace vs;

extern "C" {

void cuda_merkle_hash_leaves(const uint32_t* const* columns, uint32_t* hashes, uint32_t n_cols, uint32_t n_leaves) {
  if (!n_leaves) return;
  LeafCapped leaf{columns, nullptr, 0, n_cols};
  leaf_hash_kernel<<<blocks_for(n_leaves, 256), 256>>>(leaf, n_leaves, hashes);
  check_cuda(cudaGetLastError(), "cuda_merkle_hash_leaves");
}
void cuda_merkle_hash_nodes(const uint32_t* children, uint32_t* parents, uint32_t n_parents) {
  launch_hash_nodes(children, parents, n_parents, 0);
}
// n_nodes must be a power of two (<= 1024 in the reference).
void cuda_merkle_reduce_to_root(const uint32_t* nodes, uint32_t* root_out, uint32_t n_nodes) {
  merkle_root(LeafHashes{nodes}, n_nodes, root_out, 0);
}
void cuda_merkle_commit_small_soa4(const uint32_t* c0, const uint32_t* c1, const uint32_t* c2, const uint32_t* c3,
                                   uint32_t* root_out, uint32_t n_leaves) {
  merkle_root(LeafSoa4{c0, c1, c2, c3}, n_leaves, root_out, 0);
}
void cuda_merkle_hash_leaves_merge_soa4(const uint32_t* c0, const uint32_t* c1, const uint32_t* c2,
                                        const uint32_t* c3, uint32_t* parents, uint32_t n_leaves) {
  uint64_t pairs = n_leaves / 2;
  if (!pairs) return;
  leaves_merge_soa4_kernel<<<blocks_for(pairs, 256), 256>>>(LeafSoa4{c0, c1, c2, c3}, pairs, parents);
  check_cuda(cudaGetLastError(), "cuda_merkle_hash_leaves_merge_soa4");
}
void cuda_merkle_tiled_soa4_stream(const uint32_t* c0, const uint32_t* c1, const uint32_t* c2, const uint32_t* c3,
                                   uint32_t* subtree_roots, uint32_t n_leaves, vs_stream_t stream) {
  if (n_leaves < 1024) return;  // the reference launches n_leaves / 1024 tiles
  merkle_tile_roots(LeafSoa4{c0, c1, c2, c3}, (uint64_t)(n_leaves / 1024) * 1024, 10, subtree_roots,
                    (cudaStream_t)stream);
}
void cuda_merkle_tiled_soa4(const uint32_t* c0, const uint32_t* c1, const uint32_t* c2, const uint32_t* c3,
                            uint32_t* subtree_roots, uint32_t n_leaves) {
  cuda_merkle_tiled_soa4_stream(c0, c1, c2, c3, subtree_roots, n_leaves, 0);
}
void cuda_merkle_tiled_generic(const uint32_t* const* columns, uint32_t* subtree_roots, uint32_t n_cols,
                               uint32_t n_leaves) {
  if (n_leaves < 1024) return;
  merkle_tile_roots(LeafCapped{columns, nullptr, 0, n_cols}, (uint64_t)(n_leaves / 1024) * 1024, 10, subtree_roots, 0);
}
void cuda_build_leaves_lifted(const uint32_t* const* col_ptrs, const void* schedule, uint32_t n_chunks,
                              uint32_t lifting_log_size, uint32_t* output_hashes, uint32_t n_leaves) {
  if (!n_leaves) return;
  leaves_lifted_kernel<<<blocks_for(n_leaves, 256), 256>>>(col_ptrs, (const LeafHashChunk*)schedule, n_chunks,
                                                           lifting_log_size, output_hashes, n_leaves);
  check_cuda(cudaGetLastError(), "cuda_build_leaves_lifted");
}

int vs_merkle_root_rowpacked(const uint32_t* d_cols, uint64_t stride, uint32_t n_cols, uint32_t log_leaves,
                             uint32_t* d_root, vs_stream_t st) {
  clear_error();
  if (!d_cols || !d_root || log_leaves > 31) return set_error(VS_ERR_INVALID, "vs_merkle_root_rowpacked: bad args");
  return merkle_root(LeafRowPacked{d_cols, stride, n_cols}, 1ull << log_leaves, d_root, (cudaStream_t)st, nullptr,
                     merkle_split());
}
int vs_merkle_root_capped(const uint32_t* d_cols, uint64_t stride, uint32_t n_cols, uint32_t log_leaves,
                          uint32_t* d_root, vs_stream_t st) {
  clear_error();
  if (!d_cols || !d_root || log_leaves > 31) return set_error(VS_ERR_INVALID, "vs_merkle_root_capped: bad args");
  return merkle_root(LeafCapped{nullptr, d_cols, stride, n_cols}, 1ull << log_leaves, d_root, (cudaStream_t)st, nullptr,
                     merkle_split());
}
int vs_merkle_root_soa4(const uint32_t* c0, const uint32_t* c1, const uint32_t* c2, const uint32_t* c3,
                        uint32_t log_leaves, uint32_t* d_root, vs_stream_t st) {
  clear_error();
  if (!c0 || !c1 || !c2 || !c3 || !d_root || log_leaves > 31) return set_error(VS_ERR_INVALID, "vs_merkle_root_soa4: bad args");
  return merkle_root(LeafSoa4{c0, c1, c2, c3}, 1ull << log_leaves, d_root, (cudaStream_t)st, nullptr, merkle_split());
}

int vs_merkle_split_set(uint32_t split) {
  clear_error();
  if (split > MK_MAX_SPLIT) return set_error(VS_ERR_INVALID, "vs_merkle_split_set: split %u above %u", split, MK_MAX_SPLIT);
  g_merkle_split.store(split);
  return VS_OK;
}
uint32_t vs_merkle_split_get(void) { return merkle_split(); }

// Times the row-packed root of n_cols seeded columns of 2^log_leaves rows at every
// split (one warm-up and `reps` timed runs each, CUDA events on the stream), checks
// that every split gives the same root, and keeps the fastest split.
int vs_autotune_merkle(uint32_t log_leaves, uint32_t n_cols, uint32_t reps, uint32_t* best, float* ms_out, uint32_t cap,
                       vs_stream_t stream) {
  clear_error();
  cudaStream_t st = (cudaStream_t)stream;
  if (log_leaves < 11 || log_leaves > 28 || !n_cols || !best)
    return set_error(VS_ERR_INVALID, "vs_autotune_merkle: bad size (log %u, cols %u)", log_leaves, n_cols);
  if (!reps) reps = 3;
  const uint64_t n = 1ull << log_leaves;
  uint32_t *cols = nullptr, *scratch = nullptr, *roots = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = check_cuda(cudaMallocAsync((void**)&cols, n * n_cols * 4, st), "vs_autotune_merkle alloc");
  if (rc == VS_OK)
    rc = check_cuda(cudaMallocAsync((void**)&scratch, merkle_scratch_words_any(n) * 4, st), "vs_autotune_merkle alloc");
  if (rc == VS_OK) rc = check_cuda(cudaMallocAsync((void**)&roots, 8 * (MK_MAX_SPLIT + 1) * 4, st), "vs_autotune_merkle alloc");
  if (rc == VS_OK) rc = vs_fill_uniform_m31(cols, n * n_cols, 0x56530008ull, 0, stream);
  if (rc == VS_OK) rc = check_cuda(cudaEventCreate(&e0), "vs_autotune_merkle event");
  if (rc == VS_OK) rc = check_cuda(cudaEventCreate(&e1), "vs_autotune_merkle event");
  uint32_t best_split = merkle_split();
  float best_ms = 0.f;
  for (uint32_t sp = 0; sp <= MK_MAX_SPLIT && rc == VS_OK; sp++) {
    const LeafRowPacked leaf{cols, n, n_cols};
    rc = merkle_root(leaf, n, roots + 8 * sp, st, scratch, sp);
    if (rc == VS_OK) rc = check_cuda(cudaEventRecord(e0, st), "vs_autotune_merkle event");
    for (uint32_t k = 0; k < reps && rc == VS_OK; k++) rc = merkle_root(leaf, n, roots + 8 * sp, st, scratch, sp);
    if (rc == VS_OK) rc = check_cuda(cudaEventRecord(e1, st), "vs_autotune_merkle event");
    if (rc == VS_OK) rc = check_cuda(cudaEventSynchronize(e1), "vs_autotune_merkle sync");
    float ms = 0.f;
    if (rc == VS_OK) rc = check_cuda(cudaEventElapsedTime(&ms, e0, e1), "vs_autotune_merkle time");
    ms /= (float)reps;
    if (ms_out && sp < cap) ms_out[sp] = ms;
    if (rc == VS_OK && (sp == 0 || ms < best_ms)) {
      best_ms = ms;
      best_split = sp;
    }
  }
  uint32_t h[8 * (MK_MAX_SPLIT + 1)];
  if (rc == VS_OK) rc = check_cuda(cudaMemcpyAsync(h, roots, sizeof(h), cudaMemcpyDeviceToHost, st), "vs_autotune_merkle copy");
  if (rc == VS_OK) rc = check_cuda(cudaStreamSynchronize(st), "vs_autotune_merkle sync");
  for (uint32_t sp = 1; sp <= MK_MAX_SPLIT && rc == VS_OK; sp++)
    if (memcmp(h, h + 8 * sp, 32) != 0) rc = set_error(VS_ERR_CUDA, "vs_autotune_merkle: split %u gave another root", sp);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (cols) cudaFreeAsync(cols, st);
  if (scratch) cudaFreeAsync(scratch, st);
  if (roots) cudaFreeAsync(roots, st);
  if (rc != VS_OK) return rc;
  g_merkle_split.store(best_split);
  *best = best_split;
  return check_cuda(cudaStreamSynchronize(st), "vs_autotune_merkle");
}

}  // extern "C"
