// Host-side Merkle helpers over the generic subtree kernel (merkle_impl.cuh).
// Templates live here so other translation units can commit with fused leaf
// functors (FRI folds, constraint quotients).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>

#include "merkle_impl.cuh"
#include "vs_common.cuh"

namespace vs {

// One level of parents: parents[i] = Blake2s(children[2i] || children[2i+1]).
int launch_hash_nodes(const uint32_t* children, uint32_t* parents, uint64_t n_parents, cudaStream_t st);

// stop_log (<= TL): 2^stop_log roots per tile instead of one (merkle_subtree_kernel).
template <class Leaf>
int merkle_tile_roots(const Leaf& leaf, uint64_t n_leaves, uint32_t TL, uint32_t* roots, cudaStream_t st,
                      uint32_t stop_log = 0) {
  const unsigned smem = merkle_smem_bytes(TL);  // at most 48 KiB (TL <= 10): no opt-in needed
  const uint64_t tiles = (n_leaves + (1ull << TL) - 1) >> TL;
  if (stop_log > TL) stop_log = TL;
  merkle_subtree_kernel<Leaf><<<(unsigned)tiles, MK_THREADS, smem, st>>>(leaf, TL, n_leaves, roots, stop_log);
  VS_LAUNCHED("merkle_subtree_kernel");
  return VS_OK;
}

// Largest split merkle_root accepts: the first level may stop at 2^8 roots per
// 1024-leaf tile (the level where all 256 threads of a CTA still have a node).
constexpr uint32_t MK_MAX_SPLIT = 8;
// Process-wide split of the root-only trees (vs_merkle_split_set).
uint32_t merkle_split();

// Split of a reduction level over `cur` hashes: the leaf level takes the split
// as given; hash levels of at least 2^20 hashes (1024+ CTAs) take at most 5 (each
// step then reduces 32-fold, so the chain stays short), smaller ones reduce each
// tile to one root.
inline uint32_t merkle_level_split(uint64_t cur, uint32_t split) {
  return cur >= (1ull << 20) ? std::min<uint32_t>(split, 5) : 0u;
}

// Words of scratch merkle_root needs for n_leaves leaves with split `split` (0 when
// n_leaves <= 1024): the sum of the hash levels it writes, in the order it writes
// them (merkle_root follows the same sequence).
inline uint64_t merkle_scratch_words(uint64_t n_leaves, uint32_t split = 0) {
  if (n_leaves <= (1ull << MK_MAX_TL)) return 0;
  uint64_t cur = n_leaves >> (MK_MAX_TL - split);
  uint64_t words = cur * 8;
  while (cur > (1ull << MK_MAX_TL)) {
    cur >>= MK_MAX_TL - merkle_level_split(cur, split);
    words += cur * 8;
  }
  return words;
}
// Split used for trees that keep their 1024-leaf tile roots (prover trees of
// 2^20+ leaves): tiles stop at 2^split subtree roots and `split` node launches
// bring them up to the tile roots. Capped at 5, which bounds the extra scratch
// at 2^5 + 2^4 hashes per tile (48 hashes per 1024 leaves).
constexpr uint32_t MK_TILE_SPLIT_MAX = 5;
inline uint32_t merkle_tile_split(uint64_t n_leaves) {
  return n_leaves >= (1ull << 20) ? std::min<uint32_t>(merkle_split(), MK_TILE_SPLIT_MAX) : 0u;
}
// Subroot scratch of a tile-root tree of n_leaves leaves at split sp (0: none).
inline uint64_t merkle_tile_scratch_bytes(uint64_t n_leaves, uint32_t sp) {
  return sp ? ((n_leaves >> MK_MAX_TL) << sp) * 32 + ((n_leaves >> MK_MAX_TL) << (sp - 1)) * 32 : 0;
}
// Tile roots of a 2^TL-leaf tiling through 2^sp subtree roots per tile: the
// subtree kernel writes the subroots to sub_a, then sp node levels ping-pong
// between sub_a (2^sp hashes per tile) and sub_b (2^(sp-1)) and end in `roots`.
// Same tile roots as merkle_tile_roots(leaf, n, TL, roots).
template <class Leaf>
int merkle_tile_roots_split(const Leaf& leaf, uint64_t n_leaves, uint32_t TL, uint32_t sp, uint32_t* roots,
                            uint32_t* sub_a, uint32_t* sub_b, cudaStream_t st);

// Scratch that serves merkle_root at every split 0..MK_MAX_SPLIT.
inline uint64_t merkle_scratch_words_any(uint64_t n_leaves) {
  uint64_t w = 0;
  for (uint32_t sp = 0; sp <= MK_MAX_SPLIT; sp++) w = std::max(w, merkle_scratch_words(n_leaves, sp));
  return w;
}

// Root of a power-of-two tree whose leaves come from `leaf`. Intermediate tile
// roots go to `scratch` (merkle_scratch_words(n_leaves, split) words; when null it
// is allocated stream-ordered for the call). Each reduction level is written after
// the previous one, never in place. The first level stops at 2^split roots per
// 1024-leaf tile (split <= MK_MAX_SPLIT); the root is the same for every split.
template <class Leaf>
int merkle_root(const Leaf& leaf, uint64_t n_leaves, uint32_t* d_root, cudaStream_t st, uint32_t* scratch = nullptr,
                uint32_t split = 0) {
  if (!is_pow2(n_leaves)) return set_error(VS_ERR_INVALID, "merkle: leaf count %llu is not a power of two",
                                           (unsigned long long)n_leaves);
  if (split > MK_MAX_SPLIT) return set_error(VS_ERR_INVALID, "merkle: split %u above %u", split, MK_MAX_SPLIT);
  const uint32_t L = ilog2(n_leaves);
  if (L <= MK_MAX_TL) return merkle_tile_roots(leaf, n_leaves, L, d_root, st);
  uint32_t* buf = scratch;
  if (!buf) VS_CUDA(cudaMallocAsync((void**)&buf, merkle_scratch_words(n_leaves, split) * 4, st));
  uint64_t cur = n_leaves >> (MK_MAX_TL - split);
  int rc = merkle_tile_roots(leaf, n_leaves, MK_MAX_TL, buf, st, split);
  uint32_t* level = buf;
  while (rc == VS_OK) {
    const uint32_t Lc = ilog2(cur);
    if (Lc <= MK_MAX_TL) { rc = merkle_tile_roots(LeafHashes{level}, cur, Lc, d_root, st); break; }
    uint32_t* next = level + cur * 8;
    const uint32_t sp = merkle_level_split(cur, split);
    rc = merkle_tile_roots(LeafHashes{level}, cur, MK_MAX_TL, next, st, sp);
    level = next;
    cur >>= MK_MAX_TL - sp;
  }
  if (!scratch) {
    cudaError_t e = cudaFreeAsync(buf, st);
    if (rc == VS_OK) rc = check_cuda(e, "merkle scratch free");
  }
  return rc;
}

template <class Leaf>
int merkle_tile_roots_split(const Leaf& leaf, uint64_t n_leaves, uint32_t TL, uint32_t sp, uint32_t* roots,
                            uint32_t* sub_a, uint32_t* sub_b, cudaStream_t st) {
  if (!sp) return merkle_tile_roots(leaf, n_leaves, TL, roots, st);
  const uint64_t tiles = n_leaves >> TL;
  VS_TRY(merkle_tile_roots(leaf, n_leaves, TL, sub_a, st, sp));
  uint32_t* src = sub_a;
  uint64_t c = tiles << sp;
  for (uint32_t k = sp; k > 1; k--) {
    uint32_t* dst = src == sub_a ? sub_b : sub_a;
    VS_TRY(launch_hash_nodes(src, dst, c / 2, st));
    src = dst;
    c /= 2;
  }
  return launch_hash_nodes(src, roots, tiles, st);
}

}  // namespace vs
