// Generic Blake2s Merkle subtree kernel.
//
// A CTA owns a tile of 2^TL consecutive leaves (TL <= 10). Its 256 threads hash
// the tile's leaves with a leaf functor (coalesced: thread t takes leaves t,
// t+256, ...), then reduce the tile level by level in shared memory to one
// subtree root. Hashes are stored transposed (word w of hash i at w*2^TL + i) so
// each child pair is one conflict-free 64-bit load per word, and levels
// ping-pong between two buffers so a level needs a single barrier.
//
// Leaf functors implement
//   __device__ void operator()(uint64_t leaf, uint32_t out[8]) const;
// and may have side effects (the fused FRI fold writes its folded value), since
// each leaf is evaluated exactly once.
#pragma once
#include <cstdint>

#include "vs_blake2s.cuh"
#include "vs_mem.cuh"

namespace vs {

constexpr int MK_THREADS = 256;
constexpr int MK_MAX_TL = 10;

// Shared memory: leaf layer (8 * 2^TL words) + next layer (8 * 2^(TL-1) words).
inline unsigned merkle_smem_bytes(uint32_t TL) { return (8u << TL) * 4u + (TL ? (8u << (TL - 1)) * 4u : 0u); }

// With stop_log > 0 the reduction stops at 2^stop_log subtree roots per tile
// (written hash-major: hash j of tile b at roots[(b * 2^stop_log + j) * 8]), so a
// CTA skips the narrow top levels of its tile, where most of its warps would wait
// at barriers; the next reduction level takes them over.
template <class Leaf>
__global__ void __launch_bounds__(MK_THREADS) merkle_subtree_kernel(Leaf leaf, uint32_t TL, uint64_t n_leaves,
                                                                   uint32_t* __restrict__ roots, uint32_t stop_log) {
  extern __shared__ uint32_t mk_sm[];
  const uint32_t tile = 1u << TL;
  const uint64_t base = (uint64_t)blockIdx.x << TL;
  uint32_t* bufA = mk_sm;
  uint32_t* bufB = mk_sm + 8 * tile;
  for (uint32_t i = threadIdx.x; i < tile; i += MK_THREADS) {
    uint32_t h[8];
    if (base + i < n_leaves) leaf(base + i, h);
    else {
#pragma unroll
      for (int w = 0; w < 8; w++) h[w] = 0;
    }
#pragma unroll
    for (int w = 0; w < 8; w++) bufA[w * tile + i] = h[w];
  }
  __syncthreads();
  uint32_t* cur = bufA;
  uint32_t* nxt = bufB;
  uint32_t cur_n = tile;
  const uint32_t n_out = 1u << stop_log;
  while (cur_n > n_out) {
    const uint32_t half = cur_n >> 1;
    for (uint32_t i = threadIdx.x; i < half; i += MK_THREADS) {
      uint32_t m[16];
#pragma unroll
      for (int w = 0; w < 8; w++) {
        uint2 lr = *reinterpret_cast<const uint2*>(cur + w * cur_n + 2 * i);
        m[w] = lr.x;
        m[8 + w] = lr.y;
      }
      uint32_t h[8];
      b2s_init(h);
      b2s_compress(h, m, 64u, true);
#pragma unroll
      for (int w = 0; w < 8; w++) nxt[w * half + i] = h[w];
    }
    __syncthreads();
    uint32_t* t = cur;
    cur = nxt;
    nxt = t;
    cur_n = half;
  }
  for (uint32_t i = threadIdx.x; i < 8 * n_out; i += MK_THREADS)
    roots[((uint64_t)blockIdx.x * n_out + (i >> 3)) * 8 + (i & 7)] = cur[(i & 7) * n_out + (i >> 3)];
}

// ------------------------------------------------------------------ leaf functors
// Hash inputs that are already node hashes (8 words each).
struct LeafHashes {
  const uint32_t* h;
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    const uint4 a = ld4_ro(h + 8 * i), b = ld4_ro(h + 8 * i + 4);
    out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
    out[4] = b.x; out[5] = b.y; out[6] = b.z; out[7] = b.w;
  }
};

// Reference trace leaf: the first min(n_cols, 16) columns, t = 4*min(n_cols, 16)
// (blake2s.cu:13-62). Columns via a device pointer array or base + stride.
struct LeafCapped {
  const uint32_t* const* cols;
  const uint32_t* base;
  uint64_t stride;
  uint32_t n_cols;
  __device__ __forceinline__ const uint32_t* col(uint32_t c) const { return cols ? cols[c] : base + c * stride; }
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    // the column count is the same for every leaf: dispatch it to a compile-time
    // count so the compiler drops the additions of the zero message words
    switch (n_cols < 16 ? n_cols : 16) {
#define VS_CP(r) case r: hash<r>(i, out); break;
      VS_CP(0) VS_CP(1) VS_CP(2) VS_CP(3) VS_CP(4) VS_CP(5) VS_CP(6) VS_CP(7) VS_CP(8)
      VS_CP(9) VS_CP(10) VS_CP(11) VS_CP(12) VS_CP(13) VS_CP(14) VS_CP(15)
      default: hash<16>(i, out); break;
#undef VS_CP
    }
  }
  template <int NC>
  __device__ __forceinline__ void hash(uint64_t i, uint32_t out[8]) const {
    uint32_t m[16];
#pragma unroll
    for (int c = 0; c < 16; c++) m[c] = c < NC ? col(c)[i] : 0u;
    b2s_single(out, m, NC);
  }
};

// Single column, t = 4 (the Fibonacci trace tree).
struct LeafOne {
  const uint32_t* col;
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    uint32_t m[16] = {0};
    m[0] = col[i];
    b2s_single(out, m, 1);
  }
};

// Row-packed multi-block leaf over all n_cols columns (standard Blake2s of the
// row's LE words; merkle_leaves_lifted.cu:33-98 with equal column sizes).
struct LeafRowPacked {
  const uint32_t* base;
  uint64_t stride;
  uint32_t n_cols;
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    b2s_init(out);
    uint32_t m[16];
    uint32_t done = 0;
    const uint32_t* p = base + i;
    // Non-final blocks: only when more words follow.
    while (n_cols - done > 16) {
#pragma unroll
      for (int w = 0; w < 16; w++) m[w] = __ldg(p + (uint64_t)(done + w) * stride);
      done += 16;
      b2s_compress(out, m, done * 4u, false);
    }
    // Final block: its word count is the same for every leaf, so dispatch it to a
    // compile-time count and let the compiler drop the additions of zero words
    // (14 of 16 for 34 columns).
    switch (n_cols - done) {
#define VS_RP(r) case r: final_block<r>(out, p, done); break;
      VS_RP(0) VS_RP(1) VS_RP(2) VS_RP(3) VS_RP(4) VS_RP(5) VS_RP(6) VS_RP(7) VS_RP(8)
      VS_RP(9) VS_RP(10) VS_RP(11) VS_RP(12) VS_RP(13) VS_RP(14) VS_RP(15)
      default: final_block<16>(out, p, done); break;
#undef VS_RP
    }
  }
  template <int REM>
  __device__ __forceinline__ void final_block(uint32_t out[8], const uint32_t* p, uint32_t done) const {
    uint32_t m[16];
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = w < REM ? __ldg(p + (uint64_t)(done + w) * stride) : 0u;
    b2s_compress(out, m, n_cols * 4u, true);
  }
};

// SoA4 QM31 leaf: 4 words, t = 16 (blake2s.cu:117-133).
struct LeafSoa4 {
  const uint32_t* c0;
  const uint32_t* c1;
  const uint32_t* c2;
  const uint32_t* c3;
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    uint32_t m[16] = {0};
    m[0] = c0[i];
    m[1] = c1[i];
    m[2] = c2[i];
    m[3] = c3[i];
    b2s_single(out, m, 4);
  }
};

}  // namespace vs
