// Circle NTT for sm_100a, both reference conventions:
//  * native half_coset NTT (cuda/circle_ntt.cu, src/ntt.rs:145-243)
//  * stwo / CanonicCoset NTT (cuda/circle_ntt_stwo.cu, src/ntt.rs:249-341)
//
// Both share one butterfly network: layer j pairs (i0, i0 + 2^j) with
// i0 = h*2^(j+1) + l and twiddle t = tw_j[h]; forward (v0 + v1 t, v0 - v1 t) from
// the top layer down, inverse (v0 + v1, (v0 - v1) t) from layer 0 up, then a
// 2^((30 L) mod 31) scale. Only the twiddle lookup differs.
//
// Execution: a transform is split into passes over contiguous layer ranges
// [a, b]. A pass loads tiles of 2^(b-a+1) x 2^c elements (c low index bits kept
// for coalescing) into shared memory, runs its layers as register rounds (32
// elements per thread, no barrier inside a round) and writes the tile back once.
// By default a round above the tile's first five bits holds eight 16-byte chunks
// along three layers (128-bit shared-memory traffic, one twiddle per chunk);
// the five-layer word rounds remain as the radix-5 plan the autotuner can pick. The shared tile uses a 16-byte-chunk XOR swizzle (swz)
// that keeps every round's access pattern bank-conflict free. Pass kernels loop
// over up to 8 tiles per CTA and double-buffer them: the next tile
// streams in with 16-byte cp.async copies while the current one is transformed,
// so HBM latency hides behind the integer work. A 2^24-point transform is two
// HBM round trips instead of the reference's 24 per-layer launches.
//
// The LDE path fuses interpolate -> zero-pad -> evaluate: the top pass of the
// inverse transform keeps the coefficients in shared memory and directly runs the
// forward top pass for each of the 2^B blowup blocks (the top B forward layers
// of a zero-padded input only replicate the coefficients), so neither the
// coefficients nor the zero padding touch HBM. Its upper-tile form works on
// 16-byte chunks in three-layer rounds (128-bit shared-memory traffic, one
// twiddle per chunk, 80 registers, three CTAs per SM); with 16-byte tile rows it
// runs as CTA pairs (thread-block clusters) that store whole 32-byte sectors by
// reading each other's tiles through distributed shared memory.
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "ntt.h"
#include "twiddles.h"
#include "vs_common.cuh"
#include "vs_field.cuh"

namespace vs {

// Shared-tile swizzle: the 16-byte chunk index (word bits 2..4) is XORed with
// three higher word bits chosen per C, so chunks stay whole (16-byte async
// copies and 128-bit accesses) and every register round of a tile with C low
// bits, as well as the 16-byte tile transfers, is bank-conflict free. (C = 1 is
// not a tile shape: its round 0 cannot be made conflict free this way.)
template <int C>
__device__ __forceinline__ uint32_t swz(uint32_t a) {
  static_assert(C != 1, "no C = 1 tiles");
  constexpr int s0 = C == 2 ? 7 : 5;
  constexpr int s1 = (C == 2 || C == 3) ? 8 : 6;
  constexpr int s2 = (C >= 2 && C <= 4) ? 9 : 7;
  const uint32_t h = ((a >> s0) & 1u) | (((a >> s1) & 1u) << 1) | (((a >> s2) & 1u) << 2);
  return a ^ (h << 2);
}

// x * t mod p from tt = 2t (< 2^32): x * tt = hi * 2^32 + lo with lo even, so
// x * t = hi * 2^31 + lo / 2 == hi + lo / 2 (mod p), and both halves are < 2^31.
// Written as one 64-bit product, so both halves come from a single wide multiply
// (as two 32-bit multiplies the LDE of 34 x 2^24 took 18.2 ms; 16.8 ms like this).
__device__ __forceinline__ uint32_t mul_tt(uint32_t x, uint32_t tt) {
  const uint64_t p = (uint64_t)x * tt;  // one wide multiply gives both halves
  return canon((uint32_t)(p >> 32) + ((uint32_t)p >> 1));
}

// Butterflies take doubled twiddles (tt = 2t).
template <bool FWD>
__device__ __forceinline__ void bfly(uint32_t& v0, uint32_t& v1, uint32_t tt) {
  if (FWD) {
    uint32_t m = mul_tt(v1, tt);
    v1 = sub(v0, m);
    v0 = add(v0, m);
  } else {
    uint32_t s = v0;
    v0 = add(s, v1);
    v1 = mul_tt(sub(s, v1), tt);
  }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Tile of a pass: M layers over tile bits [C, C+M); the low C index bits stay
// contiguous for coalescing. T = M + C, 2^(T-5) threads, 32 elements each.
// Register rounds cover tile bits [C + 5r, C + 5r + R(r)).
template <int M, int C>
struct Tile {
  static constexpr int T = M + C, NT = 1 << (T - 5), SIZE = 1 << T, NR = (M + 4) / 5;
  static constexpr int P0(int r) { return C + 5 * r; }
  static constexpr int R(int r) { return 5 * (r + 1) <= M ? 5 : M - 5 * r; }
};

// Runtime part of a tile's placement in the transform.
struct TileGeo {
  uint32_t a;      // first layer of the pass
  uint32_t hi;     // index bits above the pass (the twiddle group prefix)
  uint32_t gbase;  // hi << (b+1) | lo_chunk << C
};

template <int M, int C>
__device__ __forceinline__ TileGeo tile_geo(uint32_t a, uint32_t tile) {
  constexpr int T = M + C;
  TileGeo g;
  g.a = a;
  const uint32_t lo_bits = a - C;
  g.hi = tile >> lo_bits;
  const uint32_t b1 = a + M;  // b + 1
  g.gbase = (b1 >= 32 ? 0u : (g.hi << b1)) | ((tile & ((1u << lo_bits) - 1)) << C);
  (void)T;
  return g;
}
// Global index of tile element e (requires C == 0 -> a == 0 or C >= 2 for 16-byte runs).
template <int M, int C>
__device__ __forceinline__ uint32_t gidx(const TileGeo& g, uint32_t e) {
  return g.gbase | ((e >> C) << g.a) | (e & ((1u << C) - 1));
}

// Coalesced 128-bit tile transfers between global memory and the swizzled tile.
template <int M, int C>
__device__ __forceinline__ void tile_load(uint32_t* sm, const uint32_t* __restrict__ src, const TileGeo& g,
                                          uint32_t mask) {
  using S = Tile<M, C>;
#pragma unroll
  for (int i = 0; i < S::SIZE / 4 / S::NT; i++) {
    const uint32_t e = 4 * (threadIdx.x + i * S::NT);
    *reinterpret_cast<uint4*>(sm + swz<C>(e)) = *reinterpret_cast<const uint4*>(src + (gidx<M, C>(g, e) & mask));
  }
}
// The same load as 16-byte asynchronous copies (no registers held while in flight).
template <int M, int C>
__device__ __forceinline__ void tile_load_async(uint32_t* sm, const uint32_t* __restrict__ src, const TileGeo& g,
                                                uint32_t mask) {
  using S = Tile<M, C>;
  const uint32_t base = smem_addr(sm);
#pragma unroll
  for (int i = 0; i < S::SIZE / 4 / S::NT; i++) {
    const uint32_t e = 4 * (threadIdx.x + i * S::NT);
    cp_async16(base + 4 * swz<C>(e), src + (gidx<M, C>(g, e) & mask));
  }
}
template <int M, int C>
__device__ __forceinline__ void tile_store(const uint32_t* sm, uint32_t* __restrict__ dst, const TileGeo& g) {
  using S = Tile<M, C>;
#pragma unroll
  for (int i = 0; i < S::SIZE / 4 / S::NT; i++) {
    const uint32_t e = 4 * (threadIdx.x + i * S::NT);
    *reinterpret_cast<uint4*>(dst + gidx<M, C>(g, e)) = *reinterpret_cast<const uint4*>(sm + swz<C>(e));
  }
}

// Address of element k (R bits) of subgroup o, inserted at tile bit P0.
template <int P0, int R>
__device__ __forceinline__ uint32_t ins(uint32_t o, uint32_t k) {
  return ((o >> P0) << (P0 + R)) | (k << P0) | (o & ((1u << P0) - 1));
}

// Round 0 of a C = 0 tile holds 32 consecutive words per thread: eight 128-bit
// accesses (conflict free per quarter warp under swz<0>).
template <int M, int C, int r>
__device__ __forceinline__ void rload(uint32_t (&v)[32], const uint32_t* sm) {
  using S = Tile<M, C>;
  constexpr int P0 = S::P0(r), R = S::R(r), K = 1 << R, SUB = 1 << (5 - R);
  if constexpr (C == 0 && r == 0) {
    static_assert(R == 5, "C = 0 tiles start with a five-layer round");
    const uint32_t row = threadIdx.x << 5;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint4 w = *reinterpret_cast<const uint4*>(sm + swz<C>(row | (4 * j)));
      v[4 * j] = w.x;
      v[4 * j + 1] = w.y;
      v[4 * j + 2] = w.z;
      v[4 * j + 3] = w.w;
    }
  } else {
#pragma unroll
    for (int s = 0; s < SUB; s++)
#pragma unroll
      for (int k = 0; k < K; k++) v[s * K + k] = sm[swz<C>(ins<P0, R>(threadIdx.x + s * S::NT, k))];
  }
}
template <int M, int C, int r>
__device__ __forceinline__ void rstore(const uint32_t (&v)[32], uint32_t* sm) {
  using S = Tile<M, C>;
  constexpr int P0 = S::P0(r), R = S::R(r), K = 1 << R, SUB = 1 << (5 - R);
  if constexpr (C == 0 && r == 0) {
    const uint32_t row = threadIdx.x << 5;
#pragma unroll
    for (int j = 0; j < 8; j++)
      *reinterpret_cast<uint4*>(sm + swz<C>(row | (4 * j))) = make_uint4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
  } else {
#pragma unroll
    for (int s = 0; s < SUB; s++)
#pragma unroll
      for (int k = 0; k < K; k++) sm[swz<C>(ins<P0, R>(threadIdx.x + s * S::NT, k))] = v[s * K + k];
  }
}

// Butterflies of round r (R layers, no barrier). All of the round's twiddles are
// fetched into registers first (doubled, for mul_tt) so their loads overlap
// instead of stalling each butterfly. Layer at tile bit p = P0 + q is global layer j = a + p - C; its
// group index is h = hi * 2^(T-1-p) + (address >> (p+1)).
template <bool FWD, int M, int C, int r>
__device__ __forceinline__ void rbfly(uint32_t (&v)[32], const TileGeo& g, const NttTw& tw) {
  using S = Tile<M, C>;
  constexpr int P0 = S::P0(r), R = S::R(r), K = 1 << R, SUB = 1 << (5 - R), T = S::T;
#pragma unroll
  for (int s = 0; s < SUB; s++) {
    const uint32_t base = ins<P0, R>(threadIdx.x + s * S::NT, 0);
    uint32_t t[K];  // layer q's twiddles at t[K - (K >> q) + gg]
#pragma unroll
    for (int q = 0; q < R; q++) {
      const int p = P0 + q;
      const uint32_t hb = (g.hi << (T - 1 - p)) | (base >> (p + 1));
      bool circle_stwo = false;
      if (C == 0 && r == 0 && q == 0) circle_stwo = tw.stwo && g.a == 0;
      if (circle_stwo) {  // circle_ntt_stwo.cu:202-248: [y, -y, -x, x] per pair of line layer 0
        static_assert(C != 0 || R == 5 || r != 0, "round 0 of a C = 0 tile spans five layers");
#pragma unroll
        for (int gg = 0; gg < (K >> 1); gg += 4) {  // hb is a multiple of 4 here
          const uint32_t pr = 2 * ((hb >> 2) + (gg >> 2));
          const uint32_t x = __ldg(tw.flat + pr), y = __ldg(tw.flat + pr + 1);
          t[gg] = y << 1;
          t[gg + 1] = neg(y) << 1;
          t[gg + 2] = neg(x) << 1;
          t[gg + 3] = x << 1;
        }
      } else {
        // A thread's twiddles of one layer are consecutive and start at a
        // multiple of their count (hb has zero low bits there); the host side
        // hands the kernels tables aligned to min(16 B, table size), so they are
        // fetched with 128- or 64-bit loads.
        const uint32_t* tp = tw.layer[g.a + p - C] + hb;
        const int cnt = K >> (q + 1), o = K - (K >> q);
        if (cnt >= 4) {
#pragma unroll
          for (int v = 0; v < cnt / 4; v++) {
            const uint4 w = __ldg(reinterpret_cast<const uint4*>(tp) + v);
            t[o + 4 * v] = w.x << 1;
            t[o + 4 * v + 1] = w.y << 1;
            t[o + 4 * v + 2] = w.z << 1;
            t[o + 4 * v + 3] = w.w << 1;
          }
        } else if (cnt == 2) {
          const uint2 w = __ldg(reinterpret_cast<const uint2*>(tp));
          t[o] = w.x << 1;
          t[o + 1] = w.y << 1;
        } else {
#pragma unroll
          for (int gg = 0; gg < cnt; gg++) t[o + gg] = __ldg(tp + gg) << 1;
        }
      }
    }
#pragma unroll
    for (int qq = 0; qq < R; qq++) {
      const int q = FWD ? R - 1 - qq : qq;
#pragma unroll
      for (int gg = 0; gg < (K >> (q + 1)); gg++) {
        const uint32_t tv = t[K - (K >> q) + gg];
#pragma unroll
        for (int l = 0; l < (1 << q); l++) {
          const int k0 = (gg << (q + 1)) | l;
          bfly<FWD>(v[s * K + k0], v[s * K + k0 + (1 << q)], tv);
        }
      }
    }
  }
}

// One full round through shared memory (caller provides the barrier after).
template <bool FWD, int M, int C, int r>
__device__ __forceinline__ void round_sm(uint32_t* sm, const TileGeo& g, const NttTw& tw, uint32_t scale) {
  uint32_t v[32];
  rload<M, C, r>(v, sm);
  rbfly<FWD, M, C, r>(v, g, tw);
  if (scale) {
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = mul(v[k], scale);
  }
  rstore<M, C, r>(v, sm);
}

__device__ __forceinline__ const uint32_t* col_src(const NttPass& p, uint32_t c) {
  return p.src_cols ? p.src_cols[c] : p.src + (uint64_t)c * p.src_stride;
}
__device__ __forceinline__ uint32_t* col_dst(const NttPass& p, uint32_t c) {
  return p.dst_cols ? p.dst_cols[c] : p.dst + (uint64_t)c * p.dst_stride;
}

// One pass over work items w = tile * n_cols + column, strided by the grid:
// tile-major, so the columns of one tile range run back to back and the twiddles
// of that range (the low layers' tables outgrow L2 at 2^26 points) are fetched
// from HBM once and then hit L2 for the other columns.
// Per item: NR register rounds (forward: top round first) on the shared tile,
// then the tile is stored; the next item's tile is already in flight into the
// other buffer. The inverse scale is folded into the last round of the last
// inverse pass. Every thread commits one copy group per iteration (empty at the
// end), so "wait until one group is pending" always means "this tile landed".
template <bool FWD, int M, int C>
__global__ void __launch_bounds__(1 << (M + C - 5), (FWD && C == 0) ? 3 : 2) ntt_pass_kernel(NttPass p, uint32_t n_cols,
                                                                      uint32_t total) {
  using S = Tile<M, C>;
  extern __shared__ __align__(16) uint32_t pass_sm[];
  uint32_t w = blockIdx.x;
  if (w >= total) return;
  tile_load_async<M, C>(pass_sm, col_src(p, w % n_cols), tile_geo<M, C>(p.a, w / n_cols), p.src_mask);
  cp_async_commit();
  for (uint32_t it = 0; w < total; it++, w += gridDim.x) {
    uint32_t* sm = pass_sm + (it & 1) * S::SIZE;
    const uint32_t nw = w + gridDim.x;
    if (nw < total)
      tile_load_async<M, C>(pass_sm + ((it + 1) & 1) * S::SIZE, col_src(p, nw % n_cols),
                            tile_geo<M, C>(p.a, nw / n_cols), p.src_mask);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const TileGeo g = tile_geo<M, C>(p.a, w / n_cols);
#pragma unroll
    for (int rr = 0; rr < S::NR; rr++) {
      const uint32_t sc = (!FWD && rr == S::NR - 1) ? p.scale : 0u;
      switch (FWD ? S::NR - 1 - rr : rr) {
        case 0: round_sm<FWD, M, C, 0>(sm, g, p.tw, sc); break;
        case 1: round_sm<FWD, M, C, (S::NR > 1 ? 1 : 0)>(sm, g, p.tw, sc); break;
        default: round_sm<FWD, M, C, (S::NR > 2 ? 2 : 0)>(sm, g, p.tw, sc); break;
      }
      __syncthreads();
    }
    tile_store<M, C>(sm, col_dst(p, w % n_cols), g);
    __syncthreads();  // this buffer is refilled by the next iteration's prefetch
  }
}

template <bool FWD, int M, int C>
__device__ __forceinline__ void rounds_below_top(uint32_t* sm, const TileGeo& g, const NttTw& tw) {
  // forward: rounds NR-2 .. 0 ; inverse: rounds 0 .. NR-2 (the top round is handled by the caller)
  using S = Tile<M, C>;
#pragma unroll
  for (int rr = 0; rr + 1 < S::NR; rr++) {
    const int r = FWD ? S::NR - 2 - rr : rr;
    if (r == 0) round_sm<FWD, M, C, 0>(sm, g, tw, 0);
    else round_sm<FWD, M, C, (S::NR > 2 ? 1 : 0)>(sm, g, tw, 0);
    __syncthreads();
  }
}

// Fused LDE top pass: inverse layers [a, l-1] of the trace tile with the 1/n
// scale; the coefficients are parked in a second shared tile, and for each
// blowup block q the forward layers [a, l-1] of the evaluation domain (tile
// prefix hi = q) run on them and the result is written to dst block q. This
// five-layer-round form serves C = 0 tiles (transforms of at most 13 layers);
// upper tiles (C >= 2) use the chunk-round form ntt_lde_top4_kernel below.
template <int M, int C>
__global__ void __launch_bounds__(1 << (M + C - 5), 2) ntt_lde_top_kernel(NttPass inv, NttPass fwd, uint32_t B) {
  using S = Tile<M, C>;
  constexpr int TOP = S::NR - 1;
  extern __shared__ uint32_t lde_sm[];
  uint32_t* sm = lde_sm;              // working tile
  uint32_t* cf = lde_sm + S::SIZE;    // coefficients
  const TileGeo gi = tile_geo<M, C>(inv.a, blockIdx.x);
  tile_load<M, C>(sm, col_src(inv, blockIdx.y), gi, inv.src_mask);
  __syncthreads();
  rounds_below_top<false, M, C>(sm, gi, inv.tw);
  {
    uint32_t v[32];
    rload<M, C, TOP>(v, sm);
    rbfly<false, M, C, TOP>(v, gi, inv.tw);
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = mul(v[k], inv.scale);
    rstore<M, C, TOP>(v, cf);
  }
  __syncthreads();
  uint32_t* dst = col_dst(fwd, blockIdx.y);
  for (uint32_t q = 0; q < (1u << B); q++) {
    TileGeo gf = gi;
    gf.hi = q;
    gf.gbase = (q << (gi.a + M)) | gi.gbase;
    uint32_t v[32];
    rload<M, C, TOP>(v, cf);
    rbfly<true, M, C, TOP>(v, gf, fwd.tw);
    rstore<M, C, TOP>(v, sm);  // the previous block's tile_store finished before the loop-end barrier
    __syncthreads();
    rounds_below_top<true, M, C>(sm, gf, fwd.tw);
    tile_store<M, C>(sm, dst, gf);
    __syncthreads();
  }
}

// ---- Chunk-round variant of the fused LDE top pass (tiles with C >= 2).
// A thread holds eight 16-byte chunks (the four words of tile bits 0-1) along
// three round bits, so every shared-memory access is 128-bit, and the four words
// of a chunk share each twiddle (7 twiddles per three-layer round instead of 31
// per five-layer round). Round r covers tile bits [C + 3r, C + 3r + R(r)).
// The tile uses swz<0> (chunk index XOR word bits 5-7), which keeps every
// quarter-warp of these 128-bit accesses on eight distinct chunk positions for
// every round shape with C >= 2 (round bits at or above word bit 2).
// Chunk rounds cover tile bits [S0, C + M): S0 = C for upper tiles, S0 = 5 for
// C = 0 tiles whose bits 0-4 run first as one five-layer word round.
template <int M, int C, int S0 = C>
struct Tile4 {
  static_assert(S0 >= 2 && S0 >= C, "chunk rounds need two contiguous index bits below them");
  static constexpr int T = M + C, NT = 1 << (T - 5), SIZE = 1 << T, MC = T - S0, NR = (MC + 2) / 3;
  static constexpr int P0(int r) { return S0 + 3 * r; }
  static constexpr int R(int r) { return 3 * (r + 1) <= MC ? 3 : MC - 3 * r; }
};

// Whether chunk rounds r and r + 1 of a tile give every warp the same 16-byte
// chunks, so that a warp barrier orders the two rounds: the warp bits of the thread
// index (bits 5 and up) land on chunk bit b below the round and b + R above it in
// ins4, and on chunk bit b + 3 in the word round of a C = 0 tile (32 consecutive
// words per thread). (Checked against the address maps of every tile shape, for all
// threads, on the CPU.) Tiles of fewer than 32 threads keep CTA barriers.
template <int M, int C, int S0>
__host__ __device__ constexpr bool warp_local_next(int r) {
  using S = Tile4<M, C, S0>;
  bool same = S::NT >= 32 && r + 1 < S::NR;
  for (int b = 5; same && (1 << b) < S::NT; b++) {
    const int fa = b < S::P0(r) - 2 ? b : b + S::R(r);
    const int fb = b < S::P0(r + 1) - 2 ? b : b + S::R(r + 1);
    same = fa == fb;
  }
  return same;
}
// The word round and chunk round 0 of a C = 0 tile (S0 = 5).
template <int M>
__host__ __device__ constexpr bool warp_local_word() {
  using S = Tile4<M, 0, 5>;
  return S::NT >= 32 && S::R(0) == 3;
}
__device__ __forceinline__ void round_sync(bool warp_local) {
  if (warp_local) __syncwarp();
  else __syncthreads();
}

// Thread-block cluster primitives (the LDE top pass's cluster form): split cluster
// barrier (arrive with release, wait with acquire semantics at cluster scope) and
// loads from a peer CTA's shared memory (distributed shared memory).
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
// Arrive without release semantics (it does not wait for the thread's outstanding
// stores): for arrivals that only announce that the thread's reads are complete,
// which program order already guarantees when each loaded value has been consumed
// by an instruction before the arrive.
__device__ __forceinline__ void cluster_arrive_relaxed() {
  asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// the same shared-memory offset in the CTA of cluster rank `rank`
__device__ __forceinline__ uint32_t cluster_peer(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ uint4 ld_cluster16(uint32_t addr) {
  uint4 v;
  asm volatile("ld.shared::cluster.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(addr)
               : "memory");
  return v;
}

// Word address of chunk k (R round bits at word bit P0) of chunk group o; o
// enumerates the chunk-index bits outside the round.
template <int P0, int R>
__device__ __forceinline__ uint32_t ins4(uint32_t o, uint32_t k) {
  constexpr int Q = P0 - 2;
  return (((o >> Q) << (Q + R)) | (k << Q) | (o & ((1u << Q) - 1))) << 2;
}

template <int M, int C>
__device__ __forceinline__ void tile_load4(uint32_t* sm, const uint32_t* __restrict__ src, const TileGeo& g,
                                           uint32_t mask) {
  using S = Tile<M, C>;
#pragma unroll
  for (int i = 0; i < S::SIZE / 4 / S::NT; i++) {
    const uint32_t e = 4 * (threadIdx.x + i * S::NT);
    *reinterpret_cast<uint4*>(sm + swz<0>(e)) = *reinterpret_cast<const uint4*>(src + (gidx<M, C>(g, e) & mask));
  }
}
template <int M, int C>
__device__ __forceinline__ void tile_store4(const uint32_t* sm, uint32_t* __restrict__ dst, const TileGeo& g) {
  using S = Tile<M, C>;
#pragma unroll
  for (int i = 0; i < S::SIZE / 4 / S::NT; i++) {
    const uint32_t e = 4 * (threadIdx.x + i * S::NT);
    *reinterpret_cast<uint4*>(dst + gidx<M, C>(g, e)) = *reinterpret_cast<const uint4*>(sm + swz<0>(e));
  }
}
// Tile store of a cluster of K CTAs over adjacent tiles lo0 .. lo0+K-1: each tile
// holds 2^C consecutive words of every row, the K tiles together a segment of
// K 2^C words (up to 128 bytes). CTA `rank` stores rows [rank R/K, (rank+1) R/K)
// of all K tiles, reading the other tiles' pieces from their CTAs' shared memory,
// so consecutive threads write whole segments (a tile alone can only store its
// 2^C-word pieces: with 16-byte pieces, half sectors, one memory request each).
// The caller brackets it with cluster barriers: every tile of the cluster is
// complete before, and no CTA overwrites its tile until all have read it.
template <int M, int C, int K>
__device__ __forceinline__ void tile_store4_cluster(const uint32_t* sm, uint32_t* __restrict__ dst, const TileGeo& g) {
  using S = Tile<M, C>;
  static_assert(C >= 2 && (K << C) <= 32, "a cluster covers at most one 128-byte line of every row");
  constexpr uint32_t R = 1u << M, CH = 1u << (C - 2), SEG = K * CH;  // rows; 16-byte chunks per tile row, per segment
  const uint32_t rank = cluster_rank();
  const uint32_t base = g.gbase - (rank << C);  // the cluster's first tile: lo0 << C
  const uint32_t sm0 = smem_addr(sm);
#pragma unroll 4
  for (int i = 0; i < S::SIZE / 4 / S::NT; i++) {
    const uint32_t p = threadIdx.x + i * S::NT;  // chunk of this CTA's share
    const uint32_t j = p % SEG, r = rank * (R / K) + p / SEG;
    const uint32_t e = (r << C) | ((j % CH) << 2);  // tile word of chunk j % CH of row r
    const uint4 v = ld_cluster16(cluster_peer(sm0 + 4 * swz<0>(e), j / CH));
    *reinterpret_cast<uint4*>(dst + (base | (r << g.a) | (j << 2))) = v;
  }
}

template <int M, int C, int r, int S0 = C>
__device__ __forceinline__ void rload4(uint4 (&v)[8], const uint32_t* sm) {
  using S = Tile4<M, C, S0>;
  constexpr int P0 = S::P0(r), R = S::R(r), K = 1 << R, SUB = 1 << (3 - R);
#pragma unroll
  for (int s = 0; s < SUB; s++)
#pragma unroll
    for (int k = 0; k < K; k++)
      v[s * K + k] = *reinterpret_cast<const uint4*>(sm + swz<0>(ins4<P0, R>(threadIdx.x + s * S::NT, k)));
}
template <int M, int C, int r, int S0 = C>
__device__ __forceinline__ void rstore4(const uint4 (&v)[8], uint32_t* sm) {
  using S = Tile4<M, C, S0>;
  constexpr int P0 = S::P0(r), R = S::R(r), K = 1 << R, SUB = 1 << (3 - R);
#pragma unroll
  for (int s = 0; s < SUB; s++)
#pragma unroll
    for (int k = 0; k < K; k++)
      *reinterpret_cast<uint4*>(sm + swz<0>(ins4<P0, R>(threadIdx.x + s * S::NT, k))) = v[s * K + k];
}

template <bool FWD>
__device__ __forceinline__ void bfly4(uint4& a, uint4& b, uint32_t tt) {
  bfly<FWD>(a.x, b.x, tt);
  bfly<FWD>(a.y, b.y, tt);
  bfly<FWD>(a.z, b.z, tt);
  bfly<FWD>(a.w, b.w, tt);
}


// Twiddles of chunk round r for every subgroup of the thread, doubled (for
// mul_tt): layer q of subgroup s at t[s * (K - 1) + K - (K >> q) + gg]. Split from
// the butterflies so a round's twiddles can be fetched one round ahead. A
// thread's twiddles of one layer are consecutive and start at a multiple of their
// count; tables are 16-byte aligned up to their size (host-checked), so they load
// as one 128-, 64- or 32-bit access per layer.
template <int M, int C, int r, int S0 = C>
__device__ __forceinline__ void tw4_fetch(uint32_t (&t)[8], const TileGeo& g, const NttTw& tw) {
  using S = Tile4<M, C, S0>;
  constexpr int P0 = S::P0(r), R = S::R(r), K = 1 << R, SUB = 1 << (3 - R), T = S::T;
#pragma unroll
  for (int s = 0; s < SUB; s++) {
    const uint32_t base = ins4<P0, R>(threadIdx.x + s * S::NT, 0);
#pragma unroll
    for (int q = 0; q < R; q++) {
      const int p = P0 + q;
      const uint32_t hb = (g.hi << (T - 1 - p)) | (base >> (p + 1));
      const uint32_t* tp = tw.layer[g.a + p - C] + hb;
      const int cnt = K >> (q + 1), o = s * (K - 1) + K - (K >> q);
      if (cnt == 4) {
        const uint4 w = __ldg(reinterpret_cast<const uint4*>(tp));
        t[o] = w.x << 1;
        t[o + 1] = w.y << 1;
        t[o + 2] = w.z << 1;
        t[o + 3] = w.w << 1;
      } else if (cnt == 2) {
        const uint2 w = __ldg(reinterpret_cast<const uint2*>(tp));
        t[o] = w.x << 1;
        t[o + 1] = w.y << 1;
      } else {
        t[o] = __ldg(tp) << 1;
      }
    }
  }
}
template <bool FWD, int M, int C, int r, int S0 = C>
__device__ __forceinline__ void rbfly4_t(uint4 (&v)[8], const uint32_t (&t)[8]) {
  using S = Tile4<M, C, S0>;
  constexpr int R = S::R(r), K = 1 << R, SUB = 1 << (3 - R);
#pragma unroll
  for (int s = 0; s < SUB; s++)
#pragma unroll
    for (int qq = 0; qq < R; qq++) {
      const int q = FWD ? R - 1 - qq : qq;
#pragma unroll
      for (int gg = 0; gg < (K >> (q + 1)); gg++) {
        const uint32_t tv = t[s * (K - 1) + K - (K >> q) + gg];
#pragma unroll
        for (int l = 0; l < (1 << q); l++) {
          const int k0 = (gg << (q + 1)) | l;
          bfly4<FWD>(v[s * K + k0], v[s * K + k0 + (1 << q)], tv);
        }
      }
    }
}

// Inverse chunk rounds r..TOP with round r's twiddles in t; each round fetches
// the next round's twiddles before its own shared-memory loads. The last round
// applies `scale` (if nonzero) and stores to cf (the coefficient tile of the LDE
// top pass; the working tile itself in a pass kernel).
template <int M, int C, int r, int S0 = C>
__device__ __forceinline__ void inv_rounds4(uint32_t* sm, uint32_t* cf, const TileGeo& g, const NttTw& tw,
                                            uint32_t scale, uint32_t (&t)[8], const TileGeo& gn,
                                            const NttTw& twn) {
  constexpr int TOP = Tile4<M, C, S0>::NR - 1;
  uint32_t tn[8];
  if constexpr (r < TOP) tw4_fetch<M, C, r + 1, S0>(tn, g, tw);
  uint4 v[8];
  rload4<M, C, r, S0>(v, sm);
  rbfly4_t<false, M, C, r, S0>(v, t);
  // t is free once the last round's butterflies are done: fetch the forward
  // pass's first-round twiddles into it, ahead of the scale, stores and barrier
  if constexpr (r == TOP) tw4_fetch<M, C, TOP, S0>(t, gn, twn);
  if constexpr (r == TOP) {
    if (scale) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        v[k].x = mul(v[k].x, scale);
        v[k].y = mul(v[k].y, scale);
        v[k].z = mul(v[k].z, scale);
        v[k].w = mul(v[k].w, scale);
      }
    }
    rstore4<M, C, r, S0>(v, cf);
  } else {
    rstore4<M, C, r, S0>(v, sm);
  }
  // the forward pass's first round reads cf with the last round's own map (a warp
  // barrier orders them; it waits for all warps before it overwrites sm)
  round_sync(r == TOP ? Tile4<M, C, S0>::NT >= 32 : warp_local_next<M, C, S0>(r));
  if constexpr (r < TOP) {
#pragma unroll
    for (int k = 0; k < 8; k++) t[k] = tn[k];
    inv_rounds4<M, C, r + 1, S0>(sm, cf, g, tw, scale, t, gn, twn);
  }
}
// Forward chunk rounds r..0 (round TOP reads from cf: the parked coefficients of
// the LDE top pass, the working tile in a pass kernel), twiddles fetched one round
// ahead as above.
template <int M, int C, int r, int S0 = C, int K = 1>
__device__ __forceinline__ void fwd_rounds4(uint32_t* sm, const uint32_t* cf, const TileGeo& g, const NttTw& tw,
                                            uint32_t (&t)[8], const TileGeo& gn, bool next) {
  constexpr int TOP = Tile4<M, C, S0>::NR - 1;
  uint32_t tn[8];
  if constexpr (r > 0) tw4_fetch<M, C, (r > 0 ? r - 1 : 0), S0>(tn, g, tw);
  uint4 v[8];
  rload4<M, C, r, S0>(v, r == TOP ? cf : sm);
  rbfly4_t<true, M, C, r, S0>(v, t);
  // after the block's last butterflies t is free: fetch the next block's
  // first-round twiddles into it, ahead of the stores, barrier and tile store
  // (in a cluster: after the release arrive below, which would wait for these loads)
  if constexpr (r == 0 && K == 1) {
    if (next) tw4_fetch<M, C, TOP, S0>(t, gn, tw);
  }
  // the first round reads only the parked coefficients; it waits for the previous
  // block's tile store (which reads sm) only before writing sm itself, so its loads
  // and butterflies overlap that store
  // (in a cluster: until every CTA of the cluster has stored its share, which reads
  // this tile too)
  if constexpr (r == TOP) {
    if constexpr (K > 1) cluster_wait();
    else __syncthreads();
  }
  rstore4<M, C, r, S0>(v, sm);
  if constexpr (K > 1 && r == 0) {  // the cluster's tile store reads every tile of the cluster
    cluster_arrive();
    if (next) tw4_fetch<M, C, TOP, S0>(t, gn, tw);
    cluster_wait();
  } else {
    round_sync(r > 0 && warp_local_next<M, C, S0>(r - 1));  // round 0: the tile store reads everything
  }
  if constexpr (r > 0) {
#pragma unroll
    for (int k = 0; k < 8; k++) t[k] = tn[k];
    fwd_rounds4<M, C, (r > 0 ? r - 1 : 0), S0, K>(sm, cf, g, tw, t, gn, next);
  }
}

// Same dataflow as ntt_lde_top_kernel: inverse rounds with the 1/n scale folded
// into the last one, which parks the coefficients in the second tile; then for
// each blowup block q the forward rounds from the parked tile, stored to block q.
// Each round's twiddles are loaded during the round before it (the first inverse
// round's during the tile load, a block's first forward round's during the
// previous block's tile store), so their L2 latency is off the round's critical path.
//
// Cluster form (K > 1, launched as clusters of K CTAs over adjacent tiles): the
// blocks' tiles are stored as segments of K 2^C words gathered across the cluster
// (tile_store4_cluster) instead of 2^C-word pieces. The split cluster barrier
// alternates arrive and wait on every thread: an arrive after the inverse rounds;
// per block, a wait before the first round writes
// the tile (every CTA has finished reading the previous block's tiles), an arrive
// and wait after the last round (all tiles complete; the arrive releases the tile
// to the other CTAs), an arrive after the store (relaxed: it only announces reads);
// and a last wait before exit, so no CTA leaves while its tile is still being read.
template <int M, int C>
__device__ __forceinline__ void tile_load_async4(uint32_t* sm, const uint32_t* __restrict__ src, const TileGeo& g,
                                                 uint32_t mask);
template <int M, int C, int K = 1>
__global__ void __launch_bounds__(1 << (M + C - 5), 3) ntt_lde_top4_kernel(NttPass inv, NttPass fwd, uint32_t B) {
  using S = Tile4<M, C>;
  static_assert(S::NR <= 4, "at most four chunk rounds");
  constexpr int TOP = S::NR - 1;
  extern __shared__ __align__(16) uint32_t lde4_sm[];
  uint32_t* sm = lde4_sm;            // working tile
  uint32_t* cf = lde4_sm + S::SIZE;  // coefficients
  const TileGeo gi = tile_geo<M, C>(inv.a, blockIdx.x);
  uint32_t t[8];
  // the input tile streams into shared memory by 16-byte cp.async (no registers in
  // flight) while the first round's twiddles load
  tile_load_async4<M, C>(sm, col_src(inv, blockIdx.y), gi, inv.src_mask);
  cp_async_commit();
  tw4_fetch<M, C, 0>(t, gi, inv.tw);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  uint32_t* dst = col_dst(fwd, blockIdx.y);
  TileGeo gf = gi;
  gf.hi = 0;
  gf.gbase = gi.gbase;
  // each block's first-round twiddles are fetched right after the butterflies of
  // the round before it (the last inverse round, then each block's round 0)
  inv_rounds4<M, C, 0>(sm, cf, gi, inv.tw, inv.scale, t, gf, fwd.tw);
  if constexpr (K > 1) cluster_arrive_relaxed();  // this CTA's last reads of sm are consumed
  for (uint32_t q = 0; q < (1u << B); q++) {
    const TileGeo gq = gf;
    const bool more = q + 1 < (1u << B);
    if (more) {
      gf.hi = q + 1;
      gf.gbase = ((q + 1) << (gi.a + M)) | gi.gbase;
    }
    fwd_rounds4<M, C, TOP, C, K>(sm, cf, gq, fwd.tw, t, gf, more);
    // the next block's first round waits for the store before writing sm
    if constexpr (K > 1) {
      tile_store4_cluster<M, C, K>(sm, dst, gq);
      // every value read from the cluster's tiles is already stored, so the reads
      // are complete; no release (it would wait for those global stores)
      cluster_arrive_relaxed();
    } else {
      tile_store4<M, C>(sm, dst, gq);
    }
  }
  if constexpr (K > 1) cluster_wait();
}

// One chunk round of a pass: shared-memory loads, then the round's twiddles, then
// the butterflies (and the inverse scale on the last round).
template <bool FWD, int M, int C, int r, int S0>
__device__ __forceinline__ void round4(uint32_t* sm, const TileGeo& g, const NttTw& tw, uint32_t scale) {
  uint4 v[8];
  uint32_t t[8];
  rload4<M, C, r, S0>(v, sm);
  tw4_fetch<M, C, r, S0>(t, g, tw);
  rbfly4_t<FWD, M, C, r, S0>(v, t);
  if (scale) {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      v[k].x = mul(v[k].x, scale);
      v[k].y = mul(v[k].y, scale);
      v[k].z = mul(v[k].z, scale);
      v[k].w = mul(v[k].w, scale);
    }
  }
  rstore4<M, C, r, S0>(v, sm);
}
template <bool FWD, int M, int C, int S0>
__device__ __forceinline__ void chunk_round(int r, uint32_t* sm, const TileGeo& g, const NttTw& tw, uint32_t scale) {
  using S4 = Tile4<M, C, S0>;
  switch (r) {
    case 0: round4<FWD, M, C, 0, S0>(sm, g, tw, scale); break;
    case 1: round4<FWD, M, C, (S4::NR > 1 ? 1 : 0), S0>(sm, g, tw, scale); break;
    case 2: round4<FWD, M, C, (S4::NR > 2 ? 2 : 0), S0>(sm, g, tw, scale); break;
    default: round4<FWD, M, C, (S4::NR > 3 ? 3 : 0), S0>(sm, g, tw, scale); break;
  }
}

// Chunk-round form of the pass kernel (same persistent, double-buffered
// structure as ntt_pass_kernel). C = 0 tiles run tile bits 0-4 as one five-layer
// word round and the layers above as three-layer chunk rounds; upper tiles
// (C >= 2) run chunk rounds only. Both use the swz<0> tile layout.
template <int M, int C>
__device__ __forceinline__ void tile_load_async4(uint32_t* sm, const uint32_t* __restrict__ src, const TileGeo& g,
                                                 uint32_t mask) {
  using S = Tile<M, C>;
  const uint32_t base = smem_addr(sm);
#pragma unroll
  for (int i = 0; i < S::SIZE / 4 / S::NT; i++) {
    const uint32_t e = 4 * (threadIdx.x + i * S::NT);
    cp_async16(base + 4 * swz<0>(e), src + (gidx<M, C>(g, e) & mask));
  }
}
template <bool FWD, int M, int C>
__global__ void __launch_bounds__(1 << (M + C - 5), (M + C == 13) ? 3 : 2) ntt_pass4_kernel(NttPass p, uint32_t n_cols,
                                                                     uint32_t total) {
  constexpr int S0 = C == 0 ? 5 : C;
  using S4 = Tile4<M, C, S0>;
  static_assert(S4::NR >= 1 && S4::NR <= 4, "one to four chunk rounds");
  constexpr int SIZE = 1 << (M + C);
  extern __shared__ __align__(16) uint32_t pass4_sm[];
  uint32_t w = blockIdx.x;
  if (w >= total) return;
  tile_load_async4<M, C>(pass4_sm, col_src(p, w % n_cols), tile_geo<M, C>(p.a, w / n_cols), p.src_mask);
  cp_async_commit();
  for (uint32_t it = 0; w < total; it++, w += gridDim.x) {
    uint32_t* sm = pass4_sm + (it & 1) * SIZE;
    const uint32_t nw = w + gridDim.x;
    if (nw < total)
      tile_load_async4<M, C>(pass4_sm + ((it + 1) & 1) * SIZE, col_src(p, nw % n_cols),
                             tile_geo<M, C>(p.a, nw / n_cols), p.src_mask);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const TileGeo g = tile_geo<M, C>(p.a, w / n_cols);
    // (fetching a round's twiddles one round ahead, as the LDE top pass does,
    // measured slower here: the double-buffered tiles already hide the latency)
    // warp barriers between rounds that give every warp the same chunks
    // (warp_local_next, warp_local_word), CTA barriers elsewhere
    if (!FWD) {
      if (C == 0) {
        round_sm<false, M, C, 0>(sm, g, p.tw, 0);
        round_sync(C == 0 && warp_local_word<(C == 0 ? M : 13)>());
      }
#pragma unroll
      for (int r = 0; r < S4::NR; r++) {
        chunk_round<false, M, C, S0>(r, sm, g, p.tw, r == S4::NR - 1 ? p.scale : 0u);
        round_sync(warp_local_next<M, C, S0>(r));  // false after the last round: the tile store follows
      }
    } else {
#pragma unroll
      for (int r = S4::NR - 1; r >= 0; r--) {
        chunk_round<true, M, C, S0>(r, sm, g, p.tw, 0u);
        round_sync(r > 0 ? warp_local_next<M, C, S0>(r - 1) : (C == 0 && warp_local_word<(C == 0 ? M : 13)>()));
      }
      if (C == 0) {
        round_sm<true, M, C, 0>(sm, g, p.tw, 0);
        __syncthreads();
      }
    }
    tile_store4<M, C>(sm, col_dst(p, w % n_cols), g);
    __syncthreads();  // this buffer is refilled by the next iteration's prefetch
  }
}

// Single-buffered form of ntt_pass4_kernel: one tile per CTA, half the shared
// memory and at most 64 registers, so four CTAs share an SM instead of three (the
// other CTAs' work hides a tile's load instead of the double buffer). Used for the
// 13-layer lower passes when a plan asks for one tile per CTA (the default there):
// LDE of 34 x 2^24 14.87 -> 14.72 ms, of 34 x 2^22 3.32 -> 3.25 ms.
template <bool FWD, int M, int C>
__global__ void __launch_bounds__(1 << (M + C - 5), 4) ntt_pass4s_kernel(NttPass p, uint32_t n_cols, uint32_t total) {
  constexpr int S0 = C == 0 ? 5 : C;
  using S4 = Tile4<M, C, S0>;
  extern __shared__ __align__(16) uint32_t pass4s_sm[];
  const uint32_t w = blockIdx.x;
  if (w >= total) return;
  uint32_t* sm = pass4s_sm;
  const TileGeo g = tile_geo<M, C>(p.a, w / n_cols);
  tile_load_async4<M, C>(sm, col_src(p, w % n_cols), g, p.src_mask);
  cp_async_commit();
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  if (!FWD) {
    if (C == 0) {
      round_sm<false, M, C, 0>(sm, g, p.tw, 0);
      round_sync(C == 0 && warp_local_word<(C == 0 ? M : 13)>());
    }
#pragma unroll
    for (int r = 0; r < S4::NR; r++) {
      chunk_round<false, M, C, S0>(r, sm, g, p.tw, r == S4::NR - 1 ? p.scale : 0u);
      round_sync(warp_local_next<M, C, S0>(r));
    }
  } else {
#pragma unroll
    for (int r = S4::NR - 1; r >= 0; r--) {
      chunk_round<true, M, C, S0>(r, sm, g, p.tw, 0u);
      round_sync(r > 0 ? warp_local_next<M, C, S0>(r - 1) : (C == 0 && warp_local_word<(C == 0 ? M : 13)>()));
    }
    if (C == 0) {
      round_sm<true, M, C, 0>(sm, g, p.tw, 0);
      __syncthreads();
    }
  }
  tile_store4<M, C>(sm, col_dst(p, w % n_cols), g);
}

// Launch tables: single / lower passes use C = 0 (T = M, 5 <= M <= 13); upper
// passes use T = 13 (C = 13 - M, 1 <= M <= 11).
using PassFn = void (*)(NttPass, uint32_t, uint32_t);
using TopFn = void (*)(NttPass, NttPass, uint32_t);
template <bool FWD, int M> PassFn pass_lo() { return ntt_pass_kernel<FWD, M, 0>; }
template <bool FWD, int M> PassFn pass_hi() { return ntt_pass_kernel<FWD, M, 13 - M>; }
template <bool FWD, int M> PassFn pass4_lo() { return ntt_pass4_kernel<FWD, M, 0>; }
template <bool FWD, int M> PassFn pass4_hi() { return ntt_pass4_kernel<FWD, M, 13 - M>; }
template <int M> TopFn top_lo() { return ntt_lde_top_kernel<M, 0>; }
template <int M> TopFn top_hi() { return ntt_lde_top4_kernel<M, 13 - M>; }
// The LDE top pass over M = 11 layers (tiles of 16-byte rows, traces of 2^24) runs
// as CTA pairs, which store whole 32-byte sectors. Measured on 34 x 2^24: LDE 16.31
// ms with single CTAs, 15.24 with pairs, 15.87 with clusters of 4 and 17.4 with 8
// (whole 128-byte lines, but every block waits for 8 CTAs). Rows of 32 and 64 bytes
// (M = 10, 9) are whole sectors already: pairs there measured slower (2^23: 7.23 ->
// 7.34 ms, 2^22: 3.32 -> 3.56 ms).
constexpr int kTopPair = 2;
TopFn top_hi_pair() { return ntt_lde_top4_kernel<11, 2, kTopPair>; }
template <int M> TopFn top5_hi() { return ntt_lde_top_kernel<M, 13 - M>; }

static PassFn pass_fn(bool fwd, uint32_t M, uint32_t C) {
#define VS_LO(m) case m: return fwd ? pass_lo<true, m>() : pass_lo<false, m>();
#define VS_HI(m) case m: return fwd ? pass_hi<true, m>() : pass_hi<false, m>();
  if (C == 0) {
    switch (M) { VS_LO(5) VS_LO(6) VS_LO(7) VS_LO(8) VS_LO(9) VS_LO(10) VS_LO(11) VS_LO(12) VS_LO(13) default: break; }
  } else if (M + C == 13) {
    switch (M) { VS_HI(1) VS_HI(2) VS_HI(3) VS_HI(4) VS_HI(5) VS_HI(6) VS_HI(7) VS_HI(8) VS_HI(9) VS_HI(10) VS_HI(11) default: break; }
  }
#undef VS_LO
#undef VS_HI
  return nullptr;
}
// Chunk-round passes: C = 0 with more than five layers, or upper tiles.
static PassFn pass4_fn(bool fwd, uint32_t M, uint32_t C) {
#define VS_LO(m) case m: return fwd ? pass4_lo<true, m>() : pass4_lo<false, m>();
#define VS_HI(m) case m: return fwd ? pass4_hi<true, m>() : pass4_hi<false, m>();
  if (C == 0) {
    switch (M) { VS_LO(6) VS_LO(7) VS_LO(8) VS_LO(9) VS_LO(10) VS_LO(11) VS_LO(12) VS_LO(13) default: break; }
  } else if (M + C == 13 && C >= 2) {
    switch (M) { VS_HI(1) VS_HI(2) VS_HI(3) VS_HI(4) VS_HI(5) VS_HI(6) VS_HI(7) VS_HI(8) VS_HI(9) VS_HI(10) VS_HI(11) default: break; }
  }
#undef VS_LO
#undef VS_HI
  return nullptr;
}
static TopFn top_fn(uint32_t M, uint32_t C, uint32_t radix) {
#define VS_LO(m) case m: return top_lo<m>();
#define VS_HI(m) case m: return radix == 5 ? top5_hi<m>() : top_hi<m>();
  if (C == 0) {
    switch (M) { VS_LO(5) VS_LO(6) VS_LO(7) VS_LO(8) VS_LO(9) VS_LO(10) VS_LO(11) VS_LO(12) VS_LO(13) default: break; }
  } else if (M + C == 13) {
    switch (M) { VS_HI(1) VS_HI(2) VS_HI(3) VS_HI(4) VS_HI(5) VS_HI(6) VS_HI(7) VS_HI(8) VS_HI(9) VS_HI(10) VS_HI(11) default: break; }
  }
#undef VS_LO
#undef VS_HI
  return nullptr;
}

// Twiddle of layer j, group h (scalar path for single layers and tiny transforms).
__device__ __forceinline__ uint32_t twiddle(const NttTw& tw, uint32_t j, uint32_t h) {
  if (j == 0 && tw.stwo) {
    uint32_t x = __ldg(tw.flat + 2 * (h >> 2)), y = __ldg(tw.flat + 2 * (h >> 2) + 1);
    switch (h & 3) {
      case 0: return y;
      case 1: return neg(y);
      case 2: return neg(x);
      default: return x;
    }
  }
  return __ldg(tw.layer[j] + h);
}

// Single layer (cuda_circle_ntt_layer, and transforms below 32 points).
template <bool FWD>
__global__ void ntt_layer_kernel(uint32_t* __restrict__ d, NttTw tw, uint32_t j, uint32_t half_n) {
  uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= half_n) return;
  uint32_t h = tid >> j, l = tid & ((1u << j) - 1);
  uint32_t i0 = (h << (j + 1)) + l, i1 = i0 + (1u << j);
  uint32_t v0 = d[i0], v1 = d[i1];
  bfly<FWD>(v0, v1, twiddle(tw, j, h) << 1);
  d[i0] = v0;
  d[i1] = v1;
}
__global__ void scale_kernel(uint32_t* __restrict__ d, uint32_t s, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = mul(d[i], s);
}

// ------------------------------------------------------------------ host side
static const uint32_t kMaxT = 13;  // tile of 8192 words (32 KiB), 256 threads
static const uint32_t kMinC = 2;   // >= 16-byte contiguous runs per tile row

// Per-size plans (process wide). Sizes 14..24 may move layers between the lower
// pass and the single upper pass: lower in [max(5, L - 11), 13] keeps the upper
// pass at most 11 layers on a 13-bit tile.
static std::mutex g_plan_mu;
static NttPlan g_plan[32];

static bool lower_valid(uint32_t L, uint32_t lower) {
  if (lower == 0) return true;
  if (L <= kMaxT || L > 2 * kMaxT - kMinC) return false;
  return lower >= std::max<uint32_t>(5, L - (kMaxT - kMinC)) && lower <= kMaxT;
}
bool ntt_plan_valid(uint32_t L, const NttPlan& p) {
  return L < 32 && lower_valid(L, p.lower) && p.items <= 64 && (p.radix == 0 || p.radix == 3 || p.radix == 5);
}
NttPlan ntt_plan(uint32_t L) {
  NttPlan p{};
  if (L < 32) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    p = g_plan[L];
  }
  // items stays 0 for the default: one tile per CTA in 13-layer lower passes (the
  // single-buffered kernel), 8 elsewhere
  if (!p.radix) p.radix = 3;
  return p;
}
static void set_plan(uint32_t L, const NttPlan& p) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  g_plan[L] = p;
}
std::vector<NttPlan> ntt_plan_candidates(uint32_t L) {
  std::vector<NttPlan> v;
  std::vector<uint32_t> lowers{0};
  if (L > kMaxT && L <= 2 * kMaxT - kMinC) {
    lowers.clear();
    // lower passes of at least 10 layers (CTAs of 32+ threads); smaller ones are valid but never faster
    for (uint32_t lo = std::max<uint32_t>(10, L - (kMaxT - kMinC)); lo <= kMaxT; lo++) lowers.push_back(lo);
  }
  const bool upper_tile = L > kMaxT;  // the LDE top pass runs on C >= 2 tiles only above 13 layers
  const std::vector<uint32_t> radices = upper_tile ? std::vector<uint32_t>{3u, 5u} : std::vector<uint32_t>{0u};
  for (uint32_t lo : lowers)
    for (uint32_t items : {1u, 4u, 8u, 16u})
      for (uint32_t radix : radices) v.push_back({lo == kMaxT ? 0u : lo, items, radix});
  return v;
}

std::vector<PassRange> plan_passes(uint32_t L, uint32_t lower) {
  std::vector<PassRange> v;
  if (L <= kMaxT) { v.push_back({0, L - 1, 0}); return v; }
  uint32_t lo = lower_valid(L, lower) && lower ? lower : kMaxT;
  v.push_back({0, lo - 1, 0});
  uint32_t rem = L - lo, max_u = kMaxT - kMinC;
  uint32_t k = (rem + max_u - 1) / max_u;
  uint32_t a = lo;
  for (uint32_t i = 0; i < k; i++) {
    uint32_t u = rem / k + (i < rem % k ? 1 : 0);
    uint32_t c = kMaxT - u;
    if (c > a) c = a;
    v.push_back({a, a + u - 1, c});
    a += u;
  }
  return v;
}

uint32_t inv_n_scale(uint32_t log_n) {
  uint32_t e = (30u * log_n) % 31u;
  return e == 0 ? 1u : (1u << e);
}

// Opts a kernel into more than 48 KiB of dynamic shared memory, once per
// function (so repeated and graph-captured launches make no attribute calls).
static int allow_smem(const void* fn, uint32_t bytes) {
  static std::mutex mu;
  static std::map<const void*, uint32_t> done;
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find(fn);
  if (it != done.end() && it->second >= bytes) return VS_OK;
  VS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  done[fn] = bytes;
  return VS_OK;
}

// Grid of a persistent kernel: SMs x resident CTAs per SM (queried once per
// device and function; the first query happens outside any stream capture).
static uint32_t persistent_grid(const void* fn, uint32_t threads, uint32_t smem) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, uint32_t> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find({dev, fn});
  if (it != cache.end()) return it->second;
  int sms = 0, per = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, (int)threads, smem) != cudaSuccess || per <= 0) per = 1;
  const uint32_t g = (uint32_t)(sms * per);
  cache[{dev, fn}] = g;
  return g;
}

static int launch_pass(NttPass p, bool fwd, uint32_t n_cols, cudaStream_t st) {
  const uint32_t M = p.b - p.a + 1, T = M + p.c;
  if (p.radix != 5 && p.c == 0 && M == kMaxT && p.items <= 1) {  // one tile per CTA: single-buffered kernel
    PassFn f = fwd ? ntt_pass4s_kernel<true, kMaxT, 0> : ntt_pass4s_kernel<false, kMaxT, 0>;
    const uint64_t tot = (uint64_t)n_cols << (p.log_n - T);
    if (tot > 0xFFFFFFFFull) return set_error(VS_ERR_INVALID, "ntt: %llu tiles", (unsigned long long)tot);
    VS_TRY(allow_smem((const void*)f, 4u << T));
    f<<<(uint32_t)tot, 1u << (T - 5), 4u << T, st>>>(p, n_cols, (uint32_t)tot);
    VS_LAUNCHED("ntt_pass_kernel");
    return VS_OK;
  }
  PassFn fn = p.radix == 5 ? nullptr : pass4_fn(fwd, M, p.c);
  if (!fn) fn = pass_fn(fwd, M, p.c);
  if (!fn) return set_error(VS_ERR_INVALID, "ntt: no kernel for pass shape M=%u C=%u", M, p.c);
  const uint32_t tile_bits = p.log_n - T;
  const uint64_t total = (uint64_t)n_cols << tile_bits;
  if (total > 0xFFFFFFFFull) return set_error(VS_ERR_INVALID, "ntt: %llu tiles", (unsigned long long)total);
  const uint32_t smem = 8u << T;  // two tiles
  VS_TRY(allow_smem((const void*)fn, smem));
  // At most kItemsPerCta tiles per CTA: the prefetch pipeline still hides the
  // loads, and CTAs retire every few tens of microseconds, so kernels of
  // higher-priority streams (small jobs beside a large one) get SMs promptly
  // instead of waiting for a whole-GPU persistent kernel to end.
  const uint64_t kItemsPerCta = p.items ? p.items : 8;
  const uint32_t threads = 1u << (T - 5);
  const uint64_t resident = persistent_grid((const void*)fn, threads, smem);
  const uint32_t grid = (uint32_t)std::min<uint64_t>(total, std::max(resident, (total + kItemsPerCta - 1) / kItemsPerCta));
  fn<<<grid, threads, smem, st>>>(p, n_cols, (uint32_t)total);
  VS_LAUNCHED("ntt_pass_kernel");
  return VS_OK;
}

// Small transforms (< 32 points): one launch per layer.
static int small_transform(uint32_t* d, uint32_t L, const NttTw& tw, bool fwd, uint32_t scale, cudaStream_t st) {
  const uint32_t half = 1u << (L - 1);
  if (fwd) {
    for (int j = (int)L - 1; j >= 0; j--) ntt_layer_kernel<true><<<1, 32, 0, st>>>(d, tw, (uint32_t)j, half);
  } else {
    for (uint32_t j = 0; j < L; j++) ntt_layer_kernel<false><<<1, 32, 0, st>>>(d, tw, j, half);
    if (scale) scale_kernel<<<1, 32, 0, st>>>(d, scale, 2 * half);
  }
  VS_LAUNCHED("ntt small transform");
  return VS_OK;
}

// ------------------------------------------------------------------ alignment
// The pass and LDE kernels move 16-byte chunks (cp.async, 128-bit loads and
// stores) and read twiddles with 64/128-bit loads. Entry points accept any
// 4-byte-aligned device pointer, as the reference's word-by-word kernels do, so
// the host side checks column starts, strides and twiddle tables first and, when
// one is not aligned, runs the transform on aligned copies (stream-ordered
// temporaries) instead. The kernels themselves never see an unaligned address.
namespace {
bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Stream-ordered temporaries released on the stream when the scope ends.
struct StreamScratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit StreamScratch(cudaStream_t s) : st(s) {}
  ~StreamScratch() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
  int alloc(uint32_t** out, uint64_t words) {
    VS_CUDA(cudaMallocAsync((void**)out, std::max<uint64_t>(words, 4) * 4, st));
    ptrs.push_back(*out);
    return VS_OK;
  }
};

// Twiddles the kernels can read with vector loads: tw itself when its tables
// are aligned, else copies of the read part of every layer at aligned offsets.
int aligned_twiddles(const NttTw& tw, uint32_t L, cudaStream_t st, StreamScratch& tmp, NttTw* out) {
  if (tw.vec) { *out = tw; return VS_OK; }
  if (tw.stwo) {
    uint32_t* f = nullptr;
    const uint64_t words = 1ull << (L - 1);  // the flat table: pairs of the circle layer and all line layers
    VS_TRY(tmp.alloc(&f, words));
    VS_CUDA(cudaMemcpyAsync(f, tw.flat, words * 4, cudaMemcpyDeviceToDevice, st));
    *out = stwo_tw(f, L);
  } else {
    uint64_t off[32] = {0}, total = 0;
    for (uint32_t j = 0; j < L && j < 32; j++) {
      off[j] = total;
      total += ((1ull << (L - 1 - j)) + 3) & ~3ull;  // layer j reads 2^(L-1-j) twiddles
    }
    uint32_t* base = nullptr;
    VS_TRY(tmp.alloc(&base, total));
    NttTw t{};
    t.stwo = 0;
    for (uint32_t j = 0; j < L && j < 32; j++) {
      VS_CUDA(cudaMemcpyAsync(base + off[j], tw.layer[j], (1ull << (L - 1 - j)) * 4, cudaMemcpyDeviceToDevice, st));
      t.layer[j] = base + off[j];
    }
    ntt_tw_check_alignment(t, L);
    *out = t;
  }
  if (!out->vec) return set_error(VS_ERR_INVALID, "ntt: twiddle staging left a table unaligned");
  return VS_OK;
}

// Host copies of the column pointers and whether every column start (and stride)
// is 16-byte aligned. Pointer arrays are read back from the device (the batched
// entry points that pass them synchronise anyway).
int column_pointers(const NttColumns& io, std::vector<const uint32_t*>& src, std::vector<uint32_t*>& dst, bool* ok) {
  src.resize(io.n_cols);
  dst.resize(io.n_cols);
  if (io.src_cols) VS_CUDA(cudaMemcpy(src.data(), io.src_cols, io.n_cols * sizeof(void*), cudaMemcpyDeviceToHost));
  else for (uint32_t c = 0; c < io.n_cols; c++) src[c] = io.src + c * io.src_stride;
  if (io.dst_cols) VS_CUDA(cudaMemcpy(dst.data(), io.dst_cols, io.n_cols * sizeof(void*), cudaMemcpyDeviceToHost));
  else for (uint32_t c = 0; c < io.n_cols; c++) dst[c] = io.dst + c * io.dst_stride;
  *ok = true;
  for (uint32_t c = 0; c < io.n_cols; c++) *ok = *ok && al16(src[c]) && al16(dst[c]);
  return VS_OK;
}
bool strided_aligned(const NttColumns& io) {
  if (io.src_cols || io.dst_cols) return false;  // decided from the pointer values
  const bool multi = io.n_cols > 1;
  return al16(io.src) && al16(io.dst) && (!multi || (io.src_stride % 4 == 0 && io.dst_stride % 4 == 0));
}
}  // namespace

static int ntt_transform_aligned(const NttColumns& io, uint32_t L, const NttTw& tw, bool fwd, cudaStream_t st);

int ntt_transform(const NttColumns& io, uint32_t L, const NttTw& tw, bool fwd, cudaStream_t st) {
  if (L == 0) return VS_OK;
  if (L < 5) return ntt_transform_aligned(io, L, tw, fwd, st);  // word-by-word kernels
  StreamScratch tmp(st);
  NttTw t;
  VS_TRY(aligned_twiddles(tw, L, st, tmp, &t));
  if (strided_aligned(io)) return ntt_transform_aligned(io, L, t, fwd, st);
  std::vector<const uint32_t*> src;
  std::vector<uint32_t*> dst;
  bool ok = false;
  VS_TRY(column_pointers(io, src, dst, &ok));
  if (ok) return ntt_transform_aligned(io, L, t, fwd, st);
  const uint64_t n = 1ull << L;
  uint32_t* T = nullptr;
  VS_TRY(tmp.alloc(&T, n * io.n_cols));
  for (uint32_t c = 0; c < io.n_cols; c++)
    VS_CUDA(cudaMemcpyAsync(T + c * n, src[c], n * 4, cudaMemcpyDeviceToDevice, st));
  NttColumns tio{T, T, nullptr, nullptr, n, n, io.n_cols};
  VS_TRY(ntt_transform_aligned(tio, L, t, fwd, st));
  for (uint32_t c = 0; c < io.n_cols; c++)
    VS_CUDA(cudaMemcpyAsync(dst[c], T + c * n, n * 4, cudaMemcpyDeviceToDevice, st));
  return VS_OK;
}

static int ntt_transform_aligned(const NttColumns& io, uint32_t L, const NttTw& tw, bool fwd, cudaStream_t st) {
  if (L == 0) return VS_OK;
  if (L < 5) {
    for (uint32_t c = 0; c < io.n_cols; c++) {
      if (io.src_cols || io.dst_cols) return set_error(VS_ERR_INVALID, "small NTT with pointer arrays unsupported");
      uint32_t* d = io.dst + c * io.dst_stride;
      if (io.src != d) VS_CUDA(cudaMemcpyAsync(d, io.src + c * io.src_stride, 4u << L, cudaMemcpyDeviceToDevice, st));
      VS_TRY(small_transform(d, L, tw, fwd, fwd ? 0 : inv_n_scale(L), st));
    }
    return VS_OK;
  }
  const NttPlan plan = ntt_plan(L);
  auto passes = plan_passes(L, plan.lower);
  const size_t np = passes.size();
  for (size_t i = 0; i < np; i++) {
    const PassRange& r = fwd ? passes[np - 1 - i] : passes[i];
    NttPass p{};
    p.tw = tw;
    p.items = plan.items;
    p.radix = plan.radix;
    p.log_n = L;
    p.a = r.a;
    p.b = r.b;
    p.c = r.c;
    p.src_mask = 0xFFFFFFFFu;
    bool first = i == 0;
    p.src = first ? io.src : io.dst;
    p.src_cols = first ? io.src_cols : io.dst_cols;
    p.src_stride = first ? io.src_stride : io.dst_stride;
    p.dst = io.dst;
    p.dst_cols = io.dst_cols;
    p.dst_stride = io.dst_stride;
    p.scale = (!fwd && i == np - 1) ? inv_n_scale(L) : 0;
    VS_TRY(launch_pass(p, fwd, io.n_cols, st));
  }
  return VS_OK;
}

static int ntt_lde_aligned(const NttColumns& io, uint32_t l, uint32_t B, const NttTw& tw_inv, const NttTw& tw_fwd,
                           cudaStream_t st);

int ntt_lde(const NttColumns& io, uint32_t l, uint32_t B, const NttTw& tw_inv, const NttTw& tw_fwd,
            cudaStream_t st) {
  if (l < 5) return set_error(VS_ERR_INVALID, "LDE needs log_n >= 5 (got %u)", l);
  if (io.src_cols || io.dst_cols) return set_error(VS_ERR_INVALID, "LDE takes strided columns");
  StreamScratch tmp(st);
  NttTw ti, tf;
  VS_TRY(aligned_twiddles(tw_inv, l, st, tmp, &ti));
  VS_TRY(aligned_twiddles(tw_fwd, l + B, st, tmp, &tf));
  if (strided_aligned(io)) return ntt_lde_aligned(io, l, B, ti, tf, st);
  const uint64_t n = 1ull << l, N = n << B;
  uint32_t *S = nullptr, *D = nullptr;
  VS_TRY(tmp.alloc(&S, n * io.n_cols));
  VS_TRY(tmp.alloc(&D, N * io.n_cols));
  for (uint32_t c = 0; c < io.n_cols; c++)
    VS_CUDA(cudaMemcpyAsync(S + c * n, io.src + c * io.src_stride, n * 4, cudaMemcpyDeviceToDevice, st));
  NttColumns tio{S, D, nullptr, nullptr, n, N, io.n_cols};
  VS_TRY(ntt_lde_aligned(tio, l, B, ti, tf, st));
  for (uint32_t c = 0; c < io.n_cols; c++)
    VS_CUDA(cudaMemcpyAsync(io.dst + c * io.dst_stride, D + c * N, N * 4, cudaMemcpyDeviceToDevice, st));
  return VS_OK;
}

static int ntt_lde_aligned(const NttColumns& io, uint32_t l, uint32_t B, const NttTw& tw_inv, const NttTw& tw_fwd,
                           cudaStream_t st) {
  const NttPlan plan = ntt_plan(l);
  auto passes = plan_passes(l, plan.lower);
  const size_t np = passes.size();
  // 1. inverse passes below the top one: src -> dst[0, n)
  for (size_t i = 0; i + 1 < np; i++) {
    NttPass p{};
    p.tw = tw_inv;
    p.items = plan.items;
    p.radix = plan.radix;
    p.log_n = l;
    p.a = passes[i].a;
    p.b = passes[i].b;
    p.c = passes[i].c;
    p.src_mask = 0xFFFFFFFFu;
    p.src = i == 0 ? io.src : io.dst;
    p.src_stride = i == 0 ? io.src_stride : io.dst_stride;
    p.dst = io.dst;
    p.dst_stride = io.dst_stride;
    VS_TRY(launch_pass(p, false, io.n_cols, st));
  }
  // 2. fused top pass
  {
    const PassRange& r = passes[np - 1];
    NttPass pi{}, pf{};
    pi.tw = tw_inv;
    pi.log_n = l;
    pi.a = r.a;
    pi.b = r.b;
    pi.c = r.c;
    pi.src_mask = 0xFFFFFFFFu;
    pi.src = np == 1 ? io.src : io.dst;
    pi.src_stride = np == 1 ? io.src_stride : io.dst_stride;
    pi.scale = inv_n_scale(l);
    pf = pi;
    pf.tw = tw_fwd;
    pf.log_n = l + B;
    pf.dst = io.dst;
    pf.dst_stride = io.dst_stride;
    const uint32_t M = r.b - r.a + 1, T = M + r.c;
    TopFn fn = top_fn(M, r.c, plan.radix);
    if (!fn) return set_error(VS_ERR_INVALID, "ntt: no LDE kernel for shape M=%u C=%u", M, r.c);
    const uint32_t smem = 8u << T;  // working tile + coefficient tile
    const dim3 grid(1u << (l - T), io.n_cols), block(1u << (T - 5));
    // 16-byte-row tiles run as CTA pairs (whole-sector tile stores); if the
    // cluster launch is refused, the plain kernel runs instead
    TopFn cfn = nullptr;
    const uint32_t K = kTopPair;
    if (plan.radix != 5 && M == 11 && r.c == 2) cfn = top_hi_pair();
    bool launched = false;
    if (cfn && grid.x % K == 0) {
      VS_TRY(allow_smem((const void*)cfn, smem));
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = grid;
      cfg.blockDim = block;
      cfg.dynamicSmemBytes = smem;
      cfg.stream = st;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = K;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      if (cudaLaunchKernelEx(&cfg, cfn, pi, pf, B) == cudaSuccess) launched = true;
      else cudaGetLastError();  // clear the refused launch's error
    }
    if (!launched) {
      VS_TRY(allow_smem((const void*)fn, smem));
      fn<<<grid, block, smem, st>>>(pi, pf, B);
    }
    VS_LAUNCHED("ntt_lde_top_kernel");
  }
  // 3. forward passes below the top one over the whole evaluation domain
  for (int i = (int)np - 2; i >= 0; i--) {
    NttPass p{};
    p.tw = tw_fwd;
    p.items = plan.items;
    p.radix = plan.radix;
    p.log_n = l + B;
    p.a = passes[i].a;
    p.b = passes[i].b;
    p.c = passes[i].c;
    p.src_mask = 0xFFFFFFFFu;
    p.src = io.dst;
    p.src_stride = io.dst_stride;
    p.dst = io.dst;
    p.dst_stride = io.dst_stride;
    VS_TRY(launch_pass(p, true, io.n_cols, st));
  }
  return VS_OK;
}

void ntt_tw_check_alignment(NttTw& tw, uint32_t L) {
  tw.vec = 1;
  for (uint32_t j = 0; j < L && j < 32; j++) {
    const uint64_t size = 1ull << (L - 1 - j);                 // entries of layer j
    const uint64_t need = 4 * (size >= 4 ? 4 : size);          // bytes of alignment a vector load needs
    const uint32_t* base = (j == 0 && tw.stwo) ? tw.flat : tw.layer[j];
    if (!base || (reinterpret_cast<uintptr_t>(base) % need) != 0) tw.vec = 0;
  }
}

NttTw native_tw(const uint32_t* line, const uint32_t* circle, const uint32_t* offsets, uint32_t n_line_layers) {
  NttTw tw{};
  tw.stwo = 0;
  tw.layer[0] = circle;
  for (uint32_t j = 1; j <= n_line_layers && j < 32; j++) tw.layer[j] = line + offsets[j - 1];
  ntt_tw_check_alignment(tw, n_line_layers + 1);
  return tw;
}
NttTw stwo_tw(const uint32_t* flat, uint32_t L) {
  NttTw tw{};
  tw.stwo = 1;
  tw.flat = flat;
  const uint32_t half = 1u << (L - 1);
  for (uint32_t j = 1; j < L && j < 32; j++) tw.layer[j] = flat + (half - (1u << (L - j)));
  ntt_tw_check_alignment(tw, L);
  return tw;
}

int tw_for(int kind, uint32_t L, bool forward, NttTw* out, cudaStream_t st) {
  const TwiddleSet* t = nullptr;
  VS_TRY(get_twiddles(kind, L, &t, st));
  if (kind == TW_NATIVE) *out = native_tw(forward ? t->line : t->iline, forward ? t->circle : t->icircle,
                                          t->offsets.data(), L - 1);
  else *out = stwo_tw(forward ? t->line : t->iline, L);
  return VS_OK;
}

int lde_cached(int kind, const uint32_t* src, uint64_t src_stride, uint32_t* dst, uint64_t dst_stride,
               uint32_t n_cols, uint32_t l, uint32_t B, cudaStream_t st) {
  if (!src || !dst || n_cols == 0) return set_error(VS_ERR_INVALID, "lde: null argument");
  if (l < 2 || l + B > 30) return set_error(VS_ERR_INVALID, "lde: log_n %u + blowup %u out of range", l, B);
  NttTw ti, tf;
  VS_TRY(tw_for(kind, l, false, &ti, st));
  VS_TRY(tw_for(kind, l + B, true, &tf, st));
  if (l < 5) {  // tiny: interpolate in place in dst, zero the padding, evaluate
    const uint64_t n = 1ull << l, N = n << B;
    for (uint32_t c = 0; c < n_cols; c++) {
      uint32_t* d = dst + c * dst_stride;
      VS_CUDA(cudaMemcpyAsync(d, src + c * src_stride, n * 4, cudaMemcpyDeviceToDevice, st));
      VS_CUDA(cudaMemsetAsync(d + n, 0, (N - n) * 4, st));
      NttColumns a{d, d, nullptr, nullptr, 0, 0, 1};
      VS_TRY(ntt_transform(a, l, ti, false, st));
      VS_TRY(ntt_transform(a, l + B, tf, true, st));
    }
    return VS_OK;
  }
  NttColumns io{src, dst, nullptr, nullptr, src_stride, dst_stride, n_cols};
  return ntt_lde(io, l, B, ti, tf, st);
}

// ------------------------------------------------------------------ bit reversal
__global__ void bit_reverse_m31_kernel(uint32_t* d, uint32_t log_n, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t j = brev(i, log_n);
  if (i < j) {
    uint32_t t = d[i];
    d[i] = d[j];
    d[j] = t;
  }
}
__global__ void bit_reverse_qm31_kernel(const uint4* __restrict__ in, uint4* __restrict__ out, uint32_t n,
                                        uint32_t log_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[brev(i, log_n)] = in[i];
}

// ------------------------------------------------------------------ eval at point (circle_ntt.cu:119-164)
__global__ void fold_first_kernel(const uint32_t* __restrict__ c, uint32_t* __restrict__ out,
                                  const uint32_t* __restrict__ f, uint32_t half_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  qm31 fq{{f[0], f[1], f[2], f[3]}};
  qm31 bf = qscale(fq, c[i + half_n]);
  out[4 * i + 0] = add(c[i], bf.v[0]);
  out[4 * i + 1] = bf.v[1];
  out[4 * i + 2] = bf.v[2];
  out[4 * i + 3] = bf.v[3];
}
__global__ void fold_level_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                  const uint32_t* __restrict__ f, uint32_t half_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  qm31 a{{in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]}};
  uint32_t j = 4 * (i + half_n);
  qm31 b{{in[j], in[j + 1], in[j + 2], in[j + 3]}};
  qm31 fq{{f[0], f[1], f[2], f[3]}};
  qm31 r = qadd(a, qmul(b, fq));
  out[4 * i + 0] = r.v[0];
  out[4 * i + 1] = r.v[1];
  out[4 * i + 2] = r.v[2];
  out[4 * i + 3] = r.v[3];
}

}  // namespace vs

using namespace vs;

extern "C" {

void cuda_circle_ntt_evaluate(uint32_t* d, const uint32_t* tw, const uint32_t* ctw, const uint32_t* h_off,
                              const uint32_t* /*h_sizes*/, uint32_t n_line, uint32_t n) {
  uint32_t L = ilog2(n);
  NttColumns io{d, d, nullptr, nullptr, 0, 0, 1};
  ntt_transform(io, L, native_tw(tw, ctw, h_off, n_line), true, 0);
  check_cuda(cudaDeviceSynchronize(), "cuda_circle_ntt_evaluate");
}
void cuda_circle_ntt_interpolate(uint32_t* d, const uint32_t* itw, const uint32_t* ictw, const uint32_t* h_off,
                                 const uint32_t* /*h_sizes*/, uint32_t n_line, uint32_t n) {
  uint32_t L = ilog2(n);
  NttColumns io{d, d, nullptr, nullptr, 0, 0, 1};
  ntt_transform(io, L, native_tw(itw, ictw, h_off, n_line), false, 0);
  check_cuda(cudaDeviceSynchronize(), "cuda_circle_ntt_interpolate");
}
static void batch_ntt(uint32_t** cols, const uint32_t* tw, const uint32_t* ctw, const uint32_t* h_off, uint32_t n_line,
                      uint32_t n, uint32_t n_cols, bool fwd) {
  if (!n_cols) return;
  uint32_t L = ilog2(n);
  NttTw t = native_tw(tw, ctw, h_off, n_line);
  if (L < 5) {  // tiny: per column through a host copy of the pointer table
    std::vector<uint32_t*> h(n_cols);
    if (check_cuda(cudaMemcpy(h.data(), cols, n_cols * sizeof(void*), cudaMemcpyDeviceToHost), "batch ntt") != VS_OK) return;
    for (uint32_t c = 0; c < n_cols; c++) {
      NttColumns io{h[c], h[c], nullptr, nullptr, 0, 0, 1};
      ntt_transform(io, L, t, fwd, 0);
    }
  } else {
    NttColumns io{nullptr, nullptr, (const uint32_t* const*)cols, cols, 0, 0, n_cols};
    ntt_transform(io, L, t, fwd, 0);
  }
  check_cuda(cudaDeviceSynchronize(), "cuda_circle_ntt_*_batch");
}
void cuda_circle_ntt_evaluate_batch(uint32_t** cols, const uint32_t* tw, const uint32_t* ctw, const uint32_t* h_off,
                                    const uint32_t* /*h_sizes*/, uint32_t n_line, uint32_t n, uint32_t n_cols) {
  batch_ntt(cols, tw, ctw, h_off, n_line, n, n_cols, true);
}
void cuda_circle_ntt_interpolate_batch(uint32_t** cols, const uint32_t* itw, const uint32_t* ictw,
                                       const uint32_t* h_off, const uint32_t* /*h_sizes*/, uint32_t n_line,
                                       uint32_t n, uint32_t n_cols) {
  batch_ntt(cols, itw, ictw, h_off, n_line, n, n_cols, false);
}
void cuda_circle_ntt_layer(uint32_t* d, const uint32_t* tw, uint32_t layer_idx, uint32_t n, int forward) {
  NttTw t{};
  t.layer[layer_idx] = tw;
  uint32_t half = n / 2;
  if (!half) return;
  if (forward) ntt_layer_kernel<true><<<blocks_for(half, 256), 256>>>(d, t, layer_idx, half);
  else ntt_layer_kernel<false><<<blocks_for(half, 256), 256>>>(d, t, layer_idx, half);
  check_cuda(cudaGetLastError(), "cuda_circle_ntt_layer");
}
void cuda_bit_reverse_m31(uint32_t* d, uint32_t log_n) {
  uint32_t n = 1u << log_n;
  bit_reverse_m31_kernel<<<blocks_for(n, 256), 256>>>(d, log_n, n);
  check_cuda(cudaGetLastError(), "cuda_bit_reverse_m31");
}
void cuda_bit_reverse_qm31(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t log_n) {
  if (!n) return;
  bit_reverse_qm31_kernel<<<blocks_for(n, 256), 256>>>((const uint4*)in, (uint4*)out, n, log_n);
  check_cuda(cudaGetLastError(), "cuda_bit_reverse_qm31");
}
void cuda_stwo_ntt_evaluate(uint32_t* d, const uint32_t* tw, uint32_t n) {
  uint32_t L = ilog2(n);
  NttColumns io{d, d, nullptr, nullptr, 0, 0, 1};
  ntt_transform(io, L, stwo_tw(tw, L), true, 0);
  check_cuda(cudaDeviceSynchronize(), "cuda_stwo_ntt_evaluate");
}
void cuda_stwo_ntt_interpolate(uint32_t* d, const uint32_t* itw, uint32_t n) {
  uint32_t L = ilog2(n);
  NttColumns io{d, d, nullptr, nullptr, 0, 0, 1};
  ntt_transform(io, L, stwo_tw(itw, L), false, 0);
  check_cuda(cudaDeviceSynchronize(), "cuda_stwo_ntt_interpolate");
}
void cuda_eval_at_point(const uint32_t* coeffs, const uint32_t* factors, uint32_t* h_result, uint32_t n,
                        uint32_t* s1, uint32_t* s2) {
  uint32_t log_n = ilog2(n);
  uint32_t half = n / 2;
  fold_first_kernel<<<blocks_for(half, 256), 256>>>(coeffs, s1, factors, half);
  uint32_t *in = s1, *out = s2, cur = half;
  for (uint32_t lvl = 1; lvl < log_n; lvl++) {
    half = cur / 2;
    fold_level_kernel<<<blocks_for(half, 256), 256>>>(in, out, factors + 4 * lvl, half);
    uint32_t* t = in;
    in = out;
    out = t;
    cur = half;
  }
  check_cuda(cudaMemcpy(h_result, in, 16, cudaMemcpyDeviceToHost), "cuda_eval_at_point");
}

int vs_lde_stwo(const uint32_t* src, uint64_t src_stride, uint32_t* dst, uint64_t dst_stride, uint32_t n_cols,
                uint32_t log_n, uint32_t blowup, vs_stream_t st) {
  clear_error();
  return lde_cached(TW_STWO, src, src_stride, dst, dst_stride, n_cols, log_n, blowup, (cudaStream_t)st);
}
int vs_lde_native(const uint32_t* src, uint64_t src_stride, uint32_t* dst, uint64_t dst_stride, uint32_t n_cols,
                  uint32_t log_n, uint32_t blowup, vs_stream_t st) {
  clear_error();
  return lde_cached(TW_NATIVE, src, src_stride, dst, dst_stride, n_cols, log_n, blowup, (cudaStream_t)st);
}

// ------------------------------------------------------------------ autotuner
int vs_ntt_plan_set(uint32_t log_n, uint32_t lower, uint32_t items, uint32_t radix) {
  clear_error();
  // canonical form: the default lower pass (13, or the whole transform up to 13 layers) is 0
  const uint32_t lo = (lower == kMaxT || (log_n <= kMaxT && lower == log_n)) ? 0u : lower;
  const uint32_t rx = radix;
  const NttPlan p{lo, items, rx};
  if (!ntt_plan_valid(log_n, p))
    return set_error(VS_ERR_INVALID, "vs_ntt_plan_set: no plan (lower %u, items %u, radix %u) for log_n %u", lower,
                     items, radix, log_n);
  set_plan(log_n, p);
  return VS_OK;
}
int vs_ntt_plan_get(uint32_t log_n, uint32_t* lower, uint32_t* items, uint32_t* radix) {
  clear_error();
  if (log_n >= 32 || !lower || !items || !radix) return set_error(VS_ERR_INVALID, "vs_ntt_plan_get: bad argument");
  const NttPlan p = ntt_plan(log_n);
  *lower = log_n <= kMaxT ? log_n : (p.lower ? p.lower : kMaxT);
  *items = p.items;
  *radix = p.radix;
  return VS_OK;
}
int vs_ntt_plan_candidates(uint32_t log_n, uint32_t* out, uint32_t cap, uint32_t* n_out) {
  clear_error();
  if (log_n >= 32 || !n_out) return set_error(VS_ERR_INVALID, "vs_ntt_plan_candidates: bad argument");
  const auto v = ntt_plan_candidates(log_n);
  *n_out = (uint32_t)v.size();
  for (uint32_t i = 0; i < v.size() && i < cap && out; i++) {
    out[3 * i] = v[i].lower ? v[i].lower : std::min<uint32_t>(log_n, kMaxT);
    out[3 * i + 1] = v[i].items;
    out[3 * i + 2] = v[i].radix ? v[i].radix : 3u;
  }
  return VS_OK;
}

// Times every candidate plan of log_n on an n_cols-column LDE (stwo convention,
// seeded columns, `reps` timed runs after one warm-up each, CUDA events on the
// stream) and keeps the fastest as the plan of log_n.
int vs_autotune_lde(uint32_t log_n, uint32_t n_cols, uint32_t blowup_bits, uint32_t reps, uint32_t* best,
                    float* ms_out, uint32_t cap, vs_stream_t stream) {
  clear_error();
  cudaStream_t st = (cudaStream_t)stream;
  if (log_n < 5 || log_n >= 31 || log_n + blowup_bits > 30 || !n_cols || !best)
    return set_error(VS_ERR_INVALID, "vs_autotune_lde: bad size (log_n %u, blowup %u, cols %u)", log_n, blowup_bits,
                     n_cols);
  if (!reps) reps = 3;
  const uint64_t n = 1ull << log_n, N = n << blowup_bits;
  const auto cands = ntt_plan_candidates(log_n);
  const NttPlan saved = [&] {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    return g_plan[log_n];
  }();
  uint32_t *src = nullptr, *dst = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = check_cuda(cudaMallocAsync((void**)&src, n * n_cols * 4, st), "vs_autotune_lde alloc");
  if (rc == VS_OK) rc = check_cuda(cudaMallocAsync((void**)&dst, N * n_cols * 4, st), "vs_autotune_lde alloc");
  if (rc == VS_OK) rc = vs_fill_uniform_m31(src, n * n_cols, 0x56530007ull, 0, stream);
  if (rc == VS_OK) rc = check_cuda(cudaEventCreate(&e0), "vs_autotune_lde event");
  if (rc == VS_OK) rc = check_cuda(cudaEventCreate(&e1), "vs_autotune_lde event");
  float best_ms = 0.f;
  NttPlan best_plan = saved;
  for (size_t i = 0; i < cands.size() && rc == VS_OK; i++) {
    set_plan(log_n, cands[i]);
    rc = lde_cached(TW_STWO, src, n, dst, N, n_cols, log_n, blowup_bits, st);
    if (rc == VS_OK) rc = check_cuda(cudaEventRecord(e0, st), "vs_autotune_lde event");
    for (uint32_t k = 0; k < reps && rc == VS_OK; k++)
      rc = lde_cached(TW_STWO, src, n, dst, N, n_cols, log_n, blowup_bits, st);
    if (rc == VS_OK) rc = check_cuda(cudaEventRecord(e1, st), "vs_autotune_lde event");
    if (rc == VS_OK) rc = check_cuda(cudaEventSynchronize(e1), "vs_autotune_lde sync");
    float ms = 0.f;
    if (rc == VS_OK) rc = check_cuda(cudaEventElapsedTime(&ms, e0, e1), "vs_autotune_lde time");
    ms /= (float)reps;
    if (ms_out && i < cap) ms_out[i] = ms;
    if (rc == VS_OK && (i == 0 || ms < best_ms)) {
      best_ms = ms;
      best_plan = cands[i];
    }
  }
  set_plan(log_n, rc == VS_OK ? best_plan : saved);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (src) cudaFreeAsync(src, st);
  if (dst) cudaFreeAsync(dst, st);
  if (rc != VS_OK) return rc;
  best[0] = best_plan.lower ? best_plan.lower : std::min<uint32_t>(log_n, kMaxT);
  best[1] = best_plan.items;  // 0: the default
  best[2] = best_plan.radix ? best_plan.radix : 3u;
  return check_cuda(cudaStreamSynchronize(st), "vs_autotune_lde");
}

}  // extern "C"
