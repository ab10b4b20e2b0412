// Kernels behind the reference's stwo Backend adapter (crates/cuda-backend):
// column gathers for lifted-Merkle decommitment, barycentric evaluation at a
// point, lift-and-accumulate of secure columns and the PackLeaves transpose.
// Each entry point keeps the reference symbol's arguments, default-stream launch
// and (where the reference has one) its internal device synchronisation.
//
// Indexing is 64-bit throughout; the reference computes some element offsets in
// 32 bits (gather.cu:32, barycentric_eval.cu:43, accumulate_lift.cu:29), so the
// two agree on every size where those offsets fit in 32 bits.
#include "host_math.h"
#include "twiddles.h"
#include "vs_common.cuh"
#include "vs_field.cuh"
#include "vs_mem.cuh"

namespace vs {
namespace {

constexpr unsigned kThreads = 256;

inline bool host_aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Enough CTAs to fill every SM several times over; the loops are grid-strided.
inline unsigned stride_grid(uint64_t work, unsigned threads) {
  uint64_t b = (work + threads - 1) / threads;
  uint64_t cap = (uint64_t)sm_count() * 16;
  return (unsigned)(b < cap ? (b ? b : 1) : cap);
}

// dst[i] = src[idx[i]]   (gather.cu:10-18)
__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx,
                                  uint32_t* __restrict__ dst, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = __ldg(src + __ldg(idx + i));
}

// dst[8i..8i+8) = src[8 idx[i] .. 8 idx[i] + 8)   (gather.cu:22-40)
// VEC: both arrays 16-byte aligned (checked on the host); two lanes move one
// 32-byte hash as two 128-bit accesses. Otherwise eight lanes move one word each.
template <bool VEC>
__global__ void gather_u256_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx,
                                   uint32_t* __restrict__ dst, uint64_t n) {
  constexpr uint32_t kLanes = VEC ? 2 : 8;
  uint64_t total = n * kLanes;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = t / kLanes;
    uint32_t part = (uint32_t)(t % kLanes);
    uint64_t s = (uint64_t)__ldg(idx + i) * 8;
    if (VEC) {
      uint4 v = __ldg(reinterpret_cast<const uint4*>(src + s) + part);
      reinterpret_cast<uint4*>(dst + i * 8)[part] = v;
    } else {
      dst[i * 8 + part] = __ldg(src + s + part);
    }
  }
}

__device__ __forceinline__ uint64_t fold31(uint64_t a) { return (a & VS_P) + (a >> 31); }
__device__ __forceinline__ uint32_t reduce64(uint64_t a) { return canon((uint32_t)fold31(fold31(a))); }

// Partial sums of sum_i evals[i] * weights[i] (M31 x QM31, weights AoS).
// Block b owns the 256-element chunks c with c mod gridDim.x == b, which is the
// reference's grid-stride partition with 256 threads per block
// (barycentric_eval.cu:30-46), so out[4b..4b+4) is the reference's partial sum
// for block b. Four chunks are loaded before any is accumulated; four products
// (each < 2^62) are summed in 64 bits before one reduction.
template <bool VEC>
__global__ void __launch_bounds__(kThreads) barycentric_kernel(const uint32_t* __restrict__ evals,
                                                               const uint32_t* __restrict__ w, uint64_t n,
                                                               uint32_t* __restrict__ out) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  uint32_t acc[4] = {0, 0, 0, 0};
  uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  for (; i + 3 * step < n; i += 4 * step) {
    uint32_t e[4];
    uint4 q[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint64_t j = i + k * step;
      e[k] = __ldg(evals + j);
      if (VEC) {
        q[k] = __ldg(reinterpret_cast<const uint4*>(w) + j);
      } else {
        q[k] = make_uint4(__ldg(w + 4 * j), __ldg(w + 4 * j + 1), __ldg(w + 4 * j + 2), __ldg(w + 4 * j + 3));
      }
    }
    uint64_t s[4] = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      s[0] += (uint64_t)q[k].x * e[k];
      s[1] += (uint64_t)q[k].y * e[k];
      s[2] += (uint64_t)q[k].z * e[k];
      s[3] += (uint64_t)q[k].w * e[k];
    }
#pragma unroll
    for (int l = 0; l < 4; l++) acc[l] = add(acc[l], reduce64(s[l]));
  }
  for (; i < n; i += step) {
    uint32_t e = __ldg(evals + i);
#pragma unroll
    for (int l = 0; l < 4; l++) acc[l] = add(acc[l], mul(__ldg(w + 4 * i + l), e));
  }
#pragma unroll
  for (int l = 0; l < 4; l++)
#pragma unroll
    for (int m = 16; m; m >>= 1) acc[l] = add(acc[l], __shfl_xor_sync(0xffffffffu, acc[l], m));
  __shared__ uint32_t part[kThreads / 32][4];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int l = 0; l < 4; l++) part[warp][l] = acc[l];
  __syncthreads();
  if (threadIdx.x < 4) {
    uint32_t s = 0;
#pragma unroll
    for (uint32_t k = 0; k < kThreads / 32; k++) s = add(s, part[k][threadIdx.x]);
    out[4 * (uint64_t)blockIdx.x + threadIdx.x] = s;
  }
}

// col[i] += curr[((i >> (log_ratio + 1)) << 1) | (i & 1)], QM31 AoS, in place
// (accumulate_lift.cu:16-37). VEC: both arrays 16-byte aligned (host-checked).
template <bool VEC>
__global__ void accumulate_lift_kernel(uint32_t* __restrict__ col, const uint32_t* __restrict__ curr, uint64_t col_n,
                                       uint32_t shift) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < col_n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t s = ((i >> shift) << 1) | (i & 1);
    if (VEC) {
      uint4 a = reinterpret_cast<const uint4*>(col)[i];
      uint4 b = __ldg(reinterpret_cast<const uint4*>(curr) + s);
      reinterpret_cast<uint4*>(col)[i] = make_uint4(add(a.x, b.x), add(a.y, b.y), add(a.z, b.z), add(a.w, b.w));
    } else {
#pragma unroll
      for (int l = 0; l < 4; l++) col[4 * i + l] = add(col[4 * i + l], __ldg(curr + 4 * s + l));
    }
  }
}

// out[16c + p][g] = in[c][16g + p] for c < 4, p < 16   (pack_leaves.cu:22-38).
// One thread per (c, g): it reads its 16 consecutive input words as four 128-bit
// loads (word loads where a column is not 16-byte aligned) and writes one word to
// each of 16 output columns, so a warp's stores to each column are contiguous.
// When n is not a multiple of 16 the last group writes its n mod 16 words only,
// as the reference's one-thread-per-input-word grid does.
__global__ void pack_leaves_kernel(const uint32_t* const* __restrict__ in_ptrs, uint32_t* const* __restrict__ out_ptrs,
                                   uint64_t n) {
  __shared__ const uint32_t* in_s[4];
  __shared__ uint32_t* out_s[64];
  if (threadIdx.x < 4) in_s[threadIdx.x] = in_ptrs[threadIdx.x];
  if (threadIdx.x < 64) out_s[threadIdx.x] = out_ptrs[threadIdx.x];
  __syncthreads();
  const uint64_t groups = (n + 15) / 16;
  const uint32_t c = blockIdx.y;
  const uint32_t* src = in_s[c];
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < groups; g += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t* p = src + 16 * g;
    if (16 * g + 16 <= n) {
      uint32_t v[16];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        uint4 q = ld4_ro(p + 4 * k);
        v[4 * k] = q.x;
        v[4 * k + 1] = q.y;
        v[4 * k + 2] = q.z;
        v[4 * k + 3] = q.w;
      }
#pragma unroll
      for (int k = 0; k < 16; k++) out_s[16 * c + k][g] = v[k];
    } else {
      uint32_t rem = (uint32_t)(n - 16 * g);
      for (uint32_t k = 0; k < rem; k++) out_s[16 * c + k][g] = __ldg(p + k);
    }
  }
}

// ---- domain helpers the adapter computes on the host per call (fri_ops.rs:50-56,
// 100-106; quotient_ops.rs:135-140), built on the device instead.
// step^(2^b) for b < 31, so step^e costs popcount(e) circle multiplications.
struct PowTable {
  cpt p[31];
};
PowTable pow_table(h::Pt step) {
  PowTable t;
  for (int b = 0; b < 31; b++) {
    t.p[b] = cpt{step.x, step.y};
    step = h::pmul(step, step);
  }
  return t;
}
__device__ __forceinline__ cpt pow_bits(const PowTable& t, uint32_t e) {
  cpt r{1, 0};
  for (int b = 0; e; b++, e >>= 1)
    if (e & 1) r = cpmul(r, t.p[b]);
  return r;
}

// out[i] = coord(initial * step^brev_L(2i)), i < 2^(L-1): x for line domains, y for
// the half coset of a circle domain (the domains' own at(), stwo CircleDomain::at
// and LineDomain::at, whose bit-reversed even indices all lie in the first half).
__global__ void fold_points_kernel(cpt initial, PowTable t, uint32_t L, int extract_y, uint32_t* __restrict__ out) {
  const uint32_t half = 1u << (L - 1);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < half; i += gridDim.x * blockDim.x) {
    const cpt p = cpmul(initial, pow_bits(t, brev(i << 1, L)));
    out[i] = extract_y ? p.y : p.x;
  }
}

// Row r of CanonicCoset(L)'s circle domain in bit-reversed order: j = brev_L(r);
// half_odds(L-1).at(j) for j < 2^(L-1), its conjugate at j - 2^(L-1) otherwise
// (stwo CircleDomain::at over the canonic half coset).
__global__ void canonic_domain_points_kernel(cpt initial, PowTable t, uint32_t L, uint32_t* __restrict__ xs,
                                             uint32_t* __restrict__ ys) {
  const uint32_t n = 1u << L, half = n >> 1;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const uint32_t j = brev(r, L);
    const cpt p = cpmul(initial, pow_bits(t, j & (half - 1)));
    xs[r] = p.x;
    ys[r] = j >= half ? neg(p.y) : p.y;
  }
}

}  // namespace
}  // namespace vs

using namespace vs;

extern "C" {

void cuda_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint32_t n) {
  if (!n) return;
  gather_u32_kernel<<<stride_grid(n, kThreads), kThreads>>>(src, idx, dst, n);
  check_cuda(cudaGetLastError(), "cuda_gather_u32");
}

void cuda_gather_u256(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint32_t n) {
  if (!n) return;
  if (host_aligned16(src) && host_aligned16(dst))
    gather_u256_kernel<true><<<stride_grid(2ull * n, kThreads), kThreads>>>(src, idx, dst, n);
  else
    gather_u256_kernel<false><<<stride_grid(8ull * n, kThreads), kThreads>>>(src, idx, dst, n);
  check_cuda(cudaGetLastError(), "cuda_gather_u256");
}

void cuda_barycentric_eval(const uint32_t* evals, const uint32_t* weights, uint32_t n, uint32_t* out,
                           uint32_t n_blocks) {
  if (!n_blocks) return;
  if (host_aligned16(weights))
    barycentric_kernel<true><<<n_blocks, kThreads>>>(evals, weights, n, out);
  else
    barycentric_kernel<false><<<n_blocks, kThreads>>>(evals, weights, n, out);
  check_cuda(cudaGetLastError(), "cuda_barycentric_eval");
  check_cuda(cudaDeviceSynchronize(), "cuda_barycentric_eval");
}

void cuda_accumulate_lift(uint32_t* col, const uint32_t* curr, uint32_t col_n, uint32_t log_ratio) {
  if (!col_n) return;
  uint32_t shift = log_ratio + 1;
  if (shift >= 64) shift = 63;  // i >> shift is 0 for every i < 2^32 either way
  if (host_aligned16(col) && host_aligned16(curr))
    accumulate_lift_kernel<true><<<stride_grid(col_n, kThreads), kThreads>>>(col, curr, col_n, shift);
  else
    accumulate_lift_kernel<false><<<stride_grid(col_n, kThreads), kThreads>>>(col, curr, col_n, shift);
  check_cuda(cudaGetLastError(), "cuda_accumulate_lift");
}

void cuda_pack_leaves(const uint32_t* const* input_col_ptrs, uint32_t* const* output_col_ptrs, uint32_t n) {
  if (!n) return;
  uint64_t groups = (n + 15ull) / 16;
  unsigned gx = stride_grid(groups, kThreads);
  unsigned cap = (unsigned)sm_count() * 4;
  if (gx > cap) gx = cap;
  pack_leaves_kernel<<<dim3(gx, 4), kThreads>>>(input_col_ptrs, output_col_ptrs, n);
  check_cuda(cudaGetLastError(), "cuda_pack_leaves");
}


// FRI fold twiddles of a stwo domain (fri_ops.rs:50-56 circle, :100-106 line),
// one launch plus the chunked batch inverse, stream-ordered.
int vs_fold_twiddles_stwo(uint32_t is_line, uint32_t init_x, uint32_t init_y, uint32_t step_x, uint32_t step_y,
                          uint32_t log_size, uint32_t* d_out, vs_stream_t stream) {
  clear_error();
  if (!d_out) return set_error(VS_ERR_INVALID, "vs_fold_twiddles_stwo: null output");
  if (log_size < 1 || log_size > 31) return set_error(VS_ERR_INVALID, "vs_fold_twiddles_stwo: log_size %u", log_size);
  if (init_x >= VS_P || init_y >= VS_P || step_x >= VS_P || step_y >= VS_P)
    return set_error(VS_ERR_INVALID, "vs_fold_twiddles_stwo: coordinates must be canonical M31");
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t half = 1u << (log_size - 1);
  fold_points_kernel<<<stride_grid(half, kThreads), kThreads, 0, st>>>(cpt{init_x, init_y},
                                                                      pow_table(h::Pt{step_x, step_y}), log_size,
                                                                      is_line ? 0 : 1, d_out);
  VS_LAUNCHED("fold_points_kernel");
  return launch_batch_inverse(d_out, d_out, half, st);
}

// BRT-canonic domain points of CanonicCoset(log_size) (quotient_ops.rs:135-140).
int vs_canonic_domain_points(uint32_t log_size, uint32_t* d_xs, uint32_t* d_ys, vs_stream_t stream) {
  clear_error();
  if (!d_xs || !d_ys) return set_error(VS_ERR_INVALID, "vs_canonic_domain_points: null output");
  if (log_size < 1 || log_size > 30) return set_error(VS_ERR_INVALID, "vs_canonic_domain_points: log_size %u", log_size);
  const h::Coset ho = h::half_odds(log_size - 1);
  canonic_domain_points_kernel<<<stride_grid(1ull << log_size, kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      cpt{ho.initial.x, ho.initial.y}, pow_table(ho.step), log_size, d_xs, d_ys);
  VS_LAUNCHED("canonic_domain_points_kernel");
  return VS_OK;
}

}  // extern "C"
