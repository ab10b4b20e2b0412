// The reference Cairo prover's trace-commitment chain for one column group, on
// the device (cairo_air/prover.rs:899-1047). The reference takes every column
// through the host: permute half-coset natural order to BRT-canonic order on the
// CPU, upload, interpolate (download the coefficients), zero-pad and evaluate,
// add r * Z_H to the ZK-blinded columns, download, permute back to half-coset
// order on the CPU, upload again and commit the group (at most 16 columns, the
// native leaf) with its 1024-leaf tile roots. Here the chain stays in HBM:
//
//   permute (circle.rs:192-204) -> [coefficients] -> fused stwo LDE ->
//   blinding with a cached Z_H (prover.rs:924-935) -> [half-coset copy
//   (circle.rs:207-218)] -> capped-leaf root + tile roots (merkle.rs:360-417).
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include "fri.h"
#include "host_math.h"
#include "merkle.h"
#include "ntt.h"
#include "quotient.h"
#include "twiddles.h"
#include "vs_common.cuh"
#include "vs_field.cuh"

namespace vs {

// half-coset natural index k -> canonic natural -> BRT-canonic position
__device__ __forceinline__ uint32_t hc_to_cn_brt(uint32_t k, uint32_t log_n) {
  const uint32_t n = 1u << log_n;
  const uint32_t cn = (k & 1) ? n - 1 - (k >> 1) : (k >> 1);
  return brev(cn, log_n);
}

// dst[pos(k)] = src[k] (to canonic BRT) or dst[k] = src[pos(k)] (back to half-coset natural)
template <bool TO_CANONIC>
__global__ void permute_kernel(const uint32_t* __restrict__ src, uint64_t src_stride, uint32_t* __restrict__ dst,
                               uint64_t dst_stride, uint32_t log_n) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (1u << log_n)) return;
  const uint32_t* s = src + blockIdx.y * src_stride;
  uint32_t* d = dst + blockIdx.y * dst_stride;
  const uint32_t j = hc_to_cn_brt(k, log_n);
  if (TO_CANONIC) d[j] = s[k];
  else d[k] = s[j];
}

// Tiled form of the same permutation for n = 2^L >= 2^11 words. With k = 2m + e
// (e the parity, m of L-1 bits), the canonic index is cn = e ? ~m : m over L-1
// bits with e on top, so pos(k) = 2 (brev_{L-1}(m) ^ (e ? mask : 0)) + e: the even
// words of the half-coset order are bit-reversed into the even canonic words, and
// the odd words into the odd canonic words in descending order. Split m =
// (hi | mid | lo) with 5-bit hi and lo. One CTA moves the 32 x 32 (hi, lo) tile
// of a mid value M and the tile of its complement ~M: the odd words of M's tile
// land beside the even words of ~M's tile, so each 64-word destination window is
// written whole. k-side: 32 rows per tile of 64 consecutive words (fixed hi);
// j-side: 32 windows per tile of 64 consecutive words (fixed lo). Both sides move
// 8-byte pairs per lane; the shared tile is [tile][parity][hi][lo] with a 33-word
// pitch, so the bit-reversed side reads it without bank conflicts.
// TO_CANONIC reads k-rows and writes j-windows; the reverse reads j-windows (and,
// with zh, blinds them in place: word += r_col * zh, written back) and writes
// k-rows. The host checks that every column start and stride allows 8-byte access.
constexpr uint32_t PT_BITS = 5;
struct Blind16 {
  uint32_t r[16];
};
__device__ __forceinline__ uint32_t brev5(uint32_t x) { return __brev(x) >> 27; }

// The column index varies fastest over the grid, so the CTAs that blind the
// columns of one tile run together and read that tile of Z_H from L2.
template <bool TO_CANONIC>
__global__ void __launch_bounds__(256) permute_tiled_kernel(uint32_t* src, uint64_t src_stride, uint32_t* dst,
                                                            uint64_t dst_stride, uint32_t L, uint32_t n_cols,
                                                            const uint32_t* __restrict__ zh, Blind16 bl) {
  __shared__ uint32_t S[2][2][32][33];
  const uint32_t Lm = L - 1, Md = Lm - 2 * PT_BITS;
  const uint32_t col = blockIdx.x % n_cols;
  uint32_t* s = src + col * src_stride;
  uint32_t* d = dst + col * dst_stride;
  const int ntile = Md == 0 ? 1 : 2;
  const uint32_t M = blockIdx.x / n_cols, Mb = (~M) & ((1u << Md) - 1);
  const uint32_t mids[2] = {M, Mb};
  const uint32_t brmid[2] = {brev(M, Md), brev(Mb, Md)};
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t r = (!TO_CANONIC && zh && col < 16) ? bl.r[col] : 0u;
  const uint32_t rows = ntile * 32u;
  // every warp moves rows / 8 rows (or windows): all of its loads are issued
  // before any is consumed
  constexpr int PER_WARP = 8;
  if (TO_CANONIC) {
    uint2 v[PER_WARP];
#pragma unroll
    for (int i = 0; i < PER_WARP; i++) {
      const uint32_t row = warp + 8 * i, X = row >> 5, hi = row & 31;
      const uint64_t m_row = ((uint64_t)hi << (Lm - PT_BITS)) | ((uint64_t)mids[X & 1] << PT_BITS);
      if (row < rows) v[i] = *reinterpret_cast<const uint2*>(s + 2 * m_row + 2 * lane);
    }
#pragma unroll
    for (int i = 0; i < PER_WARP; i++) {
      const uint32_t row = warp + 8 * i, X = row >> 5, hi = row & 31;
      if (row < rows) {
        S[X][0][hi][lane] = v[i].x;
        S[X][1][hi][lane] = v[i].y;
      }
    }
  } else {
    uint2 v[PER_WARP], z[PER_WARP];
#pragma unroll
    for (int i = 0; i < PER_WARP; i++) {
      const uint32_t w = warp + 8 * i, X = w >> 5, lo = w & 31;
      const uint64_t base = ((uint64_t)brev5(lo) << (Lm - PT_BITS)) | ((uint64_t)brmid[X & 1] << PT_BITS);
      if (w < rows) {
        v[i] = *reinterpret_cast<const uint2*>(s + 2 * base + 2 * lane);
        if (r) z[i] = *reinterpret_cast<const uint2*>(zh + 2 * base + 2 * lane);
      }
    }
#pragma unroll
    for (int i = 0; i < PER_WARP; i++) {
      const uint32_t w = warp + 8 * i, X = w >> 5, lo = w & 31, Xb = ntile == 2 ? 1 - X : 0;
      if (w < rows) {
        if (r) {
          const uint64_t base = ((uint64_t)brev5(lo) << (Lm - PT_BITS)) | ((uint64_t)brmid[X & 1] << PT_BITS);
          v[i].x = add(v[i].x, mul(r, z[i].x));
          v[i].y = add(v[i].y, mul(r, z[i].y));
          *reinterpret_cast<uint2*>(s + 2 * base + 2 * lane) = v[i];
        }
        S[X][0][brev5(lane)][lo] = v[i].x;
        S[Xb][1][31 - brev5(lane)][31 - lo] = v[i].y;
      }
    }
  }
  __syncthreads();
  if (TO_CANONIC) {
#pragma unroll
    for (int i = 0; i < PER_WARP; i++) {
      const uint32_t w = warp + 8 * i, X = w >> 5, lo = w & 31, Xb = ntile == 2 ? 1 - X : 0;
      if (w < rows) {
        const uint64_t base = ((uint64_t)brev5(lo) << (Lm - PT_BITS)) | ((uint64_t)brmid[X & 1] << PT_BITS);
        *reinterpret_cast<uint2*>(d + 2 * base + 2 * lane) =
            make_uint2(S[X][0][brev5(lane)][lo], S[Xb][1][31 - brev5(lane)][31 - lo]);
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < PER_WARP; i++) {
      const uint32_t row = warp + 8 * i, X = row >> 5, hi = row & 31;
      if (row < rows) {
        const uint64_t m_row = ((uint64_t)hi << (Lm - PT_BITS)) | ((uint64_t)mids[X & 1] << PT_BITS);
        *reinterpret_cast<uint2*>(d + 2 * m_row + 2 * lane) = make_uint2(S[X][0][hi][lane], S[X][1][hi][lane]);
      }
    }
  }
}

// Z_H (the vanishing polynomial of half_coset(log_n)) at the BRT-canonic points of
// the evaluation domain: point i = half_odds(log_eval - 1).at(b) for b = brev(i) <
// N/2, its conjugate at b - N/2 otherwise; Z_H(p) = x(p * R) doubled log_n - 1
// times (x -> 2x^2 - 1), R = conj(half_coset(log_n).initial) * G^(2^(30-log_n))
// (circle.rs:228-253).
__global__ void zh_kernel(cpt ho_init, cpt ho_step, cpt R, uint32_t log_eval, uint32_t log_n, uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t N = 1u << log_eval, half = N >> 1;
  if (i >= N) return;
  const uint32_t b = brev(i, log_eval);
  cpt p = cpmul(ho_init, cppow(ho_step, b < half ? b : b - half));
  if (b >= half) p.y = neg(p.y);
  uint32_t x = cpmul(p, R).x;
  for (uint32_t j = 1; j < log_n; j++) x = sub(dbl(mul(x, x)), 1u);
  out[i] = x;
}

// y += r * x over n words
__global__ void axpy_kernel(uint32_t r, const uint32_t* __restrict__ x, uint32_t* __restrict__ y, uint64_t n) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = add(y[i], mul(r, x[i]));
}

// ------------------------------------------------------------------ evaluation at OODS points
// A circle polynomial with stwo coefficients c_i (i < 2^L) at a QM31 point p is
// sum_i c_i prod_{bit b of i} m_b with m_0 = p.y, m_1 = p.x, m_b = pi(m_{b-1}),
// pi(x) = 2x^2 - 1 (oods.rs:133-161 folds the same products recursively). The
// basis splits over the low h bits and the rest, basis_i = LO[i mod 2^h] *
// HI[i >> h], so the sum is sum_lo LO[lo] * (sum_s c[s, lo] HI[s]) over segments
// s of 2^h coefficients. Each thread owns EV_PER positions lo (coalesced words)
// and accumulates c * HI[s] per limb in 64 bits over the segments it visits:
// EV_UNROLL segments per step (that many loads per position in flight, and the
// sums folded once per step, three products per fold as in the numerator kernel).
// Only at the end are the sums reduced and multiplied by LO. Each CTA writes one
// partial per point; the host adds the partials (field addition is exact, so the
// grouping does not change the result).
constexpr int EV_THREADS = 256, EV_PER = 4, EV_LOG_SEG = 10, EV_UNROLL = 3;  // 2^10 = EV_THREADS * EV_PER
constexpr int EV_MAX_POINTS = 2;
struct EvMaps {
  qm31 m[EV_MAX_POINTS][30];
};

// tables[p] = LO (2^h entries) then HI (2^(L-h) entries): products of the maps
// over the set bits of the index (bits h.. for HI).
__global__ void basis_table_kernel(EvMaps mp, uint32_t np, uint32_t h, uint32_t lo_n, uint32_t hi_n,
                                   qm31* __restrict__ tables) {
  const uint32_t per = lo_n + hi_n;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np * per) return;
  const uint32_t p = t / per, r = t % per;
  const bool hi = r >= lo_n;
  uint32_t idx = hi ? r - lo_n : r;
  uint32_t b = hi ? h : 0;
  qm31 acc{{1, 0, 0, 0}};
  for (; idx; idx >>= 1, b++)
    if (idx & 1) acc = qmul(acc, mp.m[p][b]);
  tables[t] = acc;
}

__device__ __forceinline__ uint64_t ev_fold(uint64_t a) { return (a & VS_P) + (a >> 31); }
__device__ __forceinline__ uint32_t ev_reduce(uint64_t a) { return canon((uint32_t)ev_fold(ev_fold(a))); }

template <int NP>
__global__ void __launch_bounds__(EV_THREADS, 2) eval_points_kernel(const uint32_t* const* __restrict__ cols,
                                                                    uint32_t h, uint32_t lo_n, uint32_t hi_n,
                                                                    const qm31* __restrict__ tables,
                                                                    uint32_t* __restrict__ partials) {
  const uint32_t* col = cols[blockIdx.y];
  const uint32_t seg = 1u << h, per = lo_n + hi_n;
  uint64_t acc[NP][EV_PER][4];
#pragma unroll
  for (int p = 0; p < NP; p++)
#pragma unroll
    for (int j = 0; j < EV_PER; j++)
#pragma unroll
      for (int l = 0; l < 4; l++) acc[p][j][l] = 0;
  for (uint32_t s0 = blockIdx.x * EV_UNROLL; s0 < hi_n; s0 += gridDim.x * EV_UNROLL) {
    uint32_t x[EV_UNROLL][EV_PER];
#pragma unroll
    for (int u = 0; u < EV_UNROLL; u++) {
      const bool live = s0 + u < hi_n;
#pragma unroll
      for (int j = 0; j < EV_PER; j++) {
        const uint32_t i = threadIdx.x + j * EV_THREADS;
        x[u][j] = (live && i < seg) ? __ldg(col + (uint64_t)(s0 + u) * seg + i) : 0u;
      }
    }
#pragma unroll
    for (int u = 0; u < EV_UNROLL; u++)
#pragma unroll
      for (int p = 0; p < NP; p++) {
        const qm31 hs = s0 + u < hi_n ? tables[p * per + lo_n + s0 + u] : qzero();  // same for the whole CTA
#pragma unroll
        for (int j = 0; j < EV_PER; j++)
#pragma unroll
          for (int l = 0; l < 4; l++) acc[p][j][l] += (uint64_t)x[u][j] * hs.v[l];
      }
#pragma unroll
    for (int p = 0; p < NP; p++)
#pragma unroll
      for (int j = 0; j < EV_PER; j++)
#pragma unroll
        for (int l = 0; l < 4; l++) acc[p][j][l] = ev_fold(acc[p][j][l]);
  }
  qm31 tot[NP];
#pragma unroll
  for (int p = 0; p < NP; p++) {
    tot[p] = qzero();
#pragma unroll
    for (int j = 0; j < EV_PER; j++) {
      const uint32_t i = threadIdx.x + j * EV_THREADS;
      if (i < seg) {
        const qm31 part{{ev_reduce(acc[p][j][0]), ev_reduce(acc[p][j][1]), ev_reduce(acc[p][j][2]),
                         ev_reduce(acc[p][j][3])}};
        tot[p] = qadd(tot[p], qmul(part, tables[p * per + i]));
      }
    }
  }
  __shared__ uint32_t red[EV_THREADS / 32][NP * 4];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int p = 0; p < NP; p++)
#pragma unroll
    for (int l = 0; l < 4; l++) {
      uint32_t v = tot[p].v[l];
#pragma unroll
      for (int off = 16; off; off >>= 1) v = add(v, __shfl_down_sync(0xFFFFFFFFu, v, off));
      if (lane == 0) red[warp][p * 4 + l] = v;
    }
  __syncthreads();
  if (threadIdx.x < NP * 4) {
    uint32_t v = 0;
#pragma unroll
    for (int w = 0; w < EV_THREADS / 32; w++) v = add(v, red[w][threadIdx.x]);
    partials[((uint64_t)blockIdx.y * gridDim.x + blockIdx.x) * (NP * 4) + threadIdx.x] = v;
  }
}

// The same sums with the coefficients streamed through a per-thread cp.async
// ring: thread t owns the four consecutive positions 4t..4t+3 of every segment
// (one 16-byte copy per segment), EVR_STAGES - 1 segments ahead of the one it
// multiplies; it reads back only the slots it filled, so no barrier is needed.
// Needs 16-byte aligned columns and segments of 1024 words (the host checks).
constexpr int EVR_STAGES = 8;
__device__ __forceinline__ void cp_async16_cg(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_grp() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_grp() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int NP>
__global__ void __launch_bounds__(EV_THREADS, 2) eval_points_ring_kernel(const uint32_t* const* __restrict__ cols,
                                                                         uint32_t lo_n, uint32_t hi_n,
                                                                         const qm31* __restrict__ tables,
                                                                         uint32_t* __restrict__ partials) {
  __shared__ uint4 ring[EVR_STAGES][EV_THREADS];
  const uint32_t* col = cols[blockIdx.y] + 4 * threadIdx.x;
  const uint32_t per = lo_n + hi_n;
  const uint32_t slot0 = (uint32_t)__cvta_generic_to_shared(&ring[0][threadIdx.x]);
  constexpr uint32_t SLOT_STRIDE = EV_THREADS * sizeof(uint4);
  uint64_t acc[NP][4][4];
#pragma unroll
  for (int p = 0; p < NP; p++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int l = 0; l < 4; l++) acc[p][j][l] = 0;
  // this CTA's segments: s_i = blockIdx.x + i * gridDim.x
  const uint32_t n_mine = blockIdx.x < hi_n ? (hi_n - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
#pragma unroll
  for (uint32_t i = 0; i < EVR_STAGES - 1; i++) {
    if (i < n_mine) cp_async16_cg(slot0 + i * SLOT_STRIDE, col + (uint64_t)(blockIdx.x + i * gridDim.x) * lo_n);
    cp_async_commit_grp();
  }
  for (uint32_t i = 0; i < n_mine; i++) {
    const uint32_t ni = i + EVR_STAGES - 1;
    if (ni < n_mine)
      cp_async16_cg(slot0 + (ni % EVR_STAGES) * SLOT_STRIDE, col + (uint64_t)(blockIdx.x + ni * gridDim.x) * lo_n);
    cp_async_commit_grp();
    cp_async_wait_grp<EVR_STAGES - 1>();
    const uint4 v = ring[i % EVR_STAGES][threadIdx.x];
    const uint32_t x[4] = {v.x, v.y, v.z, v.w};
    const uint32_t s = blockIdx.x + i * gridDim.x;
#pragma unroll
    for (int p = 0; p < NP; p++) {
      const qm31 hs = tables[p * per + lo_n + s];  // the same for the whole CTA
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int l = 0; l < 4; l++) acc[p][j][l] += (uint64_t)x[j] * hs.v[l];
    }
    if (i % 3 == 2) {  // at most three products since the last fold
#pragma unroll
      for (int p = 0; p < NP; p++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
          for (int l = 0; l < 4; l++) acc[p][j][l] = ev_fold(acc[p][j][l]);
    }
  }
  cp_async_wait_grp<0>();
  qm31 tot[NP];
#pragma unroll
  for (int p = 0; p < NP; p++) {
    tot[p] = qzero();
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const qm31 part{{ev_reduce(acc[p][j][0]), ev_reduce(acc[p][j][1]), ev_reduce(acc[p][j][2]),
                       ev_reduce(acc[p][j][3])}};
      tot[p] = qadd(tot[p], qmul(part, tables[p * per + 4 * threadIdx.x + j]));
    }
  }
  __shared__ uint32_t red[EV_THREADS / 32][NP * 4];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int p = 0; p < NP; p++)
#pragma unroll
    for (int l = 0; l < 4; l++) {
      uint32_t v = tot[p].v[l];
#pragma unroll
      for (int off = 16; off; off >>= 1) v = add(v, __shfl_down_sync(0xFFFFFFFFu, v, off));
      if (lane == 0) red[warp][p * 4 + l] = v;
    }
  __syncthreads();
  if (threadIdx.x < NP * 4) {
    uint32_t v = 0;
#pragma unroll
    for (int w = 0; w < EV_THREADS / 32; w++) v = add(v, red[w][threadIdx.x]);
    partials[((uint64_t)blockIdx.y * gridDim.x + blockIdx.x) * (NP * 4) + threadIdx.x] = v;
  }
}

// BRT-canonic points of CanonicCoset(L): i -> j = brev_L(i); half_odds(L-1).at(j)
// for j < 2^(L-1), its conjugate at j - 2^(L-1) otherwise (prover.rs:161-165,
// 2213-2227). step^j = T_hi[j >> k] * T_lo[j mod 2^k] from two host-built tables,
// so each point costs two circle multiplications.
__global__ void canonic_points_kernel(cpt init, const cpt* __restrict__ t_lo, const cpt* __restrict__ t_hi,
                                      uint32_t k, uint32_t L, uint32_t* __restrict__ xs, uint32_t* __restrict__ ys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (1u << L)) return;
  const uint32_t j = brev(i, L), half = 1u << (L - 1);
  const uint32_t jj = j & (half - 1);
  const cpt p = cpmul(init, cpmul(t_hi[jj >> k], t_lo[jj & ((1u << k) - 1)]));
  xs[i] = p.x;
  ys[i] = j >= half ? neg(p.y) : p.y;
}

namespace {
std::mutex g_zh_mu;
std::map<std::pair<int, uint32_t>, uint32_t*> g_zh;  // (device, log_n) -> Z_H on the 4x domain

int zh_table(uint32_t log_n, uint32_t log_eval, cudaStream_t st, const uint32_t** out) {
  int dev = 0;
  VS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_zh_mu);
  auto it = g_zh.find({dev, log_n});
  if (it != g_zh.end()) { *out = it->second; return VS_OK; }
  const uint64_t N = 1ull << log_eval;
  uint32_t* t = nullptr;
  VS_CUDA(cudaMalloc(&t, N * 4));
  const h::Coset ho = h::half_odds(log_eval - 1), hc = h::half_coset(log_n);
  const h::Pt conj_init{hc.initial.x, h::sub(0, hc.initial.y)};
  h::Pt shp{2, 1268011823u};  // G doubled 30 - log_n times
  for (uint32_t k = 0; k < 30 - log_n; k++) shp = h::pmul(shp, shp);
  const h::Pt R = h::pmul(conj_init, shp);
  zh_kernel<<<blocks_for(N, 256), 256, 0, st>>>(cpt{ho.initial.x, ho.initial.y}, cpt{ho.step.x, ho.step.y},
                                                 cpt{R.x, R.y}, log_eval, log_n, t);
  VS_LAUNCHED("zh_kernel");
  VS_CUDA(cudaStreamSynchronize(st));
  g_zh[{dev, log_n}] = t;
  *out = t;
  return VS_OK;
}
}  // namespace

void release_zh_tables() {
  std::lock_guard<std::mutex> lk(g_zh_mu);
  for (auto& kv : g_zh) cudaFree(kv.second);
  g_zh.clear();
}

// dst = src permuted to BRT-canonic order (to_canonic) or back to half-coset
// natural order, n_cols columns of 2^L words. In the reverse direction a non-null
// zh blinds column c of src in place first (src += r16[c] * zh, r16[c] != 0).
// Tiled kernel when the sizes and alignment allow 8-byte access, else word
// kernels (plus the separate blinding pass).
int launch_permute(bool to_canonic, uint32_t* src, uint64_t src_stride, uint32_t* dst, uint64_t dst_stride,
                   uint32_t n_cols, uint32_t L, const uint32_t* zh, const uint32_t* r16, cudaStream_t st) {
  if (n_cols == 0) return VS_OK;
  if (n_cols > 65535 || (zh && n_cols > 16)) return set_error(VS_ERR_INVALID, "permute: column count");
  const auto a8 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7) == 0; };
  const bool tiled = L >= 2 * PT_BITS + 1 && a8(src) && a8(dst) &&
                     (n_cols == 1 || (src_stride % 2 == 0 && dst_stride % 2 == 0));
  Blind16 bl{};
  for (uint32_t c = 0; zh && c < n_cols; c++) bl.r[c] = r16[c];
  if (tiled) {
    const uint32_t Md = L - 1 - 2 * PT_BITS;
    const uint64_t blocks = (Md == 0 ? 1ull : 1ull << (Md - 1)) * n_cols;
    if (blocks > 0x7FFFFFFFull) return set_error(VS_ERR_INVALID, "permute: grid too large");
    if (to_canonic)
      permute_tiled_kernel<true><<<(unsigned)blocks, 256, 0, st>>>(src, src_stride, dst, dst_stride, L, n_cols, nullptr, bl);
    else
      permute_tiled_kernel<false><<<(unsigned)blocks, 256, 0, st>>>(src, src_stride, dst, dst_stride, L, n_cols, zh, bl);
    VS_LAUNCHED("permute_tiled_kernel");
    return VS_OK;
  }
  const uint64_t n = 1ull << L;
  for (uint32_t c = 0; zh && c < n_cols; c++) {
    if (!bl.r[c]) continue;
    axpy_kernel<<<blocks_for(n, 256), 256, 0, st>>>(bl.r[c], zh, src + c * src_stride, n);
    VS_LAUNCHED("axpy_kernel");
  }
  const dim3 grid(blocks_for(n, 256), n_cols);
  if (to_canonic) permute_kernel<true><<<grid, 256, 0, st>>>(src, src_stride, dst, dst_stride, L);
  else permute_kernel<false><<<grid, 256, 0, st>>>(src, src_stride, dst, dst_stride, L);
  VS_LAUNCHED("permute_kernel");
  return VS_OK;
}

namespace {
// Stream-ordered allocations released (stream-ordered) when the holder goes out of scope.
struct Scratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit Scratch(cudaStream_t s) : st(s) {}
  ~Scratch() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
  template <class T>
  int alloc(T** out, uint64_t count) {
    void* p = nullptr;
    VS_CUDA(cudaMallocAsync(&p, std::max<uint64_t>(count, 1) * sizeof(T), st));
    ptrs.push_back(p);
    *out = static_cast<T*>(p);
    return VS_OK;
  }
  // device copy of a host array (pageable source: the copy is staged before return)
  template <class T>
  int upload(T** out, const T* h, uint64_t count) {
    VS_TRY(alloc(out, count));
    VS_CUDA(cudaMemcpyAsync(*out, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
    return VS_OK;
  }
};

h::Q pi_x(h::Q x) {  // 2x^2 - 1
  const h::Q x2 = h::qmul(x, x);
  return h::qsub(h::qadd(x2, x2), h::qm31_of(1));
}
}  // namespace

// out[c * np + p] = column c (2^L stwo coefficients) at point p; synchronises st.
int eval_at_points(const uint32_t* const* h_cols, uint32_t n_cols, uint32_t L, const h::Q (*pts)[2], uint32_t np,
                   h::Q* out, cudaStream_t st) {
  if (np == 0 || np > EV_MAX_POINTS) return set_error(VS_ERR_INVALID, "eval_at_points: 1 or 2 points");
  if (L > 30) return set_error(VS_ERR_INVALID, "eval_at_points: log length %u", L);
  if (n_cols == 0) return VS_OK;
  if (n_cols > 65535) return set_error(VS_ERR_INVALID, "eval_at_points: too many columns");
  EvMaps mp{};
  for (uint32_t p = 0; p < np; p++) {
    h::Q m = pts[p][0];  // x
    mp.m[p][0] = qm31{{pts[p][1].v[0], pts[p][1].v[1], pts[p][1].v[2], pts[p][1].v[3]}};
    for (uint32_t b = 1; b < L; b++) {
      mp.m[p][b] = qm31{{m.v[0], m.v[1], m.v[2], m.v[3]}};
      m = pi_x(m);
    }
  }
  const uint32_t hb = std::min<uint32_t>(L, EV_LOG_SEG);
  const uint32_t lo_n = 1u << hb, hi_n = 1u << (L - hb), per = lo_n + hi_n;
  const uint32_t gx = std::max<uint32_t>(
      1, std::min<uint32_t>((hi_n + EV_UNROLL - 1) / EV_UNROLL, (uint32_t)sm_count() * 4 / n_cols));
  Scratch s(st);
  qm31* tables = nullptr;
  uint32_t* partials = nullptr;
  const uint32_t** d_cols = nullptr;
  VS_TRY(s.alloc(&tables, (uint64_t)np * per));
  VS_TRY(s.alloc(&partials, (uint64_t)n_cols * gx * np * 4));
  std::vector<const uint32_t*> cols(h_cols, h_cols + n_cols);
  VS_TRY(s.upload(&d_cols, cols.data(), n_cols));
  basis_table_kernel<<<blocks_for((uint64_t)np * per, 256), 256, 0, st>>>(mp, np, hb, lo_n, hi_n, tables);
  VS_LAUNCHED("basis_table_kernel");
  const dim3 grid(gx, n_cols);
  bool ring = hb == EV_LOG_SEG && hi_n >= 4;
  for (uint32_t c = 0; c < n_cols; c++) ring = ring && (reinterpret_cast<uintptr_t>(h_cols[c]) & 15) == 0;
  if (ring) {
    if (np == 1) eval_points_ring_kernel<1><<<grid, EV_THREADS, 0, st>>>(d_cols, lo_n, hi_n, tables, partials);
    else eval_points_ring_kernel<2><<<grid, EV_THREADS, 0, st>>>(d_cols, lo_n, hi_n, tables, partials);
    VS_LAUNCHED("eval_points_ring_kernel");
  } else {
    if (np == 1) eval_points_kernel<1><<<grid, EV_THREADS, 0, st>>>(d_cols, hb, lo_n, hi_n, tables, partials);
    else eval_points_kernel<2><<<grid, EV_THREADS, 0, st>>>(d_cols, hb, lo_n, hi_n, tables, partials);
    VS_LAUNCHED("eval_points_kernel");
  }
  std::vector<uint32_t> hp((uint64_t)n_cols * gx * np * 4);
  VS_CUDA(cudaMemcpyAsync(hp.data(), partials, hp.size() * 4, cudaMemcpyDeviceToHost, st));
  VS_CUDA(cudaStreamSynchronize(st));
  for (uint32_t c = 0; c < n_cols; c++)
    for (uint32_t p = 0; p < np; p++) {
      h::Q acc{{0, 0, 0, 0}};
      for (uint32_t b = 0; b < gx; b++) {
        const uint32_t* v = &hp[(((uint64_t)c * gx + b) * np + p) * 4];
        acc = h::qadd(acc, h::Q{{v[0], v[1], v[2], v[3]}});
      }
      out[c * np + p] = acc;
    }
  return VS_OK;
}

// 1024-leaf tile roots of a commitment, through 2^split subtree roots per tile
// (merkle_tile_split) for trees of 2^20+ leaves; stream-ordered subroot scratch.
template <class Leaf>
int tile_roots_split(const Leaf& leaf, uint64_t N, uint32_t* tiles, cudaStream_t st) {
  const uint32_t sp = merkle_tile_split(N);
  if (!sp) return merkle_tile_roots(leaf, N, MK_MAX_TL, tiles, st);
  const uint64_t t = N >> MK_MAX_TL;
  uint32_t *a = nullptr, *b = nullptr;
  VS_CUDA(cudaMallocAsync((void**)&a, (t << sp) * 32, st));
  int rc = check_cuda(cudaMallocAsync((void**)&b, (t << (sp - 1)) * 32, st), "subroot scratch");
  if (rc == VS_OK) rc = merkle_tile_roots_split(leaf, N, MK_MAX_TL, sp, tiles, a, b, st);
  cudaFreeAsync(a, st);
  if (b) cudaFreeAsync(b, st);
  return rc;
}

}  // namespace vs

using namespace vs;

extern "C" int vs_commit_group_cairo(const uint32_t* d_cols_hc, uint64_t col_stride, uint32_t n_cols, uint32_t log_n,
                                     const uint32_t* h_blind, uint32_t* d_coeffs, uint32_t* d_eval_cn,
                                     uint32_t* d_eval_hc, uint32_t* d_root, uint32_t* d_tile_roots,
                                     vs_stream_t stream) {
  clear_error();
  cudaStream_t st = (cudaStream_t)stream;
  if (!d_cols_hc || !d_eval_cn || !d_root) return set_error(VS_ERR_INVALID, "vs_commit_group_cairo: null argument");
  if (n_cols == 0 || n_cols > 16) return set_error(VS_ERR_INVALID, "vs_commit_group_cairo: 1..16 columns per group");
  if (log_n < 2 || log_n + 2 > 30) return set_error(VS_ERR_INVALID, "vs_commit_group_cairo: log_n %u out of range", log_n);
  if (col_stride < (1ull << log_n)) return set_error(VS_ERR_INVALID, "vs_commit_group_cairo: stride below 2^log_n");
  for (uint32_t c = 0; h_blind && c < n_cols; c++)
    if (h_blind[c] >= VS_P) return set_error(VS_ERR_INVALID, "vs_commit_group_cairo: blinding scalar not canonical");
  const uint32_t log_eval = log_n + 2;
  const uint64_t n = 1ull << log_n, N = 1ull << log_eval;
  // 1. half-coset natural -> BRT-canonic (into a stream-ordered scratch)
  uint32_t* cn = nullptr;
  VS_CUDA(cudaMallocAsync((void**)&cn, n_cols * n * 4, st));
  int rc = launch_permute(true, const_cast<uint32_t*>(d_cols_hc), col_stride, cn, n, n_cols, log_n, nullptr, nullptr, st);
  // 2. stwo coefficients (the reference keeps them for the OODS evaluation)
  if (rc == VS_OK && d_coeffs) {
    rc = check_cuda(cudaMemcpyAsync(d_coeffs, cn, n_cols * n * 4, cudaMemcpyDeviceToDevice, st), "coeffs copy");
    NttTw ti;
    if (rc == VS_OK) rc = tw_for(TW_STWO, log_n, false, &ti, st);
    NttColumns io{d_coeffs, d_coeffs, nullptr, nullptr, n, n, n_cols};
    if (rc == VS_OK) rc = ntt_transform(io, log_n, ti, false, st);
  }
  // 3. LDE x4 on the canonic coset, BRT output
  if (rc == VS_OK) rc = lde_cached(TW_STWO, cn, n, d_eval_cn, N, n_cols, log_n, 2, st);
  cudaFreeAsync(cn, st);
  // 4-5. ZK blinding (column c += r_c * Z_H) and the half-coset natural copy
  // that the reference's constraint kernels read, fused into one pass when both
  // are asked for
  const uint32_t* zh = nullptr;
  bool any_blind = false;
  for (uint32_t c = 0; h_blind && c < n_cols; c++) any_blind = any_blind || h_blind[c] != 0;
  if (rc == VS_OK && any_blind) rc = zh_table(log_n, log_eval, st, &zh);
  if (rc == VS_OK && d_eval_hc) {
    rc = launch_permute(false, d_eval_cn, N, d_eval_hc, N, n_cols, log_eval, any_blind ? zh : nullptr, h_blind, st);
  } else if (rc == VS_OK && any_blind) {
    for (uint32_t c = 0; c < n_cols && rc == VS_OK; c++) {
      if (!h_blind[c]) continue;
      axpy_kernel<<<blocks_for(N, 256), 256, 0, st>>>(h_blind[c], zh, d_eval_cn + c * N, N);
      rc = check_cuda(cudaGetLastError(), "blinding");
      count_launch();
    }
  }
  // 6. commitment: native capped leaf over the group's columns, root + 1024-leaf tile roots
  if (rc == VS_OK) {
    const LeafCapped leaf{nullptr, d_eval_cn, N, n_cols};
    if (N < 1024) {
      rc = merkle_root(leaf, N, d_root, st);
      if (rc == VS_OK && d_tile_roots)
        rc = check_cuda(cudaMemcpyAsync(d_tile_roots, d_root, 32, cudaMemcpyDeviceToDevice, st), "tile root");
    } else {
      uint32_t* tiles = d_tile_roots;
      if (!tiles) rc = check_cuda(cudaMallocAsync((void**)&tiles, (N / 1024) * 32, st), "tile roots");
      if (rc == VS_OK) rc = tile_roots_split(leaf, N, tiles, st);
      if (rc == VS_OK) rc = merkle_root(LeafHashes{tiles}, N / 1024, d_root, st);
      if (!d_tile_roots && tiles) cudaFreeAsync(tiles, st);
    }
  }
  return rc;
}

extern "C" int vs_eval_at_oods_points(const uint32_t* const* h_cols, uint32_t n_cols, uint32_t log_len,
                                      const uint32_t* h_points, uint32_t n_points, uint32_t* h_out,
                                      vs_stream_t stream) {
  clear_error();
  if (!h_points || (n_cols && (!h_cols || !h_out))) return set_error(VS_ERR_INVALID, "vs_eval_at_oods_points: null");
  if (n_points == 0 || n_points > EV_MAX_POINTS) return set_error(VS_ERR_INVALID, "vs_eval_at_oods_points: 1 or 2 points");
  for (uint32_t c = 0; c < n_cols; c++)
    if (!h_cols[c]) return set_error(VS_ERR_INVALID, "vs_eval_at_oods_points: null column %u", c);
  h::Q pts[EV_MAX_POINTS][2];
  for (uint32_t p = 0; p < n_points; p++)
    for (int l = 0; l < 4; l++) {
      pts[p][0].v[l] = h_points[8 * p + l];
      pts[p][1].v[l] = h_points[8 * p + 4 + l];
      if (pts[p][0].v[l] >= VS_P || pts[p][1].v[l] >= VS_P)
        return set_error(VS_ERR_INVALID, "vs_eval_at_oods_points: point not canonical");
    }
  std::vector<h::Q> out((uint64_t)n_cols * n_points);
  VS_TRY(eval_at_points(h_cols, n_cols, log_len, pts, n_points, out.data(), (cudaStream_t)stream));
  for (uint64_t i = 0; i < out.size(); i++) std::memcpy(h_out + 4 * i, out[i].v, 16);
  return VS_OK;
}

namespace {
// SoA4 commitment with 1024-leaf tile roots (merkle.rs:294-330): the root alone
// (copied into tiles) below 1024 leaves.
int commit_soa4_tiles(uint32_t* const c[4], uint64_t N, uint32_t* d_root, uint32_t* tiles, cudaStream_t st) {
  const LeafSoa4 leaf{c[0], c[1], c[2], c[3]};
  if (N < 1024) {
    VS_TRY(merkle_root(leaf, N, d_root, st));
    VS_CUDA(cudaMemcpyAsync(tiles, d_root, 32, cudaMemcpyDeviceToDevice, st));
    return VS_OK;
  }
  VS_TRY(tile_roots_split(leaf, N, tiles, st));
  return merkle_root(LeafHashes{tiles}, N / 1024, d_root, st);
}
int read_hash(const uint32_t* d, h::Hash& out, cudaStream_t st) {
  VS_CUDA(cudaMemcpyAsync(out.data(), d, 32, cudaMemcpyDeviceToHost, st));
  VS_CUDA(cudaStreamSynchronize(st));
  return VS_OK;
}
// fri.rs:294-336: 8 BRT-ordered line evaluations on half_odds(3) -> natural
// coefficients (bit-reverse, line iFFT with 1/x twiddles, scale by 1/n, bit-reverse)
std::vector<h::Q> line_coeffs_from_evals(std::vector<h::Q> e) {
  const uint32_t n = (uint32_t)e.size(), lg = ilog2(n);
  auto brev_all = [&](std::vector<h::Q>& v) {
    for (uint32_t i = 0; i < n; i++) {
      const uint32_t j = (uint32_t)h::brev(i, lg);
      if (i < j) std::swap(v[i], v[j]);
    }
  };
  brev_all(e);
  for (uint32_t chunk = n, dl = lg; chunk > 1; chunk >>= 1, dl--) {
    const h::Coset dom = h::half_odds(dl);
    const uint32_t half = chunk / 2;
    for (uint32_t base = 0; base < n; base += chunk)
      for (uint32_t i = 0; i < half; i++) {
        const uint32_t xi = h::inv(dom.at(i).x);
        const h::Q l = e[base + i], r = e[base + half + i];
        e[base + i] = h::qadd(l, r);
        e[base + half + i] = h::qscale(h::qsub(l, r), xi);
      }
  }
  const uint32_t ninv = h::inv(n);
  for (auto& v : e) v = h::qscale(v, ninv);
  brev_all(e);
  return e;
}
void put_q(uint32_t* dst, const h::Q& q) { std::memcpy(dst, q.v, 16); }
}  // namespace

extern "C" int vs_cairo_oods_fri(void* channel, vs_cairo_oods_fri_io* io, vs_stream_t stream) {
  clear_error();
  auto* ch = static_cast<h::Channel*>(channel);
  cudaStream_t st = (cudaStream_t)stream;
  if (!ch || !io) return set_error(VS_ERR_INVALID, "vs_cairo_oods_fri: null argument");
  const uint32_t log_n = io->log_n, nt = io->n_trace, ni = io->n_interaction;
  if (log_n < 2 || log_n > 26) return set_error(VS_ERR_INVALID, "vs_cairo_oods_fri: log_n %u outside [2, 26]", log_n);
  if (nt == 0 || nt > 1024 || ni > 1024) return set_error(VS_ERR_INVALID, "vs_cairo_oods_fri: column counts");
  if (!io->trace_coeffs || !io->trace_evals || (ni && !io->interaction_evals))
    return set_error(VS_ERR_INVALID, "vs_cairo_oods_fri: null column table");
  for (uint32_t c = 0; c < nt; c++) {
    if (!io->trace_coeffs[c] || !io->trace_evals[c]) return set_error(VS_ERR_INVALID, "vs_cairo_oods_fri: null trace column");
    if (io->zk_scalars && io->zk_scalars[c] >= VS_P) return set_error(VS_ERR_INVALID, "vs_cairo_oods_fri: blinding scalar");
  }
  for (uint32_t c = 0; c < ni; c++)
    if (!io->interaction_evals[c]) return set_error(VS_ERR_INVALID, "vs_cairo_oods_fri: null interaction column");
  for (int k = 0; k < 4; k++)
    if (!io->quotient_hc[k]) return set_error(VS_ERR_INVALID, "vs_cairo_oods_fri: null quotient limb");
  const uint32_t log_eval = log_n + 2;
  const uint64_t N = 1ull << log_eval;
  const uint64_t n_tiles = N < 1024 ? 1 : N / 1024;
  Scratch s(st);
  uint32_t* d_root = nullptr;
  VS_TRY(s.alloc(&d_root, 8));
  h::Hash root;

  // AIR quotient: half-coset natural -> BRT-canonic, SoA4 commitment (prover.rs:1937-1971)
  uint32_t* qcn[4];
  for (int k = 0; k < 4; k++) {
    qcn[k] = io->quotient_cn[k];
    if (!qcn[k]) VS_TRY(s.alloc(&qcn[k], N));
    VS_TRY(launch_permute(true, const_cast<uint32_t*>(io->quotient_hc[k]), N, qcn[k], N, 1, log_eval, nullptr, nullptr,
                          st));
  }
  uint32_t* qtiles = io->quotient_tile_roots;
  if (!qtiles) VS_TRY(s.alloc(&qtiles, n_tiles * 8));
  VS_TRY(commit_soa4_tiles(qcn, N, d_root, qtiles, st));
  VS_TRY(read_hash(d_root, root, st));
  std::memcpy(io->quotient_root, root.data(), 32);
  ch->mix_digest(root);

  // OODS point z and z_next = z + one trace step (oods.rs:44-81; prover.rs:1978-1984)
  const h::Q t = ch->draw_felt(), one = h::qm31_of(1);
  const h::Q t2 = h::qmul(t, t), di = h::qinv(h::qadd(one, t2));
  const h::Q zx = h::qmul(h::qsub(one, t2), di), zy = h::qmul(h::qadd(t, t), di);
  h::Pt step{2, 1268011823u};
  for (uint32_t i = 0; i < 31 - log_n; i++) step = h::pmul(step, step);
  const h::Q nx = h::qsub(h::qscale(zx, step.x), h::qscale(zy, step.y));
  const h::Q ny = h::qadd(h::qscale(zx, step.y), h::qscale(zy, step.x));
  h::Q zh_z = zx, zh_n = nx;  // oods.rs:285-291
  for (uint32_t i = 1; i < log_n; i++) { zh_z = pi_x(zh_z); zh_n = pi_x(zh_n); }
  const h::Q pts[2][2] = {{zx, zy}, {nx, ny}};

  // trace columns at z and z_next from their coefficients, plus r * Z_H (prover.rs:1987-2001)
  std::vector<h::Q> tv(2 * nt), iv(2 * ni);
  VS_TRY(eval_at_points(io->trace_coeffs, nt, log_n, pts, 2, tv.data(), st));
  if (io->zk_scalars)
    for (uint32_t c = 0; c < nt; c++)
      if (const uint32_t r = io->zk_scalars[c]) {
        tv[2 * c] = h::qadd(tv[2 * c], h::qscale(zh_z, r));
        tv[2 * c + 1] = h::qadd(tv[2 * c + 1], h::qscale(zh_n, r));
      }
  // interaction columns: first 2^log_n stwo coefficients of their evaluations (prover.rs:2037-2048)
  NttTw ti;
  VS_TRY(tw_for(TW_STWO, log_eval, false, &ti, st));
  const uint32_t B = std::min<uint32_t>(std::max<uint32_t>(ni, 4), 8);
  uint32_t* coef = nullptr;
  VS_TRY(s.alloc(&coef, B * N));
  std::vector<const uint32_t*> cp(B);
  for (uint32_t j = 0; j < B; j++) cp[j] = coef + j * N;
  for (uint32_t c0 = 0; c0 < ni; c0 += B) {
    const uint32_t nb = std::min(B, ni - c0);
    for (uint32_t j = 0; j < nb; j++)
      VS_CUDA(cudaMemcpyAsync(coef + j * N, io->interaction_evals[c0 + j], N * 4, cudaMemcpyDeviceToDevice, st));
    VS_TRY(ntt_transform(NttColumns{coef, coef, nullptr, nullptr, N, N, nb}, log_eval, ti, false, st));
    VS_TRY(eval_at_points(cp.data(), nb, log_n, pts, 2, iv.data() + 2 * c0, st));
  }
  // quotient limbs at z from all their coefficients (prover.rs:2053-2065)
  h::Q qv[4];
  for (int k = 0; k < 4; k++)
    VS_CUDA(cudaMemcpyAsync(coef + k * N, qcn[k], N * 4, cudaMemcpyDeviceToDevice, st));
  VS_TRY(ntt_transform(NttColumns{coef, coef, nullptr, nullptr, N, N, 4}, log_eval, ti, false, st));
  VS_TRY(eval_at_points(cp.data(), 4, log_eval, pts, 1, qv, st));

  // sampled values in flatten_cols order, then the OODS alpha (prover.rs:2067-2095)
  {
    std::vector<h::Q> all;
    all.reserve(2 * nt + 2 * ni + 4);
    for (uint32_t c = 0; c < nt; c++) { all.push_back(tv[2 * c]); all.push_back(tv[2 * c + 1]); }
    for (uint32_t c = 0; c < ni; c++) { all.push_back(iv[2 * c]); all.push_back(iv[2 * c + 1]); }
    for (int k = 0; k < 4; k++) all.push_back(qv[k]);
    ch->mix_felts(all);
  }
  const h::Q alpha = ch->draw_felt();

  // alpha-weighted line coefficients (prover.rs:2095-2150; oods.rs compute_line_coeffs)
  std::vector<uint32_t> bz, cz, bn, cn;
  h::Q lin_z{{0, 0, 0, 0}}, lin_n{{0, 0, 0, 0}}, ap = one;
  auto push = [&](const h::Q& py, const h::Q& v, std::vector<uint32_t>& bv, std::vector<uint32_t>& cv, h::Q& lin) {
    const h::Q b = h::qmul(h::qsub(v, h::qconj(v)), h::qinv(h::qsub(py, h::qconj(py))));
    const h::Q a = h::qsub(v, h::qmul(b, py));
    const h::Q wa = h::qmul(ap, a);
    bv.insert(bv.end(), wa.v, wa.v + 4);
    cv.insert(cv.end(), ap.v, ap.v + 4);
    lin = h::qadd(lin, h::qmul(ap, b));
    ap = h::qmul(ap, alpha);
  };
  for (uint32_t c = 0; c < nt; c++) push(zy, tv[2 * c], bz, cz, lin_z);
  for (int k = 0; k < 4; k++) push(zy, qv[k], bz, cz, lin_z);
  for (uint32_t c = 0; c < ni; c++) push(zy, iv[2 * c], bz, cz, lin_z);
  for (uint32_t c = 0; c < nt; c++) push(ny, tv[2 * c + 1], bn, cn, lin_n);
  for (uint32_t c = 0; c < ni; c++) push(ny, iv[2 * c + 1], bn, cn, lin_n);

  // DEEP numerators over [trace, quotient, interaction] (prover.rs:2152-2207)
  const uint32_t n_all = nt + 4 + ni;
  std::vector<const uint32_t*> cols;
  cols.reserve(n_all);
  for (uint32_t c = 0; c < nt; c++) cols.push_back(io->trace_evals[c]);
  for (int k = 0; k < 4; k++) cols.push_back(qcn[k]);
  for (uint32_t c = 0; c < ni; c++) cols.push_back(io->interaction_evals[c]);
  bool vec = N % 4 == 0;
  for (const uint32_t* p : cols) vec = vec && (reinterpret_cast<uintptr_t>(p) & 15) == 0;
  std::vector<uint32_t> idx_z(n_all), idx_n;
  for (uint32_t i = 0; i < n_all; i++) idx_z[i] = i;
  for (uint32_t i = 0; i < nt; i++) idx_n.push_back(i);
  for (uint32_t i = 0; i < ni; i++) idx_n.push_back(nt + 4 + i);
  const uint32_t** d_cols = nullptr;
  uint32_t *d_iz, *d_in, *d_bz, *d_cz, *d_bn, *d_cn, *numer;
  VS_TRY(s.upload(&d_cols, cols.data(), n_all));
  VS_TRY(s.upload(&d_iz, idx_z.data(), idx_z.size()));
  VS_TRY(s.upload(&d_in, idx_n.data(), idx_n.size()));
  VS_TRY(s.upload(&d_bz, bz.data(), bz.size()));
  VS_TRY(s.upload(&d_cz, cz.data(), cz.size()));
  VS_TRY(s.upload(&d_bn, bn.data(), bn.size()));
  VS_TRY(s.upload(&d_cn, cn.data(), cn.size()));
  VS_TRY(s.alloc(&numer, 8 * N));
  uint32_t* const num_z[4] = {numer, numer + N, numer + 2 * N, numer + 3 * N};
  uint32_t* const num_n[4] = {numer + 4 * N, numer + 5 * N, numer + 6 * N, numer + 7 * N};
  if (vec) {  // one pass over the columns for both samples
    std::vector<uint32_t> cb(4 * n_all, 0u);
    std::copy(cn.begin(), cn.begin() + 4 * nt, cb.begin());
    std::copy(cn.begin() + 4 * nt, cn.end(), cb.begin() + 4 * (nt + 4));
    uint32_t* d_cb;
    VS_TRY(s.upload(&d_cb, cb.data(), cb.size()));
    h::Q sa{{0, 0, 0, 0}}, sb{{0, 0, 0, 0}};
    for (size_t i = 0; i < bz.size(); i += 4) sa = h::qadd(sa, h::Q{{bz[i], bz[i + 1], bz[i + 2], bz[i + 3]}});
    for (size_t i = 0; i < bn.size(); i += 4) sb = h::qadd(sb, h::Q{{bn[i], bn[i + 1], bn[i + 2], bn[i + 3]}});
    VS_TRY(launch_accumulate_numerators2(d_cols, d_cz, d_cb, sa.v, sb.v, n_all, (uint32_t)N, num_z, num_n, st));
  } else {
    VS_TRY(launch_accumulate_numerators(d_cols, d_iz, d_bz, d_cz, n_all, (uint32_t)N, num_z, false, st));
    VS_TRY(launch_accumulate_numerators(d_cols, d_in, d_bn, d_cn, nt + ni, (uint32_t)N, num_n, false, st));
  }

  // BRT-canonic domain points and the combination (prover.rs:2213-2266)
  uint32_t *xs, *ys;
  VS_TRY(s.alloc(&xs, N));
  VS_TRY(s.alloc(&ys, N));
  {
    const h::Coset ho = h::half_odds(log_eval - 1);
    const uint32_t k = (log_eval - 1) / 2;
    std::vector<cpt> tlo(1u << k), thi(1u << (log_eval - 1 - k));
    h::Pt a{1, 0};
    for (auto& e : tlo) { e = cpt{a.x, a.y}; a = h::pmul(a, ho.step); }
    const h::Pt big = h::ppow(ho.step, 1ull << k);
    a = h::Pt{1, 0};
    for (auto& e : thi) { e = cpt{a.x, a.y}; a = h::pmul(a, big); }
    cpt *d_lo, *d_hi;
    VS_TRY(s.upload(&d_lo, tlo.data(), tlo.size()));
    VS_TRY(s.upload(&d_hi, thi.data(), thi.size()));
    canonic_points_kernel<<<blocks_for(N, 256), 256, 0, st>>>(cpt{ho.initial.x, ho.initial.y}, d_lo, d_hi, k,
                                                              log_eval, xs, ys);
    VS_LAUNCHED("canonic_points_kernel");
  }
  uint32_t meta[4 * 2 * 3 + 2];  // spx[8] spy[8] fla[8] acc_log[2]
  std::memcpy(meta, zx.v, 16);
  std::memcpy(meta + 4, nx.v, 16);
  std::memcpy(meta + 8, zy.v, 16);
  std::memcpy(meta + 12, ny.v, 16);
  std::memcpy(meta + 16, lin_z.v, 16);
  std::memcpy(meta + 20, lin_n.v, 16);
  meta[24] = meta[25] = log_eval;
  const uint32_t* nptr[8] = {num_z[0], num_n[0], num_z[1], num_n[1], num_z[2], num_n[2], num_z[3], num_n[3]};
  uint32_t* d_meta;
  const uint32_t** d_np;
  VS_TRY(s.upload(&d_meta, meta, 26));
  VS_TRY(s.upload(&d_np, nptr, 8));
  uint32_t* oq[4];
  for (int k = 0; k < 4; k++) {
    oq[k] = io->oods_quotient[k];
    if (!oq[k]) VS_TRY(s.alloc(&oq[k], N));
  }
  VS_TRY(launch_quotients_combine(d_meta, d_meta + 8, d_meta + 16, d_np, d_np + 2, d_np + 4, d_np + 6, d_meta + 24, 2,
                                  xs, ys, log_eval, (uint32_t)N, oq, st));
  uint32_t* otiles = io->oods_tile_roots;
  if (!otiles) VS_TRY(s.alloc(&otiles, n_tiles * 8));
  VS_TRY(commit_soa4_tiles(oq, N, d_root, otiles, st));
  VS_TRY(read_hash(d_root, root, st));
  std::memcpy(io->oods_root, root.data(), 32);
  ch->mix_digest(root);

  // FRI: circle fold with 1/y of the canonic points, then committed line folds
  // down to 8 values; each fold is fused with the commitment of its output
  // (prover.rs:2321-2381)
  uint32_t *fri = nullptr, *mscratch = nullptr;
  VS_TRY(s.alloc(&fri, 4 * N));
  VS_TRY(s.alloc(&mscratch, merkle_scratch_words_any(N / 2)));
  const uint32_t split = merkle_split();
  uint32_t* src[4] = {oq[0], oq[1], oq[2], oq[3]};
  uint32_t* dst[4];
  uint64_t off = 0;
  h::Q fa = ch->draw_felt();
  std::vector<h::Q> alphas{fa};
  std::vector<h::Hash> roots;
  const uint32_t* tw = nullptr;
  VS_TRY(get_fold_twiddles(FOLD_CANONIC_CIRCLE, log_eval, &tw, st));
  uint64_t half = N / 2;
  for (int k = 0; k < 4; k++) dst[k] = fri + off + k * half;
  off += 4 * half;
  VS_TRY(fold_commit_layer(src, dst, tw, fa.v, nullptr, false, half, d_root, mscratch, st, split));
  for (uint32_t cur = log_eval - 1; cur > 3; cur--) {
    VS_TRY(read_hash(d_root, root, st));
    ch->mix_digest(root);
    roots.push_back(root);
    fa = ch->draw_felt();
    alphas.push_back(fa);
    VS_TRY(get_fold_twiddles(COSET_HALF_ODDS, cur, &tw, st));
    for (int k = 0; k < 4; k++) src[k] = dst[k];
    half >>= 1;
    for (int k = 0; k < 4; k++) dst[k] = fri + off + k * half;
    off += 4 * half;
    VS_TRY(fold_commit_layer(src, dst, tw, fa.v, nullptr, false, half, d_root, mscratch, st, split));
  }
  std::vector<uint32_t> planes(32);
  for (int k = 0; k < 4; k++)
    VS_CUDA(cudaMemcpyAsync(planes.data() + 8 * k, dst[k], 32, cudaMemcpyDeviceToHost, st));
  VS_CUDA(cudaStreamSynchronize(st));
  std::vector<h::Q> last(8);
  for (int i = 0; i < 8; i++) last[i] = h::Q{{planes[i], planes[8 + i], planes[16 + i], planes[24 + i]}};
  const std::vector<h::Q> nat = line_coeffs_from_evals(last);
  std::vector<h::Q> brt(8);
  for (uint32_t i = 0; i < 8; i++) brt[h::brev(i, 3)] = nat[i];
  ch->mix_felts(brt);

  // results
  for (uint32_t c = 0; c < nt; c++) {
    if (io->trace_at_z) put_q(io->trace_at_z + 4 * c, tv[2 * c]);
    if (io->trace_at_z_next) put_q(io->trace_at_z_next + 4 * c, tv[2 * c + 1]);
  }
  for (uint32_t c = 0; c < ni; c++) {
    if (io->interaction_at_z) put_q(io->interaction_at_z + 4 * c, iv[2 * c]);
    if (io->interaction_at_z_next) put_q(io->interaction_at_z_next + 4 * c, iv[2 * c + 1]);
  }
  put_q(io->oods_point, zx);
  put_q(io->oods_point + 4, zy);
  for (int k = 0; k < 4; k++) put_q(io->quotient_at_z + 4 * k, qv[k]);
  put_q(io->oods_alpha, alpha);
  io->n_fri_roots = (uint32_t)roots.size();
  for (size_t i = 0; i < roots.size(); i++) std::memcpy(io->fri_roots + 8 * i, roots[i].data(), 32);
  for (size_t i = 0; i < alphas.size(); i++) put_q(io->fri_alphas + 4 * i, alphas[i]);
  for (int i = 0; i < 8; i++) {
    put_q(io->last_layer + 4 * i, last[i]);
    put_q(io->last_layer_coeffs + 4 * i, brt[i]);
  }
  return VS_OK;
}
