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
#include <map>
#include <memory>
#include <mutex>
#include <utility>

#include "host_math.h"
#include "merkle.h"
#include "ntt.h"
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
  int rc = VS_OK;
  permute_kernel<true><<<dim3(blocks_for(n, 256), n_cols), 256, 0, st>>>(d_cols_hc, col_stride, cn, n, log_n);
  rc = check_cuda(cudaGetLastError(), "permute to canonic");
  count_launch();
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
  // 4. ZK blinding: column c += r_c * Z_H
  if (rc == VS_OK && h_blind) {
    const uint32_t* zh = nullptr;
    for (uint32_t c = 0; c < n_cols && rc == VS_OK; c++) {
      if (!h_blind[c]) continue;
      if (!zh) rc = zh_table(log_n, log_eval, st, &zh);
      if (rc == VS_OK) {
        axpy_kernel<<<blocks_for(N, 256), 256, 0, st>>>(h_blind[c], zh, d_eval_cn + c * N, N);
        rc = check_cuda(cudaGetLastError(), "blinding");
        count_launch();
      }
    }
  }
  // 5. half-coset natural copy of the evaluations (the reference's constraint kernels read it)
  if (rc == VS_OK && d_eval_hc) {
    permute_kernel<false><<<dim3(blocks_for(N, 256), n_cols), 256, 0, st>>>(d_eval_cn, N, d_eval_hc, N, log_eval);
    rc = check_cuda(cudaGetLastError(), "permute to half-coset");
    count_launch();
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
      if (rc == VS_OK) rc = merkle_tile_roots(leaf, N, 10, tiles, st);
      if (rc == VS_OK) rc = merkle_root(LeafHashes{tiles}, N / 1024, d_root, st);
      if (!d_tile_roots && tiles) cudaFreeAsync(tiles, st);
    }
  }
  return rc;
}
