// FRI folds (drop-in for cuda/fri.cu) and the fused fold -> commit chain.
//
// A fold layer is one pass: each leaf of the new layer's Merkle tree is the
// folded value itself, so the fold runs inside the Merkle subtree kernel's leaf
// functor (it writes the folded value and hashes it in registers) and the layer
// is never re-read for its commitment.
#include <algorithm>

#include "fri.h"
#include "fri_impl.cuh"
#include "merkle.h"
#include "twiddles.h"
#include "vs_field.cuh"

namespace vs {

__global__ void fold_line_kernel(Soa4Ptrs in, const uint32_t* __restrict__ tw, Soa4Out out, qm31 alpha,
                                 uint32_t half_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  qm31 f0 = load_q(in.c, 2 * (uint64_t)i), f1 = load_q(in.c, 2 * (uint64_t)i + 1);
  qm31 r = fold_pair(f0, f1, alpha, tw[i]);
#pragma unroll
  for (int k = 0; k < 4; k++) out.c[k][i] = r.v[k];
}
__global__ void fold_circle_kernel(Soa4Out dst, Soa4Ptrs src, const uint32_t* __restrict__ tw, qm31 alpha, qm31 alpha_sq,
                                   uint32_t half_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  qm31 f0 = load_q(src.c, 2 * (uint64_t)i), f1 = load_q(src.c, 2 * (uint64_t)i + 1);
  qm31 fp = fold_pair(f0, f1, alpha, tw[i]);
  qm31 prev{{dst.c[0][i], dst.c[1][i], dst.c[2][i], dst.c[3][i]}};
  qm31 r = qadd(qmul(prev, alpha_sq), fp);
#pragma unroll
  for (int k = 0; k < 4; k++) dst.c[k][i] = r.v[k];
}

// One fold layer + its Merkle root. src/dst are SoA4 plane pointers; `half_n`
// = output size (power of two); twiddles of length half_n.
int fold_commit_layer(const uint32_t* const src[4], uint32_t* const dst[4], const uint32_t* tw, const uint32_t* alpha,
                      const uint32_t* alpha_sq, bool circle_accumulate, uint64_t half_n, uint32_t* d_root,
                      uint32_t* scratch, cudaStream_t st, uint32_t split) {
  LeafFold leaf{};
  for (int k = 0; k < 4; k++) { leaf.src.c[k] = src[k]; leaf.dst.c[k] = dst[k]; }
  leaf.tw = tw;
  for (int k = 0; k < 4; k++) { leaf.alpha.v[k] = alpha[k]; leaf.alpha_sq.v[k] = alpha_sq ? alpha_sq[k] : 0; }
  leaf.accumulate = circle_accumulate ? 1 : 0;
  return merkle_root(leaf, half_n, d_root, st, scratch, split);
}

}  // namespace vs

using namespace vs;

extern "C" {

void cuda_fold_line_soa(const uint32_t* in0, const uint32_t* in1, const uint32_t* in2, const uint32_t* in3,
                        const uint32_t* tw, uint32_t* out0, uint32_t* out1, uint32_t* out2, uint32_t* out3,
                        const uint32_t* alpha, uint32_t half_n) {
  if (!half_n) return;
  fold_line_kernel<<<blocks_for(half_n, 256), 256>>>(Soa4Ptrs{{in0, in1, in2, in3}}, tw, Soa4Out{{out0, out1, out2, out3}},
                                                     qm31{{alpha[0], alpha[1], alpha[2], alpha[3]}}, half_n);
  check_cuda(cudaGetLastError(), "cuda_fold_line_soa");
}

void cuda_fold_circle_into_line_soa(uint32_t* dst0, uint32_t* dst1, uint32_t* dst2, uint32_t* dst3,
                                    const uint32_t* src0, const uint32_t* src1, const uint32_t* src2,
                                    const uint32_t* src3, const uint32_t* tw, const uint32_t* alpha,
                                    const uint32_t* alpha_sq, uint32_t half_n) {
  if (!half_n) return;
  fold_circle_kernel<<<blocks_for(half_n, 256), 256>>>(Soa4Out{{dst0, dst1, dst2, dst3}}, Soa4Ptrs{{src0, src1, src2, src3}},
                                                       tw, qm31{{alpha[0], alpha[1], alpha[2], alpha[3]}},
                                                       qm31{{alpha_sq[0], alpha_sq[1], alpha_sq[2], alpha_sq[3]}}, half_n);
  check_cuda(cudaGetLastError(), "cuda_fold_circle_into_line_soa");
}

int vs_fri_fold_commit(const uint32_t* d_src, uint32_t log_n, const uint32_t* h_alphas, uint32_t* d_work,
                       uint32_t* d_roots, uint32_t* d_last, vs_stream_t stream) {
  clear_error();
  cudaStream_t st = (cudaStream_t)stream;
  if (!d_src || !h_alphas || !d_work || !d_roots || !d_last) return set_error(VS_ERR_INVALID, "vs_fri_fold_commit: null");
  if (log_n < 4 || log_n > 30) return set_error(VS_ERR_INVALID, "vs_fri_fold_commit: log_n %u out of range", log_n);
  const uint64_t N = 1ull << log_n;
  uint32_t* scratch = nullptr;
  VS_CUDA(cudaMallocAsync((void**)&scratch, (merkle_scratch_words_any(N / 2) + 8) * 4, st));
  // FRI layer trees are fastest at a split of at most 5 (34 x 2^24 step: FRI 6.68 ms
  // at split 0, 6.09 at 5, 6.22 at 8, the row-packed root's tuned value; this fold +
  // commit of 2^26 alone: 6.59 / 6.44 / 6.35 / 6.28 / 6.30 / 6.31 / 6.38 ms at splits
  // 2..8); the roots are the same for every split
  const uint32_t split = std::min<uint32_t>(merkle_split(), 5);
  const uint32_t* src[4] = {d_src, d_src + N, d_src + 2 * N, d_src + 3 * N};
  uint32_t* bufs[2] = {d_work, d_work + 2 * N};  // each holds 4 planes of <= N/2 words
  int rc = VS_OK;
  uint32_t cl = log_n;
  for (uint32_t layer = 0; cl > 3 && rc == VS_OK; layer++) {
    const uint64_t half = 1ull << (cl - 1);
    uint32_t* base = bufs[layer & 1];
    uint32_t* dst[4] = {base, base + half, base + 2 * half, base + 3 * half};
    const uint32_t* tw = nullptr;
    rc = get_fold_twiddles(layer == 0 ? COSET_HALF_COSET : COSET_HALF_ODDS, cl, &tw, st);
    if (rc != VS_OK) break;
    rc = fold_commit_layer(src, dst, tw, h_alphas + 4 * layer, nullptr, false, half, d_roots + 8 * layer, scratch, st,
                           split);
    for (int k = 0; k < 4; k++) src[k] = dst[k];
    cl--;
  }
  if (rc == VS_OK) {  // last layer (8 values) to AoS
    for (int k = 0; k < 4; k++)
      rc = rc == VS_OK ? check_cuda(cudaMemcpy2DAsync(d_last + k, 16, src[k], 4, 4, 8, cudaMemcpyDeviceToDevice, st),
                                    "fri last layer")
                       : rc;
  }
  cudaError_t e = cudaFreeAsync(scratch, st);
  if (rc == VS_OK) rc = check_cuda(e, "fri scratch free");
  return rc;
}

}  // extern "C"
