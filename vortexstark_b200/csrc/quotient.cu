// Constraint and OODS quotient kernels: drop-in for cuda/constraint.cu and
// cuda/quotient.cu, plus the elementwise helpers of cuda/fields.cu.
#include <algorithm>
#include <vector>

#include "quotient.h"
#include "vs_common.cuh"
#include "vs_field.cuh"
#include "vs_mem.cuh"

namespace vs {

// q[i] = alpha * (t[(i+2)%n] - (t[(i+1)%n] + t[i]))   (constraint.cu:10-64)
__global__ void fib_quotient_kernel(const uint32_t* __restrict__ t, uint32_t* __restrict__ o0, uint32_t* __restrict__ o1,
                                    uint32_t* __restrict__ o2, uint32_t* __restrict__ o3, qm31 alpha, uint32_t offset,
                                    uint32_t chunk_n, uint32_t global_n) {
  uint32_t li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= chunk_n) return;
  uint32_t i = offset + li;
  uint32_t i1 = i + 1 == global_n ? 0 : i + 1;
  uint32_t i2 = i1 + 1 == global_n ? 0 : i1 + 1;
  uint32_t c = sub(t[i2], add(t[i1], t[i]));
  qm31 r = qscale(alpha, c);
  o0[li] = r.v[0];
  o1[li] = r.v[1];
  o2[li] = r.v[2];
  o3[li] = r.v[3];
}

__global__ void zero_pad_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t src_n,
                                uint32_t dst_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < dst_n) dst[i] = i < src_n ? src[i] : 0u;
}
__global__ void interleave_kernel(const uint32_t* __restrict__ e, const uint32_t* __restrict__ o,
                                  uint32_t* __restrict__ out, uint32_t half_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < half_n) st2(out + 2 * (uint64_t)i, make_uint2(e[i], o[i]));
}

// numer[row] = sum_i (c_i * f_i[row] - b_i)   (quotient.cu:25-68), computed as
// sum_i c_i f_i - sum_i b_i. Products c_i * f_i (< 2^62) are accumulated per limb
// with 64-bit multiply-adds; every three terms the sum is folded to < 2^34
// (2^31 == 1 mod p), so it never overflows (a fold leaves < 2^34, plus at most
// three products < 2^62 each), and it is reduced once at the end. sum_i b_i is
// formed once per CTA. Each thread takes AN_ROWS rows and a three-column group
// keeps 3 loads per row in flight. VEC: the rows are consecutive and read and
// written with 128-bit accesses (the host has checked that every column, output
// and the row count allow it); otherwise the rows are strided by the grid and
// every access is a coalesced word. Same canonical result as the term-by-term
// reference.
constexpr int AN_ROWS = 4;
__device__ __forceinline__ uint64_t fold31(uint64_t a) { return (a & VS_P) + (a >> 31); }
__device__ __forceinline__ uint32_t reduce64(uint64_t a) {
  a = fold31(fold31(a));  // < 2^31 + 8
  return canon((uint32_t)a);
}
template <bool VEC>
__global__ void accumulate_numerators_kernel(const uint32_t* const* __restrict__ cols, const uint32_t* __restrict__ idx,
                                             const uint32_t* __restrict__ b, const uint32_t* __restrict__ c,
                                             uint32_t n_batch, uint32_t n_rows, uint32_t* __restrict__ o0,
                                             uint32_t* __restrict__ o1, uint32_t* __restrict__ o2,
                                             uint32_t* __restrict__ o3) {
  __shared__ uint32_t bsum[4];
  if (threadIdx.x < 4) {
    uint32_t acc = 0;
    for (uint32_t k = 0; k < n_batch; k++) acc = add(acc, __ldg(b + 4 * k + threadIdx.x));
    bsum[threadIdx.x] = acc;
  }
  __syncthreads();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t stride = VEC ? 1u : gridDim.x * blockDim.x;   // between a thread's rows
  const uint32_t t0 = VEC ? tid * AN_ROWS : tid;
  if (t0 >= n_rows) return;
  uint64_t acc[AN_ROWS][4];
#pragma unroll
  for (int r = 0; r < AN_ROWS; r++)
#pragma unroll
    for (int l = 0; l < 4; l++) acc[r][l] = 0;
  auto load = [&](uint32_t k, uint32_t (&f)[AN_ROWS]) {
    const uint32_t* col = cols[idx[k]];
    if (VEC) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(col + t0));
      f[0] = v.x; f[1] = v.y; f[2] = v.z; f[3] = v.w;
    } else {
#pragma unroll
      for (int r = 0; r < AN_ROWS; r++) {
        const uint32_t row = t0 + r * stride;
        f[r] = row < n_rows ? __ldg(col + row) : 0u;
      }
    }
  };
  auto mac = [&](uint32_t k, const uint32_t (&f)[AN_ROWS]) {
    const uint32_t cl[4] = {__ldg(c + 4 * k), __ldg(c + 4 * k + 1), __ldg(c + 4 * k + 2), __ldg(c + 4 * k + 3)};
#pragma unroll
    for (int r = 0; r < AN_ROWS; r++)
#pragma unroll
      for (int l = 0; l < 4; l++) acc[r][l] += (uint64_t)cl[l] * f[r];
  };
  auto fold_all = [&]() {
#pragma unroll
    for (int r = 0; r < AN_ROWS; r++)
#pragma unroll
      for (int l = 0; l < 4; l++) acc[r][l] = fold31(acc[r][l]);
  };
  uint32_t k = 0;
  for (; k + 3 <= n_batch; k += 3) {
    uint32_t f0[AN_ROWS], f1[AN_ROWS], f2[AN_ROWS];
    load(k, f0);
    load(k + 1, f1);
    load(k + 2, f2);
    mac(k, f0);
    mac(k + 1, f1);
    mac(k + 2, f2);
    fold_all();
  }
  for (; k < n_batch; k++) {  // at most two: no fold needed before the final reduction
    uint32_t f0[AN_ROWS];
    load(k, f0);
    mac(k, f0);
  }
  uint32_t* out[4] = {o0, o1, o2, o3};
  if (VEC) {
#pragma unroll
    for (int l = 0; l < 4; l++)
      *reinterpret_cast<uint4*>(out[l] + t0) =
          make_uint4(sub(reduce64(acc[0][l]), bsum[l]), sub(reduce64(acc[1][l]), bsum[l]),
                     sub(reduce64(acc[2][l]), bsum[l]), sub(reduce64(acc[3][l]), bsum[l]));
  } else {
#pragma unroll
    for (int r = 0; r < AN_ROWS; r++) {
      const uint32_t row = t0 + r * stride;
      if (row < n_rows) {
#pragma unroll
        for (int l = 0; l < 4; l++) out[l][row] = sub(reduce64(acc[r][l]), bsum[l]);
      }
    }
  }
}

// Two numerators in one pass over the columns (the DEEP quotient's z and z_next
// samples read mostly the same columns): numer_a = sum_k ca_k f_k - sum b_a and
// numer_b = sum_k cb_k f_k - sum b_b, with cb_k = 0 for a column the second
// sample does not open. Same accumulation as above (64-bit multiply-adds folded
// every three columns, six columns' loads in flight); each thread takes two
// consecutive rows with 64-bit accesses (the host checks alignment).
struct Numer2Out {
  uint32_t* o[8];  // a limbs 0..3, then b limbs 0..3
};
constexpr int AN2_ROWS = 2;
__global__ void __launch_bounds__(256, 3) accumulate_numerators2_kernel(
    const uint32_t* const* __restrict__ cols, const uint32_t* __restrict__ ca, const uint32_t* __restrict__ cb,
    uint32_t bsum_a0, uint32_t bsum_a1, uint32_t bsum_a2, uint32_t bsum_a3, uint32_t bsum_b0, uint32_t bsum_b1,
    uint32_t bsum_b2, uint32_t bsum_b3, uint32_t n_cols, uint32_t n_rows, Numer2Out out) {
  const uint32_t t0 = (blockIdx.x * blockDim.x + threadIdx.x) * AN2_ROWS;
  if (t0 >= n_rows) return;
  uint64_t acc[2][AN2_ROWS][4];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int r = 0; r < AN2_ROWS; r++)
#pragma unroll
      for (int l = 0; l < 4; l++) acc[a][r][l] = 0;
  auto mac = [&](uint32_t k, uint2 f) {
    const uint4 xa = __ldg(reinterpret_cast<const uint4*>(ca) + k), xb = __ldg(reinterpret_cast<const uint4*>(cb) + k);
    const uint32_t la[4] = {xa.x, xa.y, xa.z, xa.w}, lb[4] = {xb.x, xb.y, xb.z, xb.w};
#pragma unroll
    for (int l = 0; l < 4; l++) {
      acc[0][0][l] += (uint64_t)la[l] * f.x;
      acc[0][1][l] += (uint64_t)la[l] * f.y;
      acc[1][0][l] += (uint64_t)lb[l] * f.x;
      acc[1][1][l] += (uint64_t)lb[l] * f.y;
    }
  };
  auto fold_all = [&]() {
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int r = 0; r < AN2_ROWS; r++)
#pragma unroll
        for (int l = 0; l < 4; l++) acc[a][r][l] = fold31(acc[a][r][l]);
  };
  auto ld = [&](uint32_t k) { return __ldg(reinterpret_cast<const uint2*>(cols[k] + t0)); };
  uint32_t k = 0;
  for (; k + 6 <= n_cols; k += 6) {  // six columns in flight, folded every three
    const uint2 f0 = ld(k), f1 = ld(k + 1), f2 = ld(k + 2), f3 = ld(k + 3), f4 = ld(k + 4), f5 = ld(k + 5);
    mac(k, f0);
    mac(k + 1, f1);
    mac(k + 2, f2);
    fold_all();
    mac(k + 3, f3);
    mac(k + 4, f4);
    mac(k + 5, f5);
    fold_all();
  }
  for (; k + 3 <= n_cols; k += 3) {
    const uint2 f0 = ld(k), f1 = ld(k + 1), f2 = ld(k + 2);
    mac(k, f0);
    mac(k + 1, f1);
    mac(k + 2, f2);
    fold_all();
  }
  for (; k < n_cols; k++) mac(k, ld(k));  // at most two more: no fold needed before the reduction
  const uint32_t bs[2][4] = {{bsum_a0, bsum_a1, bsum_a2, bsum_a3}, {bsum_b0, bsum_b1, bsum_b2, bsum_b3}};
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int l = 0; l < 4; l++)
      *reinterpret_cast<uint2*>(out.o[4 * a + l] + t0) =
          make_uint2(sub(reduce64(acc[a][0][l]), bs[a][l]), sub(reduce64(acc[a][1][l]), bs[a][l]));
}

// q[row] = sum_j (numer_j[lift(row)] - A_j * y) * D_j(row)^-1 with
// D = (Re sx - x) Im sy - (Re sy - y) Im sx in CM31   (quotient.cu:101-197).
// The reference inverts every D with a Fermat power; here each thread takes
// QC_ROWS rows (strided by the grid for coalescing) and inverts their D_j with
// one inverse and a Montgomery product chain. A zero D is left out of the chain
// and gets inverse 0, as the Fermat power gives, so results are identical.
constexpr int QC_ROWS = 4;
__device__ __forceinline__ bool czero(cm31 x) { return (x.a | x.b) == 0; }
__global__ void quotients_combine_kernel(const uint32_t* __restrict__ spx, const uint32_t* __restrict__ spy,
                                         const uint32_t* __restrict__ fla, const uint32_t* const* __restrict__ n0,
                                         const uint32_t* const* __restrict__ n1, const uint32_t* const* __restrict__ n2,
                                         const uint32_t* const* __restrict__ n3, const uint32_t* __restrict__ acc_log,
                                         uint32_t n_accs, const uint32_t* __restrict__ dxs,
                                         const uint32_t* __restrict__ dys, uint32_t lifting_log, uint32_t n_rows,
                                         uint32_t* __restrict__ o0, uint32_t* __restrict__ o1,
                                         uint32_t* __restrict__ o2, uint32_t* __restrict__ o3) {
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t dx[QC_ROWS], dy[QC_ROWS];
  qm31 q[QC_ROWS];
#pragma unroll
  for (int i = 0; i < QC_ROWS; i++) {
    const uint32_t row = t0 + i * stride;
    const bool live = row < n_rows;
    dx[i] = live ? dxs[row] : 0u;
    dy[i] = live ? dys[row] : 0u;
    q[i] = qzero();
  }
  for (uint32_t j = 0; j < n_accs; j++) {
    const cm31 prx{spx[4 * j], spx[4 * j + 1]}, pix{spx[4 * j + 2], spx[4 * j + 3]};
    const cm31 pry{spy[4 * j], spy[4 * j + 1]}, piy{spy[4 * j + 2], spy[4 * j + 3]};
    const qm31 a{{fla[4 * j], fla[4 * j + 1], fla[4 * j + 2], fla[4 * j + 3]}};
    const uint32_t ratio = lifting_log - acc_log[j];
    const uint32_t *p0 = n0[j], *p1 = n1[j], *p2 = n2[j], *p3 = n3[j];
    cm31 den[QC_ROWS], pre[QC_ROWS];
    cm31 run{1, 0};
#pragma unroll
    for (int i = 0; i < QC_ROWS; i++) {
      den[i] = csub(cmul(csub(prx, cm31{dx[i], 0}), piy), cmul(csub(pry, cm31{dy[i], 0}), pix));
      pre[i] = run;
      if (!czero(den[i])) run = cmul(run, den[i]);
    }
    cm31 inv = cinv(run);  // run is never zero
#pragma unroll
    for (int i = QC_ROWS - 1; i >= 0; i--) {
      const bool z = czero(den[i]);
      const cm31 di = z ? cm31{0, 0} : cmul(inv, pre[i]);
      if (!z) inv = cmul(inv, den[i]);
      const uint32_t row = t0 + i * stride;
      if (row < n_rows) {
        const uint32_t li = ((row >> (ratio + 1)) << 1) + (row & 1);
        const qm31 pn{{p0[li], p1[li], p2[li], p3[li]}};
        q[i] = qadd(q[i], qscale_c(qsub(pn, qscale(a, dy[i])), di));
      }
    }
  }
#pragma unroll
  for (int i = 0; i < QC_ROWS; i++) {
    const uint32_t row = t0 + i * stride;
    if (row < n_rows) {
      o0[row] = q[i].v[0];
      o1[row] = q[i].v[1];
      o2[row] = q[i].v[2];
      o3[row] = q[i].v[3];
    }
  }
}

__global__ void m31_binop_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                 uint32_t* __restrict__ out, uint32_t n, int is_mul) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = is_mul ? mul(a[i], b[i]) : add(a[i], b[i]);
}

// SplitMix64 counter stream -> uniform M31 (see vs_fill_uniform_m31).
__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t counter) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * counter;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__global__ void fill_uniform_kernel(uint32_t* __restrict__ out, uint64_t n, uint64_t seed, uint64_t offset) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) {
    uint64_t k = offset + i;
    uint32_t v = (uint32_t)(splitmix_at(seed, k + 1) >> 33);
    if (v == VS_P) {
      v = (uint32_t)(splitmix_at(seed, k + 2) >> 33);
      if (v == VS_P) v = 0;
    }
    out[i] = v;
  }
}

int launch_accumulate_numerators(const uint32_t* const* d_cols, const uint32_t* d_idx, const uint32_t* d_b,
                                 const uint32_t* d_c, uint32_t n_batch, uint32_t n_rows, uint32_t* const o[4],
                                 bool vec, cudaStream_t st) {
  if (!n_rows) return VS_OK;
  const unsigned blocks = blocks_for((n_rows + AN_ROWS - 1) / AN_ROWS, 256);
  if (vec)
    accumulate_numerators_kernel<true><<<blocks, 256, 0, st>>>(d_cols, d_idx, d_b, d_c, n_batch, n_rows, o[0], o[1],
                                                               o[2], o[3]);
  else
    accumulate_numerators_kernel<false><<<blocks, 256, 0, st>>>(d_cols, d_idx, d_b, d_c, n_batch, n_rows, o[0], o[1],
                                                                o[2], o[3]);
  VS_LAUNCHED("accumulate_numerators_kernel");
  return VS_OK;
}
int launch_accumulate_numerators2(const uint32_t* const* d_cols, const uint32_t* d_ca, const uint32_t* d_cb,
                                  const uint32_t bsum_a[4], const uint32_t bsum_b[4], uint32_t n_cols, uint32_t n_rows,
                                  uint32_t* const oa[4], uint32_t* const ob[4], cudaStream_t st) {
  if (!n_rows) return VS_OK;
  if (n_rows % AN2_ROWS) return set_error(VS_ERR_INVALID, "numerators2: rows not a multiple of %d", AN2_ROWS);
  Numer2Out out;
  for (int l = 0; l < 4; l++) { out.o[l] = oa[l]; out.o[4 + l] = ob[l]; }
  accumulate_numerators2_kernel<<<blocks_for(n_rows / AN2_ROWS, 256), 256, 0, st>>>(
      d_cols, d_ca, d_cb, bsum_a[0], bsum_a[1], bsum_a[2], bsum_a[3], bsum_b[0], bsum_b[1], bsum_b[2], bsum_b[3],
      n_cols, n_rows, out);
  VS_LAUNCHED("accumulate_numerators2_kernel");
  return VS_OK;
}
int launch_quotients_combine(const uint32_t* spx, const uint32_t* spy, const uint32_t* fla,
                             const uint32_t* const* n0, const uint32_t* const* n1, const uint32_t* const* n2,
                             const uint32_t* const* n3, const uint32_t* acc_log, uint32_t n_accs,
                             const uint32_t* dxs, const uint32_t* dys, uint32_t lifting_log, uint32_t n_rows,
                             uint32_t* const o[4], cudaStream_t st) {
  if (!n_rows) return VS_OK;
  quotients_combine_kernel<<<blocks_for((n_rows + QC_ROWS - 1) / QC_ROWS, 256), 256, 0, st>>>(
      spx, spy, fla, n0, n1, n2, n3, acc_log, n_accs, dxs, dys, lifting_log, n_rows, o[0], o[1], o[2], o[3]);
  VS_LAUNCHED("quotients_combine_kernel");
  return VS_OK;
}

}  // namespace vs

using namespace vs;

extern "C" {

void cuda_fibonacci_quotient_chunk_stream(const uint32_t* trace, uint32_t* o0, uint32_t* o1, uint32_t* o2, uint32_t* o3,
                                          const uint32_t* alpha, uint32_t offset, uint32_t chunk_n, uint32_t global_n,
                                          vs_stream_t stream) {
  if (!chunk_n) return;
  fib_quotient_kernel<<<blocks_for(chunk_n, 256), 256, 0, (cudaStream_t)stream>>>(
      trace, o0, o1, o2, o3, qm31{{alpha[0], alpha[1], alpha[2], alpha[3]}}, offset, chunk_n, global_n);
  check_cuda(cudaGetLastError(), "cuda_fibonacci_quotient");
}
void cuda_fibonacci_quotient_chunk(const uint32_t* trace, uint32_t* o0, uint32_t* o1, uint32_t* o2, uint32_t* o3,
                                   const uint32_t* alpha, uint32_t offset, uint32_t chunk_n, uint32_t global_n) {
  cuda_fibonacci_quotient_chunk_stream(trace, o0, o1, o2, o3, alpha, offset, chunk_n, global_n, 0);
}
void cuda_fibonacci_quotient(const uint32_t* trace, uint32_t* o0, uint32_t* o1, uint32_t* o2, uint32_t* o3,
                             const uint32_t* alpha, uint32_t n) {
  cuda_fibonacci_quotient_chunk_stream(trace, o0, o1, o2, o3, alpha, 0, n, n, 0);
}
void cuda_zero_pad(const uint32_t* src, uint32_t* dst, uint32_t src_n, uint32_t dst_n) {
  if (!dst_n) return;
  zero_pad_kernel<<<blocks_for(dst_n, 256), 256>>>(src, dst, src_n, dst_n);
  check_cuda(cudaGetLastError(), "cuda_zero_pad");
}
void cuda_interleave_u32(const uint32_t* even, const uint32_t* odd, uint32_t* out, uint32_t half_n) {
  if (!half_n) return;
  interleave_kernel<<<blocks_for(half_n, 256), 256>>>(even, odd, out, half_n);
  check_cuda(cudaGetLastError(), "cuda_interleave_u32");
}
void cuda_accumulate_numerators(const uint32_t* const* cols, const uint32_t* idx, const uint32_t* b, const uint32_t* c,
                                uint32_t n_batch, uint32_t n_rows, uint32_t* o0, uint32_t* o1, uint32_t* o2,
                                uint32_t* o3) {
  if (!n_rows) return;
  // The 128-bit variant needs every column the batch reads, the outputs and the
  // row count to be multiples of 16 bytes; the column table is device memory, so
  // its used entries are read back (small, once per call) to decide.
  bool vec = n_rows % AN_ROWS == 0;
  for (uint32_t* o : {o0, o1, o2, o3}) vec = vec && (reinterpret_cast<uintptr_t>(o) & 15) == 0;
  if (vec && n_batch) {
    std::vector<uint32_t> h_idx(n_batch);
    if (check_cuda(cudaMemcpy(h_idx.data(), idx, n_batch * 4, cudaMemcpyDeviceToHost), "accumulate: indices") != VS_OK) return;
    uint32_t n_ptrs = 0;
    for (uint32_t k : h_idx) n_ptrs = std::max(n_ptrs, k + 1);
    std::vector<const uint32_t*> h_cols(n_ptrs);
    if (check_cuda(cudaMemcpy(h_cols.data(), cols, n_ptrs * sizeof(void*), cudaMemcpyDeviceToHost), "accumulate: columns") != VS_OK) return;
    for (uint32_t k : h_idx) vec = vec && (reinterpret_cast<uintptr_t>(h_cols[k]) & 15) == 0;
  }
  const unsigned blocks = blocks_for((n_rows + AN_ROWS - 1) / AN_ROWS, 256);
  if (vec) accumulate_numerators_kernel<true><<<blocks, 256>>>(cols, idx, b, c, n_batch, n_rows, o0, o1, o2, o3);
  else accumulate_numerators_kernel<false><<<blocks, 256>>>(cols, idx, b, c, n_batch, n_rows, o0, o1, o2, o3);
  check_cuda(cudaGetLastError(), "cuda_accumulate_numerators");
}
void cuda_compute_quotients_combine(const uint32_t* spx, const uint32_t* spy, const uint32_t* fla,
                                    const uint32_t* const* n0, const uint32_t* const* n1, const uint32_t* const* n2,
                                    const uint32_t* const* n3, const uint32_t* acc_log, uint32_t n_accs,
                                    const uint32_t* dxs, const uint32_t* dys, uint32_t lifting_log, uint32_t n_rows,
                                    uint32_t* o0, uint32_t* o1, uint32_t* o2, uint32_t* o3) {
  if (!n_rows) return;
  quotients_combine_kernel<<<blocks_for((n_rows + QC_ROWS - 1) / QC_ROWS, 256), 256>>>(
      spx, spy, fla, n0, n1, n2, n3, acc_log, n_accs, dxs, dys, lifting_log, n_rows, o0, o1, o2, o3);
  check_cuda(cudaGetLastError(), "cuda_compute_quotients_combine");
}
void cuda_m31_add(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n) {
  if (!n) return;
  m31_binop_kernel<<<blocks_for(n, 256), 256>>>(a, b, out, n, 0);
  check_cuda(cudaGetLastError(), "cuda_m31_add");
}
void cuda_m31_mul(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n) {
  if (!n) return;
  m31_binop_kernel<<<blocks_for(n, 256), 256>>>(a, b, out, n, 1);
  check_cuda(cudaGetLastError(), "cuda_m31_mul");
}
void cuda_device_sync(void) { check_cuda(cudaDeviceSynchronize(), "cuda_device_sync"); }

int vs_fill_uniform_m31(uint32_t* d_out, uint64_t n, uint64_t seed, uint64_t offset, vs_stream_t stream) {
  clear_error();
  if (!d_out) return set_error(VS_ERR_INVALID, "vs_fill_uniform_m31: null output");
  if (!n) return VS_OK;
  unsigned blocks = (unsigned)((n + 255) / 256);
  unsigned cap = (unsigned)sm_count() * 16;
  if (blocks > cap) blocks = cap;
  fill_uniform_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(d_out, n, seed, offset);
  VS_LAUNCHED("fill_uniform_kernel");
  return VS_OK;
}

}  // extern "C"
