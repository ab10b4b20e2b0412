// Internal, stream-ordered launchers of the OODS numerator and quotient-combine
// kernels (quotient.cu), for device-resident callers that know their pointers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace vs {

// numer[row] = sum_i (c_i * cols[idx_i][row] - b_i), SoA outputs o[0..3]. All
// tables are device memory. vec: every column read, every output and n_rows
// allow 128-bit access (16-byte aligned, n_rows a multiple of 4).
int launch_accumulate_numerators(const uint32_t* const* d_cols, const uint32_t* d_idx, const uint32_t* d_b,
                                 const uint32_t* d_c, uint32_t n_batch, uint32_t n_rows, uint32_t* const o[4],
                                 bool vec, cudaStream_t st);
// Two numerators from one pass over the columns: oa = sum_k ca_k cols[k] - bsum_a,
// ob = sum_k cb_k cols[k] - bsum_b (cb_k = 0 where the second sample does not
// open column k). ca, cb: device QM31 per column (16-byte aligned); bsums: host.
// Every column and output must allow 64-bit access and n_rows must be even.
int launch_accumulate_numerators2(const uint32_t* const* d_cols, const uint32_t* d_ca, const uint32_t* d_cb,
                                  const uint32_t bsum_a[4], const uint32_t bsum_b[4], uint32_t n_cols, uint32_t n_rows,
                                  uint32_t* const oa[4], uint32_t* const ob[4], cudaStream_t st);
// q[row] = sum_j (numer_j[lift(row)] - A_j y) / D_j(row), tables in device memory.
int launch_quotients_combine(const uint32_t* spx, const uint32_t* spy, const uint32_t* fla,
                             const uint32_t* const* n0, const uint32_t* const* n1, const uint32_t* const* n2,
                             const uint32_t* const* n3, const uint32_t* acc_log, uint32_t n_accs,
                             const uint32_t* dxs, const uint32_t* dys, uint32_t lifting_log, uint32_t n_rows,
                             uint32_t* const o[4], cudaStream_t st);

}  // namespace vs
