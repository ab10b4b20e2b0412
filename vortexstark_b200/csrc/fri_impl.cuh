// Device-side FRI fold helpers shared by the fold kernels and the prover.
#pragma once
#include <cstdint>

#include "vs_blake2s.cuh"
#include "vs_field.cuh"
#include "vs_mem.cuh"

namespace vs {

__device__ __forceinline__ qm31 load_q(const uint32_t* const s[4], uint64_t i) {
  return {{s[0][i], s[1][i], s[2][i], s[3][i]}};
}

// r = (f0 + f1) + alpha * tw * (f0 - f1)   (fri.cu:10-39)
__device__ __forceinline__ qm31 fold_pair(qm31 f0, qm31 f1, qm31 alpha, uint32_t tw) {
  return qadd(qadd(f0, f1), qmul(alpha, qscale(qsub(f0, f1), tw)));
}

struct Soa4Ptrs {
  const uint32_t* c[4];
};
struct Soa4Out {
  uint32_t* c[4];
};

// Folded SoA4 layer as Merkle leaves: leaf i = fold(src[2i], src[2i+1]); written to dst.
// circle = true also accumulates dst = dst * alpha^2 + f' when accumulate is set
// (fri.cu:44-78); the prover's destination starts at zero, so accumulate = false
// there and dst is not read.
struct LeafFold {
  Soa4Ptrs src;
  Soa4Out dst;
  const uint32_t* tw;
  qm31 alpha, alpha_sq;
  int accumulate;
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    uint2 a0 = ld2(src.c[0] + 2 * i);
    uint2 a1 = ld2(src.c[1] + 2 * i);
    uint2 a2 = ld2(src.c[2] + 2 * i);
    uint2 a3 = ld2(src.c[3] + 2 * i);
    qm31 f0{{a0.x, a1.x, a2.x, a3.x}}, f1{{a0.y, a1.y, a2.y, a3.y}};
    qm31 r = fold_pair(f0, f1, alpha, __ldg(tw + i));
    if (accumulate) {
      qm31 prev{{dst.c[0][i], dst.c[1][i], dst.c[2][i], dst.c[3][i]}};
      r = qadd(qmul(prev, alpha_sq), r);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) dst.c[k][i] = r.v[k];
    uint32_t m[16] = {0};
    m[0] = r.v[0];
    m[1] = r.v[1];
    m[2] = r.v[2];
    m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};

}  // namespace vs
