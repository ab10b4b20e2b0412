// Internal FRI API.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace vs {

// One fold layer (circle or line, per the twiddles given) fused with its SoA4
// Merkle commitment. alpha / alpha_sq are host QM31 (4 words). The fold of a
// circle layer into a zeroed destination equals the plain fold, so the prover
// passes circle_accumulate = false.
int fold_commit_layer(const uint32_t* const src[4], uint32_t* const dst[4], const uint32_t* tw, const uint32_t* alpha,
                      const uint32_t* alpha_sq, bool circle_accumulate, uint64_t half_n, uint32_t* d_root,
                      uint32_t* scratch, cudaStream_t st, uint32_t split = 0);

}  // namespace vs
