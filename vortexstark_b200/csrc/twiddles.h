// Internal twiddle-table API shared by the NTT, FRI and prover paths.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "vs_field.cuh"

namespace vs {

enum { TW_NATIVE = 0, TW_STWO = 1 };
enum { COSET_HALF_COSET = 0, COSET_HALF_ODDS = 1, COSET_SUBGROUP = 2 };
// Fold twiddles only: the circle fold of a BRT-canonic evaluation on
// CanonicCoset(L), 1/y(half_odds(L-1).at(brev_{L-1}(i))) (cairo_air/prover.rs:2327-2335).
enum { FOLD_CANONIC_CIRCLE = 3 };

struct TwiddleSet {
  int kind = 0;
  uint32_t log_n = 0;
  uint32_t* mem = nullptr;
  // native: line/iline (n-1 words, reference layout), circle/icircle (n/2),
  //         each table 16-byte aligned
  // stwo:   line = forward flat table (n/2), iline = inverse flat table (n/2)
  uint32_t* line = nullptr;
  uint32_t* iline = nullptr;
  uint32_t* circle = nullptr;
  uint32_t* icircle = nullptr;
  std::vector<uint32_t> offsets, sizes;  // native per-line-layer (host)
  uint64_t bytes = 0;                    // device bytes of mem
};

struct HostCoset {
  cpt initial, step;
  uint32_t log_size;
};
HostCoset host_coset(int which, uint32_t log_size);
cpt host_repeated_double(cpt p, uint32_t k);

// Cached per (device, kind, log_n); built on the device on first use.
int get_twiddles(int kind, uint32_t log_n, const TwiddleSet** out, cudaStream_t st);
// FRI fold twiddles 1/coord(domain.at(bitrev(2i))) for the coset `which`
// (half_coset -> y, half_odds -> x, FOLD_CANONIC_CIRCLE -> y), cached per
// (device, which, log_n).
int get_fold_twiddles(int which, uint32_t log_n, const uint32_t** out, cudaStream_t st);
int release_twiddles();
// Device bytes held by the cached twiddle and fold-twiddle tables of a device.
uint64_t twiddle_cache_bytes(int device);
// Bytes get_twiddles(kind, log_n) (kind < 16) or get_fold_twiddles(kind - 16, log_n)
// would allocate on `device`: 0 when the table is cached.
uint64_t twiddle_bytes_if_missing(int device, int kind, uint32_t log_n);
// Frees the cached vanishing-polynomial tables of the Cairo group commit (cairo.cu).
void release_zh_tables();

int launch_batch_inverse(const uint32_t* in, uint32_t* out, uint64_t n, cudaStream_t st);
int launch_coset_points(cpt initial, cpt step, uint32_t* ox, uint32_t* oy, uint64_t n, cudaStream_t st);

}  // namespace vs
