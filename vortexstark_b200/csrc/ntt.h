// Internal NTT API (tiled multi-layer passes, both reference conventions).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace vs {

// Per-layer twiddle tables: layer[j][h] is the twiddle of layer j, group h.
// For the stwo convention the circle layer (j = 0) reads (x, y) pairs from
// `flat` (the first line layer) instead.
struct NttTw {
  const uint32_t* layer[32];
  const uint32_t* flat;
  int stwo;
  int vec;  // every layer table is aligned to min(16 B, its size): twiddles may be read with vector loads
};
// Sets tw.vec from the table pointers of a transform of 2^log_n points.
void ntt_tw_check_alignment(NttTw& tw, uint32_t log_n);

struct NttPass {
  const uint32_t* src;
  uint32_t* dst;
  const uint32_t* const* src_cols;  // optional device pointer arrays (one per column)
  uint32_t* const* dst_cols;
  uint64_t src_stride, dst_stride;  // column strides in words when no pointer arrays
  uint32_t log_n;                   // log2 of the domain the layer indices refer to
  uint32_t a, b, c;                 // layers [a, b]; c low index bits per tile row
  uint32_t src_mask;
  uint32_t scale;                   // inverse scale applied after the last layer (0: none)
  uint32_t items;                   // tiles per CTA before it retires (host side; 0: 8)
  uint32_t radix;                   // 3: chunk-round kernels, 5: word-round kernels (host side; 0: 3)
  NttTw tw;
};

struct NttColumns {
  const uint32_t* src;
  uint32_t* dst;
  const uint32_t* const* src_cols;
  uint32_t* const* dst_cols;
  uint64_t src_stride, dst_stride;
  uint32_t n_cols;
};

struct PassRange { uint32_t a, b, c; };

// Launch shape of the transforms of one size, set by the autotuner
// (vs_autotune_lde) or vs_ntt_plan_set. Zero fields take the defaults. A plan
// changes how the butterfly layers are grouped into kernels, never the result.
struct NttPlan {
  uint32_t lower;      // layers of the first (lower) pass; default 13
  uint32_t items;      // tiles a pass CTA transforms before retiring; default 8
  uint32_t radix;      // layers per register round above the first five: 3 (16-byte chunks) or 5 (words); default 3
};
NttPlan ntt_plan(uint32_t log_n);
bool ntt_plan_valid(uint32_t log_n, const NttPlan& p);
std::vector<NttPlan> ntt_plan_candidates(uint32_t log_n);
std::vector<PassRange> plan_passes(uint32_t log_n, uint32_t lower = 0);
uint32_t inv_n_scale(uint32_t log_n);
NttTw native_tw(const uint32_t* line, const uint32_t* circle, const uint32_t* offsets, uint32_t n_line_layers);
NttTw stwo_tw(const uint32_t* flat, uint32_t log_n);
int tw_for(int kind, uint32_t log_n, bool forward, NttTw* out, cudaStream_t st);

// Full transform (in place when src == dst).
int ntt_transform(const NttColumns& io, uint32_t log_n, const NttTw& tw, bool forward, cudaStream_t st);
// interpolate(log_n) -> zero-pad -> evaluate(log_n + B); src is left untouched.
int ntt_lde(const NttColumns& io, uint32_t log_n, uint32_t B, const NttTw& tw_inv, const NttTw& tw_fwd,
            cudaStream_t st);
int lde_cached(int kind, const uint32_t* src, uint64_t src_stride, uint32_t* dst, uint64_t dst_stride,
               uint32_t n_cols, uint32_t log_n, uint32_t B, cudaStream_t st);

}  // namespace vs
