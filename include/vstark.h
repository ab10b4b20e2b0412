/*
 * vstark.h — C ABI of libvstark, a B200-native (sm_100a) implementation of the
 * VortexSTARK polynomial-commitment hot path.
 *
 * Two groups of entry points:
 *
 * 1. Drop-in symbols with the exact names, argument meaning, ownership and
 *    synchronisation of the reference's CUDA static library (declared in the
 *    reference at src/cuda/ffi.rs, defined in cuda/*.cu). Each cites the
 *    reference declaration it replaces. As in the reference: all pointers are
 *    device pointers unless named h_* or documented "host"; the caller owns all
 *    device memory; launches go to the legacy default stream unless a stream is
 *    passed; functions return void. A failed launch is recorded and can be read
 *    with vs_last_error() (the reference surfaces it through cudaGetLastError).
 *
 * 2. vs_* entry points (no reference counterpart) returning a vs_status, used by
 *    the batched / served paths and by bench.py.
 *
 * All field values are canonical M31 residues (< 2^31 - 1), as in the reference.
 */
#ifndef VSTARK_H
#define VSTARK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* vs_stream_t; /* == cudaStream_t */

enum {
  VS_OK = 0,
  VS_ERR_INVALID = 1,  /* bad argument (size not a power of two, null pointer, ...) */
  VS_ERR_CUDA = 2,     /* CUDA runtime error */
  VS_ERR_OOM = 3,      /* device allocation failed */
  VS_ERR_BUDGET = 4,   /* job does not fit the configured HBM budget */
  VS_ERR_TIMEOUT = 5,  /* a bounded wait gave up */
  VS_ERR_CANCELLED = 6,
  VS_ERR_BUSY = 7      /* queue full / retry later */
};

/* Last error message of the calling thread ("" when none). */
const char* vs_last_error(void);
/* Library version string. */
const char* vs_version(void);
/* Number of kernels the vs_* entry points of this process have launched so far. */
uint64_t vs_launch_count(void);

/* ===================================================================== */
/* 1. Reference-compatible drop-in entry points                           */
/* ===================================================================== */

/* --- native circle NTT (src/cuda/ffi.rs:243-283; cuda/circle_ntt.cu:181-343) ---
 * Twiddles in the reference layout: line twiddles concatenated per line layer,
 * layer l at d_twiddles + h_layer_offsets[l] (host array), circle twiddles
 * separate. In place; synchronises the device before returning (as the
 * reference does). */
void cuda_circle_ntt_evaluate(uint32_t* d_data, const uint32_t* d_twiddles, const uint32_t* d_circle_twids,
                              const uint32_t* h_layer_offsets, const uint32_t* h_layer_sizes, uint32_t n_line_layers,
                              uint32_t n);
void cuda_circle_ntt_interpolate(uint32_t* d_data, const uint32_t* d_itwiddles, const uint32_t* d_circle_itwids,
                                 const uint32_t* h_layer_offsets, const uint32_t* h_layer_sizes,
                                 uint32_t n_line_layers, uint32_t n);
/* d_columns: device array of n_cols device pointers (src/cuda/ffi.rs:263-283). */
void cuda_circle_ntt_evaluate_batch(uint32_t** d_columns, const uint32_t* d_twiddles, const uint32_t* d_circle_twids,
                                    const uint32_t* h_layer_offsets, const uint32_t* h_layer_sizes,
                                    uint32_t n_line_layers, uint32_t n, uint32_t n_cols);
void cuda_circle_ntt_interpolate_batch(uint32_t** d_columns, const uint32_t* d_itwiddles,
                                       const uint32_t* d_circle_itwids, const uint32_t* h_layer_offsets,
                                       const uint32_t* h_layer_sizes, uint32_t n_line_layers, uint32_t n,
                                       uint32_t n_cols);
/* One butterfly layer, stride 2^layer_idx (src/cuda/ffi.rs:285-291; circle_ntt.cu:318-333). Async. */
void cuda_circle_ntt_layer(uint32_t* d_data, const uint32_t* d_twiddles, uint32_t layer_idx, uint32_t n, int forward);
/* In-place bit reversal of 2^log_n words (src/cuda/ffi.rs:293; circle_ntt.cu:338-343). Async. */
void cuda_bit_reverse_m31(uint32_t* data, uint32_t log_n);
/* Evaluate a polynomial at a QM31 point by folding (src/cuda/ffi.rs:295-302; circle_ntt.cu:345-384).
 * d_folding_factors: log2(n) QM31 factors (4 words each); h_result: host[4]; scratch: 2 x (n/2*4) words. */
void cuda_eval_at_point(const uint32_t* d_coeffs, const uint32_t* d_folding_factors, uint32_t* h_result, uint32_t n,
                        uint32_t* d_scratch1, uint32_t* d_scratch2);

/* --- stwo / CanonicCoset NTT (src/cuda/ffi.rs:234-239; cuda/circle_ntt_stwo.cu:268-402) ---
 * Flat stwo twiddle table of n/2 words (src/ntt.rs:262-325 layout). Output of
 * evaluate is in bit-reversed canonic order. Synchronises before returning. */
void cuda_stwo_ntt_evaluate(uint32_t* d_data, const uint32_t* d_twiddles, uint32_t n);
void cuda_stwo_ntt_interpolate(uint32_t* d_data, const uint32_t* d_itwiddles, uint32_t n);

/* --- twiddles (src/cuda/ffi.rs:327-363; cuda/twiddles.cu, cuda/batch_inverse.cu) --- */
void cuda_compute_fold_twiddle_sources(uint32_t initial_x, uint32_t initial_y, uint32_t step_x, uint32_t step_y,
                                       uint32_t* output, uint32_t n, uint32_t log_n, int extract_y);
void cuda_compute_fold_twiddle_sources_stream(uint32_t initial_x, uint32_t initial_y, uint32_t step_x,
                                              uint32_t step_y, uint32_t* output, uint32_t n, uint32_t log_n,
                                              int extract_y, vs_stream_t stream);
/* Montgomery-trick inverse over 64-element chunks; 0 -> 0, and a chunk whose
 * first element is 0 comes out all zero (batch_inverse.cu:8-41). */
void cuda_batch_inverse_m31(const uint32_t* input, uint32_t* output, uint32_t n);
void cuda_batch_inverse_m31_stream(const uint32_t* input, uint32_t* output, uint32_t n, vs_stream_t stream);
void cuda_compute_coset_points(uint32_t initial_x, uint32_t initial_y, uint32_t step_x, uint32_t step_y,
                               uint32_t* output_x, uint32_t* output_y, uint32_t n);
void cuda_squash_x(const uint32_t* input, uint32_t* output, uint32_t out_n);
void cuda_extract_and_squash(const uint32_t* input, uint32_t* twiddle_out, uint32_t* squash_out, uint32_t half_n);

/* --- Fibonacci constraint / LDE helpers (src/cuda/ffi.rs:367-398; cuda/constraint.cu:93-165) ---
 * alpha: host[4] QM31. Outputs are four SoA columns. */
void cuda_fibonacci_quotient(const uint32_t* trace, uint32_t* out0, uint32_t* out1, uint32_t* out2, uint32_t* out3,
                             const uint32_t* alpha, uint32_t n);
void cuda_zero_pad(const uint32_t* src, uint32_t* dst, uint32_t src_n, uint32_t dst_n);
void cuda_fibonacci_quotient_chunk(const uint32_t* trace, uint32_t* out0, uint32_t* out1, uint32_t* out2,
                                   uint32_t* out3, const uint32_t* alpha, uint32_t offset, uint32_t chunk_n,
                                   uint32_t global_n);
void cuda_fibonacci_quotient_chunk_stream(const uint32_t* trace, uint32_t* out0, uint32_t* out1, uint32_t* out2,
                                          uint32_t* out3, const uint32_t* alpha, uint32_t offset, uint32_t chunk_n,
                                          uint32_t global_n, vs_stream_t stream);
void cuda_interleave_u32(const uint32_t* even, const uint32_t* odd, uint32_t* output, uint32_t half_n);

/* --- FRI folds, SoA QM31 (src/cuda/ffi.rs:305-324; cuda/fri.cu:80-121) ---
 * alpha, alpha_sq: host[4]. */
void cuda_fold_line_soa(const uint32_t* in0, const uint32_t* in1, const uint32_t* in2, const uint32_t* in3,
                        const uint32_t* twiddles, uint32_t* out0, uint32_t* out1, uint32_t* out2, uint32_t* out3,
                        const uint32_t* alpha, uint32_t half_n);
void cuda_fold_circle_into_line_soa(uint32_t* dst0, uint32_t* dst1, uint32_t* dst2, uint32_t* dst3,
                                    const uint32_t* src0, const uint32_t* src1, const uint32_t* src2,
                                    const uint32_t* src3, const uint32_t* twiddles, const uint32_t* alpha,
                                    const uint32_t* alpha_sq, uint32_t half_n);

/* --- Blake2s Merkle (src/cuda/ffi.rs:643-697; cuda/blake2s.cu:522-632) ---
 * Leaf hash of up to 16 columns (t = min(n_cols,16)*4); SoA4 leaf t = 16;
 * node = Blake2s(left||right). columns: device array of device pointers.
 * Tiled variants emit one root per 1024-leaf tile. */
void cuda_merkle_hash_leaves(const uint32_t* const* columns, uint32_t* hashes, uint32_t n_cols, uint32_t n_leaves);
void cuda_merkle_hash_nodes(const uint32_t* children, uint32_t* parents, uint32_t n_parents);
void cuda_merkle_reduce_to_root(const uint32_t* nodes, uint32_t* root_out, uint32_t n_nodes);
void cuda_merkle_commit_small_soa4(const uint32_t* col0, const uint32_t* col1, const uint32_t* col2,
                                   const uint32_t* col3, uint32_t* root_out, uint32_t n_leaves);
void cuda_merkle_hash_leaves_merge_soa4(const uint32_t* col0, const uint32_t* col1, const uint32_t* col2,
                                        const uint32_t* col3, uint32_t* parents, uint32_t n_leaves);
void cuda_merkle_tiled_soa4(const uint32_t* col0, const uint32_t* col1, const uint32_t* col2, const uint32_t* col3,
                            uint32_t* subtree_roots, uint32_t n_leaves);
void cuda_merkle_tiled_soa4_stream(const uint32_t* col0, const uint32_t* col1, const uint32_t* col2,
                                   const uint32_t* col3, uint32_t* subtree_roots, uint32_t n_leaves,
                                   vs_stream_t stream);
void cuda_merkle_tiled_generic(const uint32_t* const* columns, uint32_t* subtree_roots, uint32_t n_cols,
                               uint32_t n_leaves);
/* Row-packed multi-block leaf over any number of columns of mixed sizes
 * (src/cuda/ffi.rs:769-776; cuda/merkle_leaves_lifted.cu:107-122).
 * schedule: device array of LeafHashChunk { uint32_t col_indices[16]; uint32_t n_cols; uint32_t log_size; }. */
void cuda_build_leaves_lifted(const uint32_t* const* col_ptrs, const void* schedule, uint32_t n_chunks,
                              uint32_t lifting_log_size, uint32_t* output_hashes, uint32_t n_leaves);

/* --- OODS / DEEP quotient (src/cuda/ffi.rs:850-898; cuda/quotient.cu:199-251) --- */
void cuda_accumulate_numerators(const uint32_t* const* col_ptrs, const uint32_t* col_indices, const uint32_t* b_coeffs,
                                const uint32_t* c_coeffs, uint32_t n_batch_cols, uint32_t n_rows, uint32_t* out0,
                                uint32_t* out1, uint32_t* out2, uint32_t* out3);
void cuda_compute_quotients_combine(const uint32_t* sample_points_x, const uint32_t* sample_points_y,
                                    const uint32_t* first_linear_acc, const uint32_t* const* numer_ptrs0,
                                    const uint32_t* const* numer_ptrs1, const uint32_t* const* numer_ptrs2,
                                    const uint32_t* const* numer_ptrs3, const uint32_t* acc_log_sizes,
                                    uint32_t n_accs, const uint32_t* domain_xs, const uint32_t* domain_ys,
                                    uint32_t lifting_log_size, uint32_t n_rows, uint32_t* out0, uint32_t* out1,
                                    uint32_t* out2, uint32_t* out3);

/* --- proof-of-work grinding (src/cuda/ffi.rs:632-638, 970-976; cuda/grind.cu, cuda/grind_m31_output.cu) ---
 * Nonces batch_offset .. batch_offset + n_threads - 1 are tried; the smallest one
 * whose Blake2s(prefix || nonce_LE) has >= pow_bits trailing zeros in its first 16
 * bytes is atomicMin'd into *result (device, initialised to UINT64_MAX by the
 * caller). Asynchronous on the default stream. */
void cuda_grind_pow(const uint32_t* prefixed_digest, uint64_t* result, uint32_t pow_bits, uint64_t batch_offset,
                    uint32_t n_threads);
void cuda_grind_pow_m31_output(const uint32_t* prefixed_digest, uint64_t* result, uint32_t pow_bits,
                               uint64_t batch_offset, uint32_t n_threads);

/* --- misc (src/cuda/ffi.rs:203-207, 946; cuda/fields.cu, cuda/bit_reverse_wide.cu) --- */
void cuda_bit_reverse_qm31(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t log_n);
void cuda_m31_add(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n);
void cuda_m31_mul(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n);
void cuda_device_sync(void);

/* --- kernels behind the stwo Backend adapter (crates/cuda-backend) ---
 * All device pointers; asynchronous on the default stream unless noted. */
/* dst[i] = src[idx[i]] for i < n (src/cuda/ffi.rs:812; cuda/gather.cu:44-53;
 * caller crates/cuda-backend/src/column.rs:489). */
void cuda_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint32_t n);
/* dst[8i .. 8i+8) = src[8 idx[i] .. 8 idx[i]+8): 32-byte hashes (src/cuda/ffi.rs:816;
 * cuda/gather.cu:55-64; caller column.rs:504). */
void cuda_gather_u256(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint32_t n);
/* Partial sums of sum_i evals[i] * weights[i] (M31 times QM31, weights 4 words per
 * element): out[4b .. 4b+4) is the sum over the 256-element chunks c with
 * c mod n_blocks == b; the caller adds the n_blocks partials. Synchronises the device
 * (src/cuda/ffi.rs:828-834; cuda/barycentric_eval.cu:84-95; caller poly_ops.rs:332). */
void cuda_barycentric_eval(const uint32_t* evals, const uint32_t* weights, uint32_t n, uint32_t* out,
                           uint32_t n_blocks);
/* In place, QM31 elements of 4 words: col[i] += curr[((i >> (log_ratio+1)) << 1) | (i & 1)]
 * for i < col_n (src/cuda/ffi.rs:958; cuda/accumulate_lift.cu:41-50). */
void cuda_accumulate_lift(uint32_t* col, const uint32_t* curr, uint32_t col_n, uint32_t log_ratio);
/* output_col_ptrs[16c + p][g] = input_col_ptrs[c][16g + p] for c < 4, p < 16; both are
 * device arrays of device pointers (4 and 64 of them) (src/cuda/ffi.rs:960-964;
 * cuda/pack_leaves.cu:44-52; caller merkle_ops.rs:193). */
void cuda_pack_leaves(const uint32_t* const* input_col_ptrs, uint32_t* const* output_col_ptrs, uint32_t n);
/* FRI fold twiddles of a stwo domain, built on the device (the adapter builds them
 * on the host for every fold: crates/cuda-backend/src/fri_ops.rs:50-56 for the
 * circle fold, :100-106 for line folds). With is_line = 0 the domain is the source
 * evaluation's CircleDomain of 2^log_size points, given by its half coset (initial
 * point, step): d_out[i] = 1 / y(half_coset.at(bit_reverse_index(2i, log_size))).
 * With is_line = 1 it is a LineDomain of 2^log_size points given by its coset:
 * d_out[i] = 1 / x(coset.at(bit_reverse_index(2i, log_size))). i < 2^(log_size-1);
 * a zero coordinate maps to 0 (chunked batch inverse). Stream-ordered. */
int vs_fold_twiddles_stwo(uint32_t is_line, uint32_t init_x, uint32_t init_y, uint32_t step_x, uint32_t step_y,
                          uint32_t log_size, uint32_t* d_out, vs_stream_t stream);
/* Domain points of CanonicCoset(log_size)'s circle domain in bit-reversed row
 * order, d_xs[r], d_ys[r] = domain.at(bit_reverse_index(r, log_size)), built on the
 * device (the adapter builds them on the host per call: quotient_ops.rs:135-140). */
int vs_canonic_domain_points(uint32_t log_size, uint32_t* d_xs, uint32_t* d_ys, vs_stream_t stream);

/* ===================================================================== */
/* 2. vs_* entry points (no reference counterpart)                        */
/* ===================================================================== */

/* Fill `n` words with the seeded uniform-M31 stream used by the benchmarks:
 * word k = splitmix64(seed + (k+1+offset)*0x9E3779B97F4A7C15) >> 33, re-drawn once
 * from counter k+2+offset when it equals 2^31-1 (0 if that is 2^31-1 too). */
int vs_fill_uniform_m31(uint32_t* d_out, uint64_t n, uint64_t seed, uint64_t offset, vs_stream_t stream);

/* Fused LDE in the stwo / CanonicCoset convention: for each of n_cols columns
 * (column c at d_src + c*src_stride, 2^log_n BRT-canonic evaluations) compute
 * interpolate -> zero-pad -> evaluate on CanonicCoset(log_n + blowup_bits),
 * writing column c at d_dst + c*dst_stride (bit-reversed canonic order).
 * Equivalent to the reference's interpolate_stwo / cuda_zero_pad /
 * evaluate_stwo chain (src/cairo_air/prover.rs:954-965) without materialising
 * the zero padding. d_src is not modified. Twiddles are cached per size. */
int vs_lde_stwo(const uint32_t* d_src, uint64_t src_stride, uint32_t* d_dst, uint64_t dst_stride, uint32_t n_cols,
                uint32_t log_n, uint32_t blowup_bits, vs_stream_t stream);
/* Same for the native half_coset convention (src/prover.rs:1745-1762). */
int vs_lde_native(const uint32_t* d_src, uint64_t src_stride, uint32_t* d_dst, uint64_t dst_stride, uint32_t n_cols,
                  uint32_t log_n, uint32_t blowup_bits, vs_stream_t stream);

/* NTT launch-shape autotuner (no counterpart in the reference, which launches one
 * kernel per butterfly layer). A plan per transform size log_n (process wide, used
 * by every NTT and LDE of that size, native and stwo; an LDE uses the plan of its
 * trace size):
 *   lower      layers of the first (lower) pass; 14 <= log_n <= 24 accepts
 *              max(5, log_n - 11) .. 13, other sizes only their default
 *              (13, or log_n below 14);
 *   items      tiles a pass CTA transforms before it retires, 1..64; 1 runs 13-layer
 *              lower passes in a single-buffered kernel (four CTAs per SM, one
 *              tile each); 0: the default (1 for 13-layer lower passes, 8 elsewhere);
 *   radix      layers per register round above a C = 0 tile's first five:
 *              3 (16-byte chunk rounds, the default) or 5 (word rounds); 0: default.
 *              The LDE of at most 13 layers has the word-round form only.
 * Plans change only how layers are grouped into launches; results are identical.
 * vs_ntt_plan_set(log_n, 0, 0, 0) restores the defaults. */
int vs_ntt_plan_set(uint32_t log_n, uint32_t lower, uint32_t items, uint32_t radix);
int vs_ntt_plan_get(uint32_t log_n, uint32_t* lower, uint32_t* items, uint32_t* radix);
/* The plans the autotuner tries for log_n, 3 words each (lower, items, radix);
 * *n_out = their number (host only, no device calls). */
int vs_ntt_plan_candidates(uint32_t log_n, uint32_t* out, uint32_t cap, uint32_t* n_out);
/* Times every candidate plan on an n_cols-column stwo LDE of 2^log_n rows (seeded
 * columns, one warm-up and `reps` timed runs each, CUDA events on `stream`), keeps the
 * fastest as the plan of log_n and writes it to best[3]; ms[i] (i < cap) receives
 * candidate i's time per LDE. Allocates its scratch columns on `stream`. */
int vs_autotune_lde(uint32_t log_n, uint32_t n_cols, uint32_t blowup_bits, uint32_t reps, uint32_t* best,
                    float* ms, uint32_t cap, vs_stream_t stream);
/* Merkle subtree shape of the root-only trees (no counterpart in the reference):
 * the first reduction level stops at 2^split roots per 1024-leaf tile (0..8), so a
 * CTA skips the narrow top levels of its tile, and the next level reduces them.
 * Roots are identical for every split. Process wide; applies to vs_commit_columns,
 * vs_merkle_root_rowpacked / _capped / _soa4, vs_fri_fold_commit, the Cairo FRI and
 * the engine's commitment jobs (their scratch is sized for split 8). */
int vs_merkle_split_set(uint32_t split);
uint32_t vs_merkle_split_get(void);
/* Times the row-packed root of n_cols seeded columns x 2^log_leaves rows (11..28) at
 * every split (one warm-up and `reps` timed runs each, CUDA events on `stream`),
 * checks that all splits give one root, keeps the fastest split and writes it to
 * *best; ms[s] (s < cap) receives split s's time per root. Allocates its scratch on
 * `stream`. */
int vs_autotune_merkle(uint32_t log_leaves, uint32_t n_cols, uint32_t reps, uint32_t* best, float* ms, uint32_t cap,
                       vs_stream_t stream);

/* Merkle root over n_cols columns of 2^log_leaves rows with the row-packed
 * multi-block leaf (all columns, merkle_leaves_lifted.cu semantics with equal
 * sizes). Column c at d_cols + c*stride. root written to d_root (device, 8 words). */
int vs_merkle_root_rowpacked(const uint32_t* d_cols, uint64_t stride, uint32_t n_cols, uint32_t log_leaves,
                             uint32_t* d_root, vs_stream_t stream);
/* Same root as vs_merkle_root_rowpacked, but allocates no device memory: its
 * intermediate subtree roots live in a fixed 2.1 MB array inside the library
 * (held by every GPU that loads it, until exit), for callers that cannot allocate
 * at that point (a server whose HBM is fully reserved by its admission budget, a
 * framework whose allocator owns device memory, a step that must not risk an
 * allocation failure or sync). No counterpart in the reference. Accepts at most
 * 2^26 leaves (VS_ERR_INVALID beyond). The first call on a device, and the first
 * after the device's context was recreated, looks up the array's device address;
 * make it before any stream capture. All calls share the array: calls whose work
 * overlaps on the GPU race. */
int vs_merkle_root_rowpacked_noalloc(const uint32_t* d_cols, uint64_t stride, uint32_t n_cols, uint32_t log_leaves,
                                     uint32_t* d_root, vs_stream_t stream);
/* Merkle root with the reference's <=16-column leaf (blake2s.cu leaf semantics). */
int vs_merkle_root_capped(const uint32_t* d_cols, uint64_t stride, uint32_t n_cols, uint32_t log_leaves,
                          uint32_t* d_root, vs_stream_t stream);
/* Merkle root of a SoA4 QM31 column (leaf t = 16). */
int vs_merkle_root_soa4(const uint32_t* d_c0, const uint32_t* d_c1, const uint32_t* d_c2, const uint32_t* d_c3,
                        uint32_t log_leaves, uint32_t* d_root, vs_stream_t stream);

/* Commitment-layer step: LDE (stwo convention) of n_cols columns of 2^log_n
 * rows into d_lde (n_cols x 2^(log_n+blowup), column-major), then the
 * row-packed Blake2s Merkle root into d_root (device, 8 words). */
int vs_commit_columns(const uint32_t* d_cols, uint32_t n_cols, uint32_t log_n, uint32_t blowup_bits, uint32_t* d_lde,
                      uint32_t* d_root, vs_stream_t stream);

/* FRI chain on one QM31 evaluation vector (SoA4 in d_src, 4 planes of 2^log_n
 * words at d_src + k*2^log_n): circle fold on half_coset(log_n), then line folds
 * on half_odds down to 2^3 values, committing every folded layer (SoA4 leaf).
 * h_alphas: host, (log_n - 3) QM31 fold challenges. d_work: device scratch of
 * 4 * 2^log_n words. Writes (log_n - 3) roots (8 words each) to d_roots and the
 * 8 last-layer QM31 values (AoS) to d_last. */
int vs_fri_fold_commit(const uint32_t* d_src, uint32_t log_n, const uint32_t* h_alphas, uint32_t* d_work,
                       uint32_t* d_roots, uint32_t* d_last, vs_stream_t stream);

/* Fibonacci prover (src/prover.rs:192-209 prove(); stage order of
 * prove_with_cache, src/prover.rs:1721-1978). Writes the proof in the KRAK v1
 * wire format (src/bin/stark_cli.rs:907-976) into h_out (host) when cap is large
 * enough; *out_len receives the proof length. */
int vs_prove_fib(uint32_t a, uint32_t b, uint32_t log_n, uint8_t* h_out, uint64_t cap, uint64_t* out_len,
                 vs_stream_t stream);
/* Verifier (src/verifier.rs:39-236) over a KRAK proof. Returns VS_OK when
 * accepted, VS_ERR_INVALID otherwise with the reason in err (host). */
int vs_verify_fib(const uint8_t* h_proof, uint64_t len, char* err, uint64_t err_cap);

/* Graph-captured Fibonacci prover for one trace size (2^log_n rows): the whole
 * proof (trace, LDE, commitments, device-side Fiat-Shamir channel, FRI, queries,
 * decommitment) is one CUDA graph launch on the prover's own stream; same KRAK v1
 * bytes as vs_prove_fib. One proof in flight per handle. */
int vs_prover_create(uint32_t log_n, void** prover);
int vs_prover_prove(void* prover, uint32_t a, uint32_t b, uint8_t* h_out, uint64_t cap, uint64_t* out_len);
int vs_prover_destroy(void* prover);

/* Batched / served execution (no reference counterpart: the reference proves a
 * batch one proof after another, ProverPipeline::prove_batch, src/prover.rs:2265-2270).
 * An engine owns n_slots workers (host thread + CUDA streams) and a pool of cached
 * device workspaces (batched provers, graph-captured provers, commitment buffers).
 * Submitted jobs queue in FIFO order; a free slot takes the head job together with
 * the queued Fibonacci jobs of the same trace size (log_n <= 22), up to that size's
 * batch capacity, and proves them as one batch (one CUDA graph launch, one kernel
 * per stage for all of them). A job runs when a cached workspace of its shape is
 * idle or a new one keeps the engine's device memory (every cached workspace plus
 * the library's twiddle tables) within hbm_budget_bytes (0 = unlimited); idle
 * workspaces of other shapes are freed, least recently used first, to make room.
 * A job whose workspace does not fit the budget even on an idle engine fails with
 * VS_ERR_BUDGET. Results: a KRAK proof for VS_JOB_FIB, the 32-byte row-packed root
 * of the seeded columns' x4 stwo LDE for VS_JOB_COMMIT; each result depends only
 * on its job. Times are seconds since engine creation. */
enum { VS_JOB_FIB = 0, VS_JOB_COMMIT = 1 };
typedef struct {
  uint32_t kind;   /* VS_JOB_FIB or VS_JOB_COMMIT */
  uint32_t log_n;  /* log2 of the trace rows */
  uint32_t a, b;   /* Fibonacci public inputs (t0, t1) */
  uint32_t n_cols; /* commitment: number of columns */
  uint32_t pad;
  uint64_t seed;   /* commitment: seed of the uniform-M31 columns (vs_fill_uniform_m31) */
} vs_job;
typedef struct {
  int status;
  uint32_t pad;
  uint64_t out_len;
  double t_submit, t_start, t_end;
} vs_job_result;
int vs_engine_create(uint32_t n_slots, uint64_t hbm_budget_bytes, void** engine);
/* As vs_engine_create with flags: VS_ENGINE_FIFO_PRIORITY runs every job at the
 * same stream priority; by default (flags 0, and vs_engine_create) jobs run at
 * one of three CUDA stream priorities by working-set size, smallest first, which
 * shortens small jobs' latency at some cost to large jobs' tails. Results are the
 * same either way. */
#define VS_ENGINE_FIFO_PRIORITY 1u
int vs_engine_create_ex(uint32_t n_slots, uint64_t hbm_budget_bytes, uint32_t flags, void** engine);
int vs_engine_destroy(void* engine);
/* Builds the workspace for this job shape in every slot (outside any timing; for
 * batched Fibonacci sizes a full-capacity one, which serves batches of any size). */
int vs_engine_prepare(void* engine, const vs_job* shape);
int vs_engine_submit(void* engine, const vs_job* job, uint64_t* ticket);
/* Queues n jobs at once (all or none), so slots see them together and batch
 * them fully; tickets[i] receives job i's ticket. */
int vs_engine_submit_many(void* engine, const vs_job* jobs, uint32_t n, uint64_t* tickets);
/* Blocks until the job is done. With h_out == NULL only the result record is
 * filled (the bytes stay available); otherwise the bytes are copied and the
 * ticket is retired. */
int vs_engine_wait(void* engine, uint64_t ticket, vs_job_result* result, uint8_t* h_out, uint64_t cap);
/* As vs_engine_wait, giving up after timeout_s seconds (negative: no limit) with
 * VS_ERR_TIMEOUT; the ticket stays valid. A failed, cancelled or rejected job
 * returns its status (VS_ERR_CANCELLED, VS_ERR_BUDGET, VS_ERR_OOM, ...); with
 * h_out != NULL its ticket is retired. */
int vs_engine_wait_for(void* engine, uint64_t ticket, double timeout_s, vs_job_result* result, uint8_t* h_out,
                       uint64_t cap);
/* Cancels a job that has not started: VS_OK, and its wait returns
 * VS_ERR_CANCELLED. A running or finished job cannot be cancelled (VS_ERR_BUSY). */
int vs_engine_cancel(void* engine, uint64_t ticket);
int vs_engine_drain(void* engine);
double vs_engine_now(void* engine);
/* At most max_jobs proofs per batch (0 = each size's default capacity, 1 = one
 * proof per graph launch). Takes effect for workspaces created afterwards. */
int vs_engine_set_batch_limit(void* engine, uint32_t max_jobs);
/* Device bytes of the largest workspace a job of this shape runs in (for small
 * Fibonacci proofs the full-capacity batch workspace; a batch that finds no idle
 * workspace gets one sized to it, at most this), not counting twiddle tables. */
int vs_engine_workspace_bytes(void* engine, const vs_job* shape, uint64_t* bytes);
/* Host-side fault injection for tests: the next `count` workspace creations fail
 * with VS_ERR_OOM before allocating anything; the engine stays usable. */
int vs_engine_inject_alloc_failures(void* engine, uint32_t count);
typedef struct {
  uint64_t budget_bytes;        /* 0: unlimited */
  uint64_t resident_bytes;      /* cached workspaces, idle and in use */
  uint64_t twiddle_bytes;       /* the library's twiddle tables on the engine's device */
  uint64_t peak_held_bytes;     /* largest resident + twiddle bytes admitted so far */
  uint64_t evictions;           /* idle workspaces freed to make room */
  uint64_t workspaces_created;
  uint32_t idle_workspaces, busy_workspaces;
  uint32_t queued, running;     /* jobs */
} vs_engine_stats;
int vs_engine_get_stats(void* engine, vs_engine_stats* out);

/* Release cached twiddles and scratch of the current device. */
int vs_release_caches(void);

/* One column group of the reference Cairo prover's trace commitment
 * (cairo_air/prover.rs:899-1047) with every step on the device: columns in
 * half-coset natural order (d_cols_hc, n_cols <= 16 at col_stride words) are
 * permuted to BRT-canonic order (circle.rs:192-204), optionally interpolated to
 * stwo coefficients (d_coeffs, n_cols x 2^log_n), extended x4 (d_eval_cn, n_cols x
 * 2^(log_n+2), BRT-canonic), ZK-blinded as column c += h_blind[c] * Z_H for every
 * nonzero h_blind[c] (prover.rs:924-993; h_blind may be NULL), optionally copied
 * back to half-coset order (d_eval_hc), and committed with the native leaf of the
 * group's columns: root (d_root) and 1024-leaf tile roots (d_tile_roots, 2^(log_n+2)
 * / 1024 hashes, or the root alone below 1024 leaves; may be NULL), as
 * MerkleTree::commit_root_only_with_subtrees (merkle.rs:360-417). */
int vs_commit_group_cairo(const uint32_t* d_cols_hc, uint64_t col_stride, uint32_t n_cols, uint32_t log_n,
                          const uint32_t* h_blind, uint32_t* d_coeffs, uint32_t* d_eval_cn, uint32_t* d_eval_hc,
                          uint32_t* d_root, uint32_t* d_tile_roots, vs_stream_t stream);

/* Decommitment of a tree committed with 1024-leaf tile roots
 * (merkle.rs:603-619,721-800, cairo_air/prover.rs:2520-2560,4087-4130): for each
 * leaf index, the leaf's column values (h_values, n_indices x n_cols words; may
 * be NULL) and its sibling path from leaf to root (h_paths, n_indices x
 * log_n_leaves hashes). The queried tiles are recomputed on the device from the
 * columns; the levels above come from d_tile_roots (max(1, 2^log_n_leaves / 1024)
 * hashes; the root alone for smaller trees). Leaves: VS_LEAF_CAPPED (1..16
 * columns, the native leaf) or VS_LEAF_SOA4 (4 columns, one QM31 per leaf).
 * h_cols: host array of device pointers. Synchronises the stream. */
enum { VS_LEAF_CAPPED = 0, VS_LEAF_SOA4 = 1 };
int vs_tile_tree_paths(uint32_t leaf_kind, const uint32_t* const* h_cols, uint32_t n_cols, uint32_t log_n_leaves,
                       const uint32_t* d_tile_roots, const uint64_t* h_indices, uint32_t n_indices,
                       uint32_t* h_values, uint32_t* h_paths, vs_stream_t stream);

/* stwo wire-format helpers (src/stwo_export.rs:160-330, 700-790), host only.
 * Positions may come in any order and repeat (the first occurrence counts).
 * hash witness: from per-query auth paths (h_paths, n x height hashes, leaf level
 * first) the sibling hashes a verifier cannot compute, level by level in
 * ascending position order; the fold-pair form opens both members of each
 * queried pair (FRI layers). fri witness: the partner values (h_sibling_values, 4
 * words per query, the value at position ^ 1) of queried positions whose partner
 * is not queried. root from witness: rebuilds the root from the queried rows
 * (n x n_cols words, leaf = Blake2s of the row's words) and a hash witness,
 * failing when the witness is short or not used up. out_len counts hashes or
 * QM31 values written (at most cap). */
int vs_stwo_hash_witness(const uint64_t* h_positions, uint32_t n, const uint32_t* h_paths, uint32_t height,
                         uint32_t* h_out, uint32_t cap_hashes, uint32_t* out_len);
int vs_stwo_fold_pair_hash_witness(const uint64_t* h_positions, uint32_t n, const uint32_t* h_paths, uint32_t height,
                                   uint32_t* h_out, uint32_t cap_hashes, uint32_t* out_len);
int vs_stwo_fri_witness(const uint64_t* h_positions, uint32_t n, const uint32_t* h_sibling_values, uint32_t* h_out,
                        uint32_t cap, uint32_t* out_len);
int vs_stwo_root_from_witness(uint32_t log_height, const uint64_t* h_positions, uint32_t n, const uint32_t* h_rows,
                              uint32_t n_cols, const uint32_t* h_witness, uint32_t n_witness, uint32_t* h_root);

/* The stwo wire-format proof (src/stwo_export.rs:415-660 cairo_proof_to_stwo and
 * :687-690 cairo_proof_to_json): the seven commitment trees in channel order
 * (trace columns 0-15, 16-30 and 31-33, the LogUp, RC and S_dict interaction trees,
 * the composition quotient), their OODS samples, column-major queried values and
 * deduplicated hash witnesses (the trace trees over the query rows and, when next-row
 * paths are given, the next rows), and the FRI proof (the OODS quotient as first
 * layer with its fold-pair witness, then each line-fold layer). All arrays are host
 * memory; auth paths are [query][level][8 words], leaf level first, with
 * height = log_trace_size + 2 (FRI layer i: height - i - 1). */
typedef struct {
  uint32_t log_trace_size;
  uint32_t n_queries;
  const uint64_t* query_indices;            /* n_queries positions in the evaluation domain */
  uint64_t pow_nonce;
  uint32_t commitments[7][8];
  uint32_t n_trace_cols;                    /* >= 16; columns past 34 are not exported */
  const uint32_t* trace_values_at_queries;  /* [n_queries][n_trace_cols] */
  uint32_t n_oods, n_oods_next;             /* trace columns sampled at z and at z_next */
  const uint32_t* oods_trace_at_z;          /* [n_oods][4] */
  const uint32_t* oods_trace_at_z_next;     /* [n_oods_next][4] */
  uint32_t oods_interaction_at_z[3][4][4];  /* all zero: not sampled */
  uint32_t oods_interaction_at_z_next[3][4][4];
  uint32_t oods_quotient_at_z[4][4];        /* all zero: not sampled */
  const uint32_t* trace_auth_paths[3];      /* trees 0-2 at the query rows */
  const uint32_t* trace_auth_paths_next[3]; /* at the next rows, or NULL */
  const uint32_t* decom_values[4];          /* trees 3-6: [n_queries][4] */
  const uint32_t* decom_auth_paths[4];
  uint32_t oods_quotient_commitment[8];
  const uint32_t* oods_quotient_sibling_values;  /* [n_queries][4] at position ^ 1 */
  const uint32_t* oods_quotient_auth_paths;
  uint32_t n_fri;
  const uint32_t* fri_commitments;          /* [n_fri][8] */
  const uint32_t* const* fri_sibling_values; /* n_fri host arrays [n_queries][4] */
  const uint32_t* const* fri_auth_paths;    /* n_fri host arrays [n_queries][height - i - 1][8] */
  uint32_t n_last;
  const uint32_t* last_layer_poly;          /* [n_last][4] */
} vs_stwo_proof_parts;
/* Writes the proof as serde_json's pretty JSON into h_out (when cap suffices);
 * *out_len receives its length (h_out NULL: length query). */
int vs_stwo_proof_json(const vs_stwo_proof_parts* parts, char* h_out, uint64_t cap, uint64_t* out_len);

/* Circle polynomials in the stwo coefficient basis evaluated at QM31 points
 * (oods.rs:133-161, eval_at_oods_from_coeffs, which the reference runs on the
 * host per column). h_cols: host array of n_cols device pointers, 2^log_len
 * coefficients each; h_points: n_points (<= 2) points as 8 words (x QM31, y
 * QM31); h_out: n_cols x n_points QM31 (4 words), column-major over points.
 * Synchronises the stream. */
int vs_eval_at_oods_points(const uint32_t* const* h_cols, uint32_t n_cols, uint32_t log_len,
                           const uint32_t* h_points, uint32_t n_points, uint32_t* h_out, vs_stream_t stream);

/* The reference Cairo prover's tail after the trace and interaction commitments
 * (cairo_air/prover.rs:1937-2438), device-resident:
 *   AIR quotient (4 limbs, half-coset natural) -> BRT-canonic -> SoA4 commitment
 *   with 1024-leaf tile roots, mixed; OODS point z from the channel, z_next one
 *   trace step on; trace columns at z / z_next from their coefficients (plus
 *   r * Z_H at the point for blinded columns), interaction columns from the first
 *   2^log_n stwo coefficients of their evaluations, quotient limbs from all
 *   coefficients; sampled values mixed in flatten_cols order; OODS alpha drawn;
 *   DEEP quotient numerators over [trace, quotient, interaction] columns for z
 *   and [trace, interaction] for z_next with alpha-power line coefficients;
 *   combination on the BRT-canonic domain; SoA4 commitment with tile roots,
 *   mixed; FRI circle fold (twiddles 1/y of the canonic points) and committed
 *   line folds down to 8 values; last-layer line-polynomial coefficients (BRT
 *   order) mixed.
 * The channel is advanced exactly as the reference's. Device outputs left NULL
 * are kept internally; host arrays left NULL are not written. */
typedef struct {
  uint32_t log_n;         /* trace rows 2^log_n (2..26); evaluation domain 2^(log_n+2) */
  uint32_t n_trace;       /* trace columns (1..1024) */
  uint32_t n_interaction; /* interaction component columns (0..1024) */
  uint32_t pad;
  const uint32_t* const* trace_coeffs;      /* host array of device pointers: 2^log_n stwo coefficients */
  const uint32_t* zk_scalars;               /* host: blinding scalar per trace column (0 = none), or NULL */
  const uint32_t* const* trace_evals;       /* host array of device pointers: BRT-canonic evaluations */
  const uint32_t* const* interaction_evals; /* host array of device pointers: BRT-canonic evaluations */
  const uint32_t* quotient_hc[4];           /* device: AIR quotient limbs, half-coset natural order */
  uint32_t* quotient_cn[4];                 /* device out (optional): quotient limbs, BRT-canonic */
  uint32_t* oods_quotient[4];               /* device out (optional): DEEP quotient limbs, BRT-canonic */
  uint32_t* quotient_tile_roots;            /* device out (optional): max(1, N/1024) hashes */
  uint32_t* oods_tile_roots;                /* device out (optional): max(1, N/1024) hashes */
  uint32_t* trace_at_z;                     /* host out (optional): 4 x n_trace */
  uint32_t* trace_at_z_next;                /* host out (optional): 4 x n_trace */
  uint32_t* interaction_at_z;               /* host out (optional): 4 x n_interaction */
  uint32_t* interaction_at_z_next;          /* host out (optional): 4 x n_interaction */
  uint32_t quotient_root[8];
  uint32_t oods_point[8];     /* z.x then z.y (QM31 each) */
  uint32_t quotient_at_z[16]; /* 4 limbs x QM31 */
  uint32_t oods_alpha[4];
  uint32_t oods_root[8];
  uint32_t n_fri_roots;       /* committed line layers: log_n - 2 */
  uint32_t fri_roots[32 * 8];
  uint32_t fri_alphas[32 * 4]; /* [0] circle fold, then one per line fold (log_n - 1 in all) */
  uint32_t last_layer[8 * 4];  /* the 8 final evaluations */
  uint32_t last_layer_coeffs[8 * 4];
} vs_cairo_oods_fri_io;
int vs_cairo_oods_fri(void* channel, vs_cairo_oods_fri_io* io, vs_stream_t stream);

/* Fiat–Shamir channel (src/channel.rs:15-185): a Blake2s transcript with the
 * reference's byte layouts. Digests are 8 LE words; felts are QM31 as 4 words
 * [a.a, a.b, b.a, b.b]. Host-only state; grind_pow runs the nonce search on the
 * GPU in batches of 2^26 and returns the smallest passing nonce below max_nonces
 * (it does not mix the nonce in: call mix_u64, as the reference does). */
int vs_channel_create(void** channel);
int vs_channel_destroy(void* channel);
int vs_channel_state(void* channel, uint8_t* h_state32, uint32_t* n_draws);
int vs_channel_mix_digest(void* channel, const uint32_t* h_digest8);          /* channel.rs:29-40 */
int vs_channel_mix_felts(void* channel, const uint32_t* h_felts, uint64_t n_felts); /* channel.rs:44-58 */
int vs_channel_mix_u64(void* channel, uint64_t value);                          /* channel.rs:120-129 */
int vs_channel_draw_felt(void* channel, uint32_t* h_out4);                      /* channel.rs:60-86 */
int vs_channel_draw_number(void* channel, uint64_t bound, uint64_t* out);       /* channel.rs:88-99 */
int vs_channel_draw_query_indices(void* channel, uint32_t log_domain_size, uint32_t n, uint32_t* h_out); /* :102-116 */
int vs_channel_pow_prefix(void* channel, uint32_t pow_bits, uint32_t* h_out8);  /* channel.rs:144-152 */
int vs_channel_verify_pow_nonce(void* channel, uint32_t pow_bits, uint64_t nonce); /* :144-168; 1 valid, 0 not, -1 error */
int vs_channel_grind_pow(void* channel, uint32_t pow_bits, uint64_t max_nonces, uint64_t* nonce, vs_stream_t stream);
/* Sets the release threshold of the current device's default stream-ordered
 * memory pool (bytes kept cached across synchronisations; UINT64_MAX never
 * releases). Replaces init_memory_pool (2 GiB) / init_memory_pool_greedy
 * (src/cuda/ffi.rs:165-207); vs_prove_fib and the FRI scratch allocate from this
 * pool, as the reference's DeviceBuffer does (src/device/buffer.rs:16-87). */
int vs_init_memory_pool(uint64_t release_threshold_bytes);

#ifdef __cplusplus
}
#endif
#endif /* VSTARK_H */
