// CPU oracle for the VortexSTARK polynomial-commitment hot path.
//
// TEST INFRASTRUCTURE ONLY. This is a plain C++17 restatement of the
// reference prover's arithmetic (garrick99/VortexSTARK), used by tests/ as
// the parity checker and by bench.py as the timed CPU baseline. The product
// library (vortexstark_b200) never links, loads or calls it.
//
// Every function cites the reference file:line it restates. All arithmetic is
// exact mod p = 2^31 - 1; values are canonical (< p) everywhere.
//
// Parity pins: field/circle known answers from the reference's own tests,
// Blake2s-256 against Python hashlib, and the reference's CUDA kernels built
// from its sources (oracle/build_ref.sh) run on a B200 to produce the golden
// vectors under tests/golden/.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace vso {

constexpr uint32_t P = 0x7FFFFFFFu;

// ---------------------------------------------------------------- M31
// src/field/m31.rs:23-54, 83-164; cuda/include/m31.cuh:9-53
inline uint32_t m31_reduce(uint64_t v) {
  uint32_t lo = (uint32_t)(v & P);
  uint32_t hi = (uint32_t)(v >> 31);
  uint32_t r = lo + hi;
  return r >= P ? r - P : r;
}
inline uint32_t m31_add(uint32_t a, uint32_t b) { uint32_t r = a + b; return r >= P ? r - P : r; }
inline uint32_t m31_sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P - b; }
inline uint32_t m31_mul(uint32_t a, uint32_t b) { return m31_reduce((uint64_t)a * b); }
inline uint32_t m31_neg(uint32_t a) { return a == 0 ? 0 : P - a; }
inline uint32_t m31_double(uint32_t a) { uint32_t r = a << 1; return r >= P ? r - P : r; }
uint32_t m31_pow(uint32_t a, uint32_t e);
inline uint32_t m31_inv(uint32_t a) { return m31_pow(a, P - 2); }

// ---------------------------------------------------------------- CM31 / QM31
// src/field/cm31.rs:8-113; src/field/qm31.rs:10-170
struct CM31 { uint32_t a, b; };
inline CM31 cm_add(CM31 x, CM31 y) { return {m31_add(x.a, y.a), m31_add(x.b, y.b)}; }
inline CM31 cm_sub(CM31 x, CM31 y) { return {m31_sub(x.a, y.a), m31_sub(x.b, y.b)}; }
inline CM31 cm_mul(CM31 x, CM31 y) {
  return {m31_sub(m31_mul(x.a, y.a), m31_mul(x.b, y.b)), m31_add(m31_mul(x.a, y.b), m31_mul(x.b, y.a))};
}
inline CM31 cm_neg(CM31 x) { return {m31_neg(x.a), m31_neg(x.b)}; }
inline CM31 cm_scale(CM31 x, uint32_t s) { return {m31_mul(x.a, s), m31_mul(x.b, s)}; }
CM31 cm_inv(CM31 x);

// QM31 = a + b*u, u^2 = 2 + i. Limb order [a.a, a.b, b.a, b.b] (qm31.rs:44-47).
struct QM31 { uint32_t v[4]; };
inline bool operator==(const QM31& x, const QM31& y) {
  return x.v[0] == y.v[0] && x.v[1] == y.v[1] && x.v[2] == y.v[2] && x.v[3] == y.v[3];
}
inline QM31 qm_from(CM31 a, CM31 b) { return {{a.a, a.b, b.a, b.b}}; }
inline CM31 qm_a(QM31 x) { return {x.v[0], x.v[1]}; }
inline CM31 qm_b(QM31 x) { return {x.v[2], x.v[3]}; }
inline QM31 qm_m31(uint32_t x) { return {{x, 0, 0, 0}}; }
inline QM31 qm_add(QM31 x, QM31 y) { return qm_from(cm_add(qm_a(x), qm_a(y)), cm_add(qm_b(x), qm_b(y))); }
inline QM31 qm_sub(QM31 x, QM31 y) { return qm_from(cm_sub(qm_a(x), qm_a(y)), cm_sub(qm_b(x), qm_b(y))); }
// (a + bu)(c + du) = (ac + bd(2+i)) + (ad + bc)u   (qm31.rs:112-131)
inline QM31 qm_mul(QM31 x, QM31 y) {
  CM31 ac = cm_mul(qm_a(x), qm_a(y)), bd = cm_mul(qm_b(x), qm_b(y));
  CM31 ad = cm_mul(qm_a(x), qm_b(y)), bc = cm_mul(qm_b(x), qm_a(y));
  CM31 bdu = {m31_sub(m31_double(bd.a), bd.b), m31_add(bd.a, m31_double(bd.b))};
  return qm_from(cm_add(ac, bdu), cm_add(ad, bc));
}
inline QM31 qm_scale(QM31 x, uint32_t s) { return {{m31_mul(x.v[0], s), m31_mul(x.v[1], s), m31_mul(x.v[2], s), m31_mul(x.v[3], s)}}; }
inline QM31 qm_scale_cm(QM31 x, CM31 s) { return qm_from(cm_mul(qm_a(x), s), cm_mul(qm_b(x), s)); }
inline QM31 qm_neg(QM31 x) { return {{m31_neg(x.v[0]), m31_neg(x.v[1]), m31_neg(x.v[2]), m31_neg(x.v[3])}}; }
inline QM31 qm_conj(QM31 x) { return qm_from(qm_a(x), cm_neg(qm_b(x))); }
QM31 qm_inv(QM31 x);

// ---------------------------------------------------------------- circle group
// src/circle.rs:11-268
struct CPoint { uint32_t x, y; };
inline bool operator==(const CPoint& a, const CPoint& b) { return a.x == b.x && a.y == b.y; }
constexpr CPoint CP_IDENTITY{1, 0};
constexpr CPoint CP_GENERATOR{2, 1268011823u};  // circle.rs:26-29
inline CPoint cp_mul(CPoint a, CPoint b) {
  return {m31_sub(m31_mul(a.x, b.x), m31_mul(a.y, b.y)), m31_add(m31_mul(a.x, b.y), m31_mul(a.y, b.x))};
}
inline CPoint cp_conj(CPoint a) { return {a.x, m31_neg(a.y)}; }
CPoint cp_repeated_double(CPoint p, uint32_t n);
CPoint cp_mul_scalar(CPoint p, uint64_t k);

struct Coset {
  CPoint initial, step;
  uint32_t log_size;
  uint64_t size() const { return 1ull << log_size; }
  CPoint at(uint64_t i) const { return cp_mul(initial, cp_mul_scalar(step, i)); }  // circle.rs:189
};
Coset coset_subgroup(uint32_t log_size);    // circle.rs:101-110
Coset coset_half_coset(uint32_t log_size);  // circle.rs:114-123
Coset coset_half_odds(uint32_t log_size);   // circle.rs:133-144 (log 30 -> G^1)
std::vector<CPoint> coset_points(const Coset& c);  // all points, natural order

inline uint32_t bit_reverse(uint64_t v, uint32_t bits) {
  uint64_t r = 0;
  for (uint32_t i = 0; i < bits; i++) { r = (r << 1) | (v & 1); v >>= 1; }
  return (uint32_t)r;
}
// circle.rs:196-208 (BRT-canonic position of a natural half-coset index)
uint64_t hc_natural_to_canonic_brt_index(uint64_t k, uint32_t log_n);
std::vector<uint32_t> permute_hc_natural_to_canonic_brt(const std::vector<uint32_t>& d, uint32_t log_n);
std::vector<uint32_t> permute_canonic_brt_to_hc_natural(const std::vector<uint32_t>& d, uint32_t log_n);

// ---------------------------------------------------------------- batch inverse
// cuda/batch_inverse.cu:8-41 — Montgomery trick over 64-element chunks.
// Quirk kept: zero inputs map to zero; if a chunk starts with zero the whole
// chunk comes out zero (its running prefix starts at zero).
std::vector<uint32_t> batch_inverse_chunked(const std::vector<uint32_t>& in);

// ---------------------------------------------------------------- native twiddles
// src/circle.rs:277-340 with cuda/twiddles.cu:80-142 semantics.
struct NativeTwiddles {
  uint32_t log_n;
  std::vector<uint32_t> line, circle;            // forward
  std::vector<uint32_t> iline, icircle;          // inverse (batch-inverted)
  std::vector<uint32_t> offsets, sizes;          // per line layer (host arrays)
};
NativeTwiddles native_twiddles(const Coset& coset);

// ---------------------------------------------------------------- native NTT
// cuda/circle_ntt.cu:8-50,181-249 (in place).
void native_evaluate(std::vector<uint32_t>& d, const NativeTwiddles& t);
void native_interpolate(std::vector<uint32_t>& d, const NativeTwiddles& t);
// One butterfly layer (cuda/circle_ntt.cu:22-50, 318-333).
void ntt_layer(uint32_t* d, uint64_t n, const uint32_t* tw, uint32_t layer_idx, bool forward);
inline uint32_t inv_n_scale(uint32_t log_n) {  // circle_ntt.cu:239-243
  uint32_t e = (30u * log_n) % 31u;
  return e == 0 ? 1u : (1u << e);
}
void bit_reverse_inplace(std::vector<uint32_t>& d, uint32_t log_n);  // circle_ntt.cu:167-177

// ---------------------------------------------------------------- stwo NTT
// src/ntt.rs:262-325 twiddle layout; cuda/circle_ntt_stwo.cu:30-402 transform.
struct StwoTwiddles { uint32_t log_n; std::vector<uint32_t> fwd, inv; };
StwoTwiddles stwo_twiddles(uint32_t log_n);  // coset = half_coset(log_n)
void stwo_evaluate(std::vector<uint32_t>& d, const StwoTwiddles& t);
void stwo_interpolate(std::vector<uint32_t>& d, const StwoTwiddles& t);
// 34-column style LDE: BRT-canonic evals on CanonicCoset(log_n) -> stwo iNTT ->
// zero-pad to 2^(log_n+blowup) -> stwo NTT (BRT-canonic output).
std::vector<uint32_t> stwo_lde(const std::vector<uint32_t>& evals, uint32_t log_n, uint32_t blowup_bits,
                               const StwoTwiddles& tt, const StwoTwiddles& te);

// ---------------------------------------------------------------- Blake2s-256
// cuda/include/blake2s.cuh:29-95; src/channel.rs:222-298 (no personalisation).
using Hash = std::array<uint32_t, 8>;
void blake2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t, uint32_t f);
Hash blake2s_words(const uint32_t* words, size_t n_words);   // standard Blake2s of LE words
std::array<uint8_t, 32> blake2s_bytes(const uint8_t* data, size_t len);
Hash hash_node(const Hash& l, const Hash& r);                  // blake2s.cu:65-89

// ---------------------------------------------------------------- Merkle
// Leaf hashes: blake2s.cu:13-62 (<= 16 columns, t = min(n,16)*4),
// SoA4 leaf t = 16 (blake2s.cu:117-133), row-packed multi-block leaf
// (merkle_leaves_lifted.cu:33-98).
Hash leaf_hash_capped(const uint32_t* vals, uint32_t n_cols);
Hash leaf_hash_rowpacked(const uint32_t* vals, uint32_t n_cols);
// layers[0] = leaves ... layers.back() = {root}  (merkle.rs:804-842)
std::vector<std::vector<Hash>> merkle_layers(std::vector<Hash> leaves);
Hash merkle_root(std::vector<Hash> leaves);
std::vector<Hash> auth_path(const std::vector<std::vector<Hash>>& layers, uint64_t idx);  // merkle.rs:846-861
bool verify_auth_path(const Hash& root, const Hash& leaf, uint64_t idx, const std::vector<Hash>& path);  // merkle.rs:494-534
// Roots of common column layouts (multithreaded over leaves).
Hash merkle_root_columns_capped(const std::vector<const uint32_t*>& cols, uint64_t n_leaves, int threads = 1);
Hash merkle_root_columns_rowpacked(const std::vector<const uint32_t*>& cols, uint64_t n_leaves, int threads = 1);
Hash merkle_root_soa4(const uint32_t* const c[4], uint64_t n_leaves, int threads = 1);
// Lifted leaves (merkle_leaves_lifted.cu:33-98): columns of mixed log sizes.
std::vector<Hash> lifted_leaves(const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& col_log,
                                uint32_t lifting_log);

// ---------------------------------------------------------------- channel
// src/channel.rs:15-185
struct Channel {
  std::array<uint8_t, 32> state{};
  uint32_t n_draws = 0;
  void mix_digest(const Hash& d);
  void mix_felts(const std::vector<QM31>& felts);
  void mix_u64(uint64_t v);
  std::array<uint8_t, 32> squeeze();
  QM31 draw_felt();
  uint64_t draw_number(uint64_t bound);
  std::vector<uint64_t> draw_query_indices(uint32_t log_domain, size_t n);
  Hash state_words() const;
  // PoW (channel.rs:140-168): prefix = Blake2s(0x12345678_LE || 0^12 || state || pow_bits_LE)
  Hash pow_prefix(uint32_t pow_bits) const;
  bool verify_pow_nonce(uint32_t pow_bits, uint64_t nonce) const;
};

// Trailing zeros of the first 16 bytes (u128 LE) of Blake2s(prefix || nonce_LE)
// (grind.cu:16-79); m31_output reduces each word mod p first (grind_m31_output.cu).
uint32_t pow_trailing_zeros(const Hash& prefix, uint64_t nonce, bool m31_output);
// Smallest nonce in [offset, offset + n) with >= pow_bits trailing zeros, or UINT64_MAX.
uint64_t pow_grind_min(const Hash& prefix, uint32_t pow_bits, uint64_t offset, uint64_t n, bool m31_output, int threads);

// ---------------------------------------------------------------- FRI
// Fold twiddles: fri.rs:112-139 + twiddles.cu:23-52 (1/coord(domain.at(bitrev(2i)))).
std::vector<uint32_t> fold_twiddles(const Coset& domain, bool extract_y);
// fri.cu:44-78 — dst = dst*alpha^2 + (f0+f1) + alpha*tw*(f0-f1)
void fold_circle_into_line(QM31* dst, const QM31* src, const uint32_t* tw, QM31 alpha, uint64_t half_n);
// fri.cu:10-39 / fri.rs:411-427
void fold_line(QM31* dst, const QM31* src, const uint32_t* tw, QM31 alpha, uint64_t half_n);
std::vector<QM31> last_layer_poly_coeffs(std::vector<QM31> eval);             // fri.rs:294-336
QM31 eval_last_layer_poly(const std::vector<QM31>& coeffs, uint64_t idx, uint32_t log_size);  // fri.rs:346-384

// ---------------------------------------------------------------- quotients
// constraint.cu:10-37 — q[i] = alpha * (t[(i+2)%n] - (t[(i+1)%n] + t[i]))
QM31 fib_quotient_at(const uint32_t* t, uint64_t n, uint64_t i, QM31 alpha);
// quotient.cu:25-68
void accumulate_numerators(const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& col_idx,
                           const std::vector<QM31>& b, const std::vector<QM31>& c, uint64_t n_rows, QM31* out);
// quotient.cu:101-197
struct QuotAcc { QM31 spx, spy, first_linear; const QM31* numer; uint32_t log_size; };
void quotients_combine(const std::vector<QuotAcc>& accs, const uint32_t* dxs, const uint32_t* dys,
                       uint32_t lifting_log, uint64_t n_rows, QM31* out);
// oods.rs:33-75, 133-161, 340-367
struct OodsPoint { QM31 x, y; };
OodsPoint oods_point_from_channel(Channel& ch);
QM31 eval_at_oods_from_coeffs(const std::vector<uint32_t>& coeffs, OodsPoint z);
void compute_line_coeffs(OodsPoint z, QM31 v, QM31& a, QM31& b);
CPoint canonic_domain_point(uint64_t j, uint32_t log_eval);  // cairo_air/prover.rs:161-165

// ---------------------------------------------------------------- Cairo group commitment
// circle.rs:232-253: vanishing polynomial of a coset at a point
uint32_t coset_vanishing_at(const Coset& c, CPoint p);
// cairo_air/prover.rs:924-935: Z_H of half_coset(log_n) at the BRT-canonic points of the 4x domain
std::vector<uint32_t> zh_eval_domain(uint32_t log_n);
// cairo_air/prover.rs:955-1047 for one group (<= 16 columns), with merkle.rs:360-417
struct GroupCommit {
  std::vector<std::vector<uint32_t>> coeffs, eval_cn, eval_hc;
  Hash root;
  std::vector<Hash> tile_roots;
};
GroupCommit commit_group_cairo(const std::vector<std::vector<uint32_t>>& cols_hc, uint32_t log_n,
                               const std::vector<uint32_t>& blind, int threads);

// ---------------------------------------------------------------- Cairo OODS + FRI tail
// cairo_air/prover.rs:1937-2438: AIR quotient commitment, OODS sampling of the
// trace / interaction / quotient columns, DEEP (OODS) quotient, its commitment
// and the FRI fold chain down to 8 values, ending with the mix of the last-layer
// line-polynomial coefficients.
struct CairoOodsFri {
  Hash quotient_root;
  std::vector<Hash> quotient_tiles;
  OodsPoint z;
  std::vector<QM31> trace_at_z, trace_at_z_next, inter_at_z, inter_at_z_next;
  QM31 quotient_at_z[4];
  QM31 oods_alpha;
  std::vector<uint32_t> oods_q[4];  // BRT-canonic SoA
  Hash oods_root;
  std::vector<Hash> oods_tiles;
  std::vector<QM31> fri_alphas;     // [0] = circle fold
  std::vector<Hash> fri_roots;      // committed line layers, log_eval - 1 down to 4
  std::vector<QM31> last_layer, last_layer_coeffs;  // 8 evaluations; 8 coefficients in BRT order
};
CairoOodsFri cairo_oods_fri(Channel& ch, uint32_t log_n, const std::vector<std::vector<uint32_t>>& trace_coeffs,
                            const std::vector<uint32_t>& zk, const std::vector<std::vector<uint32_t>>& trace_evals,
                            const std::vector<std::vector<uint32_t>>& inter_evals,
                            const std::vector<std::vector<uint32_t>>& quot_hc, int threads);

// ---------------------------------------------------------------- Fibonacci AIR + prover
// air.rs:16-25 (additive recurrence, t0 = a, t1 = b)
std::vector<uint32_t> fibonacci_trace(uint32_t a, uint32_t b, uint32_t log_n);

constexpr uint32_t BLOWUP_BITS = 2;  // prover.rs:86
constexpr uint32_t N_QUERIES = 80;   // prover.rs:90
constexpr uint32_t LOG_LAST_LAYER = 3;  // fri.rs:265

template <class T> struct Decommit {
  std::vector<T> values, sibling_values;
  std::vector<std::vector<Hash>> auth_paths, sibling_auth_paths;
};
using Q4 = std::array<uint32_t, 4>;
struct StarkProof {  // prover.rs:116-137
  Hash trace_commitment{}, quotient_commitment{};
  std::vector<Hash> fri_commitments;
  std::vector<QM31> fri_last_layer;
  uint32_t log_trace_size = 0, a = 0, b = 0;
  std::vector<uint64_t> query_indices;
  Decommit<uint32_t> trace_decommitment;
  Decommit<Q4> quotient_decommitment;
  std::vector<Decommit<Q4>> fri_decommitments;
};
// prover.rs:1721-1978 (prove_with_cache stage order). threads = host threads for hashing.
StarkProof prove(uint32_t a, uint32_t b, uint32_t log_n, int threads = 1);
// verifier.rs:39-236. Returns "" when the proof is accepted, else the reason.
std::string verify(const StarkProof& p);
// stark_cli.rs:907-976 ("KRAK" v1, little-endian u32 words)
std::vector<uint8_t> serialize_proof(const StarkProof& p);
bool deserialize_proof(const uint8_t* data, size_t len, StarkProof& out);

// ---------------------------------------------------------------- stwo Backend adapter kernels
// gather.cu:10-18: dst[i] = src[idx[i]]
void gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint64_t n);
// gather.cu:22-40: dst[8i..8i+8) = src[8 idx[i] .. 8 idx[i]+8)
void gather_u256(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint64_t n);
// barycentric_eval.cu:30-83 with 256 threads per block: out[4b..4b+4) = sum of
// evals[i] * weights[i] (QM31 weights, 4 words each) over i with (i / 256) mod n_blocks == b.
void barycentric_partials(const uint32_t* evals, const uint32_t* weights, uint64_t n, uint32_t n_blocks, uint32_t* out);
// accumulate_lift.cu:16-37: col[i] += curr[((i >> (log_ratio + 1)) << 1) | (i & 1)], QM31 elements of 4 words.
void accumulate_lift(uint32_t* col, const uint32_t* curr, uint64_t col_n, uint32_t log_ratio);
// pack_leaves.cu:22-38: out[16c + p][j] = in[c][16j + p] for every input word 16j + p < n.
void pack_leaves(const uint32_t* const in[4], uint32_t* const out[64], uint64_t n);

// ---------------------------------------------------------------- seeded inputs
// SplitMix64; uniform M31 = (u64 >> 33) rejecting P.
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  uint32_t m31() {
    for (;;) { uint32_t v = (uint32_t)(next() >> 33); if (v != P) return v; }
  }
};

}  // namespace vso
