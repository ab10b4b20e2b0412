// C entry points of the CPU oracle, loaded by tests/ and bench.py (cpu baseline)
// through ctypes. TEST INFRASTRUCTURE ONLY — the product library never calls this.
#include <chrono>
#include <cstring>
#include <thread>

#include "oracle.h"

using namespace vso;

namespace {
Coset make_coset(uint32_t kind, uint32_t log_n) {
  switch (kind) {
    case 0: return coset_half_coset(log_n);
    case 1: return coset_half_odds(log_n);
    default: return coset_subgroup(log_n);
  }
}
QM31 q(const uint32_t* v) { return {{v[0], v[1], v[2], v[3]}}; }
void put(uint32_t* o, const QM31& x) { std::memcpy(o, x.v, 16); }
void put_hash(uint32_t* o, const Hash& h) { std::memcpy(o, h.data(), 32); }
std::vector<QM31> soa_to_aos(const uint32_t* const c[4], uint64_t n) {
  std::vector<QM31> v(n);
  for (uint64_t i = 0; i < n; i++) v[i] = {{c[0][i], c[1][i], c[2][i], c[3][i]}};
  return v;
}
void aos_to_soa(const std::vector<QM31>& v, uint32_t* const c[4]) {
  for (uint64_t i = 0; i < v.size(); i++)
    for (int k = 0; k < 4; k++) c[k][i] = v[i].v[k];
}
struct ChState { uint8_t state[32]; uint32_t n_draws; };
Channel load(const ChState* s) { Channel c; std::memcpy(c.state.data(), s->state, 32); c.n_draws = s->n_draws; return c; }
void store(ChState* s, const Channel& c) { std::memcpy(s->state, c.state.data(), 32); s->n_draws = c.n_draws; }
}  // namespace

extern "C" {

void oracle_coset(uint32_t kind, uint32_t log_n, uint32_t* out4) {
  Coset c = make_coset(kind, log_n);
  out4[0] = c.initial.x; out4[1] = c.initial.y; out4[2] = c.step.x; out4[3] = c.step.y;
}
void oracle_coset_points(uint32_t ix, uint32_t iy, uint32_t sx, uint32_t sy, uint64_t n, uint32_t* ox, uint32_t* oy) {
  CPoint cur{ix, iy}, st{sx, sy};
  for (uint64_t i = 0; i < n; i++) { ox[i] = cur.x; oy[i] = cur.y; cur = cp_mul(cur, st); }
}
uint32_t oracle_m31_mul(uint32_t a, uint32_t b) { return m31_mul(a, b); }
uint32_t oracle_m31_inv(uint32_t a) { return m31_inv(a); }
void oracle_qm31_mul(const uint32_t* a, const uint32_t* b, uint32_t* o) { put(o, qm_mul(q(a), q(b))); }
void oracle_qm31_inv(const uint32_t* a, uint32_t* o) { put(o, qm_inv(q(a))); }
void oracle_cm31_mul(const uint32_t* a, const uint32_t* b, uint32_t* o) {
  CM31 r = cm_mul({a[0], a[1]}, {b[0], b[1]});
  o[0] = r.a; o[1] = r.b;
}
void oracle_cp_repeated_double(uint32_t x, uint32_t y, uint32_t n, uint32_t* o) {
  CPoint p = cp_repeated_double({x, y}, n);
  o[0] = p.x; o[1] = p.y;
}

void oracle_batch_inverse(const uint32_t* in, uint32_t* out, uint64_t n) {
  std::vector<uint32_t> v(in, in + n);
  auto r = batch_inverse_chunked(v);
  std::memcpy(out, r.data(), n * 4);
}

// Native twiddles for half_coset(log_n) (kind 0) or another coset kind.
// Buffers: line/iline n-1, circle/icircle n/2, offsets/sizes log_n-1.
void oracle_native_twiddles(uint32_t kind, uint32_t log_n, uint32_t* line, uint32_t* circle, uint32_t* iline,
                            uint32_t* icircle, uint32_t* offsets, uint32_t* sizes) {
  NativeTwiddles t = native_twiddles(make_coset(kind, log_n));
  std::memcpy(line, t.line.data(), t.line.size() * 4);
  std::memcpy(iline, t.iline.data(), t.iline.size() * 4);
  std::memcpy(circle, t.circle.data(), t.circle.size() * 4);
  std::memcpy(icircle, t.icircle.data(), t.icircle.size() * 4);
  std::memcpy(offsets, t.offsets.data(), t.offsets.size() * 4);
  std::memcpy(sizes, t.sizes.data(), t.sizes.size() * 4);
}
void oracle_native_evaluate(uint32_t* d, uint32_t log_n) {
  std::vector<uint32_t> v(d, d + (1ull << log_n));
  native_evaluate(v, native_twiddles(coset_half_coset(log_n)));
  std::memcpy(d, v.data(), v.size() * 4);
}
void oracle_native_interpolate(uint32_t* d, uint32_t log_n) {
  std::vector<uint32_t> v(d, d + (1ull << log_n));
  native_interpolate(v, native_twiddles(coset_half_coset(log_n)));
  std::memcpy(d, v.data(), v.size() * 4);
}
void oracle_ntt_layer(uint32_t* d, uint64_t n, const uint32_t* tw, uint32_t layer_idx, int fwd) {
  ntt_layer(d, n, tw, layer_idx, fwd != 0);
}
void oracle_bit_reverse(uint32_t* d, uint32_t log_n) {
  std::vector<uint32_t> v(d, d + (1ull << log_n));
  bit_reverse_inplace(v, log_n);
  std::memcpy(d, v.data(), v.size() * 4);
}
void oracle_stwo_twiddles(uint32_t log_n, uint32_t* fwd, uint32_t* inv) {
  StwoTwiddles t = stwo_twiddles(log_n);
  std::memcpy(fwd, t.fwd.data(), t.fwd.size() * 4);
  std::memcpy(inv, t.inv.data(), t.inv.size() * 4);
}
void oracle_stwo_evaluate(uint32_t* d, uint32_t log_n) {
  std::vector<uint32_t> v(d, d + (1ull << log_n));
  stwo_evaluate(v, stwo_twiddles(log_n));
  std::memcpy(d, v.data(), v.size() * 4);
}
void oracle_stwo_interpolate(uint32_t* d, uint32_t log_n) {
  std::vector<uint32_t> v(d, d + (1ull << log_n));
  stwo_interpolate(v, stwo_twiddles(log_n));
  std::memcpy(d, v.data(), v.size() * 4);
}
// LDE of n_cols columns (column-major, each 2^log_n BRT-canonic evals) into
// out (column-major, each 2^(log_n+blowup)); columns run on `threads` threads.
void oracle_stwo_lde_columns(const uint32_t* in, uint32_t n_cols, uint32_t log_n, uint32_t blowup, uint32_t* out,
                             int threads) {
  StwoTwiddles tt = stwo_twiddles(log_n), te = stwo_twiddles(log_n + blowup);
  const uint64_t n = 1ull << log_n, N = n << blowup;
  auto work = [&](uint32_t c0, uint32_t c1) {
    for (uint32_t c = c0; c < c1; c++) {
      std::vector<uint32_t> ev(in + c * n, in + (c + 1) * n);
      auto e = stwo_lde(ev, log_n, blowup, tt, te);
      std::memcpy(out + c * N, e.data(), N * 4);
    }
  };
  if (threads <= 1) { work(0, n_cols); return; }
  std::vector<std::thread> ts;
  uint32_t per = (n_cols + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    uint32_t c0 = t * per, c1 = std::min(n_cols, c0 + per);
    if (c0 < c1) ts.emplace_back(work, c0, c1);
  }
  for (auto& t : ts) t.join();
}

void oracle_blake2s_bytes(const uint8_t* d, uint64_t len, uint8_t* out32) {
  auto h = blake2s_bytes(d, len);
  std::memcpy(out32, h.data(), 32);
}
void oracle_blake2s_words(const uint32_t* w, uint64_t n, uint32_t* out8) { put_hash(out8, blake2s_words(w, n)); }

// Merkle helpers. `cols` is column-major (n_cols x n_leaves).
void oracle_leaf_hashes_capped(const uint32_t* cols, uint32_t n_cols, uint64_t n_leaves, uint32_t* out) {
  uint32_t row[16] = {0};
  uint32_t nc = n_cols < 16 ? n_cols : 16;
  for (uint64_t i = 0; i < n_leaves; i++) {
    for (uint32_t c = 0; c < nc; c++) row[c] = cols[c * n_leaves + i];
    put_hash(out + 8 * i, leaf_hash_capped(row, n_cols));
  }
}
void oracle_hash_nodes(const uint32_t* children, uint64_t n_parents, uint32_t* out) {
  for (uint64_t i = 0; i < n_parents; i++) {
    Hash l, r;
    std::memcpy(l.data(), children + 16 * i, 32);
    std::memcpy(r.data(), children + 16 * i + 8, 32);
    put_hash(out + 8 * i, hash_node(l, r));
  }
}
void oracle_merkle_root_hashes(const uint32_t* hashes, uint64_t n, uint32_t* out8) {
  std::vector<Hash> v(n);
  for (uint64_t i = 0; i < n; i++) std::memcpy(v[i].data(), hashes + 8 * i, 32);
  put_hash(out8, merkle_root(std::move(v)));
}
void oracle_merkle_root_capped(const uint32_t* cols, uint32_t n_cols, uint64_t n_leaves, int threads, uint32_t* out8) {
  std::vector<const uint32_t*> c;
  for (uint32_t i = 0; i < n_cols; i++) c.push_back(cols + i * n_leaves);
  put_hash(out8, merkle_root_columns_capped(c, n_leaves, threads));
}
void oracle_merkle_root_rowpacked(const uint32_t* cols, uint32_t n_cols, uint64_t n_leaves, int threads, uint32_t* out8) {
  std::vector<const uint32_t*> c;
  for (uint32_t i = 0; i < n_cols; i++) c.push_back(cols + i * n_leaves);
  put_hash(out8, merkle_root_columns_rowpacked(c, n_leaves, threads));
}
void oracle_merkle_root_soa4(const uint32_t* c0, const uint32_t* c1, const uint32_t* c2, const uint32_t* c3,
                             uint64_t n_leaves, int threads, uint32_t* out8) {
  const uint32_t* c[4] = {c0, c1, c2, c3};
  put_hash(out8, merkle_root_soa4(c, n_leaves, threads));
}
void oracle_lifted_leaves(const uint32_t* const* cols, const uint32_t* col_log, uint32_t n_cols, uint32_t lifting_log,
                          uint32_t* out) {
  std::vector<const uint32_t*> c(cols, cols + n_cols);
  std::vector<uint32_t> l(col_log, col_log + n_cols);
  auto h = lifted_leaves(c, l, lifting_log);
  for (size_t i = 0; i < h.size(); i++) put_hash(out + 8 * i, h[i]);
}

// Channel (state = 32 bytes + u32 draw counter).
void oracle_ch_mix_digest(ChState* s, const uint32_t* d8) {
  Channel c = load(s); Hash h; std::memcpy(h.data(), d8, 32); c.mix_digest(h); store(s, c);
}
void oracle_ch_mix_felts(ChState* s, const uint32_t* f, uint64_t n) {
  Channel c = load(s); std::vector<QM31> v(n);
  for (uint64_t i = 0; i < n; i++) v[i] = q(f + 4 * i);
  c.mix_felts(v); store(s, c);
}
void oracle_ch_mix_u64(ChState* s, uint64_t v) { Channel c = load(s); c.mix_u64(v); store(s, c); }
void oracle_ch_draw_felt(ChState* s, uint32_t* o4) { Channel c = load(s); put(o4, c.draw_felt()); store(s, c); }
uint64_t oracle_ch_draw_number(ChState* s, uint64_t bound) { Channel c = load(s); uint64_t r = c.draw_number(bound); store(s, c); return r; }
void oracle_ch_pow_prefix(const ChState* s, uint32_t pow_bits, uint32_t* out8) {
  Hash h = load(s).pow_prefix(pow_bits);
  for (int k = 0; k < 8; k++) out8[k] = h[k];
}
int oracle_ch_verify_pow(const ChState* s, uint32_t pow_bits, uint64_t nonce) {
  return load(s).verify_pow_nonce(pow_bits, nonce) ? 1 : 0;
}
uint32_t oracle_pow_trailing_zeros(const uint32_t* prefix8, uint64_t nonce, int m31_output) {
  Hash h{};
  for (int k = 0; k < 8; k++) h[k] = prefix8[k];
  return pow_trailing_zeros(h, nonce, m31_output != 0);
}
uint64_t oracle_pow_grind_min(const uint32_t* prefix8, uint32_t pow_bits, uint64_t offset, uint64_t n, int m31_output,
                              int threads) {
  Hash h{};
  for (int k = 0; k < 8; k++) h[k] = prefix8[k];
  return pow_grind_min(h, pow_bits, offset, n, m31_output != 0, threads);
}
void oracle_ch_draw_queries(ChState* s, uint32_t log_domain, uint64_t n, uint64_t* out) {
  Channel c = load(s); auto r = c.draw_query_indices(log_domain, n); std::memcpy(out, r.data(), n * 8); store(s, c);
}

// FRI
void oracle_fold_twiddles(uint32_t kind, uint32_t log_n, int extract_y, uint32_t* out) {
  auto t = fold_twiddles(make_coset(kind, log_n), extract_y != 0);
  std::memcpy(out, t.data(), t.size() * 4);
}
// Row r of CanonicCoset(log_size)'s circle domain at bit_reverse_index(r): the
// domain points the stwo adapter builds per call (crates/cuda-backend/src/
// quotient_ops.rs:135-140; CircleDomain::at over half_odds(log_size - 1)).
void oracle_canonic_domain_points(uint32_t log_size, uint32_t* xs, uint32_t* ys) {
  const uint64_t n = 1ull << log_size;
  for (uint64_t r = 0; r < n; r++) {
    const CPoint p = canonic_domain_point(bit_reverse(r, log_size), log_size);
    xs[r] = p.x;
    ys[r] = p.y;
  }
}
// Generic coset (matches cuda_compute_fold_twiddle_sources + cuda_batch_inverse_m31).
void oracle_fold_twiddles_generic(uint32_t ix, uint32_t iy, uint32_t sx, uint32_t sy, uint32_t log_n, int extract_y,
                                  uint32_t* out) {
  Coset c{{ix, iy}, {sx, sy}, log_n};
  auto t = fold_twiddles(c, extract_y != 0);
  std::memcpy(out, t.data(), t.size() * 4);
}
void oracle_fold_circle_into_line(uint32_t* const dst[4], const uint32_t* const src[4], const uint32_t* tw,
                                  const uint32_t* alpha, const uint32_t* alpha_sq, uint64_t half_n) {
  QM31 a = q(alpha), a2 = q(alpha_sq);
  for (uint64_t i = 0; i < half_n; i++) {
    QM31 f0{{src[0][2 * i], src[1][2 * i], src[2][2 * i], src[3][2 * i]}};
    QM31 f1{{src[0][2 * i + 1], src[1][2 * i + 1], src[2][2 * i + 1], src[3][2 * i + 1]}};
    QM31 fp = qm_add(qm_add(f0, f1), qm_mul(a, qm_scale(qm_sub(f0, f1), tw[i])));
    QM31 prev{{dst[0][i], dst[1][i], dst[2][i], dst[3][i]}};
    QM31 r = qm_add(qm_mul(prev, a2), fp);
    for (int k = 0; k < 4; k++) dst[k][i] = r.v[k];
  }
}
void oracle_fold_line(const uint32_t* const src[4], const uint32_t* tw, uint32_t* const dst[4], const uint32_t* alpha,
                      uint64_t half_n) {
  std::vector<QM31> s = soa_to_aos(src, 2 * half_n), d(half_n);
  fold_line(d.data(), s.data(), tw, q(alpha), half_n);
  aos_to_soa(d, dst);
}
void oracle_last_layer_poly_coeffs(const uint32_t* evals, uint64_t n, uint32_t* out) {
  std::vector<QM31> e(n);
  for (uint64_t i = 0; i < n; i++) e[i] = q(evals + 4 * i);
  auto c = last_layer_poly_coeffs(e);
  for (size_t i = 0; i < c.size(); i++) put(out + 4 * i, c[i]);
}
void oracle_eval_last_layer_poly(const uint32_t* coeffs, uint64_t n, uint64_t idx, uint32_t log_size, uint32_t* out) {
  std::vector<QM31> c(n);
  for (uint64_t i = 0; i < n; i++) c[i] = q(coeffs + 4 * i);
  put(out, eval_last_layer_poly(c, idx, log_size));
}

// Quotients
void oracle_fib_quotient(const uint32_t* t, uint64_t n, const uint32_t* alpha, uint32_t* const out[4]) {
  for (uint64_t i = 0; i < n; i++) {
    QM31 r = fib_quotient_at(t, n, i, q(alpha));
    for (int k = 0; k < 4; k++) out[k][i] = r.v[k];
  }
}
void oracle_accumulate_numerators(const uint32_t* const* cols, const uint32_t* col_idx, const uint32_t* b,
                                  const uint32_t* c, uint32_t n_batch, uint64_t n_rows, uint32_t* const out[4]) {
  uint32_t max_idx = 0;
  for (uint32_t i = 0; i < n_batch; i++) max_idx = col_idx[i] > max_idx ? col_idx[i] : max_idx;
  std::vector<const uint32_t*> cv(cols, cols + (n_batch ? max_idx + 1 : 0));
  std::vector<uint32_t> ci(col_idx, col_idx + n_batch);
  std::vector<QM31> bv(n_batch), cvv(n_batch), o(n_rows);
  for (uint32_t i = 0; i < n_batch; i++) { bv[i] = q(b + 4 * i); cvv[i] = q(c + 4 * i); }
  accumulate_numerators(cv, ci, bv, cvv, n_rows, o.data());
  aos_to_soa(o, out);
}
void oracle_quotients_combine(const uint32_t* spx, const uint32_t* spy, const uint32_t* fla,
                              const uint32_t* const* n0, const uint32_t* const* n1, const uint32_t* const* n2,
                              const uint32_t* const* n3, const uint32_t* acc_log, uint32_t n_accs,
                              const uint32_t* dxs, const uint32_t* dys, uint32_t lifting_log, uint64_t n_rows,
                              uint32_t* const out[4]) {
  std::vector<std::vector<QM31>> numer(n_accs);
  std::vector<QuotAcc> accs(n_accs);
  for (uint32_t j = 0; j < n_accs; j++) {
    uint64_t sz = 1ull << acc_log[j];
    const uint32_t* c[4] = {n0[j], n1[j], n2[j], n3[j]};
    numer[j] = soa_to_aos(c, sz);
    accs[j] = {q(spx + 4 * j), q(spy + 4 * j), q(fla + 4 * j), numer[j].data(), acc_log[j]};
  }
  std::vector<QM31> o(n_rows);
  quotients_combine(accs, dxs, dys, lifting_log, n_rows, o.data());
  aos_to_soa(o, out);
}
void oracle_oods_point(ChState* s, uint32_t* out8) {
  Channel c = load(s);
  OodsPoint z = oods_point_from_channel(c);
  put(out8, z.x); put(out8 + 4, z.y);
  store(s, c);
}
void oracle_eval_at_oods(const uint32_t* coeffs, uint64_t n, const uint32_t* z8, uint32_t* out4) {
  std::vector<uint32_t> c(coeffs, coeffs + n);
  put(out4, eval_at_oods_from_coeffs(c, {q(z8), q(z8 + 4)}));
}
void oracle_line_coeffs(const uint32_t* z8, const uint32_t* v, uint32_t* a4, uint32_t* b4) {
  QM31 a, b;
  compute_line_coeffs({q(z8), q(z8 + 4)}, q(v), a, b);
  put(a4, a); put(b4, b);
}

// AIR / prover / verifier / serialization
void oracle_fib_trace(uint32_t a, uint32_t b, uint32_t log_n, uint32_t* out) {
  auto t = fibonacci_trace(a, b, log_n);
  std::memcpy(out, t.data(), t.size() * 4);
}
// Returns the KRAK byte length; writes at most `cap` bytes into out.
uint64_t oracle_prove(uint32_t a, uint32_t b, uint32_t log_n, int threads, uint8_t* out, uint64_t cap) {
  auto bytes = serialize_proof(prove(a, b, log_n, threads));
  if (out) std::memcpy(out, bytes.data(), std::min<uint64_t>(cap, bytes.size()));
  return bytes.size();
}
// 0 = accepted, 1 = rejected (reason in err), 2 = undecodable.
int oracle_verify(const uint8_t* data, uint64_t len, char* err, uint64_t cap) {
  StarkProof p;
  if (!deserialize_proof(data, len, p)) { if (err && cap) std::snprintf(err, cap, "undecodable proof"); return 2; }
  std::string e = verify(p);
  if (err && cap) std::snprintf(err, cap, "%s", e.c_str());
  return e.empty() ? 0 : 1;
}

// Seeded inputs: SplitMix64 counter stream, uniform M31 (see oracle.h and the
// product's generator, which must agree).
void oracle_seeded_m31(uint64_t seed, uint64_t offset, uint64_t n, uint32_t* out) {
  for (uint64_t k = 0; k < n; k++) {
    uint64_t c = offset + k;
    SplitMix64 g(seed + 0x9E3779B97F4A7C15ull * c);
    uint32_t v = (uint32_t)(g.next() >> 33);
    if (v == P) { v = (uint32_t)(g.next() >> 33); if (v == P) v = 0; }
    out[k] = v;
  }
}

// CPU baseline for the commitment-layer workload: LDE + row-packed root of
// n_cols columns (column-major, BRT-canonic evals), on `threads` threads.
// Returns wall seconds.
double oracle_bench_commit(const uint32_t* cols, uint32_t n_cols, uint32_t log_n, uint32_t blowup, int threads,
                           uint32_t* root8) {
  auto t0 = std::chrono::steady_clock::now();
  const uint64_t N = 1ull << (log_n + blowup);
  std::vector<uint32_t> lde((uint64_t)n_cols * N);
  oracle_stwo_lde_columns(cols, n_cols, log_n, blowup, lde.data(), threads);
  oracle_merkle_root_rowpacked(lde.data(), n_cols, N, threads, root8);
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
// CPU baseline for the FRI fold+commit chain on one QM31 vector (SoA4):
// circle fold on half_coset(log_n), line folds on half_odds down to 2^3,
// committing every folded layer. alphas: (log_n - 3) QM31. roots: (log_n - 3) x 8.
double oracle_bench_fri(const uint32_t* const src[4], uint32_t log_n, const uint32_t* alphas, int threads,
                        uint32_t* roots, uint32_t* last8x4) {
  auto t0 = std::chrono::steady_clock::now();
  std::vector<QM31> cur = soa_to_aos(src, 1ull << log_n);
  uint32_t cl = log_n;
  for (uint32_t layer = 0; cl > LOG_LAST_LAYER; layer++) {
    bool circle = layer == 0;
    auto tw = fold_twiddles(circle ? coset_half_coset(cl) : coset_half_odds(cl), circle);
    std::vector<QM31> nx(cur.size() / 2, QM31{{0, 0, 0, 0}});
    if (circle) fold_circle_into_line(nx.data(), cur.data(), tw.data(), q(alphas + 4 * layer), nx.size());
    else fold_line(nx.data(), cur.data(), tw.data(), q(alphas + 4 * layer), nx.size());
    cl--;
    std::vector<uint32_t> s[4];
    for (int k = 0; k < 4; k++) { s[k].resize(nx.size()); for (size_t i = 0; i < nx.size(); i++) s[k][i] = nx[i].v[k]; }
    const uint32_t* c[4] = {s[0].data(), s[1].data(), s[2].data(), s[3].data()};
    put_hash(roots + 8 * layer, merkle_root_soa4(c, nx.size(), threads));
    cur.swap(nx);
  }
  for (size_t i = 0; i < cur.size(); i++) put(last8x4 + 4 * i, cur[i]);
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"

extern "C" void oracle_commit_group_cairo(const uint32_t* cols_hc, uint32_t n_cols, uint32_t log_n, const uint32_t* blind,
                                          uint32_t* coeffs, uint32_t* eval_cn, uint32_t* eval_hc, uint32_t* root,
                                          uint32_t* tile_roots, int threads) {
  const uint64_t n = 1ull << log_n, N = n << 2;
  std::vector<std::vector<uint32_t>> cols(n_cols);
  for (uint32_t c = 0; c < n_cols; c++) cols[c].assign(cols_hc + c * n, cols_hc + (c + 1) * n);
  std::vector<uint32_t> b(blind, blind + n_cols);
  GroupCommit g = commit_group_cairo(cols, log_n, b, threads);
  for (uint32_t c = 0; c < n_cols; c++) {
    std::copy(g.coeffs[c].begin(), g.coeffs[c].end(), coeffs + c * n);
    std::copy(g.eval_cn[c].begin(), g.eval_cn[c].end(), eval_cn + c * N);
    std::copy(g.eval_hc[c].begin(), g.eval_hc[c].end(), eval_hc + c * N);
  }
  for (int k = 0; k < 8; k++) root[k] = g.root[k];
  for (size_t t = 0; t < g.tile_roots.size(); t++)
    for (int k = 0; k < 8; k++) tile_roots[8 * t + k] = g.tile_roots[t][k];
}
extern "C" void oracle_zh_eval_domain(uint32_t log_n, uint32_t* out) {
  auto z = zh_eval_domain(log_n);
  std::copy(z.begin(), z.end(), out);
}
extern "C" uint32_t oracle_coset_vanishing_half_coset(uint32_t log_n, uint32_t x, uint32_t y) {
  return coset_vanishing_at(coset_half_coset(log_n), CPoint{x, y});
}

// Cairo OODS + FRI tail. Flat inputs: trace_coeffs nt x 2^log_n, trace_evals nt x N,
// inter_evals ni x N, quot_hc 4 x N (N = 2^(log_n+2)). Outputs as in CairoOodsFri;
// tiles hold max(1, N/1024) hashes, fri_roots log_n - 2, fri_alphas log_n - 1.
extern "C" void oracle_cairo_oods_fri(ChState* s, uint32_t log_n, const uint32_t* trace_coeffs, uint32_t nt,
                                      const uint32_t* zk, const uint32_t* trace_evals, const uint32_t* inter_evals,
                                      uint32_t ni, const uint32_t* quot_hc, uint32_t* quotient_root,
                                      uint32_t* quotient_tiles, uint32_t* z8, uint32_t* trace_at_z,
                                      uint32_t* trace_at_zn, uint32_t* inter_at_z, uint32_t* inter_at_zn,
                                      uint32_t* quot_at_z16, uint32_t* alpha4, uint32_t* oods_q, uint32_t* oods_root,
                                      uint32_t* oods_tiles, uint32_t* fri_roots, uint32_t* fri_alphas,
                                      uint32_t* last32, uint32_t* coeffs32, int threads) {
  const uint64_t n = 1ull << log_n, N = n << 2;
  std::vector<std::vector<uint32_t>> tc(nt), te(nt), ie(ni), qh(4);
  for (uint32_t c = 0; c < nt; c++) {
    tc[c].assign(trace_coeffs + c * n, trace_coeffs + (c + 1) * n);
    te[c].assign(trace_evals + c * N, trace_evals + (c + 1) * N);
  }
  for (uint32_t c = 0; c < ni; c++) ie[c].assign(inter_evals + c * N, inter_evals + (c + 1) * N);
  for (int k = 0; k < 4; k++) qh[k].assign(quot_hc + k * N, quot_hc + (k + 1) * N);
  std::vector<uint32_t> z(zk, zk + nt);
  Channel ch = load(s);
  CairoOodsFri r = cairo_oods_fri(ch, log_n, tc, z, te, ie, qh, threads);
  store(s, ch);
  put_hash(quotient_root, r.quotient_root);
  for (size_t t = 0; t < r.quotient_tiles.size(); t++) put_hash(quotient_tiles + 8 * t, r.quotient_tiles[t]);
  put(z8, r.z.x);
  put(z8 + 4, r.z.y);
  for (uint32_t c = 0; c < nt; c++) { put(trace_at_z + 4 * c, r.trace_at_z[c]); put(trace_at_zn + 4 * c, r.trace_at_z_next[c]); }
  for (uint32_t c = 0; c < ni; c++) { put(inter_at_z + 4 * c, r.inter_at_z[c]); put(inter_at_zn + 4 * c, r.inter_at_z_next[c]); }
  for (int k = 0; k < 4; k++) put(quot_at_z16 + 4 * k, r.quotient_at_z[k]);
  put(alpha4, r.oods_alpha);
  for (int k = 0; k < 4; k++) std::copy(r.oods_q[k].begin(), r.oods_q[k].end(), oods_q + k * N);
  put_hash(oods_root, r.oods_root);
  for (size_t t = 0; t < r.oods_tiles.size(); t++) put_hash(oods_tiles + 8 * t, r.oods_tiles[t]);
  for (size_t i = 0; i < r.fri_roots.size(); i++) put_hash(fri_roots + 8 * i, r.fri_roots[i]);
  for (size_t i = 0; i < r.fri_alphas.size(); i++) put(fri_alphas + 4 * i, r.fri_alphas[i]);
  for (int i = 0; i < 8; i++) { put(last32 + 4 * i, r.last_layer[i]); put(coeffs32 + 4 * i, r.last_layer_coeffs[i]); }
}

// Full-tree auth paths (merkle.rs:846-861) of a capped-leaf (kind 0, <= 16 used
// columns) or SoA4 (kind 1) tree over flat columns (n_cols x 2^log_n).
extern "C" void oracle_tree_paths(uint32_t kind, const uint32_t* cols, uint32_t n_cols, uint32_t log_n,
                                  const uint64_t* idx, uint32_t n_idx, uint32_t* out_paths, int threads) {
  const uint64_t n = 1ull << log_n;
  std::vector<Hash> leaves(n);
  for (uint64_t i = 0; i < n; i++) {
    uint32_t row[16] = {0};
    const uint32_t used = std::min<uint32_t>(n_cols, 16);
    for (uint32_t c = 0; c < used; c++) row[c] = cols[c * n + i];
    leaves[i] = kind == 1 ? blake2s_words(row, 4) : leaf_hash_capped(row, n_cols);
  }
  (void)threads;
  auto layers = merkle_layers(std::move(leaves));
  for (uint32_t q = 0; q < n_idx; q++) {
    auto p = auth_path(layers, idx[q]);
    for (size_t k = 0; k < p.size(); k++) put_hash(out_paths + ((uint64_t)q * log_n + k) * 8, p[k]);
  }
}

// stwo Backend adapter kernels (gather.cu, barycentric_eval.cu, accumulate_lift.cu, pack_leaves.cu).
extern "C" void oracle_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint64_t n) {
  gather_u32(src, idx, dst, n);
}
extern "C" void oracle_gather_u256(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint64_t n) {
  gather_u256(src, idx, dst, n);
}
extern "C" void oracle_barycentric_partials(const uint32_t* evals, const uint32_t* weights, uint64_t n,
                                            uint32_t n_blocks, uint32_t* out) {
  barycentric_partials(evals, weights, n, n_blocks, out);
}
extern "C" void oracle_accumulate_lift(uint32_t* col, const uint32_t* curr, uint64_t col_n, uint32_t log_ratio) {
  accumulate_lift(col, curr, col_n, log_ratio);
}
// in_flat: 4 columns of n words back to back; out_flat: 64 columns of out_len words.
extern "C" void oracle_pack_leaves(const uint32_t* in_flat, uint64_t n, uint32_t* out_flat, uint64_t out_len) {
  const uint32_t* in[4];
  uint32_t* out[64];
  for (int c = 0; c < 4; c++) in[c] = in_flat + c * n;
  for (int c = 0; c < 64; c++) out[c] = out_flat + c * out_len;
  pack_leaves(in, out, n);
}
