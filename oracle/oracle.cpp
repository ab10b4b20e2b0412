// CPU oracle for the VortexSTARK polynomial-commitment hot path.
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); see oracle.h.
#include "oracle.h"

#include <algorithm>
#include <cstring>
#include <functional>
#include <mutex>
#include <stdexcept>
#include <thread>

namespace vso {

// ------------------------------------------------------------------ helpers
static void parallel_for(uint64_t n, int threads, const std::function<void(uint64_t, uint64_t)>& fn) {
  if (threads <= 1 || n < 4096) { fn(0, n); return; }
  std::vector<std::thread> ts;
  uint64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    uint64_t lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    ts.emplace_back(fn, lo, hi);
  }
  for (auto& t : ts) t.join();
}

// ------------------------------------------------------------------ field
uint32_t m31_pow(uint32_t a, uint32_t e) {  // m31.rs:40-52
  uint32_t r = 1, b = a;
  while (e) { if (e & 1) r = m31_mul(r, b); b = m31_mul(b, b); e >>= 1; }
  return r;
}
CM31 cm_inv(CM31 x) {  // cm31.rs:41-50
  uint32_t inv_norm = m31_inv(m31_add(m31_mul(x.a, x.a), m31_mul(x.b, x.b)));
  return {m31_mul(x.a, inv_norm), m31_mul(m31_neg(x.b), inv_norm)};
}
QM31 qm_inv(QM31 x) {  // qm31.rs:56-80
  CM31 a2 = cm_mul(qm_a(x), qm_a(x)), b2 = cm_mul(qm_b(x), qm_b(x));
  CM31 b2u = {m31_sub(m31_double(b2.a), b2.b), m31_add(b2.a, m31_double(b2.b))};
  CM31 inv_norm = cm_inv(cm_sub(a2, b2u));
  QM31 c = qm_conj(x);
  return qm_from(cm_mul(qm_a(c), inv_norm), cm_mul(qm_b(c), inv_norm));
}

// ------------------------------------------------------------------ circle
CPoint cp_repeated_double(CPoint p, uint32_t n) {  // circle.rs:57-63
  for (uint32_t i = 0; i < n; i++) p = cp_mul(p, p);
  return p;
}
CPoint cp_mul_scalar(CPoint p, uint64_t k) {  // circle.rs:66-77
  CPoint r = CP_IDENTITY, b = p;
  while (k) { if (k & 1) r = cp_mul(r, b); b = cp_mul(b, b); k >>= 1; }
  return r;
}
Coset coset_subgroup(uint32_t log_size) {
  return {CP_IDENTITY, cp_repeated_double(CP_GENERATOR, 31 - log_size), log_size};
}
Coset coset_half_coset(uint32_t log_size) {
  if (log_size > 30) throw std::invalid_argument("half_coset: log_size > 30");
  return {cp_repeated_double(CP_GENERATOR, 30 - log_size), cp_repeated_double(CP_GENERATOR, 31 - log_size), log_size};
}
Coset coset_half_odds(uint32_t log_size) {
  if (log_size > 30) throw std::invalid_argument("half_odds: log_size > 30");
  uint32_t d = log_size >= 29 ? 0 : 29 - log_size;  // saturating_sub (circle.rs:141)
  return {cp_repeated_double(CP_GENERATOR, d), cp_repeated_double(CP_GENERATOR, 31 - log_size), log_size};
}
std::vector<CPoint> coset_points(const Coset& c) {  // circle.rs:258-267
  std::vector<CPoint> pts(c.size());
  CPoint cur = c.initial;
  for (uint64_t i = 0; i < c.size(); i++) { pts[i] = cur; cur = cp_mul(cur, c.step); }
  return pts;
}
uint64_t hc_natural_to_canonic_brt_index(uint64_t k, uint32_t log_n) {
  uint64_t n = 1ull << log_n;
  uint64_t cn = (k % 2 == 0) ? k / 2 : n - 1 - k / 2;
  return bit_reverse(cn, log_n);
}
std::vector<uint32_t> permute_hc_natural_to_canonic_brt(const std::vector<uint32_t>& d, uint32_t log_n) {
  std::vector<uint32_t> out(d.size());
  for (uint64_t k = 0; k < d.size(); k++) out[hc_natural_to_canonic_brt_index(k, log_n)] = d[k];
  return out;
}
std::vector<uint32_t> permute_canonic_brt_to_hc_natural(const std::vector<uint32_t>& d, uint32_t log_n) {
  std::vector<uint32_t> out(d.size());
  for (uint64_t k = 0; k < d.size(); k++) out[k] = d[hc_natural_to_canonic_brt_index(k, log_n)];
  return out;
}

// ------------------------------------------------------------------ batch inverse
std::vector<uint32_t> batch_inverse_chunked(const std::vector<uint32_t>& in) {
  const uint64_t n = in.size();
  std::vector<uint32_t> out(n);
  for (uint64_t start = 0; start < n; start += 64) {
    uint64_t count = std::min<uint64_t>(64, n - start);
    uint32_t prefix[64];
    prefix[0] = in[start];
    for (uint64_t i = 1; i < count; i++) {
      uint32_t v = in[start + i];
      prefix[i] = v == 0 ? prefix[i - 1] : m31_mul(prefix[i - 1], v);
    }
    uint32_t inv = m31_inv(prefix[count - 1]);
    for (uint64_t i = count - 1; i > 0; i--) {
      uint32_t v = in[start + i];
      if (v == 0) out[start + i] = 0;
      else { out[start + i] = m31_mul(inv, prefix[i - 1]); inv = m31_mul(inv, v); }
    }
    out[start] = in[start] == 0 ? 0 : inv;
  }
  return out;
}

// ------------------------------------------------------------------ native twiddles
NativeTwiddles native_twiddles(const Coset& coset) {
  NativeTwiddles t;
  t.log_n = coset.log_size;
  const uint64_t n = coset.size();
  const uint32_t n_line = coset.log_size > 0 ? coset.log_size - 1 : 0;
  std::vector<CPoint> pts = coset_points(coset);
  std::vector<uint32_t> cur(n);
  t.circle.resize(n / 2);
  for (uint64_t i = 0; i < n; i++) cur[i] = pts[i].x;
  for (uint64_t i = 0; i < n / 2; i++) t.circle[i] = pts[i].y;
  // n - 1 slots; the layers fill n - 2 of them and the last slot stays zero.
  t.line.assign(n > 0 ? n - 1 : 0, 0);
  uint64_t off = 0, cur_n = n;
  for (uint32_t l = 0; l < n_line; l++) {
    uint64_t ls = cur_n / 2;
    t.offsets.push_back((uint32_t)off);
    t.sizes.push_back((uint32_t)ls);
    std::vector<uint32_t> sq(ls);
    for (uint64_t i = 0; i < ls; i++) {  // twiddles.cu:127-142
      uint32_t x = cur[2 * i];
      t.line[off + i] = x;
      uint32_t x2 = m31_mul(x, x);
      sq[i] = m31_sub(m31_add(x2, x2), 1);
    }
    off += ls;
    cur.swap(sq);
    cur_n = ls;
  }
  t.iline = batch_inverse_chunked(t.line);
  t.icircle = batch_inverse_chunked(t.circle);
  return t;
}

// ------------------------------------------------------------------ NTT layers
void ntt_layer(uint32_t* d, uint64_t n, const uint32_t* tw, uint32_t j, bool fwd) {
  const uint64_t half = n / 2, stride = 1ull << j;
  for (uint64_t tid = 0; tid < half; tid++) {
    uint64_t h = tid >> j, l = tid & (stride - 1);
    uint64_t i0 = (h << (j + 1)) + l, i1 = i0 + stride;
    uint32_t v0 = d[i0], v1 = d[i1], t = tw[h];
    if (fwd) {  // circle_ntt.cu:8-12
      uint32_t m = m31_mul(v1, t);
      d[i0] = m31_add(v0, m);
      d[i1] = m31_sub(v0, m);
    } else {    // circle_ntt.cu:15-19
      d[i0] = m31_add(v0, v1);
      d[i1] = m31_mul(m31_sub(v0, v1), t);
    }
  }
}
void native_evaluate(std::vector<uint32_t>& d, const NativeTwiddles& t) {  // circle_ntt.cu:181-210
  const uint64_t n = 1ull << t.log_n;
  if (d.size() != n) throw std::invalid_argument("native_evaluate: size");
  for (int l = (int)t.offsets.size() - 1; l >= 0; l--) ntt_layer(d.data(), n, t.line.data() + t.offsets[l], l + 1, true);
  ntt_layer(d.data(), n, t.circle.data(), 0, true);
}
void native_interpolate(std::vector<uint32_t>& d, const NativeTwiddles& t) {  // circle_ntt.cu:212-249
  const uint64_t n = 1ull << t.log_n;
  if (d.size() != n) throw std::invalid_argument("native_interpolate: size");
  ntt_layer(d.data(), n, t.icircle.data(), 0, false);
  for (uint32_t l = 0; l < t.offsets.size(); l++) ntt_layer(d.data(), n, t.iline.data() + t.offsets[l], l + 1, false);
  uint32_t s = inv_n_scale(t.log_n);
  for (auto& v : d) v = m31_mul(v, s);
}
void bit_reverse_inplace(std::vector<uint32_t>& d, uint32_t log_n) {
  for (uint64_t i = 0; i < d.size(); i++) {
    uint64_t j = bit_reverse(i, log_n);
    if (i < j) std::swap(d[i], d[j]);
  }
}

// ------------------------------------------------------------------ stwo NTT
StwoTwiddles stwo_twiddles(uint32_t log_n) {  // ntt.rs:262-325
  if (log_n < 2) throw std::invalid_argument("stwo_twiddles: log_n < 2");
  StwoTwiddles t;
  t.log_n = log_n;
  Coset cur = coset_half_odds(log_n - 1);
  const uint64_t tc = cur.size();
  while (cur.log_size > 0) {
    uint64_t half = cur.size() / 2;
    uint32_t layer_log = 0;
    while ((1ull << layer_log) < half) layer_log++;
    std::vector<uint32_t> xs(half), brt(half);
    CPoint pt = cur.initial;
    for (uint64_t j = 0; j < half; j++) { xs[j] = pt.x; pt = cp_mul(pt, cur.step); }
    for (uint64_t i = 0; i < half; i++) brt[layer_log == 0 ? 0 : bit_reverse(i, layer_log)] = xs[i];
    t.fwd.insert(t.fwd.end(), brt.begin(), brt.end());
    cur = Coset{cp_mul(cur.initial, cur.initial), cp_mul(cur.step, cur.step), cur.log_size - 1};
  }
  t.fwd.push_back(1);
  while (t.fwd.size() < tc) t.fwd.push_back(0);
  t.fwd.resize(tc);
  // Full-array Montgomery inverse (ntt.rs:308-318); the table has no zeros.
  t.inv.resize(tc);
  std::vector<uint32_t> prefix(tc);
  prefix[0] = t.fwd[0];
  for (uint64_t i = 1; i < tc; i++) prefix[i] = m31_mul(prefix[i - 1], t.fwd[i]);
  uint32_t ip = m31_inv(prefix[tc - 1]);
  for (uint64_t i = tc - 1; i > 0; i--) { t.inv[i] = m31_mul(ip, prefix[i - 1]); ip = m31_mul(ip, t.fwd[i]); }
  t.inv[0] = ip;
  return t;
}
static void stwo_circle_layer(uint32_t* d, uint64_t n, const uint32_t* tw, bool fwd) {  // circle_ntt_stwo.cu:202-248
  for (uint64_t p = 0; p < n / 2; p++) {
    uint32_t x = tw[2 * (p / 4)], y = tw[2 * (p / 4) + 1], t;
    switch (p % 4) { case 0: t = y; break; case 1: t = m31_neg(y); break; case 2: t = m31_neg(x); break; default: t = x; }
    uint32_t v0 = d[2 * p], v1 = d[2 * p + 1];
    if (fwd) { uint32_t m = m31_mul(v1, t); d[2 * p] = m31_add(v0, m); d[2 * p + 1] = m31_sub(v0, m); }
    else { d[2 * p] = m31_add(v0, v1); d[2 * p + 1] = m31_mul(m31_sub(v0, v1), t); }
  }
}
void stwo_evaluate(std::vector<uint32_t>& d, const StwoTwiddles& t) {  // circle_ntt_stwo.cu:268-337
  const uint64_t n = 1ull << t.log_n, half = n / 2;
  const uint32_t nl = t.log_n - 1;
  if (d.size() != n) throw std::invalid_argument("stwo_evaluate: size");
  for (int k = (int)nl - 1; k >= 0; k--) ntt_layer(d.data(), n, t.fwd.data() + (half - (1ull << (nl - k))), k + 1, true);
  stwo_circle_layer(d.data(), n, t.fwd.data(), true);
}
void stwo_interpolate(std::vector<uint32_t>& d, const StwoTwiddles& t) {  // circle_ntt_stwo.cu:340-402
  const uint64_t n = 1ull << t.log_n, half = n / 2;
  const uint32_t nl = t.log_n - 1;
  if (d.size() != n) throw std::invalid_argument("stwo_interpolate: size");
  stwo_circle_layer(d.data(), n, t.inv.data(), false);
  for (uint32_t k = 0; k < nl; k++) ntt_layer(d.data(), n, t.inv.data() + (half - (1ull << (nl - k))), k + 1, false);
  uint32_t s = inv_n_scale(t.log_n);
  for (auto& v : d) v = m31_mul(v, s);
}
std::vector<uint32_t> stwo_lde(const std::vector<uint32_t>& evals, uint32_t log_n, uint32_t blowup_bits,
                               const StwoTwiddles& tt, const StwoTwiddles& te) {
  // cairo_air/prover.rs:954-965: interpolate_stwo -> zero_pad -> evaluate_stwo
  std::vector<uint32_t> c = evals;
  stwo_interpolate(c, tt);
  std::vector<uint32_t> e(1ull << (log_n + blowup_bits), 0);
  std::copy(c.begin(), c.end(), e.begin());
  stwo_evaluate(e, te);
  return e;
}

// ------------------------------------------------------------------ Blake2s
static const uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                               0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
static const uint8_t SIGMA[10][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0}};
static inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
void blake2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t, uint32_t f) {
  uint32_t v[16];
  for (int i = 0; i < 8; i++) { v[i] = h[i]; v[i + 8] = IV[i]; }
  v[12] ^= t;
  v[14] ^= f;
  auto G = [&](int a, int b, int c, int d, uint32_t x, uint32_t y) {
    v[a] = v[a] + v[b] + x; v[d] = rotr(v[d] ^ v[a], 16); v[c] = v[c] + v[d]; v[b] = rotr(v[b] ^ v[c], 12);
    v[a] = v[a] + v[b] + y; v[d] = rotr(v[d] ^ v[a], 8);  v[c] = v[c] + v[d]; v[b] = rotr(v[b] ^ v[c], 7);
  };
  for (int r = 0; r < 10; r++) {
    const uint8_t* s = SIGMA[r];
    G(0, 4, 8, 12, m[s[0]], m[s[1]]);   G(1, 5, 9, 13, m[s[2]], m[s[3]]);
    G(2, 6, 10, 14, m[s[4]], m[s[5]]);  G(3, 7, 11, 15, m[s[6]], m[s[7]]);
    G(0, 5, 10, 15, m[s[8]], m[s[9]]);  G(1, 6, 11, 12, m[s[10]], m[s[11]]);
    G(2, 7, 8, 13, m[s[12]], m[s[13]]); G(3, 4, 9, 14, m[s[14]], m[s[15]]);
  }
  for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
}
// Standard Blake2s-256 (unkeyed, 32-byte digest) of n_words LE u32 words. Non-final
// blocks use t = bytes so far, f = 0; the last block (possibly full) is final.
Hash blake2s_words(const uint32_t* w, size_t n_words) {
  uint32_t h[8];
  for (int i = 0; i < 8; i++) h[i] = IV[i];
  h[0] ^= 0x01010020u;
  size_t pos = 0;
  uint32_t m[16];
  while (n_words - pos > 16) {
    std::memcpy(m, w + pos, 64);
    pos += 16;
    blake2s_compress(h, m, (uint32_t)(pos * 4), 0);
  }
  std::memset(m, 0, 64);
  if (n_words > pos) std::memcpy(m, w + pos, (n_words - pos) * 4);
  blake2s_compress(h, m, (uint32_t)(n_words * 4), 0xFFFFFFFFu);
  Hash out;
  for (int i = 0; i < 8; i++) out[i] = h[i];
  return out;
}
std::array<uint8_t, 32> blake2s_bytes(const uint8_t* data, size_t len) {
  uint32_t h[8];
  for (int i = 0; i < 8; i++) h[i] = IV[i];
  h[0] ^= 0x01010020u;
  size_t pos = 0;
  uint32_t m[16];
  uint8_t blk[64];
  while (len - pos > 64) {
    std::memcpy(blk, data + pos, 64);
    for (int i = 0; i < 16; i++) m[i] = blk[4 * i] | (blk[4 * i + 1] << 8) | (blk[4 * i + 2] << 16) | ((uint32_t)blk[4 * i + 3] << 24);
    pos += 64;
    blake2s_compress(h, m, (uint32_t)pos, 0);
  }
  std::memset(blk, 0, 64);
  if (len > pos) std::memcpy(blk, data + pos, len - pos);
  for (int i = 0; i < 16; i++) m[i] = blk[4 * i] | (blk[4 * i + 1] << 8) | (blk[4 * i + 2] << 16) | ((uint32_t)blk[4 * i + 3] << 24);
  blake2s_compress(h, m, (uint32_t)len, 0xFFFFFFFFu);
  std::array<uint8_t, 32> out;
  for (int i = 0; i < 8; i++)
    for (int k = 0; k < 4; k++) out[4 * i + k] = (uint8_t)(h[i] >> (8 * k));
  return out;
}
Hash hash_node(const Hash& l, const Hash& r) {
  uint32_t w[16];
  for (int i = 0; i < 8; i++) { w[i] = l[i]; w[8 + i] = r[i]; }
  return blake2s_words(w, 16);
}

// ------------------------------------------------------------------ Merkle
Hash leaf_hash_capped(const uint32_t* vals, uint32_t n_cols) { return blake2s_words(vals, std::min<uint32_t>(n_cols, 16)); }
Hash leaf_hash_rowpacked(const uint32_t* vals, uint32_t n_cols) { return blake2s_words(vals, n_cols); }

std::vector<std::vector<Hash>> merkle_layers(std::vector<Hash> leaves) {
  std::vector<std::vector<Hash>> layers;
  layers.push_back(std::move(leaves));
  while (layers.back().size() > 1) {
    const auto& prev = layers.back();
    std::vector<Hash> par(prev.size() / 2);
    for (size_t i = 0; i < par.size(); i++) par[i] = hash_node(prev[2 * i], prev[2 * i + 1]);
    layers.push_back(std::move(par));
  }
  return layers;
}
static Hash reduce_parallel(std::vector<Hash> cur, int threads) {
  while (cur.size() > 1) {
    std::vector<Hash> par(cur.size() / 2);
    parallel_for(par.size(), threads, [&](uint64_t lo, uint64_t hi) {
      for (uint64_t i = lo; i < hi; i++) par[i] = hash_node(cur[2 * i], cur[2 * i + 1]);
    });
    cur.swap(par);
  }
  return cur[0];
}
Hash merkle_root(std::vector<Hash> leaves) { return reduce_parallel(std::move(leaves), 1); }
std::vector<Hash> auth_path(const std::vector<std::vector<Hash>>& layers, uint64_t idx) {
  std::vector<Hash> path;
  for (size_t l = 0; l + 1 < layers.size(); l++) { path.push_back(layers[l][idx ^ 1]); idx >>= 1; }
  return path;
}
bool verify_auth_path(const Hash& root, const Hash& leaf, uint64_t idx, const std::vector<Hash>& path) {
  Hash cur = leaf;
  for (const Hash& s : path) { cur = (idx % 2 == 0) ? hash_node(cur, s) : hash_node(s, cur); idx >>= 1; }
  return cur == root;
}
Hash merkle_root_columns_capped(const std::vector<const uint32_t*>& cols, uint64_t n, int threads) {
  std::vector<Hash> leaves(n);
  const uint32_t nc = (uint32_t)std::min<size_t>(cols.size(), 16);
  parallel_for(n, threads, [&](uint64_t lo, uint64_t hi) {
    uint32_t row[16];
    for (uint64_t i = lo; i < hi; i++) {
      for (uint32_t c = 0; c < nc; c++) row[c] = cols[c][i];
      leaves[i] = leaf_hash_capped(row, (uint32_t)cols.size());
    }
  });
  return reduce_parallel(std::move(leaves), threads);
}
Hash merkle_root_columns_rowpacked(const std::vector<const uint32_t*>& cols, uint64_t n, int threads) {
  std::vector<Hash> leaves(n);
  parallel_for(n, threads, [&](uint64_t lo, uint64_t hi) {
    std::vector<uint32_t> row(cols.size());
    for (uint64_t i = lo; i < hi; i++) {
      for (size_t c = 0; c < cols.size(); c++) row[c] = cols[c][i];
      leaves[i] = leaf_hash_rowpacked(row.data(), (uint32_t)cols.size());
    }
  });
  return reduce_parallel(std::move(leaves), threads);
}
Hash merkle_root_soa4(const uint32_t* const c[4], uint64_t n, int threads) {
  std::vector<Hash> leaves(n);
  parallel_for(n, threads, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; i++) {
      uint32_t w[4] = {c[0][i], c[1][i], c[2][i], c[3][i]};
      leaves[i] = blake2s_words(w, 4);
    }
  });
  return reduce_parallel(std::move(leaves), threads);
}
std::vector<Hash> lifted_leaves(const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& col_log,
                                uint32_t S) {
  const uint64_t n = 1ull << S;
  std::vector<Hash> out(n);
  std::vector<uint32_t> row(cols.size());
  for (uint64_t leaf = 0; leaf < n; leaf++) {
    for (size_t c = 0; c < cols.size(); c++) {
      uint32_t L = col_log[c];
      uint64_t r = (L == S) ? leaf : (((leaf >> (S - L + 1)) << 1) | (leaf & 1));  // merkle_leaves_lifted.cu:26-31
      row[c] = cols[c][r];
    }
    out[leaf] = blake2s_words(row.data(), row.size());
  }
  return out;
}

// ------------------------------------------------------------------ channel
void Channel::mix_digest(const Hash& d) {  // channel.rs:30-38
  uint8_t in[64];
  std::memcpy(in, state.data(), 32);
  for (int i = 0; i < 8; i++)
    for (int k = 0; k < 4; k++) in[32 + 4 * i + k] = (uint8_t)(d[i] >> (8 * k));
  state = blake2s_bytes(in, 64);
  n_draws = 0;
}
void Channel::mix_felts(const std::vector<QM31>& f) {  // channel.rs:46-59 (multi-block blake2s)
  if (f.empty()) return;
  std::vector<uint8_t> in(32 + 16 * f.size());
  std::memcpy(in.data(), state.data(), 32);
  for (size_t j = 0; j < f.size(); j++)
    for (int l = 0; l < 4; l++)
      for (int k = 0; k < 4; k++) in[32 + 16 * j + 4 * l + k] = (uint8_t)(f[j].v[l] >> (8 * k));
  state = blake2s_bytes(in.data(), in.size());
  n_draws = 0;
}
void Channel::mix_u64(uint64_t v) {  // channel.rs:120-129
  uint8_t in[40];
  std::memcpy(in, state.data(), 32);
  for (int k = 0; k < 8; k++) in[32 + k] = (uint8_t)(v >> (8 * k));
  state = blake2s_bytes(in, 40);
  n_draws = 0;
}
std::array<uint8_t, 32> Channel::squeeze() {  // channel.rs:177-184
  uint8_t in[37];
  std::memcpy(in, state.data(), 32);
  for (int k = 0; k < 4; k++) in[32 + k] = (uint8_t)(n_draws >> (8 * k));
  in[36] = 0;
  n_draws++;
  return blake2s_bytes(in, 37);
}
static inline uint32_t le32(const uint8_t* b) { return b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24); }
QM31 Channel::draw_felt() {  // channel.rs:66-83
  for (;;) {
    auto b = squeeze();
    uint32_t u[8];
    bool ok = true;
    for (int i = 0; i < 8; i++) { u[i] = le32(&b[4 * i]); ok = ok && u[i] < 2 * P; }
    if (ok) return {{u[0] % P, u[1] % P, u[2] % P, u[3] % P}};
  }
}
uint64_t Channel::draw_number(uint64_t bound) {  // channel.rs:91-95
  auto b = squeeze();
  uint64_t raw = 0;
  for (int k = 7; k >= 0; k--) raw = (raw << 8) | b[k];
  return raw % bound;
}
std::vector<uint64_t> Channel::draw_query_indices(uint32_t log_domain, size_t n) {  // channel.rs:102-116
  uint32_t mask = (uint32_t)((1ull << log_domain) - 1);
  std::vector<uint64_t> r;
  while (r.size() < n) {
    auto b = squeeze();
    for (int i = 0; i < 8 && r.size() < n; i++) r.push_back(le32(&b[4 * i]) & mask);
  }
  return r;
}
Hash Channel::state_words() const {
  Hash h;
  for (int i = 0; i < 8; i++) h[i] = le32(&state[4 * i]);
  return h;
}

Hash Channel::pow_prefix(uint32_t pow_bits) const {  // channel.rs:144-152
  uint8_t in[52] = {0};
  const uint32_t magic = 0x12345678u;
  std::memcpy(in, &magic, 4);
  std::memcpy(in + 16, state.data(), 32);
  std::memcpy(in + 48, &pow_bits, 4);
  const auto d = blake2s_bytes(in, 52);
  Hash h{};
  std::memcpy(h.data(), d.data(), 32);
  return h;
}
uint32_t pow_trailing_zeros(const Hash& prefix, uint64_t nonce, bool m31_output) {
  uint32_t w[10];
  for (int k = 0; k < 8; k++) w[k] = prefix[k];
  w[8] = (uint32_t)nonce;
  w[9] = (uint32_t)(nonce >> 32);
  Hash r = blake2s_words(w, 10);
  uint32_t tz = 0;
  for (int k = 0; k < 4; k++) {
    uint32_t v = r[k];
    if (m31_output) v = m31_reduce(v);  // grind_m31_output.cu:47-52 (m31.cuh:9-14)
    if (v) return tz + (uint32_t)__builtin_ctz(v);
    tz += 32;
  }
  return tz;
}
bool Channel::verify_pow_nonce(uint32_t pow_bits, uint64_t nonce) const {  // channel.rs:144-168
  return pow_trailing_zeros(pow_prefix(pow_bits), nonce, false) >= pow_bits;
}
uint64_t pow_grind_min(const Hash& prefix, uint32_t pow_bits, uint64_t offset, uint64_t n, bool m31_output,
                       int threads) {
  std::vector<uint64_t> best(std::max(threads, 1), UINT64_MAX);
  parallel_for(n, threads, [&](uint64_t lo, uint64_t hi) {
    uint64_t b = UINT64_MAX;
    for (uint64_t i = lo; i < hi && b == UINT64_MAX; i++)
      if (pow_trailing_zeros(prefix, offset + i, m31_output) >= pow_bits) b = offset + i;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    best[0] = std::min(best[0], b);
  });
  return best[0];
}

// ------------------------------------------------------------------ FRI
std::vector<uint32_t> fold_twiddles(const Coset& dom, bool extract_y) {
  const uint64_t n = dom.size(), half = n / 2;
  std::vector<uint32_t> src(half);
  for (uint64_t i = 0; i < half; i++) {  // twiddles.cu:23-52
    CPoint p = dom.at(bit_reverse(i << 1, dom.log_size));
    src[i] = extract_y ? p.y : p.x;
  }
  return batch_inverse_chunked(src);
}
void fold_circle_into_line(QM31* dst, const QM31* src, const uint32_t* tw, QM31 alpha, uint64_t half_n) {
  QM31 a2 = qm_mul(alpha, alpha);
  for (uint64_t i = 0; i < half_n; i++) {
    QM31 f0 = src[2 * i], f1 = src[2 * i + 1];
    QM31 fp = qm_add(qm_add(f0, f1), qm_mul(alpha, qm_scale(qm_sub(f0, f1), tw[i])));
    dst[i] = qm_add(qm_mul(dst[i], a2), fp);
  }
}
void fold_line(QM31* dst, const QM31* src, const uint32_t* tw, QM31 alpha, uint64_t half_n) {
  for (uint64_t i = 0; i < half_n; i++) {
    QM31 f0 = src[2 * i], f1 = src[2 * i + 1];
    dst[i] = qm_add(qm_add(f0, f1), qm_mul(alpha, qm_scale(qm_sub(f0, f1), tw[i])));
  }
}
static void bit_reverse_qm(std::vector<QM31>& v, uint32_t log_n) {
  for (uint64_t i = 0; i < v.size(); i++) {
    uint64_t j = bit_reverse(i, log_n);
    if (i < j) std::swap(v[i], v[j]);
  }
}
std::vector<QM31> last_layer_poly_coeffs(std::vector<QM31> e) {
  const uint64_t n = e.size();
  uint32_t log_n = 0;
  while ((1ull << log_n) < n) log_n++;
  bit_reverse_qm(e, log_n);
  uint64_t chunk = n;
  uint32_t dl = log_n;
  while (chunk > 1) {
    Coset dom = coset_half_odds(dl);
    uint64_t half = chunk / 2;
    for (uint64_t base = 0; base < n; base += chunk)
      for (uint64_t i = 0; i < half; i++) {
        uint32_t xi = m31_inv(dom.at(i).x);
        QM31 l = e[base + i], r = e[base + half + i];
        e[base + i] = qm_add(l, r);
        e[base + half + i] = qm_scale(qm_sub(l, r), xi);
      }
    dl--;
    chunk = half;
  }
  uint32_t ninv = m31_inv((uint32_t)n);
  for (auto& v : e) v = qm_scale(v, ninv);
  bit_reverse_qm(e, log_n);
  e.resize(1ull << LOG_LAST_LAYER);
  return e;
}
static QM31 fold_eval(const QM31* c, uint64_t n, const uint32_t* dbl) {
  if (n == 1) return c[0];
  QM31 l = fold_eval(c, n / 2, dbl + 1), r = fold_eval(c + n / 2, n / 2, dbl + 1);
  return qm_add(l, qm_scale(r, dbl[0]));
}
QM31 eval_last_layer_poly(const std::vector<QM31>& coeffs, uint64_t idx, uint32_t log_size) {
  Coset dom = coset_half_odds(log_size);
  uint32_t x = dom.at(bit_reverse(idx, log_size)).x;
  const uint64_t n = coeffs.size();
  if (n == 1) return coeffs[0];
  uint32_t log_n = 0;
  while ((1ull << log_n) < n) log_n++;
  std::vector<uint32_t> dbl;
  uint32_t xi = x;
  for (uint32_t k = 0; k < log_n; k++) { dbl.push_back(xi); xi = m31_sub(m31_mul(m31_mul(2, xi), xi), 1); }
  std::vector<QM31> brt(n);
  for (uint64_t i = 0; i < n; i++) brt[bit_reverse(i, log_n)] = coeffs[i];
  return fold_eval(brt.data(), n, dbl.data());
}

// ------------------------------------------------------------------ quotients / OODS
QM31 fib_quotient_at(const uint32_t* t, uint64_t n, uint64_t i, QM31 alpha) {
  uint32_t c = m31_sub(t[(i + 2) % n], m31_add(t[(i + 1) % n], t[i]));
  return qm_scale(alpha, c);
}
void accumulate_numerators(const std::vector<const uint32_t*>& cols, const std::vector<uint32_t>& col_idx,
                           const std::vector<QM31>& b, const std::vector<QM31>& c, uint64_t n_rows, QM31* out) {
  for (uint64_t r = 0; r < n_rows; r++) {
    QM31 acc{{0, 0, 0, 0}};
    for (size_t i = 0; i < col_idx.size(); i++)
      acc = qm_add(acc, qm_sub(qm_scale(c[i], cols[col_idx[i]][r]), b[i]));
    out[r] = acc;
  }
}
void quotients_combine(const std::vector<QuotAcc>& accs, const uint32_t* dxs, const uint32_t* dys,
                       uint32_t lifting_log, uint64_t n_rows, QM31* out) {
  for (uint64_t row = 0; row < n_rows; row++) {
    uint32_t dx = dxs[row], dy = dys[row];
    QM31 q{{0, 0, 0, 0}};
    for (const QuotAcc& a : accs) {
      CM31 prx = qm_a(a.spx), pry = qm_a(a.spy), pix = qm_b(a.spx), piy = qm_b(a.spy);
      CM31 den = cm_sub(cm_mul(cm_sub(prx, {dx, 0}), piy), cm_mul(cm_sub(pry, {dy, 0}), pix));
      CM31 di = cm_inv(den);
      uint32_t ratio = lifting_log - a.log_size;
      uint64_t li = ((row >> (ratio + 1)) << 1) + (row & 1);
      QM31 full = qm_sub(a.numer[li], qm_scale(a.first_linear, dy));
      q = qm_add(q, qm_scale_cm(full, di));
    }
    out[row] = q;
  }
}
OodsPoint oods_point_from_channel(Channel& ch) {
  QM31 t = ch.draw_felt();
  QM31 t2 = qm_mul(t, t);
  QM31 one = qm_m31(1);
  QM31 di = qm_inv(qm_add(one, t2));
  return {qm_mul(qm_sub(one, t2), di), qm_mul(qm_add(t, t), di)};
}
static QM31 fold_m31(const uint32_t* v, uint64_t n, const QM31* f) {
  if (n == 1) return qm_m31(v[0]);
  QM31 l = fold_m31(v, n / 2, f + 1), r = fold_m31(v + n / 2, n / 2, f + 1);
  return qm_add(l, qm_mul(f[0], r));
}
QM31 eval_at_oods_from_coeffs(const std::vector<uint32_t>& c, OodsPoint z) {
  const uint64_t n = c.size();
  uint32_t log_n = 0;
  while ((1ull << log_n) < n) log_n++;
  if (log_n == 0) return qm_m31(c[0]);
  std::vector<QM31> maps;
  maps.push_back(z.y);
  QM31 x = z.x;
  for (uint32_t k = 1; k < log_n; k++) {
    maps.push_back(x);
    QM31 x2 = qm_mul(x, x);
    x = qm_sub(qm_add(x2, x2), qm_m31(1));
  }
  std::reverse(maps.begin(), maps.end());
  return fold_m31(c.data(), n, maps.data());
}
void compute_line_coeffs(OodsPoint z, QM31 v, QM31& a, QM31& b) {
  QM31 den = qm_sub(z.y, qm_conj(z.y));
  b = qm_mul(qm_sub(v, qm_conj(v)), qm_inv(den));
  a = qm_sub(v, qm_mul(b, z.y));
}
CPoint canonic_domain_point(uint64_t j, uint32_t log_eval) {
  Coset ho = coset_half_odds(log_eval - 1);
  uint64_t half = 1ull << (log_eval - 1);
  return j < half ? ho.at(j) : cp_conj(ho.at(j - half));
}

// ------------------------------------------------------------------ AIR
std::vector<uint32_t> fibonacci_trace(uint32_t a, uint32_t b, uint32_t log_n) {
  std::vector<uint32_t> t(1ull << log_n);
  t[0] = a;
  t[1] = b;
  for (uint64_t i = 2; i < t.size(); i++) t[i] = m31_add(t[i - 1], t[i - 2]);
  return t;
}

// ------------------------------------------------------------------ prover
// Merkle trees of the prover keep only the levels from 2^K-leaf tile roots up
// (merkle.rs:804-842 keeps every level; the root and every auth path are the
// same): a full tree of 2^30 leaves would take 64 GB of host memory. An auth
// path recomputes its tile's leaves and inner levels from the leaf function.
struct LeanTree {
  uint32_t K = 0;                       // log2 leaves per tile
  std::vector<std::vector<Hash>> up;    // up[0] = tile roots ... up.back() = {root}
  std::function<Hash(uint64_t)> leaf;
  const Hash& root() const { return up.back()[0]; }
};
static constexpr uint32_t LEAN_TILE_LOG = 10;

static LeanTree build_tree(uint64_t n, int threads, std::function<Hash(uint64_t)> leaf) {
  LeanTree t;
  t.leaf = std::move(leaf);
  uint32_t log_n = 0;
  while ((1ull << log_n) < n) log_n++;
  t.K = std::min(log_n, LEAN_TILE_LOG);
  const uint64_t tile = 1ull << t.K, n_tiles = n >> t.K;
  std::vector<Hash> roots(n_tiles);
  parallel_for(n_tiles, threads, [&](uint64_t lo, uint64_t hi) {
    std::vector<Hash> cur(tile);
    for (uint64_t g = lo; g < hi; g++) {
      for (uint64_t j = 0; j < tile; j++) cur[j] = t.leaf(g * tile + j);
      for (uint64_t m = tile; m > 1; m >>= 1)
        for (uint64_t j = 0; j < m / 2; j++) cur[j] = hash_node(cur[2 * j], cur[2 * j + 1]);
      roots[g] = cur[0];
    }
  });
  t.up.push_back(std::move(roots));
  while (t.up.back().size() > 1) {
    const auto& prev = t.up.back();
    std::vector<Hash> par(prev.size() / 2);
    parallel_for(par.size(), threads, [&](uint64_t lo, uint64_t hi) {
      for (uint64_t i = lo; i < hi; i++) par[i] = hash_node(prev[2 * i], prev[2 * i + 1]);
    });
    t.up.push_back(std::move(par));
  }
  return t;
}
// Leaf-to-root siblings of leaf idx (merkle.rs:846-861 order).
static std::vector<Hash> auth_path(const LeanTree& t, uint64_t idx) {
  std::vector<Hash> path;
  const uint64_t tile = 1ull << t.K, g = idx >> t.K;
  std::vector<Hash> cur(tile);
  for (uint64_t j = 0; j < tile; j++) cur[j] = t.leaf(g * tile + j);
  uint64_t pos = idx & (tile - 1);
  for (uint64_t m = tile; m > 1; m >>= 1) {
    path.push_back(cur[pos ^ 1]);
    for (uint64_t j = 0; j < m / 2; j++) cur[j] = hash_node(cur[2 * j], cur[2 * j + 1]);
    pos >>= 1;
  }
  pos = g;
  for (size_t l = 0; l + 1 < t.up.size(); l++) { path.push_back(t.up[l][pos ^ 1]); pos >>= 1; }
  return path;
}
static Hash soa4_leaf(const std::vector<QM31>& v, uint64_t i) { return blake2s_words(v[i].v, 4); }
static Q4 q4(const QM31& x) { return {x.v[0], x.v[1], x.v[2], x.v[3]}; }

StarkProof prove(uint32_t a, uint32_t b, uint32_t log_n, int threads) {
  if (log_n < 4) throw std::invalid_argument("trace too small");  // prover.rs:1724
  const uint32_t log_eval = log_n + BLOWUP_BITS;
  const uint64_t N = 1ull << log_eval;

  // Steps 1-3: trace -> interpolate (half_coset(log_n)) -> zero-pad -> evaluate (half_coset(log_eval))
  std::vector<uint32_t> tr = fibonacci_trace(a, b, log_n);
  NativeTwiddles tt = native_twiddles(coset_half_coset(log_n));
  NativeTwiddles te = native_twiddles(coset_half_coset(log_eval));
  native_interpolate(tr, tt);
  std::vector<uint32_t> ev(N, 0);
  std::copy(tr.begin(), tr.end(), ev.begin());
  native_evaluate(ev, te);

  // Step 4: trace tree (single column leaf, t = 4)
  auto trace_tree = build_tree(N, threads, [&](uint64_t i) { return leaf_hash_capped(&ev[i], 1); });
  StarkProof pf;
  pf.trace_commitment = trace_tree.root();

  // Step 5: quotient
  Channel ch;
  ch.mix_digest(pf.trace_commitment);
  QM31 alpha = ch.draw_felt();
  std::vector<QM31> quot(N);
  parallel_for(N, threads, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; i++) quot[i] = fib_quotient_at(ev.data(), N, i, alpha);
  });
  auto quot_tree = build_tree(N, threads, [&](uint64_t i) { return soa4_leaf(quot, i); });
  pf.quotient_commitment = quot_tree.root();
  ch.mix_digest(pf.quotient_commitment);

  // Step 7: FRI (prover.rs:1816-1904); twiddles per fri.rs:143-160
  std::vector<std::vector<QM31>> fri_evals;
  fri_evals.reserve(64);  // leaf functions below index into it
  std::vector<LeanTree> fri_trees;
  uint32_t cur_log = log_eval;
  {
    QM31 fa = ch.draw_felt();
    std::vector<uint32_t> tw = fold_twiddles(coset_half_coset(log_eval), true);
    std::vector<QM31> line(N / 2, QM31{{0, 0, 0, 0}});
    fold_circle_into_line(line.data(), quot.data(), tw.data(), fa, N / 2);
    cur_log--;
    fri_evals.push_back(std::move(line));
    const size_t l = fri_evals.size() - 1;
    auto tree = build_tree(fri_evals[l].size(), threads, [&fri_evals, l](uint64_t i) { return soa4_leaf(fri_evals[l], i); });
    pf.fri_commitments.push_back(tree.root());
    ch.mix_digest(tree.root());
    fri_trees.push_back(std::move(tree));
  }
  while (cur_log > LOG_LAST_LAYER) {
    QM31 fa = ch.draw_felt();
    std::vector<uint32_t> tw = fold_twiddles(coset_half_odds(cur_log), false);
    const auto& prev = fri_evals.back();
    std::vector<QM31> next(prev.size() / 2);
    fold_line(next.data(), prev.data(), tw.data(), fa, next.size());
    cur_log--;
    fri_evals.push_back(std::move(next));
    const size_t l = fri_evals.size() - 1;
    auto tree = build_tree(fri_evals[l].size(), threads, [&fri_evals, l](uint64_t i) { return soa4_leaf(fri_evals[l], i); });
    pf.fri_commitments.push_back(tree.root());
    ch.mix_digest(tree.root());
    fri_trees.push_back(std::move(tree));
  }
  pf.fri_last_layer = fri_evals.back();

  // Step 8: queries and decommitments
  ch.mix_felts(pf.fri_last_layer);
  for (uint32_t q = 0; q < N_QUERIES; q++) pf.query_indices.push_back(ch.draw_number(N));
  for (uint64_t qi : pf.query_indices) {
    pf.trace_decommitment.values.push_back(ev[qi]);
    pf.trace_decommitment.sibling_values.push_back(ev[qi ^ 1]);
  }
  for (uint64_t qi : pf.query_indices) pf.trace_decommitment.auth_paths.push_back(auth_path(trace_tree, qi));
  for (uint64_t qi : pf.query_indices) pf.trace_decommitment.sibling_auth_paths.push_back(auth_path(trace_tree, qi ^ 1));
  for (uint64_t qi : pf.query_indices) {
    pf.quotient_decommitment.values.push_back(q4(quot[qi]));
    pf.quotient_decommitment.sibling_values.push_back(q4(quot[qi ^ 1]));
  }
  for (uint64_t qi : pf.query_indices) pf.quotient_decommitment.auth_paths.push_back(auth_path(quot_tree, qi));
  for (uint64_t qi : pf.query_indices) pf.quotient_decommitment.sibling_auth_paths.push_back(auth_path(quot_tree, qi ^ 1));
  std::vector<uint64_t> folded;
  for (uint64_t qi : pf.query_indices) folded.push_back(qi / 2);
  for (size_t l = 0; l < fri_evals.size(); l++) {
    Decommit<Q4> d;
    for (uint64_t f : folded) { d.values.push_back(q4(fri_evals[l][f])); d.sibling_values.push_back(q4(fri_evals[l][f ^ 1])); }
    for (uint64_t f : folded) d.auth_paths.push_back(auth_path(fri_trees[l], f));
    for (uint64_t f : folded) d.sibling_auth_paths.push_back(auth_path(fri_trees[l], f ^ 1));
    pf.fri_decommitments.push_back(std::move(d));
    for (auto& f : folded) f /= 2;
  }
  pf.log_trace_size = log_n;
  pf.a = a;
  pf.b = b;
  return pf;
}

// ------------------------------------------------------------------ verifier (verifier.rs:39-236)
static uint32_t fold_twiddle_at(const Coset& dom, uint64_t folded, bool circle) {
  CPoint p = dom.at(bit_reverse(folded << 1, dom.log_size));
  return m31_inv(circle ? p.y : p.x);
}
static QM31 fold_pair(QM31 f0, QM31 f1, QM31 alpha, uint32_t tw) {
  return qm_add(qm_add(f0, f1), qm_mul(alpha, qm_scale(qm_sub(f0, f1), tw)));
}
static QM31 from_q4(const Q4& v) { return {{v[0], v[1], v[2], v[3]}}; }
static std::string check_paths_u32(const Hash& root, const Decommit<uint32_t>& d, const std::vector<uint64_t>& idx,
                                   const std::string& label) {
  if (d.values.size() != N_QUERIES || d.auth_paths.size() != N_QUERIES) return label + " decommitment size mismatch";
  if (d.sibling_values.size() != N_QUERIES || d.sibling_auth_paths.size() != N_QUERIES) return label + " decommitment size mismatch";
  for (size_t q = 0; q < idx.size(); q++) {
    if (!verify_auth_path(root, leaf_hash_capped(&d.values[q], 1), idx[q], d.auth_paths[q])) return label + " auth path invalid";
    if (!verify_auth_path(root, leaf_hash_capped(&d.sibling_values[q], 1), idx[q] ^ 1, d.sibling_auth_paths[q]))
      return label + " sibling auth path invalid";
  }
  return "";
}
static std::string check_paths_q4(const Hash& root, const Decommit<Q4>& d, const std::vector<uint64_t>& idx,
                                  const std::string& label) {
  if (d.values.size() != N_QUERIES || d.auth_paths.size() != N_QUERIES) return label + " decommitment size mismatch";
  if (d.sibling_values.size() != N_QUERIES || d.sibling_auth_paths.size() != N_QUERIES) return label + " decommitment size mismatch";
  for (size_t q = 0; q < idx.size(); q++) {
    if (!verify_auth_path(root, blake2s_words(d.values[q].data(), 4), idx[q], d.auth_paths[q])) return label + " auth path invalid";
    if (!verify_auth_path(root, blake2s_words(d.sibling_values[q].data(), 4), idx[q] ^ 1, d.sibling_auth_paths[q]))
      return label + " sibling auth path invalid";
  }
  return "";
}
std::string verify(const StarkProof& p) {
  const uint32_t log_n = p.log_trace_size;
  if (log_n < 1 || log_n > 29) return "bad log size";
  const uint32_t log_eval = log_n + BLOWUP_BITS;
  const uint64_t N = 1ull << log_eval;
  if (p.a >= P || p.b >= P) return "Public inputs out of M31 range";
  if (p.query_indices.size() != N_QUERIES) return "Expected 80 queries";
  Channel ch;
  ch.mix_digest(p.trace_commitment);
  (void)ch.draw_felt();
  ch.mix_digest(p.quotient_commitment);
  std::vector<QM31> alphas{ch.draw_felt()};
  for (const Hash& c : p.fri_commitments) { ch.mix_digest(c); alphas.push_back(ch.draw_felt()); }
  uint32_t expected_layers = log_eval > 3 ? log_eval - 3 : 0;
  if (p.fri_commitments.size() != expected_layers) return "wrong number of FRI layers";
  if (p.fri_last_layer.size() != 8) return "wrong FRI last layer size";
  ch.mix_felts(p.fri_last_layer);
  for (uint32_t q = 0; q < N_QUERIES; q++)
    if (p.query_indices[q] != ch.draw_number(N)) return "Query indices don't match Fiat-Shamir derivation";
  Hash zero{};
  if (p.trace_commitment == zero) return "Trace commitment is zero";
  if (p.quotient_commitment == zero) return "Quotient commitment is zero";
  std::string e = check_paths_u32(p.trace_commitment, p.trace_decommitment, p.query_indices, "trace");
  if (!e.empty()) return e;
  e = check_paths_q4(p.quotient_commitment, p.quotient_decommitment, p.query_indices, "quotient");
  if (!e.empty()) return e;
  std::vector<uint64_t> folded;
  for (uint64_t qi : p.query_indices) folded.push_back(qi / 2);
  size_t n_layers = std::min(p.fri_decommitments.size(), p.fri_commitments.size());
  for (size_t l = 0; l < n_layers; l++) {
    e = check_paths_q4(p.fri_commitments[l], p.fri_decommitments[l], folded, "FRI layer " + std::to_string(l));
    if (!e.empty()) return e;
    for (auto& f : folded) f /= 2;
  }
  const size_t nfd = p.fri_decommitments.size();
  if (nfd == 0) return "no FRI decommitments";
  for (size_t q = 0; q < N_QUERIES; q++) {
    uint64_t idx = p.query_indices[q];
    uint32_t cl = log_eval;
    {
      Coset dom = cl <= 30 ? coset_half_coset(cl) : coset_subgroup(cl);
      uint64_t fi = idx / 2;
      QM31 v = from_q4(p.quotient_decommitment.values[q]), s = from_q4(p.quotient_decommitment.sibling_values[q]);
      QM31 f0 = idx % 2 == 0 ? v : s, f1 = idx % 2 == 0 ? s : v;
      if (!(fold_pair(f0, f1, alphas[0], fold_twiddle_at(dom, fi, true)) == from_q4(p.fri_decommitments[0].values[q])))
        return "Circle fold mismatch";
      idx = fi;
      cl--;
    }
    for (size_t l = 0; l + 1 < nfd; l++) {
      Coset dom = coset_half_odds(cl);
      uint64_t fi = idx / 2;
      QM31 v = from_q4(p.fri_decommitments[l].values[q]), s = from_q4(p.fri_decommitments[l].sibling_values[q]);
      QM31 f0 = idx % 2 == 0 ? v : s, f1 = idx % 2 == 0 ? s : v;
      if (l + 1 >= alphas.size()) return "missing FRI alpha";
      if (!(fold_pair(f0, f1, alphas[l + 1], fold_twiddle_at(dom, fi, false)) == from_q4(p.fri_decommitments[l + 1].values[q])))
        return "Line fold mismatch";
      idx = fi;
      cl--;
    }
    if (idx >= p.fri_last_layer.size()) return "FRI last layer index out of bounds";
    if (!(from_q4(p.fri_decommitments[nfd - 1].values[q]) == p.fri_last_layer[idx])) return "FRI last layer mismatch";
  }
  return "";
}

// ------------------------------------------------------------------ KRAK serialization
static void w32(std::vector<uint8_t>& w, uint32_t v) { for (int k = 0; k < 4; k++) w.push_back((uint8_t)(v >> (8 * k))); }
static void wpaths(std::vector<uint8_t>& w, const std::vector<std::vector<Hash>>& ps) {
  for (const auto& p : ps) { w32(w, (uint32_t)p.size()); for (const Hash& h : p) for (uint32_t x : h) w32(w, x); }
}
std::vector<uint8_t> serialize_proof(const StarkProof& p) {
  std::vector<uint8_t> w;
  w32(w, 0x4B52414Bu);
  w32(w, 1);
  w32(w, p.log_trace_size);
  w32(w, p.a);
  w32(w, p.b);
  for (uint32_t x : p.trace_commitment) w32(w, x);
  for (uint32_t x : p.quotient_commitment) w32(w, x);
  w32(w, (uint32_t)p.fri_commitments.size());
  for (const Hash& h : p.fri_commitments) for (uint32_t x : h) w32(w, x);
  w32(w, (uint32_t)p.fri_last_layer.size());
  for (const QM31& v : p.fri_last_layer) for (uint32_t x : v.v) w32(w, x);
  w32(w, (uint32_t)p.query_indices.size());
  for (uint64_t q : p.query_indices) w32(w, (uint32_t)q);
  const auto& t = p.trace_decommitment;
  w32(w, (uint32_t)t.values.size());
  for (uint32_t v : t.values) w32(w, v);
  for (uint32_t v : t.sibling_values) w32(w, v);
  wpaths(w, t.auth_paths);
  wpaths(w, t.sibling_auth_paths);
  auto w4 = [&](const Decommit<Q4>& d) {
    w32(w, (uint32_t)d.values.size());
    for (const Q4& v : d.values) for (uint32_t x : v) w32(w, x);
    for (const Q4& v : d.sibling_values) for (uint32_t x : v) w32(w, x);
    wpaths(w, d.auth_paths);
    wpaths(w, d.sibling_auth_paths);
  };
  w4(p.quotient_decommitment);
  w32(w, (uint32_t)p.fri_decommitments.size());
  for (const auto& d : p.fri_decommitments) w4(d);
  return w;
}
namespace {
struct Reader {
  const uint8_t* d; size_t n, pos = 0; bool ok = true;
  uint32_t u() {
    if (pos + 4 > n) { ok = false; return 0; }
    uint32_t v = le32(d + pos); pos += 4; return v;
  }
  std::vector<std::vector<Hash>> paths(uint32_t count) {
    std::vector<std::vector<Hash>> ps;
    for (uint32_t i = 0; i < count && ok; i++) {
      uint32_t depth = u();
      if (depth > 64) { ok = false; break; }
      std::vector<Hash> p(depth);
      for (auto& h : p) for (auto& x : h) x = u();
      ps.push_back(std::move(p));
    }
    return ps;
  }
};
}  // namespace
bool deserialize_proof(const uint8_t* data, size_t len, StarkProof& p) {
  Reader r{data, len};
  if (r.u() != 0x4B52414Bu || r.u() != 1) return false;
  p = StarkProof{};
  p.log_trace_size = r.u();
  p.a = r.u();
  p.b = r.u();
  for (auto& x : p.trace_commitment) x = r.u();
  for (auto& x : p.quotient_commitment) x = r.u();
  uint32_t nf = r.u();
  if (nf > 64) return false;
  p.fri_commitments.resize(nf);
  for (auto& h : p.fri_commitments) for (auto& x : h) x = r.u();
  uint32_t nl = r.u();
  if (nl > 1024) return false;
  p.fri_last_layer.resize(nl);
  for (auto& v : p.fri_last_layer) for (auto& x : v.v) x = r.u();
  uint32_t nq = r.u();
  if (nq > 4096) return false;
  for (uint32_t i = 0; i < nq; i++) p.query_indices.push_back(r.u());
  uint32_t tn = r.u();
  if (tn > 4096) return false;
  for (uint32_t i = 0; i < tn; i++) p.trace_decommitment.values.push_back(r.u());
  for (uint32_t i = 0; i < tn; i++) p.trace_decommitment.sibling_values.push_back(r.u());
  p.trace_decommitment.auth_paths = r.paths(tn);
  p.trace_decommitment.sibling_auth_paths = r.paths(tn);
  auto r4 = [&](Decommit<Q4>& d) {
    uint32_t k = r.u();
    if (k > 4096) { r.ok = false; return; }
    d.values.resize(k);
    d.sibling_values.resize(k);
    for (auto& v : d.values) for (auto& x : v) x = r.u();
    for (auto& v : d.sibling_values) for (auto& x : v) x = r.u();
    d.auth_paths = r.paths(k);
    d.sibling_auth_paths = r.paths(k);
  };
  r4(p.quotient_decommitment);
  uint32_t nd = r.u();
  if (nd > 64) return false;
  p.fri_decommitments.resize(nd);
  for (auto& d : p.fri_decommitments) r4(d);
  return r.ok && r.pos == len;
}

// ------------------------------------------------------------------ stwo Backend adapter kernels
void gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint64_t n) {
  for (uint64_t i = 0; i < n; i++) dst[i] = src[idx[i]];
}
void gather_u256(const uint32_t* src, const uint32_t* idx, uint32_t* dst, uint64_t n) {
  for (uint64_t i = 0; i < n; i++)
    for (int k = 0; k < 8; k++) dst[8 * i + k] = src[8 * (uint64_t)idx[i] + k];
}
void barycentric_partials(const uint32_t* evals, const uint32_t* weights, uint64_t n, uint32_t n_blocks, uint32_t* out) {
  std::vector<QM31> part(n_blocks, QM31{{0, 0, 0, 0}});
  for (uint64_t i = 0; i < n; i++) {
    QM31 w{{weights[4 * i], weights[4 * i + 1], weights[4 * i + 2], weights[4 * i + 3]}};
    QM31& acc = part[(i / 256) % n_blocks];
    acc = qm_add(acc, qm_scale(w, evals[i]));  // qm31_mul_m31: each limb times the M31 value
  }
  for (uint32_t b = 0; b < n_blocks; b++) std::memcpy(out + 4 * (uint64_t)b, part[b].v, 16);
}
void accumulate_lift(uint32_t* col, const uint32_t* curr, uint64_t col_n, uint32_t log_ratio) {
  const uint32_t shift = log_ratio + 1;
  for (uint64_t i = 0; i < col_n; i++) {
    uint64_t s = ((shift >= 64 ? 0 : (i >> shift)) << 1) | (i & 1);
    for (int k = 0; k < 4; k++) col[4 * i + k] = m31_add(col[4 * i + k], curr[4 * s + k]);
  }
}
void pack_leaves(const uint32_t* const in[4], uint32_t* const out[64], uint64_t n) {
  for (uint32_t c = 0; c < 4; c++)
    for (uint64_t k = 0; k < n; k++) out[16 * c + (k % 16)][k / 16] = in[c][k];
}

// ------------------------------------------------------------------ Cairo group commitment
uint32_t coset_vanishing_at(const Coset& c, CPoint p) {  // circle.rs:238-253
  const CPoint shp = cp_repeated_double(CP_GENERATOR, 30 - c.log_size);
  const CPoint r = cp_mul(cp_mul(p, cp_conj(c.initial)), shp);
  uint32_t x = r.x;
  for (uint32_t i = 1; i < c.log_size; i++) x = m31_sub(m31_double(m31_mul(x, x)), 1);
  return x;
}
std::vector<uint32_t> zh_eval_domain(uint32_t log_n) {  // cairo_air/prover.rs:924-935
  const uint32_t log_eval = log_n + 2;
  const uint64_t N = 1ull << log_eval, half = N / 2;
  const Coset ho = coset_half_odds(log_eval - 1), hc = coset_half_coset(log_n);
  std::vector<uint32_t> zh(N);
  for (uint64_t i = 0; i < N; i++) {
    const uint64_t b = bit_reverse(i, log_eval);
    const CPoint p = b < half ? ho.at(b) : cp_conj(ho.at(b - half));
    zh[i] = coset_vanishing_at(hc, p);
  }
  return zh;
}
GroupCommit commit_group_cairo(const std::vector<std::vector<uint32_t>>& cols_hc, uint32_t log_n,
                               const std::vector<uint32_t>& blind, int threads) {
  GroupCommit g;
  const uint32_t log_eval = log_n + 2;
  const StwoTwiddles tw = stwo_twiddles(log_n), te = stwo_twiddles(log_eval);
  std::vector<uint32_t> zh;
  for (size_t c = 0; c < cols_hc.size(); c++) {
    std::vector<uint32_t> cn = permute_hc_natural_to_canonic_brt(cols_hc[c], log_n);
    std::vector<uint32_t> co = cn;
    stwo_interpolate(co, tw);
    g.coeffs.push_back(co);
    std::vector<uint32_t> ev = stwo_lde(cn, log_n, 2, tw, te);
    if (c < blind.size() && blind[c]) {
      if (zh.empty()) zh = zh_eval_domain(log_n);
      for (size_t i = 0; i < ev.size(); i++) ev[i] = m31_add(ev[i], m31_mul(blind[c], zh[i]));
    }
    g.eval_hc.push_back(permute_canonic_brt_to_hc_natural(ev, log_eval));
    g.eval_cn.push_back(std::move(ev));
  }
  std::vector<const uint32_t*> ptrs;
  for (auto& e : g.eval_cn) ptrs.push_back(e.data());
  const uint64_t N = 1ull << log_eval;
  std::vector<Hash> leaves(N);
  parallel_for(N, threads, [&](uint64_t lo, uint64_t hi) {
    std::vector<uint32_t> row(ptrs.size());
    for (uint64_t i = lo; i < hi; i++) {
      for (size_t c = 0; c < ptrs.size(); c++) row[c] = ptrs[c][i];
      leaves[i] = leaf_hash_capped(row.data(), (uint32_t)ptrs.size());
    }
  });
  auto layers = merkle_layers(leaves);  // layers[0] = leaves
  g.root = layers.back()[0];
  if (N < 1024) g.tile_roots = {g.root};
  else g.tile_roots = layers[10];
  return g;
}


// ------------------------------------------------------------------ Cairo OODS + FRI tail
static QM31 qm_double_x(QM31 x) {  // oods.rs double_x_qm31: 2x^2 - 1
  QM31 x2 = qm_mul(x, x);
  return qm_sub(qm_add(x2, x2), qm_m31(1));
}
// merkle.rs:294-330: SoA4 leaves, root and 1024-leaf tile roots (root alone below 1024)
static void soa4_root_tiles(const std::vector<uint32_t>* c, Hash& root, std::vector<Hash>& tiles, int threads) {
  const uint64_t n = c[0].size();
  std::vector<Hash> leaves(n);
  parallel_for(n, threads, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; i++) {
      uint32_t w[4] = {c[0][i], c[1][i], c[2][i], c[3][i]};
      leaves[i] = blake2s_words(w, 4);
    }
  });
  auto layers = merkle_layers(std::move(leaves));
  root = layers.back()[0];
  tiles = n < 1024 ? std::vector<Hash>{root} : layers[10];
}
CairoOodsFri cairo_oods_fri(Channel& ch, uint32_t log_n, const std::vector<std::vector<uint32_t>>& trace_coeffs,
                            const std::vector<uint32_t>& zk, const std::vector<std::vector<uint32_t>>& trace_evals,
                            const std::vector<std::vector<uint32_t>>& inter_evals,
                            const std::vector<std::vector<uint32_t>>& quot_hc, int threads) {
  CairoOodsFri r;
  const uint32_t log_eval = log_n + 2;
  const uint64_t n = 1ull << log_n, N = 1ull << log_eval;
  const size_t nt = trace_coeffs.size(), ni = inter_evals.size();
  const StwoTwiddles te = stwo_twiddles(log_eval);
  // AIR quotient: half-coset natural -> BRT-canonic, SoA4 commitment (prover.rs:1937-1971)
  std::vector<uint32_t> hq[4];
  for (int k = 0; k < 4; k++) hq[k] = permute_hc_natural_to_canonic_brt(quot_hc[k], log_eval);
  soa4_root_tiles(hq, r.quotient_root, r.quotient_tiles, threads);
  ch.mix_digest(r.quotient_root);
  // OODS point and its successor on the trace domain (prover.rs:1975-1985)
  const OodsPoint z = oods_point_from_channel(ch);
  const CPoint step = cp_repeated_double(CP_GENERATOR, 31 - log_n);
  const OodsPoint zn{qm_sub(qm_scale(z.x, step.x), qm_scale(z.y, step.y)),
                     qm_add(qm_scale(z.x, step.y), qm_scale(z.y, step.x))};
  r.z = z;
  QM31 zh_z = z.x, zh_zn = zn.x;  // oods.rs:285-291
  for (uint32_t i = 1; i < log_n; i++) { zh_z = qm_double_x(zh_z); zh_zn = qm_double_x(zh_zn); }
  // trace columns at z and z_next, blinding added as r * Z_H (prover.rs:1987-2001)
  for (size_t c = 0; c < nt; c++) {
    QM31 vz = eval_at_oods_from_coeffs(trace_coeffs[c], z), vn = eval_at_oods_from_coeffs(trace_coeffs[c], zn);
    if (c < zk.size() && zk[c]) {
      vz = qm_add(vz, qm_scale(zh_z, zk[c]));
      vn = qm_add(vn, qm_scale(zh_zn, zk[c]));
    }
    r.trace_at_z.push_back(vz);
    r.trace_at_z_next.push_back(vn);
  }
  // interaction columns: stwo iNTT of the evaluations, first n coefficients (prover.rs:2037-2048)
  for (size_t c = 0; c < ni; c++) {
    std::vector<uint32_t> co = inter_evals[c];
    stwo_interpolate(co, te);
    co.resize(n);
    r.inter_at_z.push_back(eval_at_oods_from_coeffs(co, z));
    r.inter_at_z_next.push_back(eval_at_oods_from_coeffs(co, zn));
  }
  // AIR quotient limbs at z from all N coefficients (prover.rs:2053-2065)
  for (int k = 0; k < 4; k++) {
    std::vector<uint32_t> co = hq[k];
    stwo_interpolate(co, te);
    r.quotient_at_z[k] = eval_at_oods_from_coeffs(co, z);
  }
  {  // sampled values in flatten_cols order (prover.rs:2067-2092)
    std::vector<QM31> all;
    for (size_t c = 0; c < nt; c++) { all.push_back(r.trace_at_z[c]); all.push_back(r.trace_at_z_next[c]); }
    for (size_t c = 0; c < ni; c++) { all.push_back(r.inter_at_z[c]); all.push_back(r.inter_at_z_next[c]); }
    for (int k = 0; k < 4; k++) all.push_back(r.quotient_at_z[k]);
    ch.mix_felts(all);
  }
  const QM31 alpha = ch.draw_felt();
  r.oods_alpha = alpha;
  // line coefficients weighted by powers of alpha (prover.rs:2095-2150)
  std::vector<QM31> bz, cz, bn, cn;
  QM31 lin_z{{0, 0, 0, 0}}, lin_n{{0, 0, 0, 0}}, ap = qm_m31(1);
  auto push = [&](OodsPoint p, QM31 v, std::vector<QM31>& b, std::vector<QM31>& c, QM31& lin) {
    QM31 a, bb;
    compute_line_coeffs(p, v, a, bb);
    b.push_back(qm_mul(ap, a));
    c.push_back(ap);
    lin = qm_add(lin, qm_mul(ap, bb));
    ap = qm_mul(ap, alpha);
  };
  for (size_t c = 0; c < nt; c++) push(z, r.trace_at_z[c], bz, cz, lin_z);
  for (int k = 0; k < 4; k++) push(z, r.quotient_at_z[k], bz, cz, lin_z);
  for (size_t c = 0; c < ni; c++) push(z, r.inter_at_z[c], bz, cz, lin_z);
  for (size_t c = 0; c < nt; c++) push(zn, r.trace_at_z_next[c], bn, cn, lin_n);
  for (size_t c = 0; c < ni; c++) push(zn, r.inter_at_z_next[c], bn, cn, lin_n);
  // numerators over [trace, quotient, interaction] columns (prover.rs:2152-2207)
  std::vector<const uint32_t*> cols;
  for (auto& e : trace_evals) cols.push_back(e.data());
  for (int k = 0; k < 4; k++) cols.push_back(hq[k].data());
  for (auto& e : inter_evals) cols.push_back(e.data());
  std::vector<uint32_t> idx_z, idx_n;
  for (uint32_t i = 0; i < nt + 4 + ni; i++) idx_z.push_back(i);
  for (uint32_t i = 0; i < nt; i++) idx_n.push_back(i);
  for (uint32_t i = 0; i < ni; i++) idx_n.push_back((uint32_t)(nt + 4 + i));
  std::vector<QM31> num_z(N), num_n(N);
  parallel_for(N, threads, [&](uint64_t lo, uint64_t hi) {
    std::vector<const uint32_t*> sub(cols.size());
    for (size_t c = 0; c < cols.size(); c++) sub[c] = cols[c] + lo;
    accumulate_numerators(sub, idx_z, bz, cz, hi - lo, num_z.data() + lo);
    accumulate_numerators(sub, idx_n, bn, cn, hi - lo, num_n.data() + lo);
  });
  // BRT-canonic domain points and the combination (prover.rs:2213-2266)
  std::vector<uint32_t> dx(N), dy(N);
  for (uint64_t i = 0; i < N; i++) {
    const CPoint p = canonic_domain_point(bit_reverse(i, log_eval), log_eval);
    dx[i] = p.x;
    dy[i] = p.y;
  }
  std::vector<QuotAcc> accs{{z.x, z.y, lin_z, num_z.data(), log_eval}, {zn.x, zn.y, lin_n, num_n.data(), log_eval}};
  std::vector<QM31> oq(N);
  quotients_combine(accs, dx.data(), dy.data(), log_eval, N, oq.data());
  for (int k = 0; k < 4; k++) {
    r.oods_q[k].resize(N);
    for (uint64_t i = 0; i < N; i++) r.oods_q[k][i] = oq[i].v[k];
  }
  soa4_root_tiles(r.oods_q, r.oods_root, r.oods_tiles, threads);
  ch.mix_digest(r.oods_root);
  // FRI: circle fold with twiddles 1/y of the canonic points (prover.rs:2321-2340)
  const QM31 fa = ch.draw_felt();
  r.fri_alphas.push_back(fa);
  const Coset ho = coset_half_odds(log_eval - 1);
  const std::vector<uint32_t> ctw = fold_twiddles(Coset{ho.initial, ho.step, log_eval}, true);
  std::vector<QM31> line(N / 2, QM31{{0, 0, 0, 0}});
  fold_circle_into_line(line.data(), oq.data(), ctw.data(), fa, N / 2);
  // committed line folds down to 2^3 values (prover.rs:2353-2381)
  uint32_t cur = log_eval - 1;
  while (cur > 3) {
    std::vector<uint32_t> soa[4];
    for (int k = 0; k < 4; k++) {
      soa[k].resize(line.size());
      for (size_t i = 0; i < line.size(); i++) soa[k][i] = line[i].v[k];
    }
    const uint32_t* cp[4] = {soa[0].data(), soa[1].data(), soa[2].data(), soa[3].data()};
    const Hash root = merkle_root_soa4(cp, line.size(), threads);
    ch.mix_digest(root);
    r.fri_roots.push_back(root);
    const QM31 a = ch.draw_felt();
    r.fri_alphas.push_back(a);
    const std::vector<uint32_t> tw = fold_twiddles(coset_half_odds(cur), false);
    std::vector<QM31> nx(line.size() / 2);
    fold_line(nx.data(), line.data(), tw.data(), a, nx.size());
    line.swap(nx);
    cur--;
  }
  r.last_layer = line;
  const std::vector<QM31> nat = last_layer_poly_coeffs(line);
  r.last_layer_coeffs.assign(nat.size(), QM31{{0, 0, 0, 0}});
  uint32_t lb = 0;
  while ((1ull << lb) < nat.size()) lb++;
  for (size_t i = 0; i < nat.size(); i++) r.last_layer_coeffs[bit_reverse(i, lb)] = nat[i];
  ch.mix_felts(r.last_layer_coeffs);
  return r;
}

}  // namespace vso
