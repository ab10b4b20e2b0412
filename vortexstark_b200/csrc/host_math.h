// Host-side M31/QM31 arithmetic, circle points, Blake2s-256 and the
// Fiat-Shamir channel, used by the prover's orchestration and the verifier.
// Same canonical arithmetic as the device code (src/field/*.rs, src/circle.rs,
// src/channel.rs).
#pragma once
#include <array>
#include <cstdint>
#include <cstring>
#include <vector>

namespace vs {
namespace h {

constexpr uint32_t P = 0x7FFFFFFFu;
inline uint32_t add(uint32_t a, uint32_t b) { uint32_t r = a + b; return r >= P ? r - P : r; }
inline uint32_t sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P - b; }
inline uint32_t neg(uint32_t a) { return a ? P - a : 0; }
inline uint32_t mul(uint32_t a, uint32_t b) {
  uint64_t p = (uint64_t)a * b;
  uint32_t r = ((uint32_t)p & P) + (uint32_t)(p >> 31);
  return r >= P ? r - P : r;
}
inline uint32_t dbl(uint32_t a) { return add(a, a); }
inline uint32_t pw(uint32_t a, uint32_t e) {
  uint32_t r = 1;
  while (e) { if (e & 1) r = mul(r, a); a = mul(a, a); e >>= 1; }
  return r;
}
inline uint32_t inv(uint32_t a) { return pw(a, P - 2); }

struct Q { uint32_t v[4]; };
inline bool operator==(const Q& a, const Q& b) { return !std::memcmp(a.v, b.v, 16); }
inline Q qadd(Q a, Q b) { return {{add(a.v[0], b.v[0]), add(a.v[1], b.v[1]), add(a.v[2], b.v[2]), add(a.v[3], b.v[3])}}; }
inline Q qsub(Q a, Q b) { return {{sub(a.v[0], b.v[0]), sub(a.v[1], b.v[1]), sub(a.v[2], b.v[2]), sub(a.v[3], b.v[3])}}; }
inline Q qscale(Q a, uint32_t s) { return {{mul(a.v[0], s), mul(a.v[1], s), mul(a.v[2], s), mul(a.v[3], s)}}; }
inline Q qmul(Q x, Q y) {
  auto cm = [](uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t& re, uint32_t& im) {
    re = sub(mul(a, c), mul(b, d));
    im = add(mul(a, d), mul(b, c));
  };
  uint32_t acr, aci, bdr, bdi, adr, adi, bcr, bci;
  cm(x.v[0], x.v[1], y.v[0], y.v[1], acr, aci);
  cm(x.v[2], x.v[3], y.v[2], y.v[3], bdr, bdi);
  cm(x.v[0], x.v[1], y.v[2], y.v[3], adr, adi);
  cm(x.v[2], x.v[3], y.v[0], y.v[1], bcr, bci);
  uint32_t ur = sub(dbl(bdr), bdi), ui = add(bdr, dbl(bdi));  // bd * (2 + i)
  return {{add(acr, ur), add(aci, ui), add(adr, bcr), add(adi, bci)}};
}

inline Q qconj(Q x) { return {{x.v[0], x.v[1], neg(x.v[2]), neg(x.v[3])}}; }  // a + bu -> a - bu
// (a + bu)^-1 = (a - bu) / (a^2 - (2 + i) b^2), the denominator inverted in CM31
// as conj(d) / |d|^2 (qm31.rs inverse). Zero maps to zero.
inline Q qinv(Q x) {
  const uint32_t a2r = sub(mul(x.v[0], x.v[0]), mul(x.v[1], x.v[1])), a2i = dbl(mul(x.v[0], x.v[1]));
  const uint32_t b2r = sub(mul(x.v[2], x.v[2]), mul(x.v[3], x.v[3])), b2i = dbl(mul(x.v[2], x.v[3]));
  const uint32_t dr = sub(a2r, sub(dbl(b2r), b2i)), di = sub(a2i, add(b2r, dbl(b2i)));
  const uint32_t s = inv(add(mul(dr, dr), mul(di, di)));
  const uint32_t ir = mul(dr, s), ii = mul(neg(di), s);
  auto cm = [](uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t& re, uint32_t& im) {
    re = sub(mul(a, c), mul(b, d));
    im = add(mul(a, d), mul(b, c));
  };
  Q r;
  cm(x.v[0], x.v[1], ir, ii, r.v[0], r.v[1]);
  cm(neg(x.v[2]), neg(x.v[3]), ir, ii, r.v[2], r.v[3]);
  return r;
}
inline Q qm31_of(uint32_t a) { return {{a, 0, 0, 0}}; }

struct Pt { uint32_t x, y; };
inline Pt pmul(Pt a, Pt b) { return {sub(mul(a.x, b.x), mul(a.y, b.y)), add(mul(a.x, b.y), mul(a.y, b.x))}; }
inline Pt ppow(Pt b, uint64_t e) {
  Pt r{1, 0};
  while (e) { if (e & 1) r = pmul(r, b); b = pmul(b, b); e >>= 1; }
  return r;
}
inline uint64_t brev(uint64_t v, uint32_t bits) {
  uint64_t r = 0;
  for (uint32_t i = 0; i < bits; i++) { r = (r << 1) | (v & 1); v >>= 1; }
  return r;
}

using Hash = std::array<uint32_t, 8>;

// Standard Blake2s-256 of a byte string (unkeyed, 32-byte digest).
std::array<uint8_t, 32> blake2s(const uint8_t* data, size_t len);
Hash blake2s_words(const uint32_t* w, size_t n);
inline Hash node(const Hash& l, const Hash& r) {
  uint32_t w[16];
  for (int i = 0; i < 8; i++) { w[i] = l[i]; w[8 + i] = r[i]; }
  return blake2s_words(w, 16);
}

// Fiat-Shamir transcript (channel.rs:15-185).
struct Channel {
  std::array<uint8_t, 32> state{};
  uint32_t n_draws = 0;
  void mix_digest(const Hash& d);
  void mix_felts(const std::vector<Q>& f);
  std::array<uint8_t, 32> squeeze();
  Q draw_felt();
  uint64_t draw_number(uint64_t bound);
  // channel.rs:102-116: 8 indices per squeeze, word & (2^log_size - 1)
  std::vector<uint32_t> draw_query_indices(uint32_t log_size, uint32_t n);
  // channel.rs:120-129: state = Blake2s(state || lo_LE || hi_LE)
  void mix_u64(uint64_t v);
  // channel.rs:144-152: Blake2s(0x12345678_LE || 0^12 || state || pow_bits_LE) as words
  Hash pow_prefix(uint32_t pow_bits) const;
};

// Circle cosets (circle.rs:101-144).
struct Coset {
  Pt initial, step;
  uint32_t log_size;
  Pt at(uint64_t i) const { return pmul(initial, ppow(step, i)); }
};
Coset half_coset(uint32_t log_size);
Coset half_odds(uint32_t log_size);
Coset subgroup(uint32_t log_size);

}  // namespace h
}  // namespace vs
