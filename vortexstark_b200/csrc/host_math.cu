// Host Blake2s-256, channel and cosets (see host_math.h).
#include "host_math.h"

namespace vs {
namespace h {

namespace {
const uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                        0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
const uint8_t SG[10][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0}};
inline uint32_t ror(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
void compress(uint32_t hs[8], const uint32_t m[16], uint32_t t, bool last) {
  uint32_t v[16];
  for (int i = 0; i < 8; i++) { v[i] = hs[i]; v[8 + i] = IV[i]; }
  v[12] ^= t;
  if (last) v[14] = ~v[14];
  auto g = [&](int a, int b, int c, int d, uint32_t x, uint32_t y) {
    v[a] += v[b] + x; v[d] = ror(v[d] ^ v[a], 16); v[c] += v[d]; v[b] = ror(v[b] ^ v[c], 12);
    v[a] += v[b] + y; v[d] = ror(v[d] ^ v[a], 8);  v[c] += v[d]; v[b] = ror(v[b] ^ v[c], 7);
  };
  for (int r = 0; r < 10; r++) {
    const uint8_t* s = SG[r];
    g(0, 4, 8, 12, m[s[0]], m[s[1]]);   g(1, 5, 9, 13, m[s[2]], m[s[3]]);
    g(2, 6, 10, 14, m[s[4]], m[s[5]]);  g(3, 7, 11, 15, m[s[6]], m[s[7]]);
    g(0, 5, 10, 15, m[s[8]], m[s[9]]);  g(1, 6, 11, 12, m[s[10]], m[s[11]]);
    g(2, 7, 8, 13, m[s[12]], m[s[13]]); g(3, 4, 9, 14, m[s[14]], m[s[15]]);
  }
  for (int i = 0; i < 8; i++) hs[i] ^= v[i] ^ v[8 + i];
}
uint32_t le(const uint8_t* b) { return b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24); }
}  // namespace

std::array<uint8_t, 32> blake2s(const uint8_t* data, size_t len) {
  uint32_t hs[8];
  for (int i = 0; i < 8; i++) hs[i] = IV[i];
  hs[0] ^= 0x01010020u;
  uint32_t m[16];
  uint8_t blk[64];
  size_t pos = 0;
  while (len - pos > 64) {
    for (int i = 0; i < 16; i++) m[i] = le(data + pos + 4 * i);
    pos += 64;
    compress(hs, m, (uint32_t)pos, false);
  }
  std::memset(blk, 0, 64);
  if (len > pos) std::memcpy(blk, data + pos, len - pos);
  for (int i = 0; i < 16; i++) m[i] = le(blk + 4 * i);
  compress(hs, m, (uint32_t)len, true);
  std::array<uint8_t, 32> out;
  for (int i = 0; i < 8; i++)
    for (int k = 0; k < 4; k++) out[4 * i + k] = (uint8_t)(hs[i] >> (8 * k));
  return out;
}
Hash blake2s_words(const uint32_t* w, size_t n) {
  std::vector<uint8_t> b(4 * n);
  for (size_t i = 0; i < n; i++)
    for (int k = 0; k < 4; k++) b[4 * i + k] = (uint8_t)(w[i] >> (8 * k));
  auto d = blake2s(b.data(), b.size());
  Hash h;
  for (int i = 0; i < 8; i++) h[i] = le(&d[4 * i]);
  return h;
}

void Channel::mix_digest(const Hash& d) {
  uint8_t in[64];
  std::memcpy(in, state.data(), 32);
  for (int i = 0; i < 8; i++)
    for (int k = 0; k < 4; k++) in[32 + 4 * i + k] = (uint8_t)(d[i] >> (8 * k));
  state = blake2s(in, 64);
  n_draws = 0;
}
void Channel::mix_felts(const std::vector<Q>& f) {
  if (f.empty()) return;
  std::vector<uint8_t> in(32 + 16 * f.size());
  std::memcpy(in.data(), state.data(), 32);
  for (size_t j = 0; j < f.size(); j++)
    for (int l = 0; l < 4; l++)
      for (int k = 0; k < 4; k++) in[32 + 16 * j + 4 * l + k] = (uint8_t)(f[j].v[l] >> (8 * k));
  state = blake2s(in.data(), in.size());
  n_draws = 0;
}
std::array<uint8_t, 32> Channel::squeeze() {
  uint8_t in[37];
  std::memcpy(in, state.data(), 32);
  for (int k = 0; k < 4; k++) in[32 + k] = (uint8_t)(n_draws >> (8 * k));
  in[36] = 0;
  n_draws++;
  return blake2s(in, 37);
}
Q Channel::draw_felt() {
  for (;;) {
    auto b = squeeze();
    uint32_t u[8];
    bool ok = true;
    for (int i = 0; i < 8; i++) { u[i] = le(&b[4 * i]); ok = ok && u[i] < 2 * P; }
    if (ok) return {{u[0] % P, u[1] % P, u[2] % P, u[3] % P}};
  }
}
uint64_t Channel::draw_number(uint64_t bound) {
  auto b = squeeze();
  uint64_t raw = 0;
  for (int k = 7; k >= 0; k--) raw = (raw << 8) | b[k];
  return raw % bound;
}
std::vector<uint32_t> Channel::draw_query_indices(uint32_t log_size, uint32_t n) {
  const uint32_t mask = log_size >= 32 ? ~0u : (1u << log_size) - 1;
  std::vector<uint32_t> out;
  out.reserve(n);
  while (out.size() < n) {
    auto b = squeeze();
    for (int i = 0; i < 8 && out.size() < n; i++) out.push_back(le(&b[4 * i]) & mask);
  }
  return out;
}
void Channel::mix_u64(uint64_t v) {
  uint8_t in[40];
  std::memcpy(in, state.data(), 32);
  for (int k = 0; k < 8; k++) in[32 + k] = (uint8_t)(v >> (8 * k));
  state = blake2s(in, 40);
  n_draws = 0;
}
Hash Channel::pow_prefix(uint32_t pow_bits) const {
  uint8_t in[52] = {0};
  for (int k = 0; k < 4; k++) in[k] = (uint8_t)(0x12345678u >> (8 * k));
  std::memcpy(in + 16, state.data(), 32);
  for (int k = 0; k < 4; k++) in[48 + k] = (uint8_t)(pow_bits >> (8 * k));
  const auto d = blake2s(in, 52);
  Hash h{};
  for (int i = 0; i < 8; i++) h[i] = le(&d[4 * i]);
  return h;
}

static Pt rdouble(Pt p, uint32_t k) {
  for (uint32_t i = 0; i < k; i++) p = pmul(p, p);
  return p;
}
static const Pt G{2, 1268011823u};
Coset half_coset(uint32_t l) { return {rdouble(G, 30 - l), rdouble(G, 31 - l), l}; }
Coset half_odds(uint32_t l) { return {rdouble(G, l >= 29 ? 0 : 29 - l), rdouble(G, 31 - l), l}; }
Coset subgroup(uint32_t l) { return {{1, 0}, rdouble(G, 31 - l), l}; }

}  // namespace h
}  // namespace vs
