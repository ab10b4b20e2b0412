// Fiat-Shamir channel on the device (src/channel.rs:15-185), run by one thread,
// so the prover's stage chain needs no host round trip and can be captured in
// a CUDA graph. State: 8 words (the 32-byte digest, LE) + the draw counter.
#pragma once
#include <cstdint>

#include "vs_blake2s.cuh"

namespace vs {

struct ChanDev {
  uint32_t state[8];
  uint32_t n_draws;
  uint32_t error;  // set when a rejection loop exceeds its bound (never expected)
};

// state = Blake2s(state || digest)   (mix_digest, 64-byte input)
__device__ __forceinline__ void ch_mix_digest(ChanDev& c, const uint32_t* d) {
  uint32_t m[16], h[8];
#pragma unroll
  for (int i = 0; i < 8; i++) { m[i] = c.state[i]; m[8 + i] = d[i]; }
  b2s_init(h);
  b2s_compress(h, m, 64u, true);
#pragma unroll
  for (int i = 0; i < 8; i++) c.state[i] = h[i];
  c.n_draws = 0;
}

// Blake2s(state || n_draws_le || 0x00)   (squeeze, 37-byte input)
__device__ __forceinline__ void ch_squeeze(ChanDev& c, uint32_t out[8]) {
  uint32_t m[16] = {0};
#pragma unroll
  for (int i = 0; i < 8; i++) m[i] = c.state[i];
  m[8] = c.n_draws;
  m[9] = 0;  // the domain byte 0x00 followed by zero padding
  b2s_init(out);
  b2s_compress(out, m, 37u, true);
  c.n_draws++;
}

// draw_felt: rejection until all 8 words < 2p, then the first 4 mod p.
__device__ __forceinline__ void ch_draw_felt(ChanDev& c, uint32_t out[4]) {
  for (int tries = 0; tries < 64; tries++) {
    uint32_t w[8];
    ch_squeeze(c, w);
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 8; i++) ok = ok && w[i] < 2u * 0x7FFFFFFFu;
    if (ok) {
#pragma unroll
      for (int i = 0; i < 4; i++) out[i] = w[i] % 0x7FFFFFFFu;
      return;
    }
  }
  c.error = 1;
  for (int i = 0; i < 4; i++) out[i] = 0;
}

// draw_number for a power-of-two bound: u64_le(bytes[0..8]) mod bound.
__device__ __forceinline__ uint32_t ch_draw_pow2(ChanDev& c, uint32_t log_bound) {
  uint32_t w[8];
  ch_squeeze(c, w);
  uint64_t raw = ((uint64_t)w[1] << 32) | w[0];
  return (uint32_t)(raw & ((1ull << log_bound) - 1));
}

// mix_felts over n QM31 values given as 4 planes (multi-block Blake2s of
// state || v0 || v1 || ..., each value 4 LE words).
__device__ __forceinline__ void ch_mix_felts_planes(ChanDev& c, const uint32_t* const planes[4], uint32_t n) {
  const uint32_t total = 8 + 4 * n;  // words
  uint32_t h[8], m[16];
  b2s_init(h);
  uint32_t pos = 0, seen = 0;
  for (uint32_t wi = 0; wi < total; wi++) {
    uint32_t word = wi < 8 ? c.state[wi] : planes[(wi - 8) & 3][(wi - 8) >> 2];
    m[pos++] = word;
    seen++;
    if (pos == 16 && seen < total) {
      b2s_compress(h, m, seen * 4u, false);
      pos = 0;
    }
  }
  for (uint32_t w = pos; w < 16; w++) m[w] = 0;
  b2s_compress(h, m, total * 4u, true);
#pragma unroll
  for (int i = 0; i < 8; i++) c.state[i] = h[i];
  c.n_draws = 0;
}

}  // namespace vs
