// Blake2s-256 compression kept entirely in registers (RFC 7693; unkeyed,
// 32-byte digest, no personalisation — the parameter block only sets
// digest length 32, fanout 1, depth 1, as in the reference's leaf, node and
// channel hashing).
//
// Rotations by 16 and 8 are byte permutes (PRMT); by 12 and 7 funnel shifts.
// Part of the additions run on the FMA pipe (see VS_G).
#pragma once
#include <cstdint>

namespace vs {

__constant__ constexpr uint32_t B2S_IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                             0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
constexpr uint32_t B2S_H0 = 0x6A09E667u ^ 0x01010020u;

__device__ __forceinline__ uint32_t rotr16(uint32_t x) { return __byte_perm(x, x, 0x1032); }
__device__ __forceinline__ uint32_t rotr8(uint32_t x) { return __byte_perm(x, x, 0x0321); }
__device__ __forceinline__ uint32_t rotr12(uint32_t x) { return __funnelshift_r(x, x, 12); }
__device__ __forceinline__ uint32_t rotr7(uint32_t x) { return __funnelshift_r(x, x, 7); }

// The XORs and rotations keep the integer ALU pipe busy; three of the G
// function's six additions are issued as multiply-adds (x * 1 + y) on the FMA
// pipe instead. The 1 lives in constant memory so the compiler cannot fold the
// multiply back into an ALU add. (Measured on B200: adding b + m first and then
// a with a multiply-add was the fastest split of the variants tried.)
static __constant__ uint32_t B2S_ONE = 1u;
__device__ __forceinline__ uint32_t fma_add(uint32_t x, uint32_t y) {
  uint32_t r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(B2S_ONE), "r"(y));
  return r;
}

#define VS_G(a, b, c, d, x, y)          \
  do {                                  \
    a = fma_add(a, b + (x));            \
    d = rotr16(d ^ a);                  \
    c = fma_add(c, d);                  \
    b = rotr12(b ^ c);                  \
    a = fma_add(a, b + (y));            \
    d = rotr8(d ^ a);                   \
    c = fma_add(c, d);                  \
    b = rotr7(b ^ c);                   \
  } while (0)

#define VS_ROUND(s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
  do {                                                                                  \
    VS_G(v0, v4, v8, v12, m[s0], m[s1]);                                                \
    VS_G(v1, v5, v9, v13, m[s2], m[s3]);                                                \
    VS_G(v2, v6, v10, v14, m[s4], m[s5]);                                               \
    VS_G(v3, v7, v11, v15, m[s6], m[s7]);                                               \
    VS_G(v0, v5, v10, v15, m[s8], m[s9]);                                               \
    VS_G(v1, v6, v11, v12, m[s10], m[s11]);                                             \
    VS_G(v2, v7, v8, v13, m[s12], m[s13]);                                              \
    VS_G(v3, v4, v9, v14, m[s14], m[s15]);                                              \
  } while (0)

// h[8] updated in place; m[16] message words (LE); t = byte counter; last = final block.
__device__ __forceinline__ void b2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t, bool last) {
  uint32_t v0 = h[0], v1 = h[1], v2 = h[2], v3 = h[3], v4 = h[4], v5 = h[5], v6 = h[6], v7 = h[7];
  uint32_t v8 = 0x6A09E667u, v9 = 0xBB67AE85u, v10 = 0x3C6EF372u, v11 = 0xA54FF53Au;
  uint32_t v12 = 0x510E527Fu ^ t, v13 = 0x9B05688Cu, v14 = last ? ~0x1F83D9ABu : 0x1F83D9ABu, v15 = 0x5BE0CD19u;
  VS_ROUND(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
  VS_ROUND(14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3);
  VS_ROUND(11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4);
  VS_ROUND(7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8);
  VS_ROUND(9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13);
  VS_ROUND(2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9);
  VS_ROUND(12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11);
  VS_ROUND(13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10);
  VS_ROUND(6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5);
  VS_ROUND(10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0);
  h[0] ^= v0 ^ v8; h[1] ^= v1 ^ v9; h[2] ^= v2 ^ v10; h[3] ^= v3 ^ v11;
  h[4] ^= v4 ^ v12; h[5] ^= v5 ^ v13; h[6] ^= v6 ^ v14; h[7] ^= v7 ^ v15;
}

__device__ __forceinline__ void b2s_init(uint32_t h[8]) {
  h[0] = B2S_H0; h[1] = 0xBB67AE85u; h[2] = 0x3C6EF372u; h[3] = 0xA54FF53Au;
  h[4] = 0x510E527Fu; h[5] = 0x9B05688Cu; h[6] = 0x1F83D9ABu; h[7] = 0x5BE0CD19u;
}

// Hash of a single block of n_words (<= 16) words: t = 4 * n_words, final.
__device__ __forceinline__ void b2s_single(uint32_t out[8], const uint32_t m[16], uint32_t n_words) {
  b2s_init(out);
  b2s_compress(out, m, n_words * 4u, true);
}

// Parent node = Blake2s(left || right), t = 64 (blake2s.cu:65-89 semantics).
__device__ __forceinline__ void b2s_node(uint32_t out[8], const uint32_t l[8], const uint32_t r[8]) {
  uint32_t m[16];
#pragma unroll
  for (int i = 0; i < 8; i++) { m[i] = l[i]; m[8 + i] = r[i]; }
  b2s_init(out);
  b2s_compress(out, m, 64u, true);
}

}  // namespace vs
