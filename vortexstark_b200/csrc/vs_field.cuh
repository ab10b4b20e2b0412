// M31 / CM31 / QM31 arithmetic for sm_100a.
//
// Values are canonical (< p = 2^31 - 1) at every function boundary, so every
// result is the mathematically defined residue and matches the reference's
// canonical arithmetic (src/field/m31.rs, cm31.rs, qm31.rs) bit for bit.
// Reductions use the branch-free min(r, r - p) form: when r < p the unsigned
// subtraction wraps to a large value and min keeps r.
#pragma once
#include <cstdint>

#define VS_P 0x7FFFFFFFu

namespace vs {

__device__ __forceinline__ uint32_t canon(uint32_t r) { return min(r, r - VS_P); }  // r < 2p
__device__ __forceinline__ uint32_t add(uint32_t a, uint32_t b) { return canon(a + b); }
__device__ __forceinline__ uint32_t sub(uint32_t a, uint32_t b) { return canon(a + VS_P - b); }
__device__ __forceinline__ uint32_t neg(uint32_t a) { return canon(VS_P - a); }  // 0 -> p -> 0
__device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) {
  uint64_t p = (uint64_t)a * b;  // < 2^62
  uint32_t r = ((uint32_t)p & VS_P) + (uint32_t)(p >> 31);
  return canon(r);
}
__device__ __forceinline__ uint32_t dbl(uint32_t a) { return canon(a << 1); }
__device__ __forceinline__ uint32_t pow(uint32_t a, uint32_t e) {
  uint32_t r = 1;
  while (e) { if (e & 1) r = mul(r, a); a = mul(a, a); e >>= 1; }
  return r;
}
// a^(p-2) = a^(2^31 - 3) (Fermat; 0 -> 0) by a fixed addition chain: 30 squarings
// and 8 multiplications instead of square-and-multiply's 31 + 30.
//   e_k = a^(2^k - 1):  e2 = e1^2 e1, e4 = e2^(2^2) e2, e8 = e4^(2^4) e4,
//   e16 = e8^(2^8) e8, e24 = e16^(2^8) e8, e28 = e24^(2^4) e4, e29 = e28^2 a,
//   a^(p-2) = e29^(2^2) a   since (2^29 - 1) * 4 + 1 = 2^31 - 3.
__device__ __forceinline__ uint32_t sqn(uint32_t x, int n) {
#pragma unroll
  for (int i = 0; i < n; i++) x = mul(x, x);
  return x;
}
__device__ __forceinline__ uint32_t inv(uint32_t a) {
  const uint32_t e2 = mul(sqn(a, 1), a);
  const uint32_t e4 = mul(sqn(e2, 2), e2);
  const uint32_t e8 = mul(sqn(e4, 4), e4);
  const uint32_t e16 = mul(sqn(e8, 8), e8);
  const uint32_t e24 = mul(sqn(e16, 8), e8);
  const uint32_t e28 = mul(sqn(e24, 4), e4);
  const uint32_t e29 = mul(sqn(e28, 1), a);
  return mul(sqn(e29, 2), a);
}

struct cm31 { uint32_t a, b; };
__device__ __forceinline__ cm31 cadd(cm31 x, cm31 y) { return {add(x.a, y.a), add(x.b, y.b)}; }
__device__ __forceinline__ cm31 csub(cm31 x, cm31 y) { return {sub(x.a, y.a), sub(x.b, y.b)}; }
__device__ __forceinline__ cm31 cmul(cm31 x, cm31 y) {
  return {sub(mul(x.a, y.a), mul(x.b, y.b)), add(mul(x.a, y.b), mul(x.b, y.a))};
}
__device__ __forceinline__ cm31 cinv(cm31 x) {
  uint32_t in = inv(add(mul(x.a, x.a), mul(x.b, x.b)));
  return {mul(x.a, in), mul(neg(x.b), in)};
}

// QM31 = (a, b) = a + b*u with u^2 = 2 + i; limbs v = [a.a, a.b, b.a, b.b].
struct qm31 { uint32_t v[4]; };
__device__ __forceinline__ qm31 qzero() { return {{0, 0, 0, 0}}; }
__device__ __forceinline__ qm31 qadd(qm31 x, qm31 y) {
  return {{add(x.v[0], y.v[0]), add(x.v[1], y.v[1]), add(x.v[2], y.v[2]), add(x.v[3], y.v[3])}};
}
__device__ __forceinline__ qm31 qsub(qm31 x, qm31 y) {
  return {{sub(x.v[0], y.v[0]), sub(x.v[1], y.v[1]), sub(x.v[2], y.v[2]), sub(x.v[3], y.v[3])}};
}
__device__ __forceinline__ qm31 qscale(qm31 x, uint32_t s) {
  return {{mul(x.v[0], s), mul(x.v[1], s), mul(x.v[2], s), mul(x.v[3], s)}};
}
__device__ __forceinline__ qm31 qscale_c(qm31 x, cm31 s) {
  cm31 a = cmul({x.v[0], x.v[1]}, s), b = cmul({x.v[2], x.v[3]}, s);
  return {{a.a, a.b, b.a, b.b}};
}
__device__ __forceinline__ qm31 qmul(qm31 x, qm31 y) {
  cm31 xa{x.v[0], x.v[1]}, xb{x.v[2], x.v[3]}, ya{y.v[0], y.v[1]}, yb{y.v[2], y.v[3]};
  cm31 ac = cmul(xa, ya), bd = cmul(xb, yb), ad = cmul(xa, yb), bc = cmul(xb, ya);
  cm31 bdu{sub(dbl(bd.a), bd.b), add(bd.a, dbl(bd.b))};  // bd * (2 + i)
  cm31 ra = cadd(ac, bdu), rb = cadd(ad, bc);
  return {{ra.a, ra.b, rb.a, rb.b}};
}

// Circle group over M31: (x1,y1)*(x2,y2) = (x1x2 - y1y2, x1y2 + y1x2).
struct cpt { uint32_t x, y; };
__device__ __forceinline__ cpt cpmul(cpt a, cpt b) {
  return {sub(mul(a.x, b.x), mul(a.y, b.y)), add(mul(a.x, b.y), mul(a.y, b.x))};
}
__device__ __forceinline__ cpt cppow(cpt b, uint32_t e) {
  cpt r{1, 0};
  while (e) { if (e & 1) r = cpmul(r, b); b = cpmul(b, b); e >>= 1; }
  return r;
}

__device__ __forceinline__ uint32_t brev(uint32_t v, uint32_t bits) { return bits ? __brev(v) >> (32 - bits) : 0; }

}  // namespace vs
