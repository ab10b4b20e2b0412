// Vector accesses to caller-owned global memory. Entry points take plain device
// pointers, which are only promised to be 4-byte aligned (the reference's kernels
// read them word by word). Every 64/128-bit access here checks its address at
// run time and falls back to words when it is not aligned. The wide access is
// inline PTX (volatile): the compiler can neither speculate it past the check nor
// fuse it with the word path, and the word path's plain 32-bit accesses carry no
// alignment the compiler could widen them with.
#pragma once
#include <cstdint>

namespace vs {

__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
__device__ __forceinline__ bool aligned8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7) == 0; }

__device__ __forceinline__ uint4 ld4(const uint32_t* p) {
  uint4 v;
  if (aligned16(p)) {
    asm volatile("ld.global.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  } else {
    v.x = p[0];
    v.y = p[1];
    v.z = p[2];
    v.w = p[3];
  }
  return v;
}
// Read-only variant (the data is not written while the kernel runs).
__device__ __forceinline__ uint4 ld4_ro(const uint32_t* p) {
  uint4 v;
  if (aligned16(p)) {
    asm volatile("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  } else {
    v.x = __ldg(p);
    v.y = __ldg(p + 1);
    v.z = __ldg(p + 2);
    v.w = __ldg(p + 3);
  }
  return v;
}
__device__ __forceinline__ void st4(uint32_t* p, uint4 v) {
  if (aligned16(p)) {
    asm volatile("st.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w) : "memory");
  } else {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
    p[3] = v.w;
  }
}
__device__ __forceinline__ uint2 ld2(const uint32_t* p) {
  uint2 v;
  if (aligned8(p)) {
    asm volatile("ld.global.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
  } else {
    v.x = p[0];
    v.y = p[1];
  }
  return v;
}
__device__ __forceinline__ void st2(uint32_t* p, uint2 v) {
  if (aligned8(p)) {
    asm volatile("st.global.v2.u32 [%0], {%1, %2};" ::"l"(p), "r"(v.x), "r"(v.y) : "memory");
  } else {
    p[0] = v.x;
    p[1] = v.y;
  }
}

// Global -> shared without holding registers: one 16-byte cp.async when the
// global address is 16-byte aligned, four 4-byte ones otherwise. dst is a
// shared-space address with 16-byte alignment.
__device__ __forceinline__ void cp_async_16_or_words(uint32_t dst, const uint32_t* src) {
  if (aligned16(src)) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
  } else {
#pragma unroll
    for (int k = 0; k < 4; k++)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst + 4 * k), "l"(src + k) : "memory");
  }
}

}  // namespace vs
