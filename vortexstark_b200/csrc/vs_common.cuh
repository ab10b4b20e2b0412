// Shared host-side plumbing: status codes, error capture, launch helpers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/vstark.h"

namespace vs {

// Records a failure for vs_last_error() and returns its status code.
int set_error(int status, const char* fmt, ...);
void clear_error();

inline int check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return set_error(VS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return VS_OK;
}

#define VS_TRY(expr)                 \
  do {                               \
    int _st = (expr);                \
    if (_st != VS_OK) return _st;    \
  } while (0)

#define VS_CUDA(expr) VS_TRY(::vs::check_cuda((expr), #expr))

// Counts library kernel launches (read with vs_launch_count()).
void count_launch();

// Launch-configuration check after a kernel launch (does not synchronise).
#define VS_LAUNCHED(name)                                      \
  do {                                                         \
    ::vs::count_launch();                                      \
    VS_TRY(::vs::check_cuda(cudaGetLastError(), name));        \
  } while (0)

inline uint32_t ilog2(uint64_t n) {
  uint32_t l = 0;
  while ((1ull << l) < n) l++;
  return l;
}
inline bool is_pow2(uint64_t n) { return n && !(n & (n - 1)); }
inline unsigned blocks_for(uint64_t n, unsigned threads) { return (unsigned)((n + threads - 1) / threads); }

// Number of SMs on the current device (cached per process).
int sm_count();

}  // namespace vs
