// Fiat–Shamir channel as a C ABI (src/channel.rs: mix_digest, mix_felts,
// draw_felt, draw_number, draw_query_indices, mix_u64, verify_pow_nonce) and the
// Blake2s proof-of-work grind on the GPU (cuda/grind.cu, cuda/grind_m31_output.cu).
//
// Grinding: nonce k passes when the first 16 bytes of Blake2s(prefix || k_LE), a
// single 40-byte block, read as a little-endian u128, have at least pow_bits
// trailing zeros (with every word reduced mod 2^31 - 1 first for the M31-output
// variant). The kernel walks nonces grid-stride and keeps the smallest passing
// one with atomicMin; a thread stops as soon as a smaller nonce is recorded, so
// the answer is the minimum of the range whatever the scheduling.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "host_math.h"
#include "vs_blake2s.cuh"
#include "vs_common.cuh"

namespace vs {

template <bool M31_OUTPUT>
__device__ __forceinline__ uint32_t pow_trailing_zeros(const uint32_t prefix[8], uint64_t nonce) {
  uint32_t m[16] = {prefix[0], prefix[1], prefix[2], prefix[3], prefix[4], prefix[5], prefix[6], prefix[7],
                    (uint32_t)nonce, (uint32_t)(nonce >> 32), 0, 0, 0, 0, 0, 0};
  uint32_t h[8];
  b2s_init(h);
  b2s_compress(h, m, 40u, true);
  uint32_t tz = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint32_t v = h[k];
    if (M31_OUTPUT) {  // m31.cuh:9-14 on a 32-bit word: (v & p) + (v >> 31), then < p
      v = (v & 0x7FFFFFFFu) + (v >> 31);
      v = v >= 0x7FFFFFFFu ? v - 0x7FFFFFFFu : v;
    }
    if (v) return tz + (uint32_t)(__ffs(v) - 1);
    tz += 32;
  }
  return tz;
}

template <bool M31_OUTPUT>
__global__ void grind_pow_kernel(const uint32_t* __restrict__ prefix, unsigned long long* __restrict__ result,
                                 uint32_t pow_bits, uint64_t offset, uint64_t n) {
  uint32_t p[8];
#pragma unroll
  for (int k = 0; k < 8; k++) p[k] = __ldg(prefix + k);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t nonce = offset + i;
    if (*(volatile unsigned long long*)result < nonce) return;  // a smaller passing nonce is known
    if (pow_trailing_zeros<M31_OUTPUT>(p, nonce) >= pow_bits) {
      atomicMin(result, (unsigned long long)nonce);
      return;
    }
  }
}

static int launch_grind(const uint32_t* d_prefix, uint64_t* d_result, uint32_t pow_bits, uint64_t offset, uint64_t n,
                        bool m31, cudaStream_t st) {
  if (!n) return VS_OK;
  const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 16);
  if (m31)
    grind_pow_kernel<true><<<(unsigned)blocks, 256, 0, st>>>(d_prefix, (unsigned long long*)d_result, pow_bits, offset, n);
  else
    grind_pow_kernel<false><<<(unsigned)blocks, 256, 0, st>>>(d_prefix, (unsigned long long*)d_result, pow_bits, offset, n);
  VS_LAUNCHED("grind_pow_kernel");
  return VS_OK;
}

}  // namespace vs

using namespace vs;

extern "C" {

// ------------------------------------------------------------------ drop-ins (cuda/grind*.cu)
void cuda_grind_pow(const uint32_t* prefixed_digest, uint64_t* result, uint32_t pow_bits, uint64_t batch_offset,
                    uint32_t n_threads) {
  launch_grind(prefixed_digest, result, pow_bits, batch_offset, n_threads, false, 0);
}
void cuda_grind_pow_m31_output(const uint32_t* prefixed_digest, uint64_t* result, uint32_t pow_bits,
                               uint64_t batch_offset, uint32_t n_threads) {
  launch_grind(prefixed_digest, result, pow_bits, batch_offset, n_threads, true, 0);
}

// ------------------------------------------------------------------ channel
int vs_channel_create(void** ch) {
  clear_error();
  if (!ch) return set_error(VS_ERR_INVALID, "vs_channel_create: null handle");
  *ch = new h::Channel();
  return VS_OK;
}
int vs_channel_destroy(void* ch) {
  delete static_cast<h::Channel*>(ch);
  return VS_OK;
}
int vs_channel_state(void* ch, uint8_t* h_state32, uint32_t* n_draws) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c || !h_state32) return set_error(VS_ERR_INVALID, "vs_channel_state: null");
  std::memcpy(h_state32, c->state.data(), 32);
  if (n_draws) *n_draws = c->n_draws;
  return VS_OK;
}
int vs_channel_mix_digest(void* ch, const uint32_t* h_digest8) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c || !h_digest8) return set_error(VS_ERR_INVALID, "vs_channel_mix_digest: null");
  h::Hash d{};
  for (int i = 0; i < 8; i++) d[i] = h_digest8[i];
  c->mix_digest(d);
  return VS_OK;
}
int vs_channel_mix_felts(void* ch, const uint32_t* h_felts, uint64_t n_felts) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c || (n_felts && !h_felts)) return set_error(VS_ERR_INVALID, "vs_channel_mix_felts: null");
  std::vector<h::Q> f(n_felts);
  for (uint64_t j = 0; j < n_felts; j++)
    for (int l = 0; l < 4; l++) f[j].v[l] = h_felts[4 * j + l];
  c->mix_felts(f);
  return VS_OK;
}
int vs_channel_mix_u64(void* ch, uint64_t value) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c) return set_error(VS_ERR_INVALID, "vs_channel_mix_u64: null");
  c->mix_u64(value);
  return VS_OK;
}
int vs_channel_draw_felt(void* ch, uint32_t* h_out4) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c || !h_out4) return set_error(VS_ERR_INVALID, "vs_channel_draw_felt: null");
  const h::Q q = c->draw_felt();
  for (int l = 0; l < 4; l++) h_out4[l] = q.v[l];
  return VS_OK;
}
int vs_channel_draw_number(void* ch, uint64_t bound, uint64_t* out) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c || !out || !bound) return set_error(VS_ERR_INVALID, "vs_channel_draw_number: null or zero bound");
  *out = c->draw_number(bound);
  return VS_OK;
}
int vs_channel_draw_query_indices(void* ch, uint32_t log_domain_size, uint32_t n, uint32_t* h_out) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c || (n && !h_out) || log_domain_size > 32)
    return set_error(VS_ERR_INVALID, "vs_channel_draw_query_indices: bad arguments");
  const auto v = c->draw_query_indices(log_domain_size, n);
  std::memcpy(h_out, v.data(), v.size() * 4);
  return VS_OK;
}
int vs_channel_pow_prefix(void* ch, uint32_t pow_bits, uint32_t* h_out8) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c || !h_out8) return set_error(VS_ERR_INVALID, "vs_channel_pow_prefix: null");
  const h::Hash p = c->pow_prefix(pow_bits);
  for (int i = 0; i < 8; i++) h_out8[i] = p[i];
  return VS_OK;
}
int vs_channel_verify_pow_nonce(void* ch, uint32_t pow_bits, uint64_t nonce) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c) {
    set_error(VS_ERR_INVALID, "vs_channel_verify_pow_nonce: null");
    return -1;
  }
  const h::Hash p = c->pow_prefix(pow_bits);
  uint32_t w[10];
  for (int i = 0; i < 8; i++) w[i] = p[i];
  w[8] = (uint32_t)nonce;
  w[9] = (uint32_t)(nonce >> 32);
  const h::Hash r = h::blake2s_words(w, 10);
  uint32_t tz = 0;
  for (int k = 0; k < 4; k++) {
    if (r[k]) { tz += (uint32_t)__builtin_ctz(r[k]); break; }
    tz += 32;
  }
  return tz >= pow_bits ? 1 : 0;
}
int vs_channel_grind_pow(void* ch, uint32_t pow_bits, uint64_t max_nonces, uint64_t* nonce, vs_stream_t stream) {
  clear_error();
  auto* c = static_cast<h::Channel*>(ch);
  if (!c || !nonce || pow_bits > 128) return set_error(VS_ERR_INVALID, "vs_channel_grind_pow: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const h::Hash p = c->pow_prefix(pow_bits);
  uint32_t* dev = nullptr;  // 8 prefix words + the 64-bit result
  VS_CUDA(cudaMallocAsync((void**)&dev, 48, st));
  uint64_t* d_result = reinterpret_cast<uint64_t*>(dev + 8);
  uint32_t host[12];
  for (int i = 0; i < 8; i++) host[i] = p[i];
  host[8] = host[9] = host[10] = host[11] = 0xFFFFFFFFu;
  int rc = check_cuda(cudaMemcpyAsync(dev, host, 48, cudaMemcpyHostToDevice, st), "grind upload");
  uint64_t found = ~0ull;
  const uint64_t batch = 1ull << 26;
  for (uint64_t off = 0; rc == VS_OK && found == ~0ull && off < max_nonces; off += batch) {
    rc = launch_grind(dev, d_result, pow_bits, off, std::min(batch, max_nonces - off), false, st);
    if (rc == VS_OK) rc = check_cuda(cudaMemcpyAsync(&found, d_result, 8, cudaMemcpyDeviceToHost, st), "grind result");
    if (rc == VS_OK) rc = check_cuda(cudaStreamSynchronize(st), "grind sync");
  }
  cudaFreeAsync(dev, st);
  if (rc != VS_OK) return rc;
  if (found == ~0ull) return set_error(VS_ERR_INVALID, "vs_channel_grind_pow: no nonce below %llu", (unsigned long long)max_nonces);
  *nonce = found;
  return VS_OK;
}

}  // extern "C"
