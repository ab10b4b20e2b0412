// Twiddle generation on the device: coset points, line-twiddle squashing, FRI
// fold twiddles and the chunked batch inverse (drop-in for cuda/twiddles.cu and
// cuda/batch_inverse.cu), plus builders for the cached native and stwo twiddle
// tables used by the NTT paths.
#include <mutex>
#include <unordered_map>
#include <vector>

#include "twiddles.h"
#include "vs_common.cuh"
#include "vs_field.cuh"

namespace vs {

// ----------------------------------------------------------------- coset points
// Strided assignment: thread t owns points t, t+T, t+2T, ... so stores are
// coalesced; its first point is initial*step^t and it advances by step^T.
__global__ void coset_points_kernel(cpt initial, cpt step, cpt step_T, uint32_t* __restrict__ ox,
                                    uint32_t* __restrict__ oy, uint64_t n) {
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t T = (uint64_t)gridDim.x * blockDim.x;
  if (t >= n) return;
  cpt p = cpmul(initial, cppow(step, (uint32_t)t));
  for (uint64_t i = t; i < n; i += T) {
    ox[i] = p.x;
    oy[i] = p.y;
    p = cpmul(p, step_T);
  }
}

int launch_coset_points(cpt initial, cpt step, uint32_t* ox, uint32_t* oy, uint64_t n, cudaStream_t st) {
  if (n == 0) return VS_OK;
  unsigned threads = 256;
  uint64_t want = (uint64_t)sm_count() * 8 * threads;
  uint64_t total = n < want ? n : want;
  unsigned blocks = blocks_for(total, threads);
  uint64_t T = (uint64_t)blocks * threads;
  cpt step_T{1, 0};
  {  // host-side step^T
    auto hmul = [](cpt a, cpt b) {
      auto m = [](uint32_t x, uint32_t y) {
        uint64_t p = (uint64_t)x * y;
        uint32_t r = ((uint32_t)p & VS_P) + (uint32_t)(p >> 31);
        return r >= VS_P ? r - VS_P : r;
      };
      auto ad = [](uint32_t x, uint32_t y) { uint32_t r = x + y; return r >= VS_P ? r - VS_P : r; };
      auto sb = [](uint32_t x, uint32_t y) { return x >= y ? x - y : x + VS_P - y; };
      return cpt{sb(m(a.x, b.x), m(a.y, b.y)), ad(m(a.x, b.y), m(a.y, b.x))};
    };
    cpt b = step;
    uint64_t e = T;
    while (e) { if (e & 1) step_T = hmul(step_T, b); b = hmul(b, b); e >>= 1; }
  }
  coset_points_kernel<<<blocks, threads, 0, st>>>(initial, step, step_T, ox, oy, n);
  VS_LAUNCHED("coset_points_kernel");
  return VS_OK;
}

__global__ void extract_and_squash_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ tw,
                                          uint32_t* __restrict__ sq, uint32_t half_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  uint32_t x = in[2 * i];
  if (tw) tw[i] = x;
  uint32_t x2 = mul(x, x);
  sq[i] = sub(add(x2, x2), 1);
}

// ----------------------------------------------------------------- fold twiddle sources
// out[i] = coord(initial * step^bitrev(2i, log_n))   (twiddles.cu:23-52 semantics)
__global__ void fold_sources_kernel(cpt initial, cpt step, uint32_t* __restrict__ out, uint32_t half_n,
                                    uint32_t log_n, int extract_y) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  cpt p = cpmul(initial, cppow(step, brev(i << 1, log_n)));
  out[i] = extract_y ? p.y : p.x;
}

// ----------------------------------------------------------------- chunked batch inverse
// One thread per 64-element chunk. The CTA stages its 128 chunks through shared
// memory with a 65-word row pitch so both the coalesced global transfers and the
// per-thread sequential chunk walks are bank-conflict free.
constexpr int BI_CHUNK = 64, BI_THREADS = 128, BI_PITCH = 65;

__global__ void __launch_bounds__(BI_THREADS) batch_inverse_kernel(const uint32_t* __restrict__ in,
                                                                   uint32_t* __restrict__ out, uint64_t n) {
  __shared__ uint32_t sm[BI_THREADS * BI_PITCH];
  const uint64_t base = (uint64_t)blockIdx.x * BI_THREADS * BI_CHUNK;
  for (uint32_t e = threadIdx.x; e < BI_THREADS * BI_CHUNK; e += BI_THREADS) {
    uint64_t g = base + e;
    sm[(e / BI_CHUNK) * BI_PITCH + e % BI_CHUNK] = g < n ? in[g] : 0u;
  }
  __syncthreads();
  const uint64_t start = base + (uint64_t)threadIdx.x * BI_CHUNK;
  uint32_t* row = sm + threadIdx.x * BI_PITCH;
  if (start < n) {
    const uint32_t count = (uint32_t)((n - start) < BI_CHUNK ? (n - start) : BI_CHUNK);
    uint32_t prefix[BI_CHUNK];
    prefix[0] = row[0];
#pragma unroll
    for (uint32_t i = 1; i < BI_CHUNK; i++) {
      if (i < count) {
        uint32_t v = row[i];
        prefix[i] = v == 0 ? prefix[i - 1] : mul(prefix[i - 1], v);
      }
    }
    uint32_t acc = inv(prefix[count - 1]);
#pragma unroll
    for (int i = BI_CHUNK - 1; i > 0; i--) {
      if ((uint32_t)i < count) {
        uint32_t v = row[i];
        if (v == 0) {
          row[i] = 0;
        } else {
          row[i] = mul(acc, prefix[i - 1]);
          acc = mul(acc, v);
        }
      }
    }
    row[0] = row[0] == 0 ? 0 : acc;
  }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < BI_THREADS * BI_CHUNK; e += BI_THREADS) {
    uint64_t g = base + e;
    if (g < n) out[g] = sm[(e / BI_CHUNK) * BI_PITCH + e % BI_CHUNK];
  }
}

int launch_batch_inverse(const uint32_t* in, uint32_t* out, uint64_t n, cudaStream_t st) {
  if (n == 0) return VS_OK;
  uint64_t per_block = (uint64_t)BI_THREADS * BI_CHUNK;
  batch_inverse_kernel<<<blocks_for(n, (unsigned)per_block), BI_THREADS, 0, st>>>(in, out, n);
  VS_LAUNCHED("batch_inverse_kernel");
  return VS_OK;
}

// ----------------------------------------------------------------- cached twiddle tables
// Native layout (circle.rs:277-340): line layer l (0-based, used by NTT layer l+1)
// at offset n - n/2^l, size n/2^(l+1), entry i = squash^l(x(coset.at(2^(l+1) i)));
// the final slot (index n-2) is zero. Circle twiddles: y(coset.at(i)), i < n/2.
__global__ void native_line_kernel(cpt initial, cpt step, uint32_t log_n, uint32_t* __restrict__ line) {
  const uint32_t n = 1u << log_n;
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n - 1) return;
  if (e == n - 2 || n < 4) { line[e] = 0; return; }
  // locate layer: offsets n - n/2^l
  uint32_t l = 0, off = 0, sz = n / 2;
  while (e >= off + sz) { off += sz; sz >>= 1; l++; }
  uint32_t i = e - off;
  cpt p = cpmul(initial, cppow(step, i << (l + 1)));
  uint32_t x = p.x;
  for (uint32_t k = 0; k < l; k++) { uint32_t x2 = mul(x, x); x = sub(add(x2, x2), 1); }
  line[e] = x;
}
__global__ void native_circle_kernel(cpt initial, cpt step, uint32_t half_n, uint32_t* __restrict__ circ) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  circ[i] = cpmul(initial, cppow(step, i)).y;
}
// stwo layout (ntt.rs:262-325): for k = 0..L-2, layer k holds the x-coords of the
// first half of half_odds(L-1) doubled k times, bit-reversed within the layer;
// then a single 1. Entry count n/2.
__global__ void stwo_table_kernel(cpt initial, cpt step, uint32_t log_n, uint32_t* __restrict__ tw) {
  const uint32_t half = 1u << (log_n - 1);
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= half) return;
  if (e == half - 1) { tw[e] = 1; return; }
  uint32_t k = 0, off = 0, sz = half / 2;  // layer k has 2^(L-2-k) entries
  while (e >= off + sz) { off += sz; sz >>= 1; k++; }
  uint32_t i = e - off;
  uint32_t layer_log = (log_n - 2) - k;
  cpt ini = initial, stp = step;
  for (uint32_t d = 0; d < k; d++) { ini = cpmul(ini, ini); stp = cpmul(stp, stp); }
  tw[e] = cpmul(ini, cppow(stp, brev(i, layer_log))).x;
}

namespace {
std::mutex g_mu;
std::unordered_map<uint64_t, TwiddleSet*> g_cache;
uint64_t key(int dev, int kind, uint32_t log_n) { return ((uint64_t)dev << 40) | ((uint64_t)kind << 32) | log_n; }
}  // namespace

static cpt host_mul(cpt a, cpt b) {
  auto m = [](uint32_t x, uint32_t y) {
    uint64_t p = (uint64_t)x * y;
    uint32_t r = ((uint32_t)p & VS_P) + (uint32_t)(p >> 31);
    return r >= VS_P ? r - VS_P : r;
  };
  auto ad = [](uint32_t x, uint32_t y) { uint32_t r = x + y; return r >= VS_P ? r - VS_P : r; };
  auto sb = [](uint32_t x, uint32_t y) { return x >= y ? x - y : x + VS_P - y; };
  return {sb(m(a.x, b.x), m(a.y, b.y)), ad(m(a.x, b.y), m(a.y, b.x))};
}
cpt host_repeated_double(cpt p, uint32_t k) {
  for (uint32_t i = 0; i < k; i++) p = host_mul(p, p);
  return p;
}
HostCoset host_coset(int which, uint32_t log_size) {
  const cpt G{2, 1268011823u};
  HostCoset c;
  c.log_size = log_size;
  c.step = host_repeated_double(G, 31 - log_size);
  if (which == COSET_HALF_COSET) c.initial = host_repeated_double(G, 30 - log_size);
  else if (which == COSET_HALF_ODDS) c.initial = host_repeated_double(G, log_size >= 29 ? 0 : 29 - log_size);
  else c.initial = {1, 0};
  return c;
}

int get_twiddles(int kind, uint32_t log_n, const TwiddleSet** out, cudaStream_t st) {
  int dev = 0;
  VS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(key(dev, kind, log_n));
  if (it != g_cache.end()) { *out = it->second; return VS_OK; }
  if (log_n < 2 || log_n > 30) return set_error(VS_ERR_INVALID, "twiddles: log_n %u out of range [2,30]", log_n);
  auto* t = new TwiddleSet();
  t->kind = kind;
  t->log_n = log_n;
  const uint32_t n = 1u << log_n;
  const unsigned th = 256;
  if (kind == TW_NATIVE) {
    HostCoset c = host_coset(COSET_HALF_COSET, log_n);
    // line, iline, circle, icircle; each table starts on a 16-byte boundary so
    // the NTT can fetch a thread's consecutive twiddles with 128-bit loads
    const size_t lp = ((size_t)(n - 1) + 3) & ~(size_t)3, cp = ((size_t)(n / 2) + 3) & ~(size_t)3;
    size_t words = 2 * lp + 2 * cp;
    if (cudaMalloc(&t->mem, words * 4) != cudaSuccess) { delete t; return set_error(VS_ERR_OOM, "twiddles: alloc"); }
    t->bytes = words * 4;
    t->line = t->mem;
    t->iline = t->line + lp;
    t->circle = t->iline + lp;
    t->icircle = t->circle + cp;
    native_line_kernel<<<blocks_for(n - 1, th), th, 0, st>>>(c.initial, c.step, log_n, t->line);
    native_circle_kernel<<<blocks_for(n / 2, th), th, 0, st>>>(c.initial, c.step, n / 2, t->circle);
    VS_LAUNCHED("native twiddles");
    VS_TRY(launch_batch_inverse(t->line, t->iline, n - 1, st));
    VS_TRY(launch_batch_inverse(t->circle, t->icircle, n / 2, st));
    uint32_t off = 0, sz = n / 2;
    for (uint32_t l = 0; l + 1 < log_n; l++) { t->offsets.push_back(off); t->sizes.push_back(sz); off += sz; sz >>= 1; }
  } else {
    HostCoset c = host_coset(COSET_HALF_ODDS, log_n - 1);
    if (cudaMalloc(&t->mem, (size_t)n * 4) != cudaSuccess) { delete t; return set_error(VS_ERR_OOM, "twiddles: alloc"); }
    t->bytes = (uint64_t)n * 4;
    t->line = t->mem;
    t->iline = t->mem + n / 2;
    stwo_table_kernel<<<blocks_for(n / 2, th), th, 0, st>>>(c.initial, c.step, log_n, t->line);
    VS_LAUNCHED("stwo twiddles");
    VS_TRY(launch_batch_inverse(t->line, t->iline, n / 2, st));
  }
  VS_CUDA(cudaStreamSynchronize(st));
  g_cache[key(dev, kind, log_n)] = t;
  *out = t;
  return VS_OK;
}

int get_fold_twiddles(int which, uint32_t log_n, const uint32_t** out, cudaStream_t st) {
  int dev = 0;
  VS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_mu);
  const int kind = 16 + which;  // fold twiddles share the cache under distinct kinds
  auto it = g_cache.find(key(dev, kind, log_n));
  if (it != g_cache.end()) { *out = it->second->line; return VS_OK; }
  if (log_n < 1 || log_n > 30) return set_error(VS_ERR_INVALID, "fold twiddles: log_n %u out of range", log_n);
  auto* t = new TwiddleSet();
  t->kind = kind;
  t->log_n = log_n;
  const uint32_t half = 1u << (log_n - 1);
  if (cudaMalloc(&t->mem, (size_t)half * 2 * 4) != cudaSuccess) { delete t; return set_error(VS_ERR_OOM, "fold twiddles: alloc"); }
  t->bytes = (uint64_t)half * 2 * 4;
  HostCoset c = host_coset(which == FOLD_CANONIC_CIRCLE ? COSET_HALF_COSET : which, log_n);
  // half_odds(L-1) has half_coset(L)'s initial point and twice its step; with the
  // L-bit reversal of 2i this gives half_odds(L-1).at(brev_{L-1}(i)).
  if (which == FOLD_CANONIC_CIRCLE) c.step = host_mul(c.step, c.step);
  uint32_t* src = t->mem + half;
  fold_sources_kernel<<<blocks_for(half, 256), 256, 0, st>>>(c.initial, c.step, src, half, log_n,
                                                             (which == COSET_HALF_COSET || which == FOLD_CANONIC_CIRCLE) ? 1 : 0);
  VS_LAUNCHED("fold_sources_kernel");
  t->line = t->mem;
  VS_TRY(launch_batch_inverse(src, t->line, half, st));
  VS_CUDA(cudaStreamSynchronize(st));
  g_cache[key(dev, kind, log_n)] = t;
  *out = t->line;
  return VS_OK;
}

uint64_t twiddle_bytes_if_missing(int device, int kind, uint32_t log_n) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_cache.count(key(device, kind, log_n))) return 0;
  const uint64_t n = 1ull << log_n;
  if (kind == TW_NATIVE) {
    const uint64_t lp = (n - 1 + 3) & ~3ull, cp = (n / 2 + 3) & ~3ull;
    return (2 * lp + 2 * cp) * 4;
  }
  return n * 4;  // stwo table pair, or fold twiddles with their sources
}

uint64_t twiddle_cache_bytes(int device) {
  std::lock_guard<std::mutex> lk(g_mu);
  uint64_t b = 0;
  for (auto& kv : g_cache)
    if ((int)(kv.first >> 40) == device) b += kv.second->bytes;
  return b;
}

int release_twiddles() {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& kv : g_cache) {
    cudaFree(kv.second->mem);
    delete kv.second;
  }
  g_cache.clear();
  return VS_OK;
}

}  // namespace vs

using namespace vs;

extern "C" {

void cuda_compute_coset_points(uint32_t ix, uint32_t iy, uint32_t sx, uint32_t sy, uint32_t* ox, uint32_t* oy,
                               uint32_t n) {
  launch_coset_points({ix, iy}, {sx, sy}, ox, oy, n, 0);
}

void cuda_extract_and_squash(const uint32_t* in, uint32_t* tw, uint32_t* sq, uint32_t half_n) {
  if (!half_n) return;
  extract_and_squash_kernel<<<blocks_for(half_n, 256), 256>>>(in, tw, sq, half_n);
  check_cuda(cudaGetLastError(), "cuda_extract_and_squash");
}

void cuda_squash_x(const uint32_t* in, uint32_t* out, uint32_t out_n) {
  if (!out_n) return;
  extract_and_squash_kernel<<<blocks_for(out_n, 256), 256>>>(in, nullptr, out, out_n);
  check_cuda(cudaGetLastError(), "cuda_squash_x");
}

void cuda_compute_fold_twiddle_sources_stream(uint32_t ix, uint32_t iy, uint32_t sx, uint32_t sy, uint32_t* out,
                                              uint32_t n, uint32_t log_n, int extract_y, vs_stream_t stream) {
  uint32_t half = n / 2;
  if (!half) return;
  fold_sources_kernel<<<blocks_for(half, 256), 256, 0, (cudaStream_t)stream>>>({ix, iy}, {sx, sy}, out, half, log_n,
                                                                              extract_y);
  check_cuda(cudaGetLastError(), "cuda_compute_fold_twiddle_sources");
}
void cuda_compute_fold_twiddle_sources(uint32_t ix, uint32_t iy, uint32_t sx, uint32_t sy, uint32_t* out, uint32_t n,
                                       uint32_t log_n, int extract_y) {
  cuda_compute_fold_twiddle_sources_stream(ix, iy, sx, sy, out, n, log_n, extract_y, 0);
}

void cuda_batch_inverse_m31_stream(const uint32_t* in, uint32_t* out, uint32_t n, vs_stream_t stream) {
  launch_batch_inverse(in, out, n, (cudaStream_t)stream);
}
void cuda_batch_inverse_m31(const uint32_t* in, uint32_t* out, uint32_t n) { launch_batch_inverse(in, out, n, 0); }

}  // extern "C"
