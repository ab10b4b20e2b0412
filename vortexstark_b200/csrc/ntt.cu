// Circle NTT for sm_100a, both reference conventions:
//  * native half_coset NTT (cuda/circle_ntt.cu, src/ntt.rs:145-243)
//  * stwo / CanonicCoset NTT (cuda/circle_ntt_stwo.cu, src/ntt.rs:249-341)
//
// Both share one butterfly network: layer j pairs (i0, i0 + 2^j) with
// i0 = h*2^(j+1) + l and twiddle t = tw_j[h]; forward (v0 + v1 t, v0 - v1 t) from
// the top layer down, inverse (v0 + v1, (v0 - v1) t) from layer 0 up, then a
// 2^((30 L) mod 31) scale. Only the twiddle lookup differs.
//
// Execution: a transform is split into passes over contiguous layer ranges
// [a, b]. A pass loads tiles of 2^(b-a+1) x 2^c elements (c low index bits kept
// for coalescing) into shared memory, runs its layers as register rounds of up
// to five layers (32 elements per thread, no barrier inside a round) and writes
// the tile back once. The shared tile uses an XOR swizzle (addr ^ ((addr>>5)&31))
// that keeps every round's access pattern bank-conflict free. A 2^24-point
// transform is two HBM round trips instead of the reference's 24 per-layer
// launches.
//
// The LDE path fuses interpolate -> zero-pad -> evaluate: the top pass of the
// inverse transform keeps the coefficients in registers and directly runs the
// forward top pass for each of the 2^B blowup blocks (the top B forward layers
// of a zero-padded input only replicate the coefficients), so neither the
// coefficients nor the zero padding touch HBM.
#include <vector>

#include "ntt.h"
#include "twiddles.h"
#include "vs_common.cuh"
#include "vs_field.cuh"

namespace vs {

__device__ __forceinline__ uint32_t swz(uint32_t a) { return a ^ ((a >> 5) & 31u); }

// Twiddle for layer j at group index h.
__device__ __forceinline__ uint32_t twiddle(const NttTw& tw, uint32_t j, uint32_t h) {
  if (j == 0 && tw.stwo) {  // circle_ntt_stwo.cu:202-248: [y, -y, -x, x] from pairs of line layer 0
    uint32_t x = __ldg(tw.flat + 2 * (h >> 2)), y = __ldg(tw.flat + 2 * (h >> 2) + 1);
    switch (h & 3) {
      case 0: return y;
      case 1: return neg(y);
      case 2: return neg(x);
      default: return x;
    }
  }
  return __ldg(tw.layer[j] + h);
}

template <bool FWD>
__device__ __forceinline__ void bfly(uint32_t& v0, uint32_t& v1, uint32_t t) {
  if (FWD) {
    uint32_t m = mul(v1, t);
    v1 = sub(v0, m);
    v0 = add(v0, m);
  } else {
    uint32_t s = v0;
    v0 = add(s, v1);
    v1 = mul(sub(s, v1), t);
  }
}

// Tile geometry for one pass.
struct Geo {
  uint32_t T;       // log2 tile elements
  uint32_t c;       // low bits kept contiguous
  uint32_t a, b;    // layer range
  uint32_t hi;      // tile's index bits above b
  uint32_t gbase;   // hi << (b+1) | lo_chunk << c
  __device__ __forceinline__ uint32_t gidx(uint32_t e) const {
    return gbase | ((e >> c) << a) | (e & ((1u << c) - 1));
  }
};

// Element address k (R bits) of subgroup `o` inserted at bit p0.
__device__ __forceinline__ uint32_t ins(uint32_t o, uint32_t k, uint32_t p0, uint32_t R) {
  return ((o >> p0) << (p0 + R)) | (k << p0) | (o & ((1u << p0) - 1));
}

// Butterflies of one register round: R layers at tile bits [p0, p0+R).
// v holds SUB = 2^(5-R) subgroups of 2^R elements.
template <int R, bool FWD>
__device__ __forceinline__ void round_regs(uint32_t (&v)[32], const Geo& g, uint32_t p0, const NttTw& tw) {
  constexpr int SUB = 1 << (5 - R), K = 1 << R;
  const uint32_t nthr = 1u << (g.T - 5);
#pragma unroll
  for (int s = 0; s < SUB; s++) {
    const uint32_t o = threadIdx.x + s * nthr;
    const uint32_t base = ins(o, 0, p0, R);
#pragma unroll
    for (int qq = 0; qq < R; qq++) {
      const int q = FWD ? R - 1 - qq : qq;
      const uint32_t p = p0 + q;                 // tile bit of this layer
      const uint32_t j = g.a + p - g.c;          // global layer index
      const uint32_t hbase = (g.hi << (g.b - j)) | (base >> (p + 1));
#pragma unroll
      for (int gg = 0; gg < (K >> (q + 1)); gg++) {
        const uint32_t t = twiddle(tw, j, hbase | gg);
#pragma unroll
        for (int l = 0; l < (1 << q); l++) {
          const int k0 = (gg << (q + 1)) | l;
          bfly<FWD>(v[s * K + k0], v[s * K + k0 + (1 << q)], t);
        }
      }
    }
  }
}

template <int R>
__device__ __forceinline__ void load_round(uint32_t (&v)[32], const uint32_t* sm, const Geo& g, uint32_t p0) {
  constexpr int SUB = 1 << (5 - R), K = 1 << R;
  const uint32_t nthr = 1u << (g.T - 5);
#pragma unroll
  for (int s = 0; s < SUB; s++) {
    const uint32_t o = threadIdx.x + s * nthr;
#pragma unroll
    for (int k = 0; k < K; k++) v[s * K + k] = sm[swz(ins(o, k, p0, R))];
  }
}
template <int R>
__device__ __forceinline__ void store_round(const uint32_t (&v)[32], uint32_t* sm, const Geo& g, uint32_t p0) {
  constexpr int SUB = 1 << (5 - R), K = 1 << R;
  const uint32_t nthr = 1u << (g.T - 5);
#pragma unroll
  for (int s = 0; s < SUB; s++) {
    const uint32_t o = threadIdx.x + s * nthr;
#pragma unroll
    for (int k = 0; k < K; k++) sm[swz(ins(o, k, p0, R))] = v[s * K + k];
  }
}

template <bool FWD>
__device__ __forceinline__ void round_any(uint32_t (&v)[32], const Geo& g, uint32_t p0, uint32_t R, const NttTw& tw) {
  switch (R) {
    case 1: round_regs<1, FWD>(v, g, p0, tw); break;
    case 2: round_regs<2, FWD>(v, g, p0, tw); break;
    case 3: round_regs<3, FWD>(v, g, p0, tw); break;
    case 4: round_regs<4, FWD>(v, g, p0, tw); break;
    default: round_regs<5, FWD>(v, g, p0, tw); break;
  }
}
__device__ __forceinline__ void load_any(uint32_t (&v)[32], const uint32_t* sm, const Geo& g, uint32_t p0, uint32_t R) {
  switch (R) {
    case 1: load_round<1>(v, sm, g, p0); break;
    case 2: load_round<2>(v, sm, g, p0); break;
    case 3: load_round<3>(v, sm, g, p0); break;
    case 4: load_round<4>(v, sm, g, p0); break;
    default: load_round<5>(v, sm, g, p0); break;
  }
}
__device__ __forceinline__ void store_any(const uint32_t (&v)[32], uint32_t* sm, const Geo& g, uint32_t p0, uint32_t R) {
  switch (R) {
    case 1: store_round<1>(v, sm, g, p0); break;
    case 2: store_round<2>(v, sm, g, p0); break;
    case 3: store_round<3>(v, sm, g, p0); break;
    case 4: store_round<4>(v, sm, g, p0); break;
    default: store_round<5>(v, sm, g, p0); break;
  }
}

// Rounds: full five-layer rounds from tile bit c upward, the remainder (< 5) on top.
__device__ __forceinline__ uint32_t n_rounds(uint32_t m) { return (m + 4) / 5; }
__device__ __forceinline__ void round_span(uint32_t m, uint32_t c, uint32_t r, uint32_t& p0, uint32_t& R) {
  p0 = c + 5 * r;
  R = (5 * (r + 1) <= m) ? 5 : m - 5 * r;
}

__device__ __forceinline__ const uint32_t* col_src(const NttPass& p) {
  return p.src_cols ? p.src_cols[blockIdx.y] : p.src + (uint64_t)blockIdx.y * p.src_stride;
}
__device__ __forceinline__ uint32_t* col_dst(const NttPass& p) {
  return p.dst_cols ? p.dst_cols[blockIdx.y] : p.dst + (uint64_t)blockIdx.y * p.dst_stride;
}

__device__ __forceinline__ Geo make_geo(const NttPass& p, uint32_t tile) {
  Geo g;
  g.a = p.a;
  g.b = p.b;
  g.c = p.c;
  g.T = p.b - p.a + 1 + p.c;
  const uint32_t lo_bits = p.a - p.c;
  const uint32_t lo_chunk = tile & ((1u << lo_bits) - 1);
  g.hi = tile >> lo_bits;
  g.gbase = (g.b + 1 >= 32 ? 0u : (g.hi << (g.b + 1))) | (lo_chunk << p.c);
  return g;
}

template <bool FWD>
__global__ void __launch_bounds__(512) ntt_pass_kernel(NttPass p) {
  extern __shared__ uint32_t sm[];
  const Geo g = make_geo(p, blockIdx.x);
  const uint32_t* src = col_src(p);
  uint32_t* dst = col_dst(p);
  const uint32_t size = 1u << g.T, m = g.b - g.a + 1;
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) sm[swz(e)] = src[g.gidx(e) & p.src_mask];
  __syncthreads();
  uint32_t v[32];
  const uint32_t nr = n_rounds(m);
  for (uint32_t rr = 0; rr < nr; rr++) {
    const uint32_t r = FWD ? nr - 1 - rr : rr;
    uint32_t p0, R;
    round_span(m, g.c, r, p0, R);
    load_any(v, sm, g, p0, R);
    round_any<FWD>(v, g, p0, R, p.tw);
    if (!FWD && rr == nr - 1 && p.scale) {
#pragma unroll
      for (int k = 0; k < 32; k++) v[k] = mul(v[k], p.scale);
    }
    store_any(v, sm, g, p0, R);  // each element is loaded and stored by the same thread within a round
    __syncthreads();
  }
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) dst[g.gidx(e)] = sm[swz(e)];
}

// Fused LDE top pass. Inverse layers [a, l-1] of the trace-domain tile (with the
// 1/n scale), then for each blowup block q the forward layers [a, l-1] of the
// evaluation domain on a copy of the coefficients, written to dst block q.
// `inv` describes the trace-domain pass (src = partially interpolated trace or
// raw input), `fwd` the evaluation-domain pass (dst, log_n = l + B). Block q's
// tile has hi = q. If coeff_out != nullptr the coefficients are also stored.
__global__ void __launch_bounds__(512) ntt_lde_top_kernel(NttPass inv, NttPass fwd, uint32_t B, uint32_t* coeff_out,
                                                         uint64_t coeff_stride) {
  extern __shared__ uint32_t sm[];
  const Geo gi = make_geo(inv, blockIdx.x);
  const uint32_t* src = col_src(inv);
  uint32_t* dst = col_dst(fwd);
  const uint32_t size = 1u << gi.T, m = gi.b - gi.a + 1;
  for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) sm[swz(e)] = src[gi.gidx(e) & inv.src_mask];
  __syncthreads();
  uint32_t v[32], coef[32];
  const uint32_t nr = n_rounds(m);
  uint32_t p0t, Rt;
  round_span(m, gi.c, nr - 1, p0t, Rt);
  for (uint32_t r = 0; r < nr; r++) {
    uint32_t p0, R;
    round_span(m, gi.c, r, p0, R);
    load_any(v, sm, gi, p0, R);
    round_any<false>(v, gi, p0, R, inv.tw);
    if (r + 1 < nr) {
      store_any(v, sm, gi, p0, R);
      __syncthreads();
    }
  }
#pragma unroll
  for (int k = 0; k < 32; k++) coef[k] = mul(v[k], inv.scale);
  if (coeff_out) {
    __syncthreads();
    store_any(coef, sm, gi, p0t, Rt);
    __syncthreads();
    uint32_t* co = coeff_out + (uint64_t)blockIdx.y * coeff_stride;
    for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) co[gi.gidx(e)] = sm[swz(e)];
  }
  for (uint32_t q = 0; q < (1u << B); q++) {
    Geo gf = gi;
    gf.hi = q;
    gf.gbase = (q << (gi.b + 1)) | (gi.gbase & ((1u << (gi.b + 1)) - 1));
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = coef[k];
    round_any<true>(v, gf, p0t, Rt, fwd.tw);
    __syncthreads();
    store_any(v, sm, gf, p0t, Rt);
    __syncthreads();
    for (int r = (int)nr - 2; r >= 0; r--) {
      uint32_t p0, R;
      round_span(m, gi.c, r, p0, R);
      load_any(v, sm, gf, p0, R);
      round_any<true>(v, gf, p0, R, fwd.tw);
      store_any(v, sm, gf, p0, R);
      __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) dst[gf.gidx(e)] = sm[swz(e)];
  }
}

// Single layer (cuda_circle_ntt_layer, and transforms below 32 points).
template <bool FWD>
__global__ void ntt_layer_kernel(uint32_t* __restrict__ d, NttTw tw, uint32_t j, uint32_t half_n) {
  uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= half_n) return;
  uint32_t h = tid >> j, l = tid & ((1u << j) - 1);
  uint32_t i0 = (h << (j + 1)) + l, i1 = i0 + (1u << j);
  uint32_t v0 = d[i0], v1 = d[i1];
  bfly<FWD>(v0, v1, twiddle(tw, j, h));
  d[i0] = v0;
  d[i1] = v1;
}
__global__ void scale_kernel(uint32_t* __restrict__ d, uint32_t s, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = mul(d[i], s);
}

// ------------------------------------------------------------------ host side
static const uint32_t kMaxT = 13;  // tile of 8192 words (32 KiB), 256 threads
static const uint32_t kMinC = 2;   // >= 16-byte contiguous runs per tile row

std::vector<PassRange> plan_passes(uint32_t L) {
  std::vector<PassRange> v;
  if (L <= kMaxT) { v.push_back({0, L - 1, 0}); return v; }
  uint32_t lo = kMaxT;
  v.push_back({0, lo - 1, 0});
  uint32_t rem = L - lo, max_u = kMaxT - kMinC;
  uint32_t k = (rem + max_u - 1) / max_u;
  uint32_t a = lo;
  for (uint32_t i = 0; i < k; i++) {
    uint32_t u = rem / k + (i < rem % k ? 1 : 0);
    uint32_t c = kMaxT - u;
    if (c > a) c = a;
    v.push_back({a, a + u - 1, c});
    a += u;
  }
  return v;
}

uint32_t inv_n_scale(uint32_t log_n) {
  uint32_t e = (30u * log_n) % 31u;
  return e == 0 ? 1u : (1u << e);
}

static int set_smem(const void* fn, uint32_t bytes) {
  if (bytes > 48 * 1024) VS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return VS_OK;
}

static int launch_pass(NttPass p, bool fwd, uint32_t n_cols, cudaStream_t st) {
  const uint32_t T = p.b - p.a + 1 + p.c;
  const uint32_t tiles = 1u << (p.log_n - T);
  const uint32_t threads = 1u << (T - 5), smem = 4u << T;
  dim3 grid(tiles, n_cols);
  if (fwd) {
    VS_TRY(set_smem((const void*)ntt_pass_kernel<true>, smem));
    ntt_pass_kernel<true><<<grid, threads, smem, st>>>(p);
  } else {
    VS_TRY(set_smem((const void*)ntt_pass_kernel<false>, smem));
    ntt_pass_kernel<false><<<grid, threads, smem, st>>>(p);
  }
  VS_LAUNCHED("ntt_pass_kernel");
  return VS_OK;
}

// Small transforms (< 32 points): one launch per layer.
static int small_transform(uint32_t* d, uint32_t L, const NttTw& tw, bool fwd, uint32_t scale, cudaStream_t st) {
  const uint32_t half = 1u << (L - 1);
  if (fwd) {
    for (int j = (int)L - 1; j >= 0; j--) ntt_layer_kernel<true><<<1, 32, 0, st>>>(d, tw, (uint32_t)j, half);
  } else {
    for (uint32_t j = 0; j < L; j++) ntt_layer_kernel<false><<<1, 32, 0, st>>>(d, tw, j, half);
    if (scale) scale_kernel<<<1, 32, 0, st>>>(d, scale, 2 * half);
  }
  VS_LAUNCHED("ntt small transform");
  return VS_OK;
}

int ntt_transform(const NttColumns& io, uint32_t L, const NttTw& tw, bool fwd, cudaStream_t st) {
  if (L == 0) return VS_OK;
  if (L < 5) {
    for (uint32_t c = 0; c < io.n_cols; c++) {
      if (io.src_cols || io.dst_cols) return set_error(VS_ERR_INVALID, "small NTT with pointer arrays unsupported");
      uint32_t* d = io.dst + c * io.dst_stride;
      if (io.src != d) VS_CUDA(cudaMemcpyAsync(d, io.src + c * io.src_stride, 4u << L, cudaMemcpyDeviceToDevice, st));
      VS_TRY(small_transform(d, L, tw, fwd, fwd ? 0 : inv_n_scale(L), st));
    }
    return VS_OK;
  }
  auto passes = plan_passes(L);
  const size_t np = passes.size();
  for (size_t i = 0; i < np; i++) {
    const PassRange& r = fwd ? passes[np - 1 - i] : passes[i];
    NttPass p{};
    p.tw = tw;
    p.log_n = L;
    p.a = r.a;
    p.b = r.b;
    p.c = r.c;
    p.src_mask = 0xFFFFFFFFu;
    bool first = i == 0;
    p.src = first ? io.src : io.dst;
    p.src_cols = first ? io.src_cols : io.dst_cols;
    p.src_stride = first ? io.src_stride : io.dst_stride;
    p.dst = io.dst;
    p.dst_cols = io.dst_cols;
    p.dst_stride = io.dst_stride;
    p.scale = (!fwd && i == np - 1) ? inv_n_scale(L) : 0;
    VS_TRY(launch_pass(p, fwd, io.n_cols, st));
  }
  return VS_OK;
}

int ntt_lde(const NttColumns& io, uint32_t l, uint32_t B, const NttTw& tw_inv, const NttTw& tw_fwd,
            uint32_t* coeff_out, uint64_t coeff_stride, cudaStream_t st) {
  if (l < 5) return set_error(VS_ERR_INVALID, "LDE needs log_n >= 5 (got %u)", l);
  if (io.src_cols || io.dst_cols) return set_error(VS_ERR_INVALID, "LDE takes strided columns");
  auto passes = plan_passes(l);
  const size_t np = passes.size();
  // 1. inverse passes below the top one: src -> dst[0, n)
  for (size_t i = 0; i + 1 < np; i++) {
    NttPass p{};
    p.tw = tw_inv;
    p.log_n = l;
    p.a = passes[i].a;
    p.b = passes[i].b;
    p.c = passes[i].c;
    p.src_mask = 0xFFFFFFFFu;
    p.src = i == 0 ? io.src : io.dst;
    p.src_stride = i == 0 ? io.src_stride : io.dst_stride;
    p.dst = io.dst;
    p.dst_stride = io.dst_stride;
    VS_TRY(launch_pass(p, false, io.n_cols, st));
  }
  // 2. fused top pass
  {
    const PassRange& r = passes[np - 1];
    NttPass pi{}, pf{};
    pi.tw = tw_inv;
    pi.log_n = l;
    pi.a = r.a;
    pi.b = r.b;
    pi.c = r.c;
    pi.src_mask = 0xFFFFFFFFu;
    pi.src = np == 1 ? io.src : io.dst;
    pi.src_stride = np == 1 ? io.src_stride : io.dst_stride;
    pi.scale = inv_n_scale(l);
    pf = pi;
    pf.tw = tw_fwd;
    pf.log_n = l + B;
    pf.dst = io.dst;
    pf.dst_stride = io.dst_stride;
    const uint32_t T = r.b - r.a + 1 + r.c;
    const uint32_t tiles = 1u << (l - T), threads = 1u << (T - 5), smem = 4u << T;
    VS_TRY(set_smem((const void*)ntt_lde_top_kernel, smem));
    ntt_lde_top_kernel<<<dim3(tiles, io.n_cols), threads, smem, st>>>(pi, pf, B, coeff_out, coeff_stride);
    VS_LAUNCHED("ntt_lde_top_kernel");
  }
  // 3. forward passes below the top one over the whole evaluation domain
  for (int i = (int)np - 2; i >= 0; i--) {
    NttPass p{};
    p.tw = tw_fwd;
    p.log_n = l + B;
    p.a = passes[i].a;
    p.b = passes[i].b;
    p.c = passes[i].c;
    p.src_mask = 0xFFFFFFFFu;
    p.src = io.dst;
    p.src_stride = io.dst_stride;
    p.dst = io.dst;
    p.dst_stride = io.dst_stride;
    VS_TRY(launch_pass(p, true, io.n_cols, st));
  }
  return VS_OK;
}

NttTw native_tw(const uint32_t* line, const uint32_t* circle, const uint32_t* offsets, uint32_t n_line_layers) {
  NttTw tw{};
  tw.stwo = 0;
  tw.layer[0] = circle;
  for (uint32_t j = 1; j <= n_line_layers && j < 32; j++) tw.layer[j] = line + offsets[j - 1];
  return tw;
}
NttTw stwo_tw(const uint32_t* flat, uint32_t L) {
  NttTw tw{};
  tw.stwo = 1;
  tw.flat = flat;
  const uint32_t half = 1u << (L - 1);
  for (uint32_t j = 1; j < L && j < 32; j++) tw.layer[j] = flat + (half - (1u << (L - j)));
  return tw;
}

int tw_for(int kind, uint32_t L, bool forward, NttTw* out, cudaStream_t st) {
  const TwiddleSet* t = nullptr;
  VS_TRY(get_twiddles(kind, L, &t, st));
  if (kind == TW_NATIVE) *out = native_tw(forward ? t->line : t->iline, forward ? t->circle : t->icircle,
                                          t->offsets.data(), L - 1);
  else *out = stwo_tw(forward ? t->line : t->iline, L);
  return VS_OK;
}

int lde_cached(int kind, const uint32_t* src, uint64_t src_stride, uint32_t* dst, uint64_t dst_stride,
               uint32_t n_cols, uint32_t l, uint32_t B, cudaStream_t st) {
  if (!src || !dst || n_cols == 0) return set_error(VS_ERR_INVALID, "lde: null argument");
  if (l < 2 || l + B > 30) return set_error(VS_ERR_INVALID, "lde: log_n %u + blowup %u out of range", l, B);
  NttTw ti, tf;
  VS_TRY(tw_for(kind, l, false, &ti, st));
  VS_TRY(tw_for(kind, l + B, true, &tf, st));
  if (l < 5) {  // tiny: interpolate in place in dst, zero the padding, evaluate
    const uint64_t n = 1ull << l, N = n << B;
    for (uint32_t c = 0; c < n_cols; c++) {
      uint32_t* d = dst + c * dst_stride;
      VS_CUDA(cudaMemcpyAsync(d, src + c * src_stride, n * 4, cudaMemcpyDeviceToDevice, st));
      VS_CUDA(cudaMemsetAsync(d + n, 0, (N - n) * 4, st));
      NttColumns a{d, d, nullptr, nullptr, 0, 0, 1};
      VS_TRY(ntt_transform(a, l, ti, false, st));
      VS_TRY(ntt_transform(a, l + B, tf, true, st));
    }
    return VS_OK;
  }
  NttColumns io{src, dst, nullptr, nullptr, src_stride, dst_stride, n_cols};
  return ntt_lde(io, l, B, ti, tf, nullptr, 0, st);
}

// ------------------------------------------------------------------ bit reversal
__global__ void bit_reverse_m31_kernel(uint32_t* d, uint32_t log_n, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t j = brev(i, log_n);
  if (i < j) {
    uint32_t t = d[i];
    d[i] = d[j];
    d[j] = t;
  }
}
__global__ void bit_reverse_qm31_kernel(const uint4* __restrict__ in, uint4* __restrict__ out, uint32_t n,
                                        uint32_t log_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[brev(i, log_n)] = in[i];
}

// ------------------------------------------------------------------ eval at point (circle_ntt.cu:119-164)
__global__ void fold_first_kernel(const uint32_t* __restrict__ c, uint32_t* __restrict__ out,
                                  const uint32_t* __restrict__ f, uint32_t half_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  qm31 fq{{f[0], f[1], f[2], f[3]}};
  qm31 bf = qscale(fq, c[i + half_n]);
  out[4 * i + 0] = add(c[i], bf.v[0]);
  out[4 * i + 1] = bf.v[1];
  out[4 * i + 2] = bf.v[2];
  out[4 * i + 3] = bf.v[3];
}
__global__ void fold_level_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                  const uint32_t* __restrict__ f, uint32_t half_n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= half_n) return;
  qm31 a{{in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]}};
  uint32_t j = 4 * (i + half_n);
  qm31 b{{in[j], in[j + 1], in[j + 2], in[j + 3]}};
  qm31 fq{{f[0], f[1], f[2], f[3]}};
  qm31 r = qadd(a, qmul(b, fq));
  out[4 * i + 0] = r.v[0];
  out[4 * i + 1] = r.v[1];
  out[4 * i + 2] = r.v[2];
  out[4 * i + 3] = r.v[3];
}

}  // namespace vs

using namespace vs;

extern "C" {

void cuda_circle_ntt_evaluate(uint32_t* d, const uint32_t* tw, const uint32_t* ctw, const uint32_t* h_off,
                              const uint32_t* /*h_sizes*/, uint32_t n_line, uint32_t n) {
  uint32_t L = ilog2(n);
  NttColumns io{d, d, nullptr, nullptr, 0, 0, 1};
  ntt_transform(io, L, native_tw(tw, ctw, h_off, n_line), true, 0);
  check_cuda(cudaDeviceSynchronize(), "cuda_circle_ntt_evaluate");
}
void cuda_circle_ntt_interpolate(uint32_t* d, const uint32_t* itw, const uint32_t* ictw, const uint32_t* h_off,
                                 const uint32_t* /*h_sizes*/, uint32_t n_line, uint32_t n) {
  uint32_t L = ilog2(n);
  NttColumns io{d, d, nullptr, nullptr, 0, 0, 1};
  ntt_transform(io, L, native_tw(itw, ictw, h_off, n_line), false, 0);
  check_cuda(cudaDeviceSynchronize(), "cuda_circle_ntt_interpolate");
}
static void batch_ntt(uint32_t** cols, const uint32_t* tw, const uint32_t* ctw, const uint32_t* h_off, uint32_t n_line,
                      uint32_t n, uint32_t n_cols, bool fwd) {
  if (!n_cols) return;
  uint32_t L = ilog2(n);
  NttTw t = native_tw(tw, ctw, h_off, n_line);
  if (L < 5) {  // tiny: per column through a host copy of the pointer table
    std::vector<uint32_t*> h(n_cols);
    if (check_cuda(cudaMemcpy(h.data(), cols, n_cols * sizeof(void*), cudaMemcpyDeviceToHost), "batch ntt") != VS_OK) return;
    for (uint32_t c = 0; c < n_cols; c++) {
      NttColumns io{h[c], h[c], nullptr, nullptr, 0, 0, 1};
      ntt_transform(io, L, t, fwd, 0);
    }
  } else {
    NttColumns io{nullptr, nullptr, (const uint32_t* const*)cols, cols, 0, 0, n_cols};
    ntt_transform(io, L, t, fwd, 0);
  }
  check_cuda(cudaDeviceSynchronize(), "cuda_circle_ntt_*_batch");
}
void cuda_circle_ntt_evaluate_batch(uint32_t** cols, const uint32_t* tw, const uint32_t* ctw, const uint32_t* h_off,
                                    const uint32_t* /*h_sizes*/, uint32_t n_line, uint32_t n, uint32_t n_cols) {
  batch_ntt(cols, tw, ctw, h_off, n_line, n, n_cols, true);
}
void cuda_circle_ntt_interpolate_batch(uint32_t** cols, const uint32_t* itw, const uint32_t* ictw,
                                       const uint32_t* h_off, const uint32_t* /*h_sizes*/, uint32_t n_line,
                                       uint32_t n, uint32_t n_cols) {
  batch_ntt(cols, itw, ictw, h_off, n_line, n, n_cols, false);
}
void cuda_circle_ntt_layer(uint32_t* d, const uint32_t* tw, uint32_t layer_idx, uint32_t n, int forward) {
  NttTw t{};
  t.layer[layer_idx] = tw;
  uint32_t half = n / 2;
  if (!half) return;
  if (forward) ntt_layer_kernel<true><<<blocks_for(half, 256), 256>>>(d, t, layer_idx, half);
  else ntt_layer_kernel<false><<<blocks_for(half, 256), 256>>>(d, t, layer_idx, half);
  check_cuda(cudaGetLastError(), "cuda_circle_ntt_layer");
}
void cuda_bit_reverse_m31(uint32_t* d, uint32_t log_n) {
  uint32_t n = 1u << log_n;
  bit_reverse_m31_kernel<<<blocks_for(n, 256), 256>>>(d, log_n, n);
  check_cuda(cudaGetLastError(), "cuda_bit_reverse_m31");
}
void cuda_bit_reverse_qm31(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t log_n) {
  if (!n) return;
  bit_reverse_qm31_kernel<<<blocks_for(n, 256), 256>>>((const uint4*)in, (uint4*)out, n, log_n);
  check_cuda(cudaGetLastError(), "cuda_bit_reverse_qm31");
}
void cuda_stwo_ntt_evaluate(uint32_t* d, const uint32_t* tw, uint32_t n) {
  uint32_t L = ilog2(n);
  NttColumns io{d, d, nullptr, nullptr, 0, 0, 1};
  ntt_transform(io, L, stwo_tw(tw, L), true, 0);
  check_cuda(cudaDeviceSynchronize(), "cuda_stwo_ntt_evaluate");
}
void cuda_stwo_ntt_interpolate(uint32_t* d, const uint32_t* itw, uint32_t n) {
  uint32_t L = ilog2(n);
  NttColumns io{d, d, nullptr, nullptr, 0, 0, 1};
  ntt_transform(io, L, stwo_tw(itw, L), false, 0);
  check_cuda(cudaDeviceSynchronize(), "cuda_stwo_ntt_interpolate");
}
void cuda_eval_at_point(const uint32_t* coeffs, const uint32_t* factors, uint32_t* h_result, uint32_t n,
                        uint32_t* s1, uint32_t* s2) {
  uint32_t log_n = ilog2(n);
  uint32_t half = n / 2;
  fold_first_kernel<<<blocks_for(half, 256), 256>>>(coeffs, s1, factors, half);
  uint32_t *in = s1, *out = s2, cur = half;
  for (uint32_t lvl = 1; lvl < log_n; lvl++) {
    half = cur / 2;
    fold_level_kernel<<<blocks_for(half, 256), 256>>>(in, out, factors + 4 * lvl, half);
    uint32_t* t = in;
    in = out;
    out = t;
    cur = half;
  }
  check_cuda(cudaMemcpy(h_result, in, 16, cudaMemcpyDeviceToHost), "cuda_eval_at_point");
}

int vs_lde_stwo(const uint32_t* src, uint64_t src_stride, uint32_t* dst, uint64_t dst_stride, uint32_t n_cols,
                uint32_t log_n, uint32_t blowup, vs_stream_t st) {
  clear_error();
  return lde_cached(TW_STWO, src, src_stride, dst, dst_stride, n_cols, log_n, blowup, (cudaStream_t)st);
}
int vs_lde_native(const uint32_t* src, uint64_t src_stride, uint32_t* dst, uint64_t dst_stride, uint32_t n_cols,
                  uint32_t log_n, uint32_t blowup, vs_stream_t st) {
  clear_error();
  return lde_cached(TW_NATIVE, src, src_stride, dst, dst_stride, n_cols, log_n, blowup, (cudaStream_t)st);
}

}  // extern "C"
