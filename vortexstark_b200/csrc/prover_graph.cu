// Device-resident Fibonacci prover captured as one CUDA graph per trace size.
//
// Same arithmetic and transcript as prove_fib (prover.cu), restructured so no
// stage needs the host: the Fiat-Shamir channel runs on the device (one thread,
// channel_dev.cuh), fold challenges are read by the fused leaf functors from
// device memory, query indices are drawn on the device, and decommitment
// (values + authentication paths, one CTA per query recomputing its 1024-leaf
// tile) writes straight into a proof arena that is copied to pinned host memory
// once. A proof is therefore a single graph launch; the host only writes (a, b)
// and serialises the arena (KRAK v1, src/bin/stark_cli.rs:907-976).
//
// Slots: each GraphProver owns its buffers, stream and graph, so several slots
// prove concurrently (the batched and served paths).
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "channel_dev.cuh"
#include "fri_impl.cuh"
#include "merkle.h"
#include "ntt.h"
#include "prover.h"
#include "prover_graph.h"
#include "twiddles.h"
#include "vs_common.cuh"

namespace vs {

constexpr int MAXF = 28;  // FRI layers for log_eval <= 31

// ------------------------------------------------------------------ leaf functors with device-resident challenges
struct LeafFibQuotD {
  const uint32_t* e;
  uint64_t mask;
  const uint32_t* alpha;  // device QM31
  __device__ __forceinline__ qm31 q(uint64_t i) const {
    const qm31 a{{__ldg(alpha), __ldg(alpha + 1), __ldg(alpha + 2), __ldg(alpha + 3)}};
    return qscale(a, sub(e[(i + 2) & mask], add(e[(i + 1) & mask], e[i])));
  }
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    const qm31 r = q(i);
    uint32_t m[16] = {0};
    m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};
struct LeafFoldQuotD {
  LeafFibQuotD quot;
  const uint32_t* tw;
  const uint32_t* alpha;
  uint32_t* dst[4];
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    const qm31 a{{__ldg(alpha), __ldg(alpha + 1), __ldg(alpha + 2), __ldg(alpha + 3)}};
    const qm31 r = fold_pair(quot.q(2 * i), quot.q(2 * i + 1), a, __ldg(tw + i));
#pragma unroll
    for (int k = 0; k < 4; k++) dst[k][i] = r.v[k];
    uint32_t m[16] = {0};
    m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};
struct LeafFoldD {
  const uint32_t* src[4];
  uint32_t* dst[4];
  const uint32_t* tw;
  const uint32_t* alpha;
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    const qm31 a{{__ldg(alpha), __ldg(alpha + 1), __ldg(alpha + 2), __ldg(alpha + 3)}};
    const uint2 s0 = *reinterpret_cast<const uint2*>(src[0] + 2 * i);
    const uint2 s1 = *reinterpret_cast<const uint2*>(src[1] + 2 * i);
    const uint2 s2 = *reinterpret_cast<const uint2*>(src[2] + 2 * i);
    const uint2 s3 = *reinterpret_cast<const uint2*>(src[3] + 2 * i);
    const qm31 r = fold_pair(qm31{{s0.x, s1.x, s2.x, s3.x}}, qm31{{s0.y, s1.y, s2.y, s3.y}}, a, __ldg(tw + i));
#pragma unroll
    for (int k = 0; k < 4; k++) dst[k][i] = r.v[k];
    uint32_t m[16] = {0};
    m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};

// ------------------------------------------------------------------ device stages
__global__ void fib_trace_params_kernel(const uint32_t* __restrict__ ab, uint32_t* __restrict__ out, uint64_t n) {
  __shared__ uint32_t sm[256 * 33];
  const uint32_t a = ab[2 * blockIdx.y], b = ab[2 * blockIdx.y + 1];
  out += (uint64_t)blockIdx.y * n;
  const uint64_t base = (uint64_t)blockIdx.x * 256 * 32;
  const uint64_t s = base + (uint64_t)threadIdx.x * 32;
  uint32_t m00 = 1, m01 = 0, m11 = 1, b00 = 1, b01 = 1, b11 = 0;
  for (uint64_t e = s; e; e >>= 1) {
    if (e & 1) {
      const uint32_t t00 = add(mul(m00, b00), mul(m01, b01)), t01 = add(mul(m00, b01), mul(m01, b11));
      const uint32_t t11 = add(mul(m01, b01), mul(m11, b11));
      m00 = t00; m01 = t01; m11 = t11;
    }
    const uint32_t t00 = add(mul(b00, b00), mul(b01, b01)), t01 = add(mul(b00, b01), mul(b01, b11));
    const uint32_t t11 = add(mul(b01, b01), mul(b11, b11));
    b00 = t00; b01 = t01; b11 = t11;
  }
  uint32_t t0 = add(mul(a, m11), mul(b, m01)), t1 = add(mul(a, m01), mul(b, m00));
  uint32_t* row = sm + threadIdx.x * 33;
  row[0] = t0;
  row[1] = t1;
#pragma unroll
  for (int i = 2; i < 32; i++) { const uint32_t t2 = add(t0, t1); row[i] = t2; t0 = t1; t1 = t2; }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < 256 * 32; e += 256) {
    const uint64_t g = base + e;
    if (g < n) out[g] = sm[(e / 32) * 33 + e % 32];
  }
}

// mix a root (copying it into the proof arena) and optionally draw a challenge.
__global__ void ch_mix_draw_kernel(ChanDev* c, int reset, const uint32_t* __restrict__ root, uint32_t* arena_root,
                                   uint32_t* alpha_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  ChanDev ch = *c;
  if (reset) {
    for (int i = 0; i < 8; i++) ch.state[i] = 0;
    ch.n_draws = 0;
    ch.error = 0;
  }
  uint32_t r[8];
  for (int i = 0; i < 8; i++) { r[i] = root[i]; arena_root[i] = r[i]; }
  ch_mix_digest(ch, r);
  if (alpha_out) {
    uint32_t a[4];
    ch_draw_felt(ch, a);
    for (int i = 0; i < 4; i++) alpha_out[i] = a[i];
  }
  *c = ch;
}

// mix_felts(last layer) then the query indices (draw_number(eval_size) x N_QUERIES).
__global__ void ch_queries_kernel(ChanDev* c, const uint32_t* l0, const uint32_t* l1, const uint32_t* l2,
                                  const uint32_t* l3, uint32_t* arena_last, uint32_t* qidx, uint32_t* arena_q,
                                  uint32_t log_eval) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  ChanDev ch = *c;
  const uint32_t* planes[4] = {l0, l1, l2, l3};
  for (int i = 0; i < 8; i++)
    for (int k = 0; k < 4; k++) arena_last[4 * i + k] = planes[k][i];
  ch_mix_felts_planes(ch, planes, 8);
  for (uint32_t q = 0; q < N_QUERIES; q++) {
    const uint32_t v = ch_draw_pow2(ch, log_eval);
    qidx[q] = v;
    arena_q[q] = v;
  }
  *c = ch;
}

struct DecParams {
  const uint32_t* eval;
  uint32_t mask;
  const uint32_t* alpha;
  const uint32_t* qidx;
  uint32_t* trace_vals;  // 2 x 80
  uint32_t* quot_vals;   // 2 x 80 x 4
  uint32_t nf;
  const uint32_t* fri[MAXF][4];
  uint32_t* fri_vals;    // nf x 2 x 80 x 4
};
// Values at each query and its fold sibling (q ^ 1); FRI layer l uses q >> (l+1).
__global__ void decommit_values_kernel(DecParams p) {
  const uint32_t t = threadIdx.x;  // 0..159
  if (t >= 2 * N_QUERIES) return;
  const uint32_t qi = t % N_QUERIES;
  const uint32_t i = p.qidx[qi] ^ (t >= N_QUERIES ? 1u : 0u);
  p.trace_vals[t] = p.eval[i];
  const qm31 a{{p.alpha[0], p.alpha[1], p.alpha[2], p.alpha[3]}};
  const qm31 q = qscale(a, sub(p.eval[(i + 2) & p.mask], add(p.eval[(i + 1) & p.mask], p.eval[i])));
  for (int k = 0; k < 4; k++) p.quot_vals[4 * t + k] = q.v[k];
  for (uint32_t l = 0; l < p.nf; l++) {
    const uint32_t f = (p.qidx[qi] >> (l + 1)) ^ (t >= N_QUERIES ? 1u : 0u);
    for (int k = 0; k < 4; k++) p.fri_vals[(l * 2 * N_QUERIES + t) * 4 + k] = p.fri[l][k][f];
  }
}

// One CTA per query: recompute the query's tile, emit the full authentication
// paths of leaf f and of its sibling f ^ 1 (f = qidx >> shift): TL intra-tile
// siblings from the tile, the rest from the resident upper levels.
template <class Leaf>
__global__ void __launch_bounds__(256) paths_kernel(Leaf leaf, uint32_t TL, uint32_t shift,
                                                    const uint32_t* __restrict__ qidx,
                                                    const uint32_t* const* __restrict__ upper, uint32_t n_up,
                                                    uint32_t* __restrict__ out) {
  extern __shared__ uint32_t pk_sm[];
  const uint32_t qi = blockIdx.x;
  const uint32_t f = qidx[qi] >> shift;
  const uint32_t tile = f >> TL, n0 = 1u << TL, depth = TL + n_up;
  for (uint32_t i = threadIdx.x; i < n0; i += blockDim.x) {
    uint32_t h[8];
    leaf(((uint64_t)tile << TL) + i, h);
    for (int w = 0; w < 8; w++) pk_sm[8 * i + w] = h[w];
  }
  __syncthreads();
  uint32_t off = 0, cnt = n0;
  for (uint32_t k = 1; k <= TL; k++) {
    const uint32_t* prev = pk_sm + 8 * off;
    uint32_t* cur = pk_sm + 8 * (off + cnt);
    for (uint32_t i = threadIdx.x; i < cnt / 2; i += blockDim.x) {
      uint32_t h[8];
      b2s_node(h, prev + 16 * i, prev + 16 * i + 8);
      for (int w = 0; w < 8; w++) cur[8 * i + w] = h[w];
    }
    off += cnt;
    cnt >>= 1;
    __syncthreads();
  }
  // thread (s, k): s = 0 value path, 1 sibling path; k = level
  for (uint32_t t = threadIdx.x; t < 2 * depth; t += blockDim.x) {
    const uint32_t s = t / depth, k = t % depth;
    const uint32_t leaf_idx = f ^ s;
    uint32_t* dst = out + ((uint64_t)(s * N_QUERIES + qi) * depth + k) * 8;
    if (k < TL) {
      uint32_t lo = 0, lc = n0;
      for (uint32_t j = 0; j < k; j++) { lo += lc; lc >>= 1; }
      const uint32_t sib = ((leaf_idx & (n0 - 1)) >> k) ^ 1;
      for (int w = 0; w < 8; w++) dst[w] = pk_sm[8 * (lo + sib) + w];
    } else {
      const uint32_t u = k - TL;
      const uint32_t sib = ((leaf_idx >> TL) >> u) ^ 1;
      for (int w = 0; w < 8; w++) dst[w] = upper[u][8 * sib + w];
    }
  }
}

// ------------------------------------------------------------------ proof arena (shared with batch_prover.cu)
void ArenaLayout::plan(uint32_t ln) {
  log_n = ln;
  log_eval = ln + BLOWUP_BITS;
  nf = log_eval - LOG_LAST_LAYER;
  tree.clear();
  depth.clear();
  size_t w = 0;
  roots = w; w += 8 * (2 + nf);
  last = w; w += 32;
  q = w; w += N_QUERIES;
  tv = w; w += 2 * N_QUERIES;
  qv = w; w += 2 * N_QUERIES * 4;
  fv = w; w += (size_t)nf * 2 * N_QUERIES * 4;
  depth.push_back(log_eval);
  depth.push_back(log_eval);
  for (uint32_t l = 0; l < nf; l++) depth.push_back(log_eval - 1 - l);
  for (uint32_t d : depth) { tree.push_back(w); w += (size_t)2 * N_QUERIES * d * 8; }
  words = w;
}

// KRAK v1 from a host copy of the arena (after the stream completed). The format
// is a sequence of little-endian u32 words, so on a little-endian host each field
// is copied as words: the size is known up front and every region is one memcpy.
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "KRAK serialisation copies host words as LE bytes");
void ArenaLayout::serialize(const uint32_t* A, uint32_t a, uint32_t b, std::vector<uint8_t>& out) const {
  size_t total = 5 + 16 + 1 + 8 * (size_t)nf + 1 + 32 + 1 + N_QUERIES + 1 + 2 * N_QUERIES + 1 + 2 * N_QUERIES * 4 + 1;
  for (size_t t = 0; t < depth.size(); t++) total += 2 * N_QUERIES * (1 + (size_t)depth[t] * 8);
  total += (size_t)nf * (1 + 2 * N_QUERIES * 4);
  out.resize(total * 4);
  uint8_t* w = out.data();
  auto w32 = [&](uint32_t v) { std::memcpy(w, &v, 4); w += 4; };
  auto wn = [&](const uint32_t* p, size_t cnt) { std::memcpy(w, p, cnt * 4); w += cnt * 4; };
  auto wpaths = [&](size_t off, uint32_t d, uint32_t s) {
    for (uint32_t qi = 0; qi < N_QUERIES; qi++) { w32(d); wn(A + off + ((size_t)(s * N_QUERIES + qi) * d) * 8, (size_t)d * 8); }
  };
  w32(0x4B52414Bu); w32(1); w32(log_n); w32(a); w32(b);
  wn(A + roots, 16);
  w32(nf);
  wn(A + roots + 16, 8 * nf);
  w32(8);
  wn(A + last, 32);
  w32(N_QUERIES);
  wn(A + q, N_QUERIES);
  w32(N_QUERIES);
  wn(A + tv, 2 * N_QUERIES);
  wpaths(tree[0], depth[0], 0);
  wpaths(tree[0], depth[0], 1);
  w32(N_QUERIES);
  wn(A + qv, 2 * N_QUERIES * 4);
  wpaths(tree[1], depth[1], 0);
  wpaths(tree[1], depth[1], 1);
  w32(nf);
  for (uint32_t l = 0; l < nf; l++) {
    w32(N_QUERIES);
    wn(A + fv + (size_t)l * 2 * N_QUERIES * 4, 2 * N_QUERIES * 4);
    wpaths(tree[2 + l], depth[2 + l], 0);
    wpaths(tree[2 + l], depth[2 + l], 1);
  }
}

// ------------------------------------------------------------------ the prover
struct TreeBufs {
  uint64_t n = 0;
  uint32_t TL = 0;
  std::vector<uint32_t*> layers;  // [0] tile roots ... back() root
  const uint32_t** d_upper = nullptr;  // device copy of layers
};

struct GraphProver::Impl {
  uint32_t log_n = 0, log_eval = 0, nf = 0;
  uint64_t n = 0, N = 0;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaStream_t running = nullptr;  // stream of the proof in flight
  std::vector<void*> allocs;
  uint64_t allocated = 0;  // device bytes of allocs
  uint32_t *d_ab = nullptr, *h_ab = nullptr, *d_trace = nullptr, *d_eval = nullptr, *d_alpha = nullptr,
           *d_qidx = nullptr, *d_arena = nullptr, *h_arena = nullptr;
  ChanDev* d_ch = nullptr;
  std::vector<std::array<uint32_t*, 4>> fri_vals;
  TreeBufs trace_t, quot_t;
  std::vector<TreeBufs> fri_t;
  // subroot scratch shared by the trees (committed one after another in the graph)
  uint32_t split = 0, *sub_a = nullptr, *sub_b = nullptr;
  ArenaLayout lay;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;

  ~Impl() {
    if (running) cudaStreamSynchronize(running);
    if (st) cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void* p : allocs) cudaFree(p);
    if (h_arena) cudaFreeHost(h_arena);
    if (h_ab) cudaFreeHost(h_ab);
    if (st) cudaStreamDestroy(st);
  }
  template <class T>
  int alloc(T** p, uint64_t count) {
    void* q = nullptr;
    const uint64_t bytes = std::max<uint64_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return set_error(VS_ERR_OOM, "prover workspace: %s", cudaGetErrorString(e));
    allocated += (bytes + 511) & ~511ull;  // cudaMalloc's granularity
    allocs.push_back(q);
    *p = (T*)q;
    return VS_OK;
  }
  int tree_bufs(TreeBufs& t, uint64_t leaves) {
    t.n = leaves;
    t.TL = std::min<uint32_t>(MK_MAX_TL, ilog2(leaves));
    for (uint64_t cnt = leaves >> t.TL;; cnt /= 2) {
      uint32_t* l = nullptr;
      VS_TRY(alloc(&l, cnt * 8));
      t.layers.push_back(l);
      if (cnt == 1) break;
    }
    VS_TRY(alloc(&t.d_upper, t.layers.size()));
    VS_CUDA(cudaMemcpy(t.d_upper, t.layers.data(), t.layers.size() * sizeof(void*), cudaMemcpyHostToDevice));
    return VS_OK;
  }
  template <class Leaf>
  int commit(const Leaf& leaf, TreeBufs& t) {
    const uint32_t sp = (t.TL == MK_MAX_TL && t.n >= (1ull << 20)) ? split : 0u;
    VS_TRY(merkle_tile_roots_split(leaf, t.n, t.TL, sp, t.layers[0], sub_a, sub_b, st));
    for (size_t k = 1; k < t.layers.size(); k++)
      VS_TRY(launch_hash_nodes(t.layers[k - 1], t.layers[k], t.n >> (t.TL + k), st));
    return VS_OK;
  }
  template <class Leaf>
  int paths(const Leaf& leaf, const TreeBufs& t, uint32_t shift, size_t arena_off) {
    const unsigned smem = (unsigned)(((2u << t.TL) - 1) * 32);
    static std::once_flag attr_once;  // set before the first (uncaptured) run
    cudaError_t ae = cudaSuccess;
    std::call_once(attr_once, [&] {
      ae = cudaFuncSetAttribute(paths_kernel<Leaf>, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536);
    });
    VS_CUDA(ae);
    paths_kernel<Leaf><<<N_QUERIES, 256, smem, st>>>(leaf, t.TL, shift, d_qidx, t.d_upper,
                                                     (uint32_t)t.layers.size() - 1, d_arena + arena_off);
    VS_LAUNCHED("paths_kernel");
    return VS_OK;
  }

  int setup(uint32_t ln, int priority) {
    log_n = ln;
    log_eval = ln + BLOWUP_BITS;
    n = 1ull << ln;
    N = 1ull << log_eval;
    nf = log_eval - LOG_LAST_LAYER;
    VS_CUDA(cudaGetDevice(&device));
    VS_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, priority));
    VS_CUDA(cudaMallocHost((void**)&h_ab, 16));
    VS_TRY(alloc(&d_ab, 4));
    VS_TRY(alloc(&d_trace, n));
    VS_TRY(alloc(&d_eval, N));
    VS_TRY(alloc(&d_alpha, 4 * (2 + nf)));
    VS_TRY(alloc(&d_qidx, N_QUERIES));
    VS_TRY(alloc(&d_ch, 1));
    VS_TRY(tree_bufs(trace_t, N));
    VS_TRY(tree_bufs(quot_t, N));
    split = merkle_tile_split(N);  // fixed for the prover's lifetime (its graph is captured once)
    if (split) {
      VS_TRY(alloc(&sub_a, ((N >> MK_MAX_TL) << split) * 8));
      VS_TRY(alloc(&sub_b, ((N >> MK_MAX_TL) << (split - 1)) * 8));
    }
    fri_t.resize(nf);
    for (uint32_t l = 0; l < nf; l++) {
      const uint64_t half = N >> (l + 1);
      uint32_t* base = nullptr;
      VS_TRY(alloc(&base, 4 * half));
      fri_vals.push_back({base, base + half, base + 2 * half, base + 3 * half});
      VS_TRY(tree_bufs(fri_t[l], half));
    }
    lay.plan(log_n);
    VS_TRY(alloc(&d_arena, lay.words));
    VS_CUDA(cudaMallocHost((void**)&h_arena, lay.words * 4));
    // twiddles and fold twiddles are built (and cached) outside the capture
    const TwiddleSet* tw = nullptr;
    VS_TRY(get_twiddles(TW_NATIVE, log_n, &tw, st));
    VS_TRY(get_twiddles(TW_NATIVE, log_eval, &tw, st));
    for (uint32_t l = 0; l < nf; l++) {
      const uint32_t* ft = nullptr;
      VS_TRY(get_fold_twiddles(l == 0 ? COSET_HALF_COSET : COSET_HALF_ODDS, log_eval - l, &ft, st));
    }
    VS_CUDA(cudaStreamSynchronize(st));
    // one plain run sets kernel attributes, then the same sequence is captured
    VS_TRY(enqueue());
    VS_CUDA(cudaStreamSynchronize(st));
    VS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue();
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    VS_TRY(rc);
    VS_CUDA(e);
    VS_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    return VS_OK;
  }

  // The whole proof, stream-ordered on st.
  int enqueue() {
    VS_CUDA(cudaMemcpyAsync(d_ab, h_ab, 8, cudaMemcpyHostToDevice, st));
    fib_trace_params_kernel<<<blocks_for(n, 256 * 32), 256, 0, st>>>(d_ab, d_trace, n);
    VS_LAUNCHED("fib_trace_params_kernel");
    VS_TRY(lde_cached(TW_NATIVE, d_trace, 0, d_eval, 0, 1, log_n, BLOWUP_BITS, st));
    VS_TRY(commit(LeafOne{d_eval}, trace_t));
    ch_mix_draw_kernel<<<1, 32, 0, st>>>(d_ch, 1, trace_t.layers.back(), d_arena + lay.roots, d_alpha);
    VS_LAUNCHED("ch_mix_draw_kernel");
    const LeafFibQuotD quot{d_eval, N - 1, d_alpha};
    VS_TRY(commit(quot, quot_t));
    ch_mix_draw_kernel<<<1, 32, 0, st>>>(d_ch, 0, quot_t.layers.back(), d_arena + lay.roots + 8, d_alpha + 4);
    VS_LAUNCHED("ch_mix_draw_kernel");
    for (uint32_t l = 0; l < nf; l++) {
      const uint32_t cur = log_eval - l;
      const uint32_t* tw = nullptr;
      VS_TRY(get_fold_twiddles(l == 0 ? COSET_HALF_COSET : COSET_HALF_ODDS, cur, &tw, st));
      const uint32_t* a = d_alpha + 4 * (1 + l);
      if (l == 0) {
        LeafFoldQuotD leaf{quot, tw, a, {fri_vals[0][0], fri_vals[0][1], fri_vals[0][2], fri_vals[0][3]}};
        VS_TRY(commit(leaf, fri_t[0]));
      } else {
        LeafFoldD leaf{{fri_vals[l - 1][0], fri_vals[l - 1][1], fri_vals[l - 1][2], fri_vals[l - 1][3]},
                       {fri_vals[l][0], fri_vals[l][1], fri_vals[l][2], fri_vals[l][3]}, tw, a};
        VS_TRY(commit(leaf, fri_t[l]));
      }
      ch_mix_draw_kernel<<<1, 32, 0, st>>>(d_ch, 0, fri_t[l].layers.back(), d_arena + lay.roots + 8 * (2 + l),
                                           l + 1 < nf ? d_alpha + 4 * (2 + l) : nullptr);
      VS_LAUNCHED("ch_mix_draw_kernel");
    }
    const auto& last = fri_vals[nf - 1];
    ch_queries_kernel<<<1, 32, 0, st>>>(d_ch, last[0], last[1], last[2], last[3], d_arena + lay.last, d_qidx,
                                        d_arena + lay.q, log_eval);
    VS_LAUNCHED("ch_queries_kernel");
    DecParams dp{};
    dp.eval = d_eval;
    dp.mask = (uint32_t)(N - 1);
    dp.alpha = d_alpha;
    dp.qidx = d_qidx;
    dp.trace_vals = d_arena + lay.tv;
    dp.quot_vals = d_arena + lay.qv;
    dp.nf = nf;
    for (uint32_t l = 0; l < nf; l++)
      for (int k = 0; k < 4; k++) dp.fri[l][k] = fri_vals[l][k];
    dp.fri_vals = d_arena + lay.fv;
    decommit_values_kernel<<<1, 2 * N_QUERIES, 0, st>>>(dp);
    VS_LAUNCHED("decommit_values_kernel");
    VS_TRY(paths(LeafOne{d_eval}, trace_t, 0, lay.tree[0]));
    VS_TRY(paths(quot, quot_t, 0, lay.tree[1]));
    for (uint32_t l = 0; l < nf; l++)
      VS_TRY(paths(LeafSoa4{fri_vals[l][0], fri_vals[l][1], fri_vals[l][2], fri_vals[l][3]}, fri_t[l], l + 1,
                   lay.tree[2 + l]));
    VS_CUDA(cudaMemcpyAsync(h_arena, d_arena, lay.words * 4, cudaMemcpyDeviceToHost, st));
    return VS_OK;
  }

};

GraphProver::GraphProver() : impl(new Impl) {}
GraphProver::~GraphProver() = default;
int GraphProver::init(uint32_t log_n, int priority) {
  if (log_n < 4 || log_n + BLOWUP_BITS > 30) return set_error(VS_ERR_INVALID, "log_n %u outside [4, 28]", log_n);
  return impl->setup(log_n, priority);
}
uint32_t GraphProver::log_n() const { return impl->log_n; }
int GraphProver::device() const { return impl->device; }
cudaStream_t GraphProver::stream() const { return impl->st; }
uint64_t GraphProver::device_bytes() const { return impl->allocated; }

// An upper bound of device_bytes() for a prover of 2^log_n rows, known before it
// is created: trace, evaluation, arena and FRI layers as allocated, the tile-root
// levels of all trees (under N/2 words together) and the allocation rounding
// bounded by another 2N words, and subroot scratch at the largest tile split.
uint64_t GraphProver::bytes_estimate(uint32_t log_n) {
  ArenaLayout lay;
  lay.plan(log_n);
  const uint64_t n = 1ull << log_n, N = n << BLOWUP_BITS;
  uint64_t b = n * 4 + N * 4 * 3 + lay.words * 4 + (64u << 10);
  for (uint32_t l = 0; l < lay.nf; l++) b += (N >> (l + 1)) * 16;
  return b + merkle_tile_scratch_bytes(N, MK_TILE_SPLIT_MAX);
}
int GraphProver::launch(uint32_t a, uint32_t b, cudaStream_t on) {
  if (a >= h::P || b >= h::P) return set_error(VS_ERR_INVALID, "public inputs must be canonical M31");
  impl->h_ab[0] = a;
  impl->h_ab[1] = b;
  impl->running = on ? on : impl->st;
  VS_CUDA(cudaGraphLaunch(impl->exec, impl->running));
  return VS_OK;
}
int GraphProver::finish(uint32_t a, uint32_t b, std::vector<uint8_t>& out) {
  VS_CUDA(cudaStreamSynchronize(impl->running ? impl->running : impl->st));
  impl->running = nullptr;  // the launch stream may be reused for other work from here on
  impl->lay.serialize(impl->h_arena, a, b, out);
  return VS_OK;
}
bool GraphProver::busy() const {
  return cudaStreamQuery(impl->running ? impl->running : impl->st) == cudaErrorNotReady;
}

}  // namespace vs

using namespace vs;

extern "C" {

int vs_prover_create(uint32_t log_n, void** out) {
  clear_error();
  if (!out) return set_error(VS_ERR_INVALID, "vs_prover_create: null handle");
  auto p = std::make_unique<GraphProver>();
  VS_TRY(p->init(log_n));
  *out = p.release();
  return VS_OK;
}

int vs_prover_prove(void* h, uint32_t a, uint32_t b, uint8_t* out, uint64_t cap, uint64_t* out_len) {
  clear_error();
  auto* p = static_cast<GraphProver*>(h);
  if (!p) return set_error(VS_ERR_INVALID, "vs_prover_prove: null handle");
  std::vector<uint8_t> bytes;
  VS_TRY(p->launch(a, b));
  VS_TRY(p->finish(a, b, bytes));
  if (out_len) *out_len = bytes.size();
  if (!out || cap < bytes.size()) return set_error(VS_ERR_INVALID, "proof needs %zu bytes", bytes.size());
  std::copy(bytes.begin(), bytes.end(), out);
  return VS_OK;
}

int vs_prover_destroy(void* h) {
  delete static_cast<GraphProver*>(h);
  return VS_OK;
}

}  // extern "C"
