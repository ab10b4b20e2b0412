// Batched Fibonacci prover: many independent proofs of one trace size run as one
// CUDA graph in which every stage is a single kernel launch over all of them.
//
// The reference proves a batch one proof after another (ProverPipeline::prove_batch,
// src/prover.rs:2265-2270), and the graph-captured prover (prover_graph.cu) still
// issues one chain of small launches per proof. Here job j's buffers are the j-th
// slices of batch-wide arrays, so one launch covers every job:
//
//   * trace: blockIdx.y selects the job's public inputs;
//   * LDE: the jobs' traces are the columns of one multi-column native LDE;
//   * Merkle trees: job j's 2^m leaves are leaves [j 2^m, (j+1) 2^m) of one leaf
//     range, so tiles never straddle jobs and each stored level is the
//     concatenation of the jobs' levels (parents never straddle jobs either);
//   * fused quotient / fold leaves: the leaf functors split a global leaf index
//     into (job, index) and read the job's own challenges;
//   * Fiat-Shamir channel: one thread per job (one CTA per job for the query
//     draw, whose squeezes are independent given the state);
//   * decommitment: one warp per (job, query) gathers its authentication path.
//
// Trees keep every level from level 3 up (eight-leaf groups): an authentication
// path is a gather of the stored siblings plus the recomputation of one
// eight-leaf group, instead of one 1024-leaf tile per query and tree as in the
// tile-root provers (the reference keeps whole trees at these sizes too,
// MerkleTree::commit, src/prover.rs:1764-1766). The arithmetic, transcript and
// proof layout are the graph prover's: every proof is byte-identical to
// vs_prove_fib's for the same (a, b, log_n).
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batch_prover.h"
#include "channel_dev.cuh"
#include "fri_impl.cuh"
#include "merkle.h"
#include "ntt.h"
#include "prover.h"
#include "prover_graph.h"
#include "twiddles.h"
#include "vs_common.cuh"

namespace vs {

namespace {

constexpr int BMAXF = 24;        // FRI layers for log_eval <= 27 (log_n <= BATCH_MAX_LOG_N + 3)
constexpr uint32_t BGROUP = 3;   // lowest stored tree level: 2^3-leaf groups are recomputed
constexpr uint32_t BTOP = 10;    // tree_top_kernel takes the last levels of <= 2^10 hashes per tree

// ------------------------------------------------------------------ batched leaf functors
// Global leaf g of a batch of trees with 2^log_len leaves each: job g >> log_len,
// index g & (2^log_len - 1).
struct LeafFibQuotB {
  const uint32_t* e;      // [jobs][N] evaluations
  uint32_t log_n;         // log N
  const uint32_t* alpha;  // job j's quotient challenge at alpha + j * astride
  uint32_t astride;
  __device__ __forceinline__ qm31 q(uint64_t g) const {
    const uint64_t mask = (1ull << log_n) - 1, j = g >> log_n, i = g & mask;
    const uint32_t* ej = e + (j << log_n);
    const uint32_t* a = alpha + j * astride;
    const qm31 av{{__ldg(a), __ldg(a + 1), __ldg(a + 2), __ldg(a + 3)}};
    return qscale(av, sub(ej[(i + 2) & mask], add(ej[(i + 1) & mask], ej[i])));
  }
  __device__ __forceinline__ void operator()(uint64_t g, uint32_t out[8]) const {
    const qm31 r = q(g);
    uint32_t m[16] = {0};
    m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};

// Circle fold of the quotient (never materialised) into FRI layer 0.
struct LeafFoldQuotB {
  LeafFibQuotB quot;
  const uint32_t* tw;     // 2^log_half fold twiddles, shared by the jobs
  uint32_t log_half;
  const uint32_t* alpha;  // job j's fold challenge at alpha + j * astride
  uint32_t astride;
  uint32_t* dst[4];       // planes [jobs][2^log_half]
  __device__ __forceinline__ void operator()(uint64_t g, uint32_t out[8]) const {
    const uint64_t j = g >> log_half, i = g & ((1ull << log_half) - 1);
    const uint32_t* a = alpha + j * astride;
    const qm31 av{{__ldg(a), __ldg(a + 1), __ldg(a + 2), __ldg(a + 3)}};
    // 2g = j * 2^(log_half+1) + 2i: the job's own quotient values 2i and 2i + 1
    const qm31 r = fold_pair(quot.q(2 * g), quot.q(2 * g + 1), av, __ldg(tw + i));
#pragma unroll
    for (int k = 0; k < 4; k++) dst[k][g] = r.v[k];
    uint32_t m[16] = {0};
    m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};

// Line fold of FRI layer l - 1 (planes [jobs][2^(log_half+1)]) into layer l.
struct LeafFoldB {
  const uint32_t* src[4];
  uint32_t* dst[4];
  const uint32_t* tw;
  uint32_t log_half;
  const uint32_t* alpha;
  uint32_t astride;
  __device__ __forceinline__ void operator()(uint64_t g, uint32_t out[8]) const {
    const uint64_t j = g >> log_half, i = g & ((1ull << log_half) - 1);
    const uint32_t* a = alpha + j * astride;
    const qm31 av{{__ldg(a), __ldg(a + 1), __ldg(a + 2), __ldg(a + 3)}};
    const uint2 s0 = *reinterpret_cast<const uint2*>(src[0] + 2 * g);
    const uint2 s1 = *reinterpret_cast<const uint2*>(src[1] + 2 * g);
    const uint2 s2 = *reinterpret_cast<const uint2*>(src[2] + 2 * g);
    const uint2 s3 = *reinterpret_cast<const uint2*>(src[3] + 2 * g);
    const qm31 r = fold_pair(qm31{{s0.x, s1.x, s2.x, s3.x}}, qm31{{s0.y, s1.y, s2.y, s3.y}}, av, __ldg(tw + i));
#pragma unroll
    for (int k = 0; k < 4; k++) dst[k][g] = r.v[k];
    uint32_t m[16] = {0};
    m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};

// Stored levels of a batch of trees with 2^m leaves each: lv[k - s] is level k
// (k = s..m), [jobs][2^(m-k)] hashes of 8 words.
struct TreeLevels {
  uint32_t* lv[32];
  uint32_t s, m;
};

// ------------------------------------------------------------------ kernels
// One CTA per tree: levels k0+1..m from level k0 (2^(m-k0) <= 2^BTOP hashes per
// tree), each written to its stored level. Shared memory: two hash buffers.
__global__ void __launch_bounds__(256) tree_top_kernel(TreeLevels t, uint32_t k0) {
  extern __shared__ uint32_t tt_sm[];
  const uint32_t j = blockIdx.x;
  uint32_t cnt = 1u << (t.m - k0);
  uint32_t* a = tt_sm;
  uint32_t* b = tt_sm + 8 * cnt;
  const uint32_t* src = t.lv[k0 - t.s] + (uint64_t)j * cnt * 8;
  for (uint32_t i = threadIdx.x; i < 8 * cnt; i += blockDim.x) a[i] = src[i];
  __syncthreads();
  for (uint32_t k = k0 + 1; k <= t.m; k++) {
    cnt >>= 1;
    uint32_t* dst = t.lv[k - t.s] + (uint64_t)j * cnt * 8;
    for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
      uint32_t h[8];
      b2s_node(h, a + 16 * i, a + 16 * i + 8);
#pragma unroll
      for (int w = 0; w < 8; w++) { b[8 * i + w] = h[w]; dst[8 * i + w] = h[w]; }
    }
    __syncthreads();
    uint32_t* tmp = a;
    a = b;
    b = tmp;
  }
}

// Channel of job j (one thread each): mix a root (copied into the job's arena)
// and, when alpha_off >= 0, draw a challenge into the job's alpha slots.
__global__ void bch_mix_draw_kernel(ChanDev* ch, uint32_t jobs, int reset, const uint32_t* __restrict__ roots,
                                    uint32_t* arena, uint64_t words, uint64_t arena_off, uint32_t* alpha,
                                    uint32_t astride, int alpha_off) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= jobs) return;
  ChanDev c = ch[j];
  if (reset) {
    for (int i = 0; i < 8; i++) c.state[i] = 0;
    c.n_draws = 0;
    c.error = 0;
  }
  uint32_t r[8];
  uint32_t* ar = arena + (uint64_t)j * words + arena_off;
  for (int i = 0; i < 8; i++) { r[i] = roots[8 * j + i]; ar[i] = r[i]; }
  ch_mix_digest(c, r);
  if (alpha_off >= 0) {
    uint32_t v[4];
    ch_draw_felt(c, v);
    for (int i = 0; i < 4; i++) alpha[(uint64_t)j * astride + alpha_off + i] = v[i];
  }
  ch[j] = c;
}

// One CTA per job: mix_felts(last layer), then the N_QUERIES draw_number squeezes,
// which depend only on the state and their draw counter, in parallel.
__global__ void __launch_bounds__(96) bch_queries_kernel(ChanDev* ch, const uint32_t* l0, const uint32_t* l1,
                                                        const uint32_t* l2, const uint32_t* l3, uint32_t* arena,
                                                        uint64_t words, uint64_t a_last, uint64_t a_q,
                                                        uint32_t* qidx, uint32_t log_eval) {
  __shared__ ChanDev sc;
  const uint32_t j = blockIdx.x;
  uint32_t* ar = arena + (uint64_t)j * words;
  if (threadIdx.x == 0) {
    ChanDev c = ch[j];
    const uint32_t* planes[4] = {l0 + 8 * j, l1 + 8 * j, l2 + 8 * j, l3 + 8 * j};
    for (int i = 0; i < 8; i++)
      for (int k = 0; k < 4; k++) ar[a_last + 4 * i + k] = planes[k][i];
    ch_mix_felts_planes(c, planes, 8);
    sc = c;
  }
  __syncthreads();
  if (threadIdx.x < N_QUERIES) {
    ChanDev c = sc;
    c.n_draws = threadIdx.x;  // the q-th draw after the mix squeezes with counter q
    const uint32_t v = ch_draw_pow2(c, log_eval);
    qidx[j * N_QUERIES + threadIdx.x] = v;
    ar[a_q + threadIdx.x] = v;
  }
  if (threadIdx.x == 0) {
    ChanDev c = sc;
    c.n_draws = N_QUERIES;
    ch[j] = c;
  }
}

struct BDecParams {
  const uint32_t* eval;
  uint32_t log_eval;
  const uint32_t* alpha;
  uint32_t astride;
  const uint32_t* qidx;
  uint32_t* arena;
  uint64_t words, a_tv, a_qv, a_fv;
  uint32_t nf;
  const uint32_t* fri[BMAXF][4];  // plane k of layer l: [jobs][2^(log_eval-1-l)]
};
// One CTA per job: values at each query and its fold sibling (q ^ 1); FRI layer l
// uses q >> (l + 1).
__global__ void bdecommit_values_kernel(BDecParams p) {
  const uint32_t t = threadIdx.x, j = blockIdx.x;
  if (t >= 2 * N_QUERIES) return;
  const uint32_t qi = t % N_QUERIES, sib = t >= N_QUERIES ? 1u : 0u;
  const uint32_t q = p.qidx[j * N_QUERIES + qi];
  const uint32_t i = q ^ sib;
  const uint32_t mask = (1u << p.log_eval) - 1;
  const uint32_t* e = p.eval + ((uint64_t)j << p.log_eval);
  uint32_t* ar = p.arena + (uint64_t)j * p.words;
  ar[p.a_tv + t] = e[i];
  const uint32_t* al = p.alpha + (uint64_t)j * p.astride;
  const qm31 a{{al[0], al[1], al[2], al[3]}};
  const qm31 qv = qscale(a, sub(e[(i + 2) & mask], add(e[(i + 1) & mask], e[i])));
  for (int k = 0; k < 4; k++) ar[p.a_qv + 4 * t + k] = qv.v[k];
  for (uint32_t l = 0; l < p.nf; l++) {
    const uint32_t f = (q >> (l + 1)) ^ sib;
    const uint64_t base = (uint64_t)j << (p.log_eval - 1 - l);
    for (int k = 0; k < 4; k++) ar[p.a_fv + (l * 2 * N_QUERIES + t) * 4 + k] = p.fri[l][k][base + f];
  }
}

// One warp per (job, query): the authentication paths of leaf f = qidx >> shift and
// of its sibling f ^ 1. Levels below s come from recomputing f's 2^s-leaf group
// (side-effect-free leaf functor), levels s..m-1 from the stored levels.
template <class Leaf>
__global__ void __launch_bounds__(256) bpaths_kernel(Leaf leaf, TreeLevels t, uint32_t shift,
                                                    const uint32_t* __restrict__ qidx, uint32_t jobs,
                                                    uint32_t* __restrict__ arena, uint64_t words, uint64_t off) {
  __shared__ uint32_t sm[8][(2 << BGROUP) * 8];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t wi = blockIdx.x * 8 + warp;
  if (wi >= jobs * N_QUERIES) return;  // uniform per warp
  const uint32_t j = wi / N_QUERIES, qi = wi % N_QUERIES;
  const uint32_t s = t.s, m = t.m, g = 1u << s;
  const uint32_t f = qidx[j * N_QUERIES + qi] >> shift;
  uint32_t* S = sm[warp];
  const uint64_t gbase = ((uint64_t)j << m) + ((uint64_t)(f >> s) << s);
  if (lane < g) {
    uint32_t h[8];
    leaf(gbase + lane, h);
#pragma unroll
    for (int w = 0; w < 8; w++) S[8 * lane + w] = h[w];
  }
  __syncwarp();
  uint32_t lo = 0, cnt = g;
  for (uint32_t k = 1; k < s; k++) {
    if (lane < cnt / 2) {
      uint32_t h[8];
      b2s_node(h, S + 8 * (lo + 2 * lane), S + 8 * (lo + 2 * lane + 1));
#pragma unroll
      for (int w = 0; w < 8; w++) S[8 * (lo + cnt + lane) + w] = h[w];
    }
    __syncwarp();
    lo += cnt;
    cnt >>= 1;
  }
  uint32_t* out = arena + (uint64_t)j * words + off;
  for (uint32_t x = lane; x < 2 * m; x += 32) {
    const uint32_t sd = x / m, k = x % m;
    const uint32_t leaf_idx = f ^ sd;
    uint32_t* dst = out + ((uint64_t)(sd * N_QUERIES + qi) * m + k) * 8;
    const uint32_t* src;
    if (k < s) {
      uint32_t l0 = 0, lc = g;
      for (uint32_t z = 0; z < k; z++) { l0 += lc; lc >>= 1; }
      src = S + 8 * (l0 + (((leaf_idx & (g - 1)) >> k) ^ 1));
    } else {
      src = t.lv[k - s] + (((uint64_t)j << (m - k)) + ((leaf_idx >> k) ^ 1)) * 8;
    }
#pragma unroll
    for (int w = 0; w < 8; w++) dst[w] = src[w];
  }
}

uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

}  // namespace

// ------------------------------------------------------------------ the prover
struct BatchProver::Impl {
  uint32_t log_n = 0, log_eval = 0, nf = 0, cap = 0, astride = 0;
  uint64_t n = 0, N = 0, total = 0;
  int device = 0;
  cudaStream_t st = nullptr, running = nullptr;
  uint32_t count = 0;  // jobs of the batch in flight
  uint8_t* mem = nullptr;
  uint32_t *h_ab = nullptr, *h_arena = nullptr;
  uint32_t *d_ab = nullptr, *d_trace = nullptr, *d_eval = nullptr, *d_alpha = nullptr, *d_qidx = nullptr,
           *d_arena = nullptr;
  ChanDev* d_ch = nullptr;
  struct Tree {
    TreeLevels L{};
    uint32_t TL = 0;
  } trace_t, quot_t, fri_t[BMAXF];
  uint32_t* fri[BMAXF][4] = {};
  ArenaLayout lay;
  std::map<uint32_t, cudaGraphExec_t> exec;  // per batch size

  ~Impl() {
    if (running) cudaStreamSynchronize(running);
    if (st) cudaStreamSynchronize(st);
    for (auto& kv : exec) cudaGraphExecDestroy(kv.second);
    if (mem) cudaFree(mem);
    if (h_arena) cudaFreeHost(h_arena);
    if (h_ab) cudaFreeHost(h_ab);
    if (st) cudaStreamDestroy(st);
  }

  // Assigns every device buffer inside one allocation at `base` (sizes only when
  // null); returns the bytes used.
  uint64_t carve(uint8_t* base) {
    uint64_t off = 0;
    auto take = [&](uint64_t bytes) -> uint8_t* {
      uint8_t* p = base ? base + off : nullptr;
      off += align256(std::max<uint64_t>(bytes, 4));
      return p;
    };
    d_ab = (uint32_t*)take(8ull * cap);
    d_trace = (uint32_t*)take(4 * n * cap);
    d_eval = (uint32_t*)take(4 * N * cap);
    d_alpha = (uint32_t*)take(4ull * astride * cap);
    d_qidx = (uint32_t*)take(4ull * N_QUERIES * cap);
    d_ch = (ChanDev*)take(sizeof(ChanDev) * cap);
    d_arena = (uint32_t*)take(4ull * lay.words * cap);
    for (uint32_t l = 0; l < nf; l++) {
      const uint64_t half = N >> (l + 1);
      for (int k = 0; k < 4; k++) fri[l][k] = (uint32_t*)take(4 * half * cap);
    }
    auto tree = [&](Tree& t, uint32_t m) {
      t.L.m = m;
      t.L.s = std::min(BGROUP, m);
      t.TL = std::min<uint32_t>(MK_MAX_TL, m);
      for (uint32_t k = t.L.s; k <= m; k++) t.L.lv[k - t.L.s] = (uint32_t*)take(32ull * cap << (m - k));
    };
    tree(trace_t, log_eval);
    tree(quot_t, log_eval);
    for (uint32_t l = 0; l < nf; l++) tree(fri_t[l], log_eval - 1 - l);
    return off;
  }

  void plan(uint32_t ln, uint32_t c) {
    log_n = ln;
    log_eval = ln + BLOWUP_BITS;
    n = 1ull << ln;
    N = 1ull << log_eval;
    nf = log_eval - LOG_LAST_LAYER;
    cap = c;
    astride = 4 * (2 + nf);
    lay.plan(ln);
    total = carve(nullptr);
  }

  template <class Leaf>
  int commit(const Leaf& leaf, Tree& t, uint32_t b) {
    const uint32_t s = t.L.s, m = t.L.m;
    VS_TRY(merkle_tile_roots(leaf, (uint64_t)b << m, t.TL, t.L.lv[0], st, t.TL - s));
    uint32_t k = s;
    for (; m - k > BTOP; k++)
      VS_TRY(launch_hash_nodes(t.L.lv[k - s], t.L.lv[k + 1 - s], (uint64_t)b << (m - k - 1), st));
    if (k < m) {
      const unsigned smem = (unsigned)(((1u << (m - k)) * 3 / 2) * 32);
      tree_top_kernel<<<b, 256, smem, st>>>(t.L, k);
      VS_LAUNCHED("tree_top_kernel");
    }
    return VS_OK;
  }
  template <class Leaf>
  int paths(const Leaf& leaf, const Tree& t, uint32_t shift, size_t arena_off, uint32_t b) {
    bpaths_kernel<Leaf><<<blocks_for((uint64_t)b * N_QUERIES, 8), 256, 0, st>>>(leaf, t.L, shift, d_qidx, b, d_arena,
                                                                                 lay.words, arena_off);
    VS_LAUNCHED("bpaths_kernel");
    return VS_OK;
  }

  // The whole batch of b proofs, stream-ordered on st.
  int enqueue(uint32_t b) {
    VS_CUDA(cudaMemcpyAsync(d_ab, h_ab, 8ull * b, cudaMemcpyHostToDevice, st));
    fib_trace_params_kernel<<<dim3(blocks_for(n, 256 * 32), b), 256, 0, st>>>(d_ab, d_trace, n);
    VS_LAUNCHED("fib_trace_params_kernel");
    VS_TRY(lde_cached(TW_NATIVE, d_trace, n, d_eval, N, b, log_n, BLOWUP_BITS, st));
    const unsigned cb = blocks_for(b, 64);
    VS_TRY(commit(LeafOne{d_eval}, trace_t, b));
    bch_mix_draw_kernel<<<cb, 64, 0, st>>>(d_ch, b, 1, trace_t.L.lv[trace_t.L.m - trace_t.L.s], d_arena, lay.words,
                                           lay.roots, d_alpha, astride, 0);
    VS_LAUNCHED("bch_mix_draw_kernel");
    const LeafFibQuotB quot{d_eval, log_eval, d_alpha, astride};
    VS_TRY(commit(quot, quot_t, b));
    bch_mix_draw_kernel<<<cb, 64, 0, st>>>(d_ch, b, 0, quot_t.L.lv[quot_t.L.m - quot_t.L.s], d_arena, lay.words,
                                           lay.roots + 8, d_alpha, astride, 4);
    VS_LAUNCHED("bch_mix_draw_kernel");
    for (uint32_t l = 0; l < nf; l++) {
      const uint32_t cur = log_eval - l;
      const uint32_t* tw = nullptr;
      VS_TRY(get_fold_twiddles(l == 0 ? COSET_HALF_COSET : COSET_HALF_ODDS, cur, &tw, st));
      if (l == 0) {
        LeafFoldQuotB leaf{quot, tw, cur - 1, d_alpha + 4, astride, {fri[0][0], fri[0][1], fri[0][2], fri[0][3]}};
        VS_TRY(commit(leaf, fri_t[0], b));
      } else {
        LeafFoldB leaf{{fri[l - 1][0], fri[l - 1][1], fri[l - 1][2], fri[l - 1][3]},
                       {fri[l][0], fri[l][1], fri[l][2], fri[l][3]}, tw, cur - 1, d_alpha + 4 * (1 + l), astride};
        VS_TRY(commit(leaf, fri_t[l], b));
      }
      const Tree& t = fri_t[l];
      bch_mix_draw_kernel<<<cb, 64, 0, st>>>(d_ch, b, 0, t.L.lv[t.L.m - t.L.s], d_arena, lay.words,
                                             lay.roots + 8 * (2 + l), d_alpha, astride,
                                             l + 1 < nf ? (int)(4 * (2 + l)) : -1);
      VS_LAUNCHED("bch_mix_draw_kernel");
    }
    const auto& last = fri[nf - 1];
    bch_queries_kernel<<<b, 96, 0, st>>>(d_ch, last[0], last[1], last[2], last[3], d_arena, lay.words, lay.last,
                                         lay.q, d_qidx, log_eval);
    VS_LAUNCHED("bch_queries_kernel");
    BDecParams dp{};
    dp.eval = d_eval;
    dp.log_eval = log_eval;
    dp.alpha = d_alpha;
    dp.astride = astride;
    dp.qidx = d_qidx;
    dp.arena = d_arena;
    dp.words = lay.words;
    dp.a_tv = lay.tv;
    dp.a_qv = lay.qv;
    dp.a_fv = lay.fv;
    dp.nf = nf;
    for (uint32_t l = 0; l < nf; l++)
      for (int k = 0; k < 4; k++) dp.fri[l][k] = fri[l][k];
    bdecommit_values_kernel<<<b, 2 * N_QUERIES, 0, st>>>(dp);
    VS_LAUNCHED("bdecommit_values_kernel");
    VS_TRY(paths(LeafOne{d_eval}, trace_t, 0, lay.tree[0], b));
    VS_TRY(paths(quot, quot_t, 0, lay.tree[1], b));
    for (uint32_t l = 0; l < nf; l++)
      VS_TRY(paths(LeafSoa4{fri[l][0], fri[l][1], fri[l][2], fri[l][3]}, fri_t[l], l + 1, lay.tree[2 + l], b));
    VS_CUDA(cudaMemcpyAsync(h_arena, d_arena, 4ull * lay.words * b, cudaMemcpyDeviceToHost, st));
    return VS_OK;
  }

  int graph_for(uint32_t b, cudaGraphExec_t* out) {
    auto it = exec.find(b);
    if (it != exec.end()) { *out = it->second; return VS_OK; }
    cudaGraph_t g = nullptr;
    VS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue(b);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != VS_OK) { if (g) cudaGraphDestroy(g); return rc; }
    VS_CUDA(e);
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    VS_CUDA(e);
    exec[b] = x;
    *out = x;
    return VS_OK;
  }

  int setup(uint32_t ln, uint32_t c) {
    plan(ln, c);
    VS_CUDA(cudaGetDevice(&device));
    VS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaError_t e = cudaMalloc((void**)&mem, total);
    if (e != cudaSuccess) {
      mem = nullptr;
      return set_error(VS_ERR_OOM, "batch prover workspace (%llu bytes): %s", (unsigned long long)total,
                       cudaGetErrorString(e));
    }
    carve(mem);
    VS_CUDA(cudaMallocHost((void**)&h_ab, 8ull * cap));
    VS_CUDA(cudaMallocHost((void**)&h_arena, 4ull * lay.words * cap));
    for (uint32_t i = 0; i < 2 * cap; i++) h_ab[i] = 1;
    // twiddles and fold twiddles are built (and cached) outside the capture
    const TwiddleSet* tw = nullptr;
    VS_TRY(get_twiddles(TW_NATIVE, log_n, &tw, st));
    VS_TRY(get_twiddles(TW_NATIVE, log_eval, &tw, st));
    for (uint32_t l = 0; l < nf; l++) {
      const uint32_t* ft = nullptr;
      VS_TRY(get_fold_twiddles(l == 0 ? COSET_HALF_COSET : COSET_HALF_ODDS, log_eval - l, &ft, st));
    }
    VS_CUDA(cudaStreamSynchronize(st));
    // one plain run of a full batch sets kernel attributes before any capture;
    // then the graphs of every batch size a launch may use
    VS_TRY(enqueue(cap));
    VS_CUDA(cudaStreamSynchronize(st));
    for (uint32_t b = 1;; b = std::min(2 * b, cap)) {
      cudaGraphExec_t x = nullptr;
      VS_TRY(graph_for(b, &x));
      if (b == cap) break;
    }
    return VS_OK;
  }
  // Batch size a launch of `count` proofs runs at: the next power of two (at most
  // the capacity), so a workspace needs only log2(capacity) + 1 graphs; the
  // padding jobs prove (1, 1) and are not returned.
  uint32_t padded(uint32_t count) const {
    uint32_t b = 1;
    while (b < count) b *= 2;
    return std::min(b, cap);
  }
};

BatchProver::BatchProver() : impl(new Impl) {}
BatchProver::~BatchProver() = default;

uint32_t BatchProver::default_capacity(uint32_t log_n) {
  return log_n <= 16 ? 64u : std::max<uint32_t>(1u, 64u >> std::min<uint32_t>(log_n - 16, 6));
}

uint64_t BatchProver::bytes_for(uint32_t log_n, uint32_t capacity) {
  Impl p;
  p.plan(log_n, capacity);
  return p.total;
}

int BatchProver::init(uint32_t log_n, uint32_t capacity) {
  if (log_n < 4 || log_n > BATCH_MAX_LOG_N)
    return set_error(VS_ERR_INVALID, "batch prover: log_n %u outside [4, %u]", log_n, BATCH_MAX_LOG_N);
  if (capacity == 0 || capacity > 1024) return set_error(VS_ERR_INVALID, "batch prover: capacity %u", capacity);
  return impl->setup(log_n, capacity);
}

int BatchProver::launch(const uint32_t* ab, uint32_t count, cudaStream_t on) {
  if (count == 0 || count > impl->cap)
    return set_error(VS_ERR_INVALID, "batch of %u proofs (capacity %u)", count, impl->cap);
  for (uint32_t i = 0; i < 2 * count; i++)
    if (ab[i] >= h::P) return set_error(VS_ERR_INVALID, "public inputs must be canonical M31");
  const uint32_t b = impl->padded(count);
  cudaGraphExec_t x = nullptr;
  VS_TRY(impl->graph_for(b, &x));
  std::copy(ab, ab + 2 * count, impl->h_ab);
  std::fill(impl->h_ab + 2 * count, impl->h_ab + 2 * b, 1u);
  impl->count = count;
  impl->running = on ? on : impl->st;
  VS_CUDA(cudaGraphLaunch(x, impl->running));
  return VS_OK;
}

int BatchProver::finish(std::vector<std::vector<uint8_t>>& out) {
  VS_CUDA(cudaStreamSynchronize(impl->running ? impl->running : impl->st));
  impl->running = nullptr;  // the launch stream may be reused for other work from here on
  const uint32_t count = impl->count;
  out.resize(count);
  auto ser = [&](uint32_t j0, uint32_t step) {
    for (uint32_t j = j0; j < count; j += step)
      impl->lay.serialize(impl->h_arena + (uint64_t)j * impl->lay.words, impl->h_ab[2 * j], impl->h_ab[2 * j + 1],
                          out[j]);
  };
  // a batch's proofs are serialised on up to 8 host threads (about 0.1 ms per MB each)
  const uint32_t nt = std::min<uint32_t>(8, count / 4);
  std::vector<std::thread> th;
  for (uint32_t t = 1; t < nt; t++) th.emplace_back(ser, t, nt);
  ser(0, std::max<uint32_t>(nt, 1));
  for (auto& x : th) x.join();
  return VS_OK;
}

uint32_t BatchProver::log_n() const { return impl->log_n; }
uint32_t BatchProver::capacity() const { return impl->cap; }
uint64_t BatchProver::device_bytes() const { return impl->total; }

}  // namespace vs
