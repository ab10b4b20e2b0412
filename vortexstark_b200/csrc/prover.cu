// Fibonacci Circle-STARK prover on the device (stage order of the reference's
// prove_with_cache, src/prover.rs:1721-1978; constants src/prover.rs:86-96).
//
// B200-first layout of the same arithmetic:
//  * the trace is generated on the device (chunked Fibonacci jumps), so only
//    (a, b) crosses PCIe on the way in;
//  * interpolate -> zero-pad -> evaluate is one fused LDE (ntt.cu);
//  * the constraint quotient is never materialised: its Merkle leaves are
//    computed from the evaluation inside the tree kernel, and the circle fold
//    recomputes it from the evaluation as well (4 B/element instead of 16);
//  * every FRI fold is fused with its layer commitment;
//  * trees keep only the tile-root level and above resident; decommitment
//    recomputes the queried 1024-leaf tiles on the device and extracts the
//    sibling paths there, so only the proof's bytes come back to the host.
#include <algorithm>
#include <map>
#include <vector>

#include "fri_impl.cuh"
#include "host_math.h"
#include "merkle.h"
#include "ntt.h"
#include "prover.h"
#include "twiddles.h"
#include "vs_common.cuh"

namespace vs {

// ------------------------------------------------------------------ device helpers
// t_i = a F(i-1) + b F(i) (F(-1) = 1, F(0) = 0): each thread jumps to the start
// of its 32-element run with a 2x2 matrix power and then walks the recurrence;
// runs are staged through shared memory so stores are coalesced.
constexpr int TRACE_RUN = 32, TRACE_THREADS = 256;
__global__ void __launch_bounds__(TRACE_THREADS) fib_trace_kernel(uint32_t a, uint32_t b, uint32_t* __restrict__ out,
                                                                 uint64_t n) {
  __shared__ uint32_t sm[TRACE_THREADS * (TRACE_RUN + 1)];
  const uint64_t base = (uint64_t)blockIdx.x * TRACE_THREADS * TRACE_RUN;
  const uint64_t s = base + (uint64_t)threadIdx.x * TRACE_RUN;
  // M^s with M = [[1,1],[1,0]] = [[F(s+1), F(s)], [F(s), F(s-1)]]
  uint32_t m00 = 1, m01 = 0, m11 = 1, b00 = 1, b01 = 1, b11 = 0;
  for (uint64_t e = s; e; e >>= 1) {
    if (e & 1) {
      uint32_t t00 = add(mul(m00, b00), mul(m01, b01));
      uint32_t t01 = add(mul(m00, b01), mul(m01, b11));
      uint32_t t11 = add(mul(m01, b01), mul(m11, b11));
      m00 = t00; m01 = t01; m11 = t11;
    }
    uint32_t t00 = add(mul(b00, b00), mul(b01, b01));
    uint32_t t01 = add(mul(b00, b01), mul(b01, b11));
    uint32_t t11 = add(mul(b01, b01), mul(b11, b11));
    b00 = t00; b01 = t01; b11 = t11;
  }
  // F(s-1) = m11, F(s) = m01, F(s+1) = m00
  uint32_t t0 = add(mul(a, m11), mul(b, m01));
  uint32_t t1 = add(mul(a, m01), mul(b, m00));
  uint32_t* row = sm + threadIdx.x * (TRACE_RUN + 1);
  row[0] = t0;
  row[1] = t1;
#pragma unroll
  for (int i = 2; i < TRACE_RUN; i++) {
    uint32_t t2 = add(t0, t1);
    row[i] = t2;
    t0 = t1;
    t1 = t2;
  }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < TRACE_THREADS * TRACE_RUN; e += TRACE_THREADS) {
    uint64_t g = base + e;
    if (g < n) out[g] = sm[(e / TRACE_RUN) * (TRACE_RUN + 1) + e % TRACE_RUN];
  }
}

// Quotient leaf: hash of q(i) = alpha * (e[i+2] - (e[i+1] + e[i])) (indices mod N).
struct LeafFibQuot {
  const uint32_t* e;
  uint64_t mask;
  qm31 alpha;
  __device__ __forceinline__ qm31 q(uint64_t i) const {
    uint32_t c = sub(e[(i + 2) & mask], add(e[(i + 1) & mask], e[i]));
    return qscale(alpha, c);
  }
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    qm31 r = q(i);
    uint32_t m[16] = {0};
    m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};
// Circle fold of the (recomputed) quotient into FRI layer 0, fused with its leaf hash.
struct LeafFoldQuot {
  LeafFibQuot quot;
  const uint32_t* tw;
  qm31 alpha;
  uint32_t* dst[4];
  __device__ __forceinline__ void operator()(uint64_t i, uint32_t out[8]) const {
    qm31 r = fold_pair(quot.q(2 * i), quot.q(2 * i + 1), alpha, __ldg(tw + i));
#pragma unroll
    for (int k = 0; k < 4; k++) dst[k][i] = r.v[k];
    uint32_t m[16] = {0};
    m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
    b2s_single(out, m, 4);
  }
};

// Recompute queried tiles and emit each query's TL intra-tile siblings.
template <class Leaf>
__global__ void __launch_bounds__(256) tile_paths_kernel(Leaf leaf, uint32_t TL, const uint64_t* __restrict__ tiles,
                                                         const uint64_t* __restrict__ q, uint32_t nq,
                                                         uint32_t* __restrict__ out) {
  extern __shared__ uint32_t tp_sm[];  // levels 0..TL, row-major hashes
  const uint64_t tile = tiles[blockIdx.x];
  const uint32_t n0 = 1u << TL;
  for (uint32_t i = threadIdx.x; i < n0; i += blockDim.x) {
    uint32_t hh[8];
    leaf((tile << TL) + i, hh);
    for (int w = 0; w < 8; w++) tp_sm[8 * i + w] = hh[w];
  }
  __syncthreads();
  uint32_t off = 0, cnt = n0;
  for (uint32_t k = 1; k <= TL; k++) {
    const uint32_t* prev = tp_sm + 8 * off;
    uint32_t* cur = tp_sm + 8 * (off + cnt);
    for (uint32_t i = threadIdx.x; i < cnt / 2; i += blockDim.x) {
      uint32_t hh[8];
      b2s_node(hh, prev + 16 * i, prev + 16 * i + 8);
      for (int w = 0; w < 8; w++) cur[8 * i + w] = hh[w];
    }
    off += cnt;
    cnt >>= 1;
    __syncthreads();
  }
  for (uint32_t qi = threadIdx.x; qi < nq; qi += blockDim.x) {
    if ((q[qi] >> TL) != tile) continue;
    uint32_t intra = (uint32_t)(q[qi] & (n0 - 1));
    uint32_t lo = 0, lc = n0;
    for (uint32_t k = 0; k < TL; k++) {
      uint32_t sib = (intra >> k) ^ 1;
      for (int w = 0; w < 8; w++) out[((uint64_t)qi * TL + k) * 8 + w] = tp_sm[8 * (lo + sib) + w];
      lo += lc;
      lc >>= 1;
    }
  }
}

// Siblings above the tile level from the resident layers.
__global__ void upper_paths_kernel(const uint32_t* const* __restrict__ layers, uint32_t n_up,
                                   const uint64_t* __restrict__ q, uint32_t nq, uint32_t TL,
                                   uint32_t* __restrict__ out) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq * n_up) return;
  uint32_t qi = t / n_up, k = t % n_up;
  uint64_t sib = ((q[qi] >> TL) >> k) ^ 1;
  for (int w = 0; w < 8; w++) out[((uint64_t)qi * n_up + k) * 8 + w] = layers[k][8 * sib + w];
}

__global__ void gather_kernel(const uint32_t* __restrict__ src, const uint64_t* __restrict__ idx, uint32_t n,
                              uint32_t* __restrict__ out) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = src[idx[t]];
}

// ------------------------------------------------------------------ host helpers
// Stream-ordered device allocations released together.
struct DevMem {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit DevMem(cudaStream_t s) : st(s) {}
  ~DevMem() { for (void* p : ptrs) cudaFreeAsync(p, st); }
  template <class T>
  int alloc(T** out, uint64_t count) {
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, std::max<uint64_t>(count, 1) * sizeof(T), st);
    if (e != cudaSuccess) return set_error(VS_ERR_OOM, "device allocation of %llu bytes: %s",
                                           (unsigned long long)(count * sizeof(T)), cudaGetErrorString(e));
    ptrs.push_back(p);
    *out = (T*)p;
    return VS_OK;
  }
};

struct DevTree {
  uint64_t n = 0;
  uint32_t TL = 0;
  std::vector<uint32_t*> layers;  // [0] tile roots ... back() = root
  h::Hash root{};
};

template <class Leaf>
static int commit_tree(const Leaf& leaf, uint64_t n, DevTree& t, DevMem& mem, cudaStream_t st) {
  t.n = n;
  t.TL = std::min<uint32_t>(MK_MAX_TL, ilog2(n));
  t.layers.clear();
  uint64_t cnt = n >> t.TL;
  uint32_t* l0 = nullptr;
  VS_TRY(mem.alloc(&l0, cnt * 8));
  const uint32_t sp = t.TL == MK_MAX_TL ? merkle_tile_split(n) : 0u;
  uint32_t *sub_a = nullptr, *sub_b = nullptr;
  if (sp) {
    VS_TRY(mem.alloc(&sub_a, (cnt << sp) * 8));
    VS_TRY(mem.alloc(&sub_b, (cnt << (sp - 1)) * 8));
  }
  VS_TRY(merkle_tile_roots_split(leaf, n, t.TL, sp, l0, sub_a, sub_b, st));
  t.layers.push_back(l0);
  while (cnt > 1) {
    uint32_t* par = nullptr;
    VS_TRY(mem.alloc(&par, (cnt / 2) * 8));
    VS_TRY(launch_hash_nodes(t.layers.back(), par, cnt / 2, st));
    t.layers.push_back(par);
    cnt /= 2;
  }
  VS_CUDA(cudaMemcpyAsync(t.root.data(), t.layers.back(), 32, cudaMemcpyDeviceToHost, st));
  VS_CUDA(cudaStreamSynchronize(st));
  return VS_OK;
}

template <class Leaf>
static int tree_paths(const Leaf& leaf, const DevTree& t, const std::vector<uint64_t>& idx,
                      std::vector<std::vector<h::Hash>>& paths, DevMem& mem, cudaStream_t st) {
  const uint32_t nq = (uint32_t)idx.size();
  std::vector<uint64_t> tiles;
  for (uint64_t i : idx) tiles.push_back(i >> t.TL);
  std::sort(tiles.begin(), tiles.end());
  tiles.erase(std::unique(tiles.begin(), tiles.end()), tiles.end());
  const uint32_t n_up = (uint32_t)t.layers.size() - 1;
  uint64_t *d_q, *d_tiles;
  uint32_t *d_tp, *d_up;
  const uint32_t** d_layers;
  VS_TRY(mem.alloc(&d_q, nq));
  VS_TRY(mem.alloc(&d_tiles, tiles.size()));
  VS_TRY(mem.alloc(&d_tp, (uint64_t)nq * t.TL * 8));
  VS_TRY(mem.alloc(&d_up, (uint64_t)nq * n_up * 8));
  VS_TRY(mem.alloc(&d_layers, t.layers.size()));
  VS_CUDA(cudaMemcpyAsync(d_q, idx.data(), nq * 8, cudaMemcpyHostToDevice, st));
  VS_CUDA(cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * 8, cudaMemcpyHostToDevice, st));
  VS_CUDA(cudaMemcpyAsync(d_layers, t.layers.data(), t.layers.size() * sizeof(void*), cudaMemcpyHostToDevice, st));
  if (t.TL > 0) {
    const unsigned smem = (unsigned)(((2u << t.TL) - 1) * 32);
    if (smem > 48 * 1024)
      VS_CUDA(cudaFuncSetAttribute(tile_paths_kernel<Leaf>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    tile_paths_kernel<Leaf><<<(unsigned)tiles.size(), 256, smem, st>>>(leaf, t.TL, d_tiles, d_q, nq, d_tp);
    VS_LAUNCHED("tile_paths_kernel");
  }
  if (n_up) {
    upper_paths_kernel<<<blocks_for((uint64_t)nq * n_up, 128), 128, 0, st>>>(d_layers, n_up, d_q, nq, t.TL, d_up);
    VS_LAUNCHED("upper_paths_kernel");
  }
  std::vector<uint32_t> htp((uint64_t)nq * t.TL * 8), hup((uint64_t)nq * n_up * 8);
  if (!htp.empty()) VS_CUDA(cudaMemcpyAsync(htp.data(), d_tp, htp.size() * 4, cudaMemcpyDeviceToHost, st));
  if (!hup.empty()) VS_CUDA(cudaMemcpyAsync(hup.data(), d_up, hup.size() * 4, cudaMemcpyDeviceToHost, st));
  VS_CUDA(cudaStreamSynchronize(st));
  paths.assign(nq, {});
  for (uint32_t q = 0; q < nq; q++) {
    auto& p = paths[q];
    for (uint32_t k = 0; k < t.TL; k++) { h::Hash x; std::copy_n(&htp[((uint64_t)q * t.TL + k) * 8], 8, x.begin()); p.push_back(x); }
    for (uint32_t k = 0; k < n_up; k++) { h::Hash x; std::copy_n(&hup[((uint64_t)q * n_up + k) * 8], 8, x.begin()); p.push_back(x); }
  }
  return VS_OK;
}

static int gather(const uint32_t* src, const std::vector<uint64_t>& idx, std::vector<uint32_t>& out, DevMem& mem,
                  cudaStream_t st) {
  uint64_t* d_idx;
  uint32_t* d_out;
  const uint32_t n = (uint32_t)idx.size();
  VS_TRY(mem.alloc(&d_idx, n));
  VS_TRY(mem.alloc(&d_out, n));
  VS_CUDA(cudaMemcpyAsync(d_idx, idx.data(), n * 8, cudaMemcpyHostToDevice, st));
  gather_kernel<<<blocks_for(n, 128), 128, 0, st>>>(src, d_idx, n, d_out);
  VS_LAUNCHED("gather_kernel");
  out.resize(n);
  VS_CUDA(cudaMemcpyAsync(out.data(), d_out, n * 4, cudaMemcpyDeviceToHost, st));
  VS_CUDA(cudaStreamSynchronize(st));
  return VS_OK;
}

static qm31 to_dev(const h::Q& q) { return {{q.v[0], q.v[1], q.v[2], q.v[3]}}; }

int prove_fib(uint32_t a, uint32_t b, uint32_t log_n, FibProof& pf, cudaStream_t st) {
  if (log_n < 4 || log_n + BLOWUP_BITS > 30) return set_error(VS_ERR_INVALID, "log_n %u outside [4, 28]", log_n);
  if (a >= h::P || b >= h::P) return set_error(VS_ERR_INVALID, "public inputs must be canonical M31");
  const uint32_t log_eval = log_n + BLOWUP_BITS;
  const uint64_t n = 1ull << log_n, N = 1ull << log_eval;
  DevMem mem(st);
  pf = FibProof{};
  pf.log_n = log_n;
  pf.a = a;
  pf.b = b;

  // trace -> LDE (interpolate on half_coset(log_n), evaluate on half_coset(log_eval))
  uint32_t *d_trace, *d_eval;
  VS_TRY(mem.alloc(&d_trace, n));
  VS_TRY(mem.alloc(&d_eval, N));
  fib_trace_kernel<<<blocks_for(n, TRACE_THREADS * TRACE_RUN), TRACE_THREADS, 0, st>>>(a, b, d_trace, n);
  VS_LAUNCHED("fib_trace_kernel");
  VS_TRY(lde_cached(TW_NATIVE, d_trace, 0, d_eval, 0, 1, log_n, BLOWUP_BITS, st));

  // trace commitment (single-column leaf)
  DevTree trace_tree, quot_tree;
  VS_TRY(commit_tree(LeafOne{d_eval}, N, trace_tree, mem, st));
  pf.trace_root = trace_tree.root;
  h::Channel ch;
  ch.mix_digest(pf.trace_root);
  const h::Q alpha = ch.draw_felt();
  const LeafFibQuot quot{d_eval, N - 1, to_dev(alpha)};
  VS_TRY(commit_tree(quot, N, quot_tree, mem, st));
  pf.quot_root = quot_tree.root;
  ch.mix_digest(pf.quot_root);

  // FRI: circle fold of the quotient (recomputed from the evaluation), then line folds
  std::vector<DevTree> fri_trees;
  std::vector<std::array<uint32_t*, 4>> fri_vals;
  uint32_t cur = log_eval;
  while (cur > LOG_LAST_LAYER) {
    const h::Q fa = ch.draw_felt();
    const uint64_t half = 1ull << (cur - 1);
    std::array<uint32_t*, 4> dst;
    uint32_t* base;
    VS_TRY(mem.alloc(&base, 4 * half));
    for (int k = 0; k < 4; k++) dst[k] = base + k * half;
    const bool circle = cur == log_eval;
    const uint32_t* tw = nullptr;
    VS_TRY(get_fold_twiddles(circle ? COSET_HALF_COSET : COSET_HALF_ODDS, cur, &tw, st));
    DevTree t;
    if (circle) {
      LeafFoldQuot leaf{quot, tw, to_dev(fa), {dst[0], dst[1], dst[2], dst[3]}};
      VS_TRY(commit_tree(leaf, half, t, mem, st));
    } else {
      const auto& s = fri_vals.back();
      LeafFold leaf{};
      for (int k = 0; k < 4; k++) { leaf.src.c[k] = s[k]; leaf.dst.c[k] = dst[k]; }
      leaf.tw = tw;
      leaf.alpha = to_dev(fa);
      leaf.accumulate = 0;
      VS_TRY(commit_tree(leaf, half, t, mem, st));
    }
    pf.fri_roots.push_back(t.root);
    ch.mix_digest(t.root);
    fri_trees.push_back(std::move(t));
    fri_vals.push_back(dst);
    cur--;
  }
  {  // last layer (2^3 values)
    std::vector<uint32_t> planes(4 * 8);
    for (int k = 0; k < 4; k++)
      VS_CUDA(cudaMemcpyAsync(planes.data() + 8 * k, fri_vals.back()[k], 32, cudaMemcpyDeviceToHost, st));
    VS_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < 8; i++) pf.last.push_back({{planes[i], planes[8 + i], planes[16 + i], planes[24 + i]}});
  }
  ch.mix_felts(pf.last);
  for (uint32_t q = 0; q < N_QUERIES; q++) pf.queries.push_back(ch.draw_number(N));

  // decommitments: value at q and at its fold sibling q ^ 1, with auth paths
  std::vector<uint64_t> both;
  for (uint64_t q : pf.queries) both.push_back(q);
  for (uint64_t q : pf.queries) both.push_back(q ^ 1);
  {
    std::vector<uint32_t> v;
    VS_TRY(gather(d_eval, both, v, mem, st));
    pf.trace.values.assign(v.begin(), v.begin() + N_QUERIES);
    pf.trace.sibling_values.assign(v.begin() + N_QUERIES, v.end());
    std::vector<std::vector<h::Hash>> paths;
    VS_TRY(tree_paths(LeafOne{d_eval}, trace_tree, both, paths, mem, st));
    pf.trace.auth_paths.assign(paths.begin(), paths.begin() + N_QUERIES);
    pf.trace.sibling_auth_paths.assign(paths.begin() + N_QUERIES, paths.end());
  }
  {
    std::vector<uint64_t> pos;
    for (uint64_t i : both) for (uint64_t d = 0; d < 3; d++) pos.push_back((i + d) & (N - 1));
    std::vector<uint32_t> e;
    VS_TRY(gather(d_eval, pos, e, mem, st));
    for (size_t j = 0; j < both.size(); j++) {
      uint32_t c = h::sub(e[3 * j + 2], h::add(e[3 * j + 1], e[3 * j]));
      h::Q q = h::qscale(alpha, c);
      std::array<uint32_t, 4> w{q.v[0], q.v[1], q.v[2], q.v[3]};
      (j < N_QUERIES ? pf.quot.values : pf.quot.sibling_values).push_back(w);
    }
    std::vector<std::vector<h::Hash>> paths;
    VS_TRY(tree_paths(quot, quot_tree, both, paths, mem, st));
    pf.quot.auth_paths.assign(paths.begin(), paths.begin() + N_QUERIES);
    pf.quot.sibling_auth_paths.assign(paths.begin() + N_QUERIES, paths.end());
  }
  std::vector<uint64_t> folded;
  for (uint64_t q : pf.queries) folded.push_back(q / 2);
  for (size_t l = 0; l < fri_trees.size(); l++) {
    std::vector<uint64_t> fb(folded);
    for (uint64_t f : folded) fb.push_back(f ^ 1);
    Decommit4 d;
    std::vector<uint32_t> v[4];
    for (int k = 0; k < 4; k++) VS_TRY(gather(fri_vals[l][k], fb, v[k], mem, st));
    for (size_t j = 0; j < fb.size(); j++) {
      std::array<uint32_t, 4> w{v[0][j], v[1][j], v[2][j], v[3][j]};
      (j < N_QUERIES ? d.values : d.sibling_values).push_back(w);
    }
    std::vector<std::vector<h::Hash>> paths;
    LeafSoa4 leaf{fri_vals[l][0], fri_vals[l][1], fri_vals[l][2], fri_vals[l][3]};
    VS_TRY(tree_paths(leaf, fri_trees[l], fb, paths, mem, st));
    d.auth_paths.assign(paths.begin(), paths.begin() + N_QUERIES);
    d.sibling_auth_paths.assign(paths.begin() + N_QUERIES, paths.end());
    pf.fri.push_back(std::move(d));
    for (auto& f : folded) f /= 2;
  }
  VS_CUDA(cudaStreamSynchronize(st));
  return VS_OK;
}

// ------------------------------------------------------------------ KRAK v1 (stark_cli.rs:907-976)
static void w32(std::vector<uint8_t>& w, uint32_t v) { for (int k = 0; k < 4; k++) w.push_back((uint8_t)(v >> (8 * k))); }
static void wpaths(std::vector<uint8_t>& w, const std::vector<std::vector<h::Hash>>& ps) {
  for (const auto& p : ps) { w32(w, (uint32_t)p.size()); for (const auto& hh : p) for (uint32_t x : hh) w32(w, x); }
}
static void w4(std::vector<uint8_t>& w, const Decommit4& d) {
  w32(w, (uint32_t)d.values.size());
  for (const auto& v : d.values) for (uint32_t x : v) w32(w, x);
  for (const auto& v : d.sibling_values) for (uint32_t x : v) w32(w, x);
  wpaths(w, d.auth_paths);
  wpaths(w, d.sibling_auth_paths);
}
std::vector<uint8_t> serialize(const FibProof& p) {
  std::vector<uint8_t> w;
  w32(w, 0x4B52414Bu);
  w32(w, 1);
  w32(w, p.log_n);
  w32(w, p.a);
  w32(w, p.b);
  for (uint32_t x : p.trace_root) w32(w, x);
  for (uint32_t x : p.quot_root) w32(w, x);
  w32(w, (uint32_t)p.fri_roots.size());
  for (const auto& r : p.fri_roots) for (uint32_t x : r) w32(w, x);
  w32(w, (uint32_t)p.last.size());
  for (const auto& q : p.last) for (uint32_t x : q.v) w32(w, x);
  w32(w, (uint32_t)p.queries.size());
  for (uint64_t q : p.queries) w32(w, (uint32_t)q);
  w32(w, (uint32_t)p.trace.values.size());
  for (uint32_t v : p.trace.values) w32(w, v);
  for (uint32_t v : p.trace.sibling_values) w32(w, v);
  wpaths(w, p.trace.auth_paths);
  wpaths(w, p.trace.sibling_auth_paths);
  w4(w, p.quot);
  w32(w, (uint32_t)p.fri.size());
  for (const auto& d : p.fri) w4(w, d);
  return w;
}

}  // namespace vs

using namespace vs;

extern "C" int vs_prove_fib(uint32_t a, uint32_t b, uint32_t log_n, uint8_t* h_out, uint64_t cap, uint64_t* out_len,
                            vs_stream_t stream) {
  clear_error();
  FibProof pf;
  VS_TRY(prove_fib(a, b, log_n, pf, (cudaStream_t)stream));
  std::vector<uint8_t> bytes = serialize(pf);
  if (out_len) *out_len = bytes.size();
  if (!h_out || cap < bytes.size())
    return set_error(VS_ERR_INVALID, "proof needs %llu bytes, buffer has %llu", (unsigned long long)bytes.size(),
                     (unsigned long long)cap);
  std::copy(bytes.begin(), bytes.end(), h_out);
  return VS_OK;
}

// ------------------------------------------------------------------ decommitment of tile-rooted trees
namespace vs {
// out[q * n_cols + c] = cols[c][idx[q]]
__global__ void gather_cols_kernel(const uint32_t* const* __restrict__ cols, uint32_t n_cols,
                                   const uint64_t* __restrict__ idx, uint32_t nq, uint32_t* __restrict__ out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq * n_cols) return;
  const uint32_t q = t / n_cols, c = t % n_cols;
  out[t] = cols[c][idx[q]];
}

// Auth paths of a tree whose 1024-leaf tile roots are resident: the levels above
// the tiles are rebuilt from the tile roots, the queried tiles from their leaves.
template <class Leaf>
static int tile_tree_paths(const Leaf& leaf, uint32_t log_n, const uint32_t* d_tile_roots,
                           const std::vector<uint64_t>& idx, std::vector<std::vector<h::Hash>>& paths, DevMem& mem,
                           cudaStream_t st) {
  DevTree t;
  t.n = 1ull << log_n;
  t.TL = std::min<uint32_t>(MK_MAX_TL, log_n);
  uint64_t cnt = t.n >> t.TL;
  t.layers.push_back(const_cast<uint32_t*>(d_tile_roots));
  while (cnt > 1) {
    uint32_t* par = nullptr;
    VS_TRY(mem.alloc(&par, (cnt / 2) * 8));
    VS_TRY(launch_hash_nodes(t.layers.back(), par, cnt / 2, st));
    t.layers.push_back(par);
    cnt /= 2;
  }
  return tree_paths(leaf, t, idx, paths, mem, st);
}
}  // namespace vs

extern "C" int vs_tile_tree_paths(uint32_t leaf_kind, const uint32_t* const* h_cols, uint32_t n_cols,
                                  uint32_t log_n_leaves, const uint32_t* d_tile_roots, const uint64_t* h_indices,
                                  uint32_t n_indices, uint32_t* h_values, uint32_t* h_paths, vs_stream_t stream) {
  clear_error();
  cudaStream_t st = (cudaStream_t)stream;
  if (!h_cols || !d_tile_roots || (n_indices && (!h_indices || !h_paths)))
    return set_error(VS_ERR_INVALID, "vs_tile_tree_paths: null argument");
  if (leaf_kind == VS_LEAF_SOA4 ? n_cols != 4 : (leaf_kind != VS_LEAF_CAPPED || n_cols == 0 || n_cols > 16))
    return set_error(VS_ERR_INVALID, "vs_tile_tree_paths: leaf kind %u with %u columns", leaf_kind, n_cols);
  if (log_n_leaves > 30) return set_error(VS_ERR_INVALID, "vs_tile_tree_paths: log_n_leaves %u", log_n_leaves);
  for (uint32_t c = 0; c < n_cols; c++)
    if (!h_cols[c]) return set_error(VS_ERR_INVALID, "vs_tile_tree_paths: null column %u", c);
  const uint64_t n = 1ull << log_n_leaves;
  std::vector<uint64_t> idx(h_indices, h_indices + n_indices);
  for (uint64_t i : idx)
    if (i >= n) return set_error(VS_ERR_INVALID, "vs_tile_tree_paths: index %llu >= %llu", (unsigned long long)i,
                                 (unsigned long long)n);
  if (!n_indices) return VS_OK;
  DevMem mem(st);
  const uint32_t** d_cols = nullptr;
  VS_TRY(mem.alloc(&d_cols, n_cols));
  VS_CUDA(cudaMemcpyAsync(d_cols, h_cols, n_cols * sizeof(void*), cudaMemcpyHostToDevice, st));
  std::vector<std::vector<h::Hash>> paths;
  if (leaf_kind == VS_LEAF_SOA4)
    VS_TRY(tile_tree_paths(LeafSoa4{h_cols[0], h_cols[1], h_cols[2], h_cols[3]}, log_n_leaves, d_tile_roots, idx,
                           paths, mem, st));
  else
    VS_TRY(tile_tree_paths(LeafCapped{d_cols, nullptr, 0, n_cols}, log_n_leaves, d_tile_roots, idx, paths, mem, st));
  for (uint32_t q = 0; q < n_indices; q++)
    for (uint32_t k = 0; k < log_n_leaves; k++)
      std::copy_n(paths[q][k].data(), 8, h_paths + ((uint64_t)q * log_n_leaves + k) * 8);
  if (h_values) {
    uint64_t* d_idx;
    uint32_t* d_out;
    VS_TRY(mem.alloc(&d_idx, n_indices));
    VS_TRY(mem.alloc(&d_out, (uint64_t)n_indices * n_cols));
    VS_CUDA(cudaMemcpyAsync(d_idx, idx.data(), n_indices * 8, cudaMemcpyHostToDevice, st));
    gather_cols_kernel<<<blocks_for((uint64_t)n_indices * n_cols, 128), 128, 0, st>>>(d_cols, n_cols, d_idx, n_indices,
                                                                                   d_out);
    VS_LAUNCHED("gather_cols_kernel");
    VS_CUDA(cudaMemcpyAsync(h_values, d_out, (uint64_t)n_indices * n_cols * 4, cudaMemcpyDeviceToHost, st));
    VS_CUDA(cudaStreamSynchronize(st));
  }
  return VS_OK;
}
