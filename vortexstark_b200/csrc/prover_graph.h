// Graph-captured Fibonacci prover (one instance = one slot for one trace size).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

namespace vs {

// Proof arena: the words of one proof as the device writes them (roots, last
// layer, queries, values, authentication paths), serialised to KRAK v1
// (src/bin/stark_cli.rs:907-976) on the host. Shared by the graph-captured and
// the batched provers, so both emit the same bytes.
struct ArenaLayout {
  uint32_t log_n = 0, log_eval = 0, nf = 0;
  size_t roots = 0, last = 0, q = 0, tv = 0, qv = 0, fv = 0, words = 0;
  std::vector<size_t> tree;     // path region per tree: trace, quotient, FRI layers
  std::vector<uint32_t> depth;  // authentication-path depth per tree
  void plan(uint32_t log_n);
  void serialize(const uint32_t* arena, uint32_t a, uint32_t b, std::vector<uint8_t>& out) const;
};

// Fibonacci trace of each job y (blockIdx.y): t0 = ab[2y], t1 = ab[2y+1], written
// to out + y * n (8192 rows per block).
__global__ void fib_trace_params_kernel(const uint32_t* __restrict__ ab, uint32_t* __restrict__ out, uint64_t n);

class GraphProver {
 public:
  GraphProver();
  ~GraphProver();
  // Allocates the workspace on the current device, builds twiddles and captures the graph.
  // The proof runs on a stream of the given CUDA priority (0 = default; lower
  // numbers are served first when several streams have work queued).
  int init(uint32_t log_n, int priority = 0);
  // Starts a proof (one in flight per instance) on `on` (default: the prover's own
  // stream); finish() waits for it and serialises KRAK v1.
  int launch(uint32_t a, uint32_t b, cudaStream_t on = nullptr);
  int finish(uint32_t a, uint32_t b, std::vector<uint8_t>& out);
  bool busy() const;
  uint32_t log_n() const;
  int device() const;
  cudaStream_t stream() const;
  uint64_t device_bytes() const;  // device bytes the prover allocated
  static uint64_t bytes_estimate(uint32_t log_n);  // >= device_bytes() of a prover of this size

 private:
  struct Impl;
  std::unique_ptr<Impl> impl;
};

}  // namespace vs
