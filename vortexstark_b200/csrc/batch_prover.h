// Batched Fibonacci prover: up to `capacity` independent proofs of one trace size
// in one CUDA graph, one kernel launch per stage for all of them.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

namespace vs {

// Largest trace size proved in batches; larger proofs fill the GPU alone and keep
// the tile-root trees of GraphProver (their full trees would not fit many times).
constexpr uint32_t BATCH_MAX_LOG_N = 22;

class BatchProver {
 public:
  BatchProver();
  ~BatchProver();
  // Default jobs per batch for a trace size: 64 at log_n 16, halving per size
  // above it, so a full batch holds about the same device memory at every size.
  static uint32_t default_capacity(uint32_t log_n);
  // Device bytes a workspace of this shape allocates (exactly what init() allocates).
  static uint64_t bytes_for(uint32_t log_n, uint32_t capacity);
  // Allocates the workspace on the current device, builds twiddles and captures
  // the graphs of batches of 1, 2, 4, ... proofs up to the capacity (a launch
  // runs at the next of those sizes, the extra proofs being discarded).
  int init(uint32_t log_n, uint32_t capacity);
  // Starts proofs of (ab[2i], ab[2i+1]) for i < count <= capacity on stream `on`
  // (one batch in flight per instance); finish() waits and serialises each proof.
  int launch(const uint32_t* ab, uint32_t count, cudaStream_t on);
  int finish(std::vector<std::vector<uint8_t>>& out);
  uint32_t log_n() const;
  uint32_t capacity() const;
  uint64_t device_bytes() const;

 private:
  struct Impl;
  std::unique_ptr<Impl> impl;
};

}  // namespace vs
