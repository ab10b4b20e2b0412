// Graph-captured Fibonacci prover (one instance = one slot for one trace size).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

namespace vs {

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
  uint64_t device_bytes() const;

 private:
  struct Impl;
  std::unique_ptr<Impl> impl;
};

}  // namespace vs
