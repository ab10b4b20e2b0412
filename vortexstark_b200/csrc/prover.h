// Fibonacci prover / verifier internals (host structures of src/prover.rs:100-137).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <string>
#include <vector>

#include "host_math.h"

namespace vs {

constexpr uint32_t BLOWUP_BITS = 2;     // src/prover.rs:86
constexpr uint32_t N_QUERIES = 80;      // src/prover.rs:90
constexpr uint32_t LOG_LAST_LAYER = 3;  // src/fri.rs:265

struct Decommit1 {
  std::vector<uint32_t> values, sibling_values;
  std::vector<std::vector<h::Hash>> auth_paths, sibling_auth_paths;
};
struct Decommit4 {
  std::vector<std::array<uint32_t, 4>> values, sibling_values;
  std::vector<std::vector<h::Hash>> auth_paths, sibling_auth_paths;
};
struct FibProof {
  h::Hash trace_root{}, quot_root{};
  std::vector<h::Hash> fri_roots;
  std::vector<h::Q> last;
  uint32_t log_n = 0, a = 0, b = 0;
  std::vector<uint64_t> queries;
  Decommit1 trace;
  Decommit4 quot;
  std::vector<Decommit4> fri;
};

int prove_fib(uint32_t a, uint32_t b, uint32_t log_n, FibProof& pf, cudaStream_t st);
std::vector<uint8_t> serialize(const FibProof& p);
bool deserialize(const uint8_t* data, size_t len, FibProof& p);
std::string verify(const FibProof& p);  // "" when accepted

}  // namespace vs
