// stwo wire-format helpers for decommitments (src/stwo_export.rs): stwo's
// verifier consumes Merkle decommitments as a deduplicated `hash_witness` (the
// sibling hashes a verifier cannot compute itself, level by level from the
// leaves, in ascending position order) and FRI layers as a `fri_witness` (the
// fold-pair partner values that were not queried themselves). The prover here
// emits one auth path per query (leaf-to-root siblings); these functions turn a
// set of paths into stwo's form and rebuild a root from it. Host code.
#include <algorithm>
#include <cstring>
#include <map>
#include <set>
#include <vector>

#include "host_math.h"
#include "vs_common.cuh"

namespace vs {
namespace {

// Queried positions, sorted and deduplicated, each with the first query that has it.
std::map<uint64_t, uint32_t> first_query(const uint64_t* pos, uint32_t n) {
  std::map<uint64_t, uint32_t> m;
  for (uint32_t i = 0; i < n; i++) m.emplace(pos[i], i);
  return m;
}

// Walks the levels: a node whose sibling is also present needs nothing; otherwise
// its sibling comes from the path of the query it descends from
// (stwo_export.rs:269-320; fold pairs :208-267 start from whole pairs).
int walk(std::map<uint64_t, uint32_t> level, const uint32_t* paths, uint32_t height, uint32_t* out, uint32_t cap,
         uint32_t* out_len) {
  uint32_t w = 0;
  for (uint32_t k = 0; k < height; k++) {
    std::map<uint64_t, uint32_t> next;
    for (auto it = level.begin(); it != level.end();) {
      const uint64_t pos = it->first;
      const uint32_t q = it->second;
      auto nx = std::next(it);
      if (nx != level.end() && nx->first == (pos ^ 1)) {
        it = std::next(nx);
      } else {
        if (w >= cap) return set_error(VS_ERR_INVALID, "hash witness: output holds %u hashes", cap);
        std::memcpy(out + 8ull * w, paths + ((uint64_t)q * height + k) * 8, 32);
        w++;
        it = nx;
      }
      next.emplace(pos >> 1, q);
    }
    level.swap(next);
  }
  *out_len = w;
  return VS_OK;
}

}  // namespace
}  // namespace vs

using namespace vs;

extern "C" {

int vs_stwo_hash_witness(const uint64_t* h_positions, uint32_t n, const uint32_t* h_paths, uint32_t height,
                         uint32_t* h_out, uint32_t cap_hashes, uint32_t* out_len) {
  clear_error();
  if (!out_len || (n && (!h_positions || (height && (!h_paths || !h_out)))))
    return set_error(VS_ERR_INVALID, "vs_stwo_hash_witness: null argument");
  *out_len = 0;
  if (!n || !height) return VS_OK;
  return walk(first_query(h_positions, n), h_paths, height, h_out, cap_hashes, out_len);
}

int vs_stwo_fold_pair_hash_witness(const uint64_t* h_positions, uint32_t n, const uint32_t* h_paths, uint32_t height,
                                   uint32_t* h_out, uint32_t cap_hashes, uint32_t* out_len) {
  clear_error();
  if (!out_len || (n && (!h_positions || (height && (!h_paths || !h_out)))))
    return set_error(VS_ERR_INVALID, "vs_stwo_fold_pair_hash_witness: null argument");
  *out_len = 0;
  if (!n || !height) return VS_OK;
  // stwo opens whole fold pairs: both members of each queried pair are leaves,
  // carried by the query at either member (the member itself first).
  const auto q = first_query(h_positions, n);
  std::map<uint64_t, uint32_t> level;
  for (const auto& kv : q)
    for (uint64_t m : {kv.first & ~1ull, kv.first | 1ull}) {
      auto self = q.find(m);
      level.emplace(m, self != q.end() ? self->second : q.at(m ^ 1));
    }
  return walk(level, h_paths, height, h_out, cap_hashes, out_len);
}

int vs_stwo_fri_witness(const uint64_t* h_positions, uint32_t n, const uint32_t* h_sibling_values, uint32_t* h_out,
                        uint32_t cap, uint32_t* out_len) {
  clear_error();
  if (!out_len || (n && (!h_positions || !h_sibling_values || !h_out)))
    return set_error(VS_ERR_INVALID, "vs_stwo_fri_witness: null argument");
  // stwo_export.rs:174-203: the partner value of each queried position whose
  // partner is not queried, in ascending position order
  const auto q = first_query(h_positions, n);
  uint32_t w = 0;
  for (const auto& kv : q) {
    if (q.count(kv.first ^ 1)) continue;
    if (w >= cap) return set_error(VS_ERR_INVALID, "fri witness: output holds %u values", cap);
    std::memcpy(h_out + 4ull * w, h_sibling_values + 4ull * kv.second, 16);
    w++;
  }
  *out_len = w;
  return VS_OK;
}

// stwo_export.rs:711-790 (stwo's MerkleVerifier): leaves are Blake2s of the row's
// little-endian words (all columns), nodes Blake2s(left || right); the witness is
// consumed in ascending position order per level and must be used up exactly.
int vs_stwo_root_from_witness(uint32_t log_height, const uint64_t* h_positions, uint32_t n, const uint32_t* h_rows,
                              uint32_t n_cols, const uint32_t* h_witness, uint32_t n_witness, uint32_t* h_root) {
  clear_error();
  if (!n || !h_positions || !h_rows || !h_root || (n_witness && !h_witness))
    return set_error(VS_ERR_INVALID, "vs_stwo_root_from_witness: null argument or no positions");
  std::map<uint64_t, h::Hash> layer;
  for (uint32_t i = 0; i < n; i++)
    if (!layer.count(h_positions[i])) layer.emplace(h_positions[i], h::blake2s_words(h_rows + (uint64_t)i * n_cols, n_cols));
  uint32_t used = 0;
  for (uint32_t k = 0; k < log_height; k++) {
    std::map<uint64_t, h::Hash> next;
    for (auto it = layer.begin(); it != layer.end();) {
      const uint64_t pos = it->first;
      auto nx = std::next(it);
      h::Hash l, r;
      if (nx != layer.end() && nx->first == (pos ^ 1)) {
        l = it->second;
        r = nx->second;
        it = std::next(nx);
      } else {
        if (used >= n_witness) return set_error(VS_ERR_INVALID, "hash witness too short");
        h::Hash w;
        std::memcpy(w.data(), h_witness + 8ull * used++, 32);
        l = (pos & 1) ? w : it->second;
        r = (pos & 1) ? it->second : w;
        it = nx;
      }
      next.emplace(pos >> 1, h::node(l, r));
    }
    layer.swap(next);
  }
  if (used != n_witness) return set_error(VS_ERR_INVALID, "hash witness too long (%u of %u used)", used, n_witness);
  if (layer.size() != 1) return set_error(VS_ERR_INVALID, "expected one root, got %zu nodes", layer.size());
  std::memcpy(h_root, layer.begin()->second.data(), 32);
  return VS_OK;
}

}  // extern "C"
