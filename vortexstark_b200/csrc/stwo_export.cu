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
#include <string>
#include <vector>

#include "host_math.h"
#include "vs_common.cuh"

namespace vs {
namespace {

constexpr uint32_t BLOWUP_BITS_EXPORT = 2;  // src/prover.rs:86

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

// ------------------------------------------------------------------ whole-proof export
// stwo_export.rs:415-660 (cairo_proof_to_stwo) and :687-690 (cairo_proof_to_json):
// the seven commitment trees in channel order, their OODS samples, queried values
// and deduplicated hash witnesses, and the FRI proof, written as the JSON text
// serde_json::to_string_pretty produces for TwoStarkProof (two-space indent, one
// array element per line, "[]" / "{}" when empty, hashes as arrays of 32 bytes).
namespace vs {
namespace {

// serde_json's PrettyFormatter.
struct JsonOut {
  std::string s;
  std::vector<bool> has;  // per open container: an element was written
  void nl() {
    s += '\n';
    s.append(2 * has.size(), ' ');
  }
  void elem() {  // before a value inside an array, or before an object member
    if (has.empty()) return;
    if (has.back()) s += ',';
    has.back() = true;
    nl();
  }
  void open(char c) { s += c; has.push_back(false); }
  void close(char c) {
    const bool any = has.back();
    has.pop_back();
    if (any) nl();
    s += c;
  }
  void key(const char* k) { elem(); s += '"'; s += k; s += "\": "; }
  void num(uint64_t v) { s += std::to_string(v); }
  void str(const char* v) { s += '"'; s += v; s += '"'; }
  void hash(const uint32_t* w) {  // TwoHash: the 32 little-endian bytes
    open('[');
    for (int i = 0; i < 8; i++)
      for (int b = 0; b < 4; b++) { elem(); num((w[i] >> (8 * b)) & 0xFF); }
    close(']');
  }
  void words(const uint32_t* w, size_t n) {
    open('[');
    for (size_t i = 0; i < n; i++) { elem(); num(w[i]); }
    close(']');
  }
  void qm31s(const uint32_t* v, size_t n) {  // [[u32; 4]; n]
    open('[');
    for (size_t i = 0; i < n; i++) { elem(); words(v + 4 * i, 4); }
    close(']');
  }
  void hashes(const std::vector<uint32_t>& h) {
    open('[');
    for (size_t i = 0; i < h.size() / 8; i++) { elem(); hash(h.data() + 8 * i); }
    close(']');
  }
};

uint64_t brev64(uint64_t v, uint32_t bits) {
  uint64_t r = 0;
  for (uint32_t i = 0; i < bits; i++) r |= ((v >> i) & 1) << (bits - 1 - i);
  return r;
}
// cairo_air/prover.rs:170-179: the BRT-canonic position of the next trace row.
uint64_t canonic_next(uint64_t qi, uint32_t log_eval) {
  const uint64_t n = 1ull << log_eval, cn = brev64(qi, log_eval);
  const uint64_t k = cn < n / 2 ? 2 * cn : 2 * (n - 1 - cn) + 1;
  const uint64_t kn = (k + (1ull << BLOWUP_BITS_EXPORT)) % n;
  const uint64_t cn_next = kn % 2 == 0 ? kn / 2 : n - 1 - kn / 2;
  return brev64(cn_next, log_eval);
}

int hash_witness(const std::vector<uint64_t>& pos, const uint32_t* paths, uint32_t height, bool fold_pairs,
                 std::vector<uint32_t>& out) {
  out.assign((size_t)8 * 2 * std::max<size_t>(pos.size(), 1) * std::max<uint32_t>(height, 1), 0);
  uint32_t n = 0;
  const uint32_t cap = (uint32_t)(out.size() / 8);
  VS_TRY(fold_pairs ? vs_stwo_fold_pair_hash_witness(pos.data(), (uint32_t)pos.size(), paths, height, out.data(), cap, &n)
                    : vs_stwo_hash_witness(pos.data(), (uint32_t)pos.size(), paths, height, out.data(), cap, &n));
  out.resize((size_t)8 * n);
  return VS_OK;
}
int fri_witness(const std::vector<uint64_t>& pos, const uint32_t* sib, std::vector<uint32_t>& out) {
  out.assign(4 * std::max<size_t>(pos.size(), 1), 0);
  uint32_t n = 0;
  VS_TRY(vs_stwo_fri_witness(pos.data(), (uint32_t)pos.size(), sib, out.data(), (uint32_t)pos.size(), &n));
  out.resize((size_t)4 * n);
  return VS_OK;
}
bool all_zero(const uint32_t* w, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (w[i]) return false;
  return true;
}

}  // namespace
}  // namespace vs

extern "C" {

int vs_stwo_proof_json(const vs_stwo_proof_parts* P, char* h_out, uint64_t cap, uint64_t* out_len) {
  clear_error();
  if (!P || !out_len) return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: null argument");
  const uint32_t nq = P->n_queries, log_eval = P->log_trace_size + BLOWUP_BITS_EXPORT, H = log_eval;
  if (log_eval > 40) return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: log_trace_size %u", P->log_trace_size);
  if (nq && (!P->query_indices || !P->trace_values_at_queries))
    return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: queries without indices or trace values");
  if (nq && P->n_trace_cols < 16) return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: fewer than 16 trace columns");
  if (P->n_oods && P->n_oods_next && P->n_oods_next < std::min<uint32_t>(P->n_oods, 34))
    return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: fewer z_next samples than z samples");
  for (int t = 0; t < 3; t++)
    if (nq && !P->trace_auth_paths[t]) return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: trace tree %d paths", t);
  for (int t = 0; t < 4; t++)
    if (nq && (!P->decom_values[t] || !P->decom_auth_paths[t]))
      return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: decommitment %d", t);
  if (nq && (!P->oods_quotient_sibling_values || !P->oods_quotient_auth_paths))
    return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: OODS quotient decommitment");
  if (P->n_fri && (!P->fri_commitments || (nq && (!P->fri_sibling_values || !P->fri_auth_paths))))
    return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: FRI layers");
  if (P->n_last && !P->last_layer_poly) return set_error(VS_ERR_INVALID, "vs_stwo_proof_json: last layer");
  const std::vector<uint64_t> q(P->query_indices, P->query_indices + nq);

  JsonOut J;
  J.open('{');
  J.key("config");
  J.open('{');
  J.key("log_blowup_factor"); J.num(BLOWUP_BITS_EXPORT);
  J.key("n_queries"); J.num(80);            // prover.rs:90
  J.key("pow_bits"); J.num(26);             // prover.rs:96
  J.key("log_last_layer_degree_bound"); J.num(3);  // fri.rs:265
  J.close('}');

  static const char* names[7] = {"trace_lo", "trace_hi", "dict_trace", "interaction", "rc_interaction",
                                 "dict_interaction", "quotient"};
  static const uint32_t cols[7] = {16, 15, 3, 4, 4, 4, 4};
  J.key("tree_meta");
  J.open('[');
  for (int t = 0; t < 7; t++) {
    J.elem();
    J.open('{');
    J.key("name"); J.str(names[t]);
    J.key("n_cols"); J.num(cols[t]);
    J.key("log_eval_size"); J.num(log_eval);
    J.close('}');
  }
  J.close(']');

  J.key("commitments");
  J.open('[');
  for (int t = 0; t < 7; t++) { J.elem(); J.hash(P->commitments[t]); }
  J.close(']');

  // OODS samples: trace trees at z and z_next, interaction trees (when sampled),
  // the quotient at z (stwo_export.rs:444-505)
  J.key("sampled_values");
  J.open('[');
  const uint32_t lo_end = std::min(16u, P->n_oods), hi_end = std::min(31u, P->n_oods),
                 dict_end = std::min(34u, P->n_oods);
  const uint32_t ranges[3][2] = {{0, lo_end}, {lo_end, hi_end}, {hi_end, dict_end}};
  for (int t = 0; t < 3; t++) {
    J.elem();
    J.open('[');
    if (P->n_oods && P->n_oods_next)
      for (uint32_t c = ranges[t][0]; c < ranges[t][1]; c++) {
        J.elem();
        J.open('[');
        J.elem(); J.words(P->oods_trace_at_z + 4ull * c, 4);
        J.elem(); J.words(P->oods_trace_at_z_next + 4ull * c, 4);
        J.close(']');
      }
    J.close(']');
  }
  const bool has_int = !all_zero(&P->oods_interaction_at_z[0][0][0], 48);
  const bool has_int_next = !all_zero(&P->oods_interaction_at_z_next[0][0][0], 48);
  for (int pi = 0; pi < 3; pi++) {
    J.elem();
    J.open('[');
    if (has_int)
      for (int k = 0; k < 4; k++) {
        J.elem();
        J.open('[');
        J.elem(); J.words(P->oods_interaction_at_z[pi][k], 4);
        if (has_int_next) { J.elem(); J.words(P->oods_interaction_at_z_next[pi][k], 4); }
        J.close(']');
      }
    J.close(']');
  }
  J.elem();
  J.open('[');
  if (!all_zero(&P->oods_quotient_at_z[0][0], 16))
    for (int k = 0; k < 4; k++) {
      J.elem();
      J.open('[');
      J.elem(); J.words(P->oods_quotient_at_z[k], 4);
      J.close(']');
    }
  J.close(']');
  J.close(']');

  // merkle decommitments (stwo_export.rs:554-600): trace trees over the merged
  // current and next-row positions (:659-685), the others over the queries
  J.key("decommitments");
  J.open('[');
  std::vector<uint32_t> w;
  for (int t = 0; t < 3; t++) {
    std::map<uint64_t, const uint32_t*> pos_path;  // current rows win over next rows
    for (uint32_t i = 0; i < nq; i++) pos_path.emplace(q[i], P->trace_auth_paths[t] + (uint64_t)i * H * 8);
    if (P->trace_auth_paths_next[t])
      for (uint32_t i = 0; i < nq; i++)
        pos_path.emplace(canonic_next(q[i], log_eval), P->trace_auth_paths_next[t] + (uint64_t)i * H * 8);
    std::vector<uint64_t> mpos;
    std::vector<uint32_t> mpaths;
    for (const auto& kv : pos_path) {
      mpos.push_back(kv.first);
      mpaths.insert(mpaths.end(), kv.second, kv.second + (size_t)H * 8);
    }
    VS_TRY(hash_witness(mpos, mpaths.data(), H, false, w));
    J.elem(); J.open('{'); J.key("hash_witness"); J.hashes(w); J.close('}');
  }
  for (int t = 0; t < 4; t++) {
    VS_TRY(hash_witness(q, P->decom_auth_paths[t], H, false, w));
    J.elem(); J.open('{'); J.key("hash_witness"); J.hashes(w); J.close('}');
  }
  J.close(']');

  // queried values, column-major per tree (stwo_export.rs:522-552)
  J.key("queried_values");
  J.open('[');
  const uint32_t nt = P->n_trace_cols;
  const uint32_t hi_cols = nq ? std::min(nt, 31u) : 16, dict_cols = nq ? std::min(nt, 34u) : 31;
  const uint32_t qr[3][2] = {{0, 16}, {16, hi_cols}, {hi_cols, dict_cols}};
  for (int t = 0; t < 3; t++) {
    J.elem();
    J.open('[');
    for (uint32_t c = qr[t][0]; c < qr[t][1]; c++) {
      J.elem();
      J.open('[');
      for (uint32_t i = 0; i < nq; i++) { J.elem(); J.num(P->trace_values_at_queries[(uint64_t)i * nt + c]); }
      J.close(']');
    }
    J.close(']');
  }
  for (int t = 0; t < 4; t++) {
    J.elem();
    J.open('[');
    for (int k = 0; k < 4; k++) {
      J.elem();
      J.open('[');
      for (uint32_t i = 0; i < nq; i++) { J.elem(); J.num(P->decom_values[t][4ull * i + k]); }
      J.close(']');
    }
    J.close(']');
  }
  J.close(']');

  J.key("query_indices");
  J.open('[');
  for (uint32_t i = 0; i < nq; i++) { J.elem(); J.num(q[i]); }
  J.close(']');
  J.key("proof_of_work"); J.num(P->pow_nonce);

  // FRI: the OODS quotient as first layer, then the committed line folds, whose
  // queried positions halve per layer (stwo_export.rs:602-646)
  J.key("fri_proof");
  J.open('{');
  J.key("first_layer");
  J.open('{');
  VS_TRY(fri_witness(q, P->oods_quotient_sibling_values, w));
  J.key("fri_witness"); J.qm31s(w.data(), w.size() / 4);
  VS_TRY(hash_witness(q, P->oods_quotient_auth_paths, H, true, w));
  J.key("decommitment"); J.open('{'); J.key("hash_witness"); J.hashes(w); J.close('}');
  J.key("commitment"); J.hash(P->oods_quotient_commitment);
  J.close('}');
  J.key("inner_layers");
  J.open('[');
  for (uint32_t l = 0; l < P->n_fri; l++) {
    const uint32_t lh = H > l + 1 ? H - l - 1 : 0;
    std::vector<uint64_t> lp(nq);
    for (uint32_t i = 0; i < nq; i++) lp[i] = q[i] >> (l + 1);
    J.elem();
    J.open('{');
    VS_TRY(fri_witness(lp, nq ? P->fri_sibling_values[l] : nullptr, w));
    J.key("fri_witness"); J.qm31s(w.data(), w.size() / 4);
    VS_TRY(hash_witness(lp, nq ? P->fri_auth_paths[l] : nullptr, lh, true, w));
    J.key("decommitment"); J.open('{'); J.key("hash_witness"); J.hashes(w); J.close('}');
    J.key("commitment"); J.hash(P->fri_commitments + 8ull * l);
    J.close('}');
  }
  J.close(']');
  J.key("last_layer_poly"); J.qm31s(P->last_layer_poly, P->n_last);
  J.close('}');
  J.close('}');

  *out_len = J.s.size();
  if (!h_out || cap < J.s.size())
    return h_out ? set_error(VS_ERR_INVALID, "vs_stwo_proof_json: needs %zu bytes", J.s.size()) : VS_OK;
  std::memcpy(h_out, J.s.data(), J.s.size());
  return VS_OK;
}
}  // extern "C"
