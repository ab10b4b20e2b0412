// Fibonacci STARK verifier (src/verifier.rs:39-236) and KRAK v1 decoding
// (src/bin/stark_cli.rs:979-1100). Host code; shares host_math with the prover.
#include <string>

#include "prover.h"
#include "vs_common.cuh"

namespace vs {

namespace {
struct Reader {
  const uint8_t* d;
  size_t n, pos = 0;
  bool ok = true;
  uint32_t u() {
    if (pos + 4 > n) { ok = false; return 0; }
    uint32_t v = d[pos] | (d[pos + 1] << 8) | (d[pos + 2] << 16) | ((uint32_t)d[pos + 3] << 24);
    pos += 4;
    return v;
  }
  std::vector<std::vector<h::Hash>> paths(uint32_t count) {
    std::vector<std::vector<h::Hash>> ps;
    for (uint32_t i = 0; i < count && ok; i++) {
      uint32_t depth = u();
      if (depth > 64) { ok = false; break; }
      std::vector<h::Hash> p(depth);
      for (auto& hh : p) for (auto& x : hh) x = u();
      ps.push_back(std::move(p));
    }
    return ps;
  }
  bool d4(Decommit4& d) {
    uint32_t k = u();
    if (!ok || k > 4096) return ok = false;
    d.values.resize(k);
    d.sibling_values.resize(k);
    for (auto& v : d.values) for (auto& x : v) x = u();
    for (auto& v : d.sibling_values) for (auto& x : v) x = u();
    d.auth_paths = paths(k);
    d.sibling_auth_paths = paths(k);
    return ok;
  }
};

bool path_ok(const h::Hash& root, h::Hash cur, uint64_t idx, const std::vector<h::Hash>& path) {
  for (const auto& s : path) { cur = (idx % 2 == 0) ? h::node(cur, s) : h::node(s, cur); idx >>= 1; }
  return cur == root;
}
h::Q q4(const std::array<uint32_t, 4>& v) { return {{v[0], v[1], v[2], v[3]}}; }
h::Hash leaf4(const std::array<uint32_t, 4>& v) { return h::blake2s_words(v.data(), 4); }
uint32_t fold_twiddle_at(const h::Coset& dom, uint64_t folded, bool circle) {  // verifier.rs:30-36
  h::Pt p = dom.at(h::brev(folded << 1, dom.log_size));
  return h::inv(circle ? p.y : p.x);
}
h::Q fold_pair(h::Q f0, h::Q f1, h::Q alpha, uint32_t tw) {
  return h::qadd(h::qadd(f0, f1), h::qmul(alpha, h::qscale(h::qsub(f0, f1), tw)));
}
std::string check4(const h::Hash& root, const Decommit4& d, const std::vector<uint64_t>& idx, const std::string& label) {
  if (d.values.size() != N_QUERIES || d.auth_paths.size() != N_QUERIES || d.sibling_values.size() != N_QUERIES ||
      d.sibling_auth_paths.size() != N_QUERIES)
    return label + " decommitment size mismatch";
  for (size_t q = 0; q < idx.size(); q++) {
    if (!path_ok(root, leaf4(d.values[q]), idx[q], d.auth_paths[q])) return label + " auth path invalid";
    if (!path_ok(root, leaf4(d.sibling_values[q]), idx[q] ^ 1, d.sibling_auth_paths[q]))
      return label + " sibling auth path invalid";
  }
  return "";
}
}  // namespace

bool deserialize(const uint8_t* data, size_t len, FibProof& p) {
  Reader r{data, len};
  if (r.u() != 0x4B52414Bu || r.u() != 1) return false;
  p = FibProof{};
  p.log_n = r.u();
  p.a = r.u();
  p.b = r.u();
  for (auto& x : p.trace_root) x = r.u();
  for (auto& x : p.quot_root) x = r.u();
  uint32_t nf = r.u();
  if (nf > 64) return false;
  p.fri_roots.resize(nf);
  for (auto& hh : p.fri_roots) for (auto& x : hh) x = r.u();
  uint32_t nl = r.u();
  if (nl > 1024) return false;
  p.last.resize(nl);
  for (auto& q : p.last) for (auto& x : q.v) x = r.u();
  uint32_t nq = r.u();
  if (nq > 4096) return false;
  for (uint32_t i = 0; i < nq; i++) p.queries.push_back(r.u());
  uint32_t tn = r.u();
  if (tn > 4096) return false;
  for (uint32_t i = 0; i < tn; i++) p.trace.values.push_back(r.u());
  for (uint32_t i = 0; i < tn; i++) p.trace.sibling_values.push_back(r.u());
  p.trace.auth_paths = r.paths(tn);
  p.trace.sibling_auth_paths = r.paths(tn);
  if (!r.d4(p.quot)) return false;
  uint32_t nd = r.u();
  if (nd > 64) return false;
  p.fri.resize(nd);
  for (auto& d : p.fri) if (!r.d4(d)) return false;
  return r.ok && r.pos == len;
}

std::string verify(const FibProof& p) {
  if (p.log_n < 1 || p.log_n > 29) return "bad log size";
  const uint32_t log_eval = p.log_n + BLOWUP_BITS;
  const uint64_t N = 1ull << log_eval;
  if (p.a >= h::P || p.b >= h::P) return "Public inputs out of M31 range";
  if (p.queries.size() != N_QUERIES) return "Expected 80 queries";
  h::Channel ch;
  ch.mix_digest(p.trace_root);
  (void)ch.draw_felt();
  ch.mix_digest(p.quot_root);
  std::vector<h::Q> alphas{ch.draw_felt()};
  for (const auto& c : p.fri_roots) { ch.mix_digest(c); alphas.push_back(ch.draw_felt()); }
  if (p.fri_roots.size() != (log_eval > 3 ? log_eval - 3 : 0)) return "wrong number of FRI layers";
  if (p.last.size() != 8) return "wrong FRI last layer size";
  ch.mix_felts(p.last);
  for (uint32_t q = 0; q < N_QUERIES; q++)
    if (p.queries[q] != ch.draw_number(N)) return "Query indices don't match Fiat-Shamir derivation";
  if (p.trace_root == h::Hash{}) return "Trace commitment is zero";
  if (p.quot_root == h::Hash{}) return "Quotient commitment is zero";
  const auto& t = p.trace;
  if (t.values.size() != N_QUERIES || t.auth_paths.size() != N_QUERIES || t.sibling_values.size() != N_QUERIES ||
      t.sibling_auth_paths.size() != N_QUERIES)
    return "trace decommitment size mismatch";
  for (size_t q = 0; q < N_QUERIES; q++) {
    if (!path_ok(p.trace_root, h::blake2s_words(&t.values[q], 1), p.queries[q], t.auth_paths[q]))
      return "trace auth path invalid";
    if (!path_ok(p.trace_root, h::blake2s_words(&t.sibling_values[q], 1), p.queries[q] ^ 1, t.sibling_auth_paths[q]))
      return "trace sibling auth path invalid";
  }
  std::string e = check4(p.quot_root, p.quot, p.queries, "quotient");
  if (!e.empty()) return e;
  std::vector<uint64_t> folded;
  for (uint64_t q : p.queries) folded.push_back(q / 2);
  const size_t nl = std::min(p.fri.size(), p.fri_roots.size());
  for (size_t l = 0; l < nl; l++) {
    e = check4(p.fri_roots[l], p.fri[l], folded, "FRI layer " + std::to_string(l));
    if (!e.empty()) return e;
    for (auto& f : folded) f /= 2;
  }
  const size_t nfd = p.fri.size();
  if (nfd == 0) return "no FRI decommitments";
  for (size_t q = 0; q < N_QUERIES; q++) {
    uint64_t idx = p.queries[q];
    uint32_t cl = log_eval;
    {
      h::Coset dom = cl <= 30 ? h::half_coset(cl) : h::subgroup(cl);
      uint64_t fi = idx / 2;
      h::Q v = q4(p.quot.values[q]), s = q4(p.quot.sibling_values[q]);
      h::Q f0 = idx % 2 == 0 ? v : s, f1 = idx % 2 == 0 ? s : v;
      if (!(fold_pair(f0, f1, alphas[0], fold_twiddle_at(dom, fi, true)) == q4(p.fri[0].values[q])))
        return "Circle fold mismatch";
      idx = fi;
      cl--;
    }
    for (size_t l = 0; l + 1 < nfd; l++) {
      h::Coset dom = h::half_odds(cl);
      uint64_t fi = idx / 2;
      h::Q v = q4(p.fri[l].values[q]), s = q4(p.fri[l].sibling_values[q]);
      h::Q f0 = idx % 2 == 0 ? v : s, f1 = idx % 2 == 0 ? s : v;
      if (l + 1 >= alphas.size()) return "missing FRI alpha";
      if (!(fold_pair(f0, f1, alphas[l + 1], fold_twiddle_at(dom, fi, false)) == q4(p.fri[l + 1].values[q])))
        return "Line fold mismatch";
      idx = fi;
      cl--;
    }
    if (idx >= p.last.size()) return "FRI last layer index out of bounds";
    if (!(q4(p.fri[nfd - 1].values[q]) == p.last[idx])) return "FRI last layer mismatch";
  }
  return "";
}

}  // namespace vs

using namespace vs;

extern "C" int vs_verify_fib(const uint8_t* h_proof, uint64_t len, char* err, uint64_t err_cap) {
  clear_error();
  FibProof p;
  std::string e;
  if (!h_proof || !deserialize(h_proof, len, p)) e = "undecodable proof";
  else e = verify(p);
  if (err && err_cap) snprintf(err, err_cap, "%s", e.c_str());
  if (e.empty()) return VS_OK;
  return set_error(VS_ERR_INVALID, "%s", e.c_str());
}
