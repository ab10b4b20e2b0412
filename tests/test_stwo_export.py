"""stwo wire-format helpers (src/stwo_export.rs) in the library's C ABI against a
direct Python restatement of the reference functions, and against the oracle's
Merkle trees. These run on the host only; no GPU is needed."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

V = pytest.importorskip("vortexstark_b200")
P = 0x7FFFFFFF


@pytest.fixture(scope="module")
def L():
    return V.lib()


# ---------------------------------------------------------------- restatement (stwo_export.rs)
def ref_hash_witness(positions, paths, height):  # :269-320
    pos_to_q = {}
    for i, p in enumerate(positions):
        pos_to_q.setdefault(p, i)
    cur = dict(sorted(pos_to_q.items()))
    out = []
    for level in range(height):
        ps = list(cur)
        i = 0
        while i < len(ps):
            if i + 1 < len(ps) and ps[i + 1] == ps[i] ^ 1:
                i += 2
            else:
                out.append(paths[cur[ps[i]]][level])
                i += 1
        nxt = {}
        for p in ps:
            nxt.setdefault(p >> 1, cur[p])
        cur = dict(sorted(nxt.items()))
    return out


def ref_fold_pair_witness(positions, paths, height):  # :208-267
    pos_to_q = {}
    for i, p in enumerate(positions):
        pos_to_q.setdefault(p, i)
    pairs = sorted({p & ~1 for p in pos_to_q} | {p | 1 for p in pos_to_q})
    cur = {p: pos_to_q[p] if p in pos_to_q else pos_to_q[p ^ 1] for p in pairs}
    out = []
    for level in range(height):
        ps = sorted(cur)
        nxt = {}
        i = 0
        while i < len(ps):
            p = ps[i]
            if i + 1 < len(ps) and ps[i + 1] == p ^ 1:
                nxt.setdefault(p >> 1, cur[p])
                i += 2
            else:
                out.append(paths[cur[p]][level])
                nxt.setdefault(p >> 1, cur[p])
                i += 1
        cur = nxt
    return out


def ref_fri_witness(positions, sib_values):  # :174-203
    first = {}
    for i, p in enumerate(positions):
        first.setdefault(p, sib_values[i])
    return [first[p] for p in sorted(first) if (p ^ 1) not in first]


# ---------------------------------------------------------------- C ABI wrappers
def lib_witness(L, fn, positions, paths, height):
    n = len(positions)
    pos = (C.c_uint64 * max(1, n))(*positions)
    flat = np.ascontiguousarray(paths, np.uint32).reshape(-1)
    hp = (C.c_uint32 * max(1, flat.size))(*flat.tolist())
    out = (C.c_uint32 * max(8, n * height * 8))()
    m = C.c_uint32()
    assert fn(pos, n, hp, height, out, max(1, n * height), C.byref(m)) == 0, L.vs_last_error()
    return np.array(out, np.uint32)[: m.value * 8].reshape(-1, 8)


def lib_root(L, log_h, positions, rows, witness):
    n = len(positions)
    rows = np.ascontiguousarray(rows, np.uint32)
    w = np.ascontiguousarray(witness, np.uint32).reshape(-1)
    root = (C.c_uint32 * 8)()
    rc = L.vs_stwo_root_from_witness(log_h, (C.c_uint64 * n)(*positions), n,
                                     (C.c_uint32 * rows.size)(*rows.reshape(-1).tolist()), rows.shape[1],
                                     (C.c_uint32 * max(1, w.size))(*w.tolist()), w.size // 8, root)
    return rc, np.array(root, np.uint32)


QUERY_SETS = [
    [5],
    [0, 1],                       # a complete pair
    [7, 3, 3, 12, 13, 63],        # duplicates, a pair, the last leaf
    list(range(0, 64, 3)),
    list(range(64)),              # every leaf: an empty witness
]


@pytest.mark.parametrize("qs", QUERY_SETS)
@pytest.mark.parametrize("kind,nc", [(0, 5), (1, 4)])
def test_hash_witness_matches_reference_and_rebuilds_root(L, qs, kind, nc):
    log_n = 6
    n = 1 << log_n
    cols = np.stack([O.seeded_m31(0x7D00 + 3 * c + kind, n) for c in range(nc)])
    paths = O.tree_paths(kind, cols, qs)
    got = lib_witness(L, L.vs_stwo_hash_witness, qs, paths, log_n)
    want = ref_hash_witness(qs, paths, log_n)
    assert np.array_equal(got, np.array(want, np.uint32).reshape(-1, 8))
    root = O.merkle_root_capped(cols) if kind == 0 else O.merkle_root_soa4(cols)
    rc, rebuilt = lib_root(L, log_n, qs, cols[:, qs].T, got)
    assert rc == 0, L.vs_last_error()
    assert np.array_equal(rebuilt, root)
    if len(got):  # a corrupted witness gives another root; a short or long one is refused
        bad = got.copy()
        bad[0, 0] ^= 1
        assert not np.array_equal(lib_root(L, log_n, qs, cols[:, qs].T, bad)[1], root)
        assert lib_root(L, log_n, qs, cols[:, qs].T, got[:-1])[0] != 0
    assert lib_root(L, log_n, qs, cols[:, qs].T, np.concatenate([got.reshape(-1, 8), np.zeros((1, 8), np.uint32)]))[0] != 0


@pytest.mark.parametrize("qs", QUERY_SETS[:4])
def test_fold_pair_witness_matches_reference_and_rebuilds_root(L, qs):
    log_n = 6
    cols = np.stack([O.seeded_m31(0x7E00 + c, 1 << log_n) for c in range(4)])
    paths = O.tree_paths(1, cols, qs)
    got = lib_witness(L, L.vs_stwo_fold_pair_hash_witness, qs, paths, log_n)
    want = ref_fold_pair_witness(qs, paths, log_n)
    assert np.array_equal(got, np.array(want, np.uint32).reshape(-1, 8))
    opened = sorted({p & ~1 for p in qs} | {p | 1 for p in qs})
    rc, rebuilt = lib_root(L, log_n, opened, cols[:, opened].T, got)
    assert rc == 0 and np.array_equal(rebuilt, O.merkle_root_soa4(cols))


@pytest.mark.parametrize("qs", QUERY_SETS)
def test_fri_witness_matches_reference(L, qs):
    rng = np.random.default_rng(len(qs))
    sib = rng.integers(0, P, size=(len(qs), 4), dtype=np.uint64).astype(np.uint32)
    n = len(qs)
    out = (C.c_uint32 * (4 * n))()
    m = C.c_uint32()
    assert L.vs_stwo_fri_witness((C.c_uint64 * n)(*qs), n, (C.c_uint32 * (4 * n))(*sib.reshape(-1).tolist()), out, n,
                                 C.byref(m)) == 0
    got = np.array(out, np.uint32)[: 4 * m.value].reshape(-1, 4)
    want = ref_fri_witness(qs, [tuple(r) for r in sib])
    assert np.array_equal(got, np.array(want, np.uint32).reshape(-1, 4))


def test_witness_output_capacity_is_checked(L):
    cols = np.stack([O.seeded_m31(0x7F00 + c, 64) for c in range(4)])
    paths = np.ascontiguousarray(O.tree_paths(1, cols, [5]), np.uint32).reshape(-1)
    out = (C.c_uint32 * 8)()
    m = C.c_uint32()
    assert L.vs_stwo_hash_witness((C.c_uint64 * 1)(5), 1, (C.c_uint32 * paths.size)(*paths.tolist()), 6, out, 1,
                                  C.byref(m)) != 0


# ---------------------------------------------------------------- whole proof (stwo_export.rs:415-690)
def ref_canonic_next(qi, log_eval):  # cairo_air/prover.rs:170-179
    n = 1 << log_eval
    cn = int(format(qi, f"0{log_eval}b")[::-1], 2)
    k = 2 * cn if cn < n // 2 else 2 * (n - 1 - cn) + 1
    kn = (k + 4) % n
    cnn = kn // 2 if kn % 2 == 0 else n - 1 - kn // 2
    return int(format(cnn, f"0{log_eval}b")[::-1], 2)


def two_hash(words):
    return [b for w in words for b in int(w).to_bytes(4, "little")]


def ref_stwo_proof(pp):
    """cairo_proof_to_stwo restated over the parts dict (field order of TwoStarkProof)."""
    log_eval = pp["log_trace_size"] + 2
    H = log_eval
    q = [int(x) for x in pp["query_indices"]]
    nq = len(q)
    tv = pp["trace_values_at_queries"]
    cfg = {"log_blowup_factor": 2, "n_queries": 80, "pow_bits": 26, "log_last_layer_degree_bound": 3}
    meta = [{"name": n, "n_cols": c, "log_eval_size": log_eval} for n, c in
            (("trace_lo", 16), ("trace_hi", 15), ("dict_trace", 3), ("interaction", 4), ("rc_interaction", 4),
             ("dict_interaction", 4), ("quotient", 4))]
    z, zn = pp.get("oods_trace_at_z"), pp.get("oods_trace_at_z_next")
    nz, nzn = (0 if z is None else len(z)), (0 if zn is None else len(zn))
    lo, hi, de = min(16, nz), min(31, nz), min(nz, 34)
    sv = []
    for a, b in ((0, lo), (min(lo, 16), hi), (min(hi, 31), de)):
        sv.append([[[int(x) for x in z[c]], [int(x) for x in zn[c]]] for c in range(a, b)] if nz and nzn else [])
    iz = np.zeros((3, 4, 4), np.uint32) if pp.get("oods_interaction_at_z") is None else pp["oods_interaction_at_z"]
    izn = np.zeros((3, 4, 4), np.uint32) if pp.get("oods_interaction_at_z_next") is None else pp["oods_interaction_at_z_next"]
    has, has_n = bool(np.any(iz)), bool(np.any(izn))
    for pi in range(3):
        sv.append([[[int(x) for x in iz[pi][k]]] + ([[int(x) for x in izn[pi][k]]] if has_n else []) for k in range(4)]
                  if has else [])
    qz = np.zeros((4, 4), np.uint32) if pp.get("oods_quotient_at_z") is None else pp["oods_quotient_at_z"]
    sv.append([[[int(x) for x in qz[k]]] for k in range(4)] if np.any(qz) else [])
    dec = []
    for t in range(3):
        cur, nxt = pp["trace_auth_paths"][t], (pp.get("trace_auth_paths_next") or [None] * 3)[t]
        m = {}
        for i, pos in enumerate(q):
            m.setdefault(pos, cur[i])
        if nxt is not None:
            for i, pos in enumerate(q):
                m.setdefault(ref_canonic_next(pos, log_eval), nxt[i])
        ps = sorted(m)
        dec.append({"hash_witness": [two_hash(h) for h in ref_hash_witness(ps, [m[x] for x in ps], H)]})
    for t in range(4):
        dec.append({"hash_witness": [two_hash(h) for h in ref_hash_witness(q, pp["decom_auth_paths"][t], H)]})
    hi_cols = min(tv.shape[1], 31) if nq else 16
    dict_cols = min(tv.shape[1], 34) if nq else 31
    qv = [[[int(tv[i][c]) for i in range(nq)] for c in range(a, b)] for a, b in ((0, 16), (16, hi_cols), (hi_cols, dict_cols))]
    for t in range(4):
        qv.append([[int(pp["decom_values"][t][i][k]) for i in range(nq)] for k in range(4)])
    first = {"fri_witness": [[int(x) for x in v] for v in ref_fri_witness(q, pp["oods_quotient_sibling_values"])],
             "decommitment": {"hash_witness": [two_hash(h) for h in
                                               ref_fold_pair_witness(q, pp["oods_quotient_auth_paths"], H)]},
             "commitment": two_hash(pp["oods_quotient_commitment"])}
    inner = []
    for i, c in enumerate(pp.get("fri_commitments", [])):
        lp = [x >> (i + 1) for x in q]
        inner.append({"fri_witness": [[int(x) for x in v] for v in ref_fri_witness(lp, pp["fri_sibling_values"][i])],
                      "decommitment": {"hash_witness": [two_hash(h) for h in
                                                        ref_fold_pair_witness(lp, pp["fri_auth_paths"][i], max(H - i - 1, 0))]},
                      "commitment": two_hash(c)})
    last = pp.get("last_layer_poly")
    return {"config": cfg, "tree_meta": meta, "commitments": [two_hash(c) for c in pp["commitments"]],
            "sampled_values": sv, "decommitments": dec, "queried_values": qv, "query_indices": q,
            "proof_of_work": int(pp.get("pow_nonce", 0)),
            "fri_proof": {"first_layer": first, "inner_layers": inner,
                          "last_layer_poly": [] if last is None else [[int(x) for x in v] for v in last]}}


def make_parts(log_n, qs, n_trace=34, oods=True, interaction=True, next_paths=True, seed=1):
    """Proof parts for trees of 2^(log_n+2) leaves with real Merkle paths: trace
    trees over capped leaves of seeded columns, quotient and FRI layers over SoA4
    leaves (so hash witnesses rebuild the committed roots)."""
    rng = np.random.default_rng(seed)
    H = log_n + 2
    n = 1 << H
    qs = list(qs)
    nq = len(qs)
    trace = np.stack([O.seeded_m31(0x8100 + c + seed, n) for c in range(n_trace)])
    groups = [(0, 16), (16, min(31, n_trace)), (min(31, n_trace), min(34, n_trace))]
    commitments, tpaths, tnext = [], [], []
    nxt = [ref_canonic_next(x, H) for x in qs]
    for a, b in groups:
        cols = trace[a:b] if b > a else np.zeros((1, n), np.uint32)
        commitments.append(O.merkle_root_capped(cols))
        tpaths.append(O.tree_paths(0, cols, qs))
        tnext.append(O.tree_paths(0, cols, nxt))
    dvals, dpaths = [], []
    for t in range(4):
        c4 = np.stack([O.seeded_m31(0x8200 + 4 * t + k + seed, n) for k in range(4)])
        commitments.append(O.merkle_root_soa4(c4))
        dvals.append(c4[:, qs].T.copy())
        dpaths.append(O.tree_paths(1, c4, qs))
    oq = np.stack([O.seeded_m31(0x8300 + k + seed, n) for k in range(4)])
    fri_c, fri_sv, fri_ap = [], [], []
    for i in range(H - 3):
        m = n >> (i + 1)
        layer = np.stack([O.seeded_m31(0x8400 + 16 * i + k + seed, m) for k in range(4)])
        fri_c.append(O.merkle_root_soa4(layer))
        lp = [x >> (i + 1) for x in qs]
        fri_sv.append(layer[:, [x ^ 1 for x in lp]].T.copy())
        fri_ap.append(O.tree_paths(1, layer, lp))
    r4 = lambda *s: rng.integers(0, P, size=s, dtype=np.uint64).astype(np.uint32)  # noqa: E731
    parts = {"log_trace_size": log_n, "query_indices": np.array(qs, np.uint64), "pow_nonce": 123456789012,
             "commitments": commitments, "trace_values_at_queries": trace[:, qs].T.copy(),
             "oods_trace_at_z": r4(n_trace, 4) if oods else None,
             "oods_trace_at_z_next": r4(n_trace, 4) if oods else None,
             "oods_interaction_at_z": r4(3, 4, 4) if interaction else None,
             "oods_interaction_at_z_next": r4(3, 4, 4) if interaction else None,
             "oods_quotient_at_z": r4(4, 4) if oods else None,
             "trace_auth_paths": tpaths, "trace_auth_paths_next": tnext if next_paths else None,
             "decom_values": dvals, "decom_auth_paths": dpaths,
             "oods_quotient_commitment": O.merkle_root_soa4(oq),
             "oods_quotient_sibling_values": oq[:, [x ^ 1 for x in qs]].T.copy(),
             "oods_quotient_auth_paths": O.tree_paths(1, oq, qs),
             "fri_commitments": fri_c, "fri_sibling_values": fri_sv, "fri_auth_paths": fri_ap,
             "last_layer_poly": r4(8, 4)}
    return parts


@pytest.mark.parametrize("log_n,qs,kw", [
    (4, [5, 7, 3, 3, 12, 13, 63, 0, 1], {}),
    (4, list(range(0, 64, 5)), {"next_paths": False}),
    (5, [17, 16, 100, 101, 2, 127], {"oods": False, "interaction": False}),
    (4, [9, 40], {"n_trace": 20}),
    (6, [], {}),
])
def test_stwo_proof_json_matches_reference_restatement(L, log_n, qs, kw):
    import json

    from vortexstark_b200 import api
    parts = make_parts(log_n, qs, **kw)
    got = api.stwo_proof_json(parts)
    assert got == json.dumps(ref_stwo_proof(parts), indent=2)
    proof = json.loads(got)
    H = log_n + 2
    if qs:  # the quotient tree's witness rebuilds its commitment from the queried values
        rows = np.array(proof["queried_values"][6], np.uint32).T
        w = np.array([[int.from_bytes(bytes(h[4 * k:4 * k + 4]), "little") for k in range(8)]
                      for h in proof["decommitments"][6]["hash_witness"]], np.uint32).reshape(-1, 8)
        rc, root = lib_root(L, H, qs, rows, w)
        assert rc == 0 and two_hash(root) == proof["commitments"][6]


def test_stwo_proof_json_rejects_bad_parts(L):
    from vortexstark_b200 import api
    parts = make_parts(4, [3, 4])
    parts["trace_values_at_queries"] = parts["trace_values_at_queries"][:, :10]
    with pytest.raises(V.VstarkError):
        api.stwo_proof_json(parts)
