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
